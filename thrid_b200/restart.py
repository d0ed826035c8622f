"""State record (restart) files in the reference's format, from and to the
device state.

write_sta restates wrsta.F90:8-180: header keys (#npoly, #nwater, #nmatom,
#natom, #mchain, #xcel/#ycel/#zcel in m, #nstep), one line per atom
(I10, 6E24.16, A3: running index, x y z in m, vx vy vz in m/s, atom type)
in the sections #poly / #water / #matom, then #nhc (xlogs, vlogs in 1/s),
#andersen (vlogv in 1/s, pint in Pa), #andersen_aniso (vboxg in 1/s, pintt
in Pa) and #end.  read_sta restates rdstarec.F90:8-393 (free-format fields,
conversion back to reduced units, atoms numbered in file order).

Values are written with 16 significant digits (Fortran E24.16), so a round
trip reproduces a double to about one unit in the 16th digit, as the
reference does.
"""
from __future__ import annotations

import numpy as np

from thrid_b200 import abi
from thrid_b200 import systems as S


def fortran_e(v: float, w: int = 24, d: int = 16) -> str:
    """Fortran Ew.d edit descriptor: 0.ddd...dE+xx, right-justified in w."""
    v = float(v)
    if v == 0.0:
        body = "0." + "0" * d + "E+00"
    else:
        s = f"{abs(v):.{d - 1}e}"                      # d1.d2...dd e+XX
        mant, ex = s.split("e")
        digits = mant.replace(".", "")
        e = int(ex) + 1
        if abs(e) <= 99:
            es = f"E{'+' if e >= 0 else '-'}{abs(e):02d}"
        else:
            es = f"{'+' if e >= 0 else '-'}{abs(e):03d}"
        body = ("-" if v < 0 else "") + "0." + digits + es
    return body.rjust(w)


def _section_atoms(system, npoly_mol):
    """Atom order of the file: molecules in molept_index order (poly first,
    then water, then monatomic), atoms of each in molept_list order."""
    mi, ml = system.molept_index, system.molept_list
    return [[int(a) for a in ml[mi[m]:mi[m + 1]]] for m in range(system.nmole)]


def header_lines(npoly, nwater, nmatom, natom, mchain, box_si, nstep):
    """Header of a state record (wrsta.F90:56-73), each line followed by the
    empty record of a bare list-directed write."""
    L = [f"#npoly{npoly:8d}", f"#nwater{nwater:8d}", f"#nmatom{nmatom:8d}", f"#natom{natom:10d}",
         f"#mchain{mchain:3d}", "#xcel" + fortran_e(box_si[0]), "#ycel" + fortran_e(box_si[1]),
         "#zcel" + fortran_e(box_si[2]), f"#nstep{int(nstep):12d}"]
    out = []
    for ln in L:
        out += [ln, ""]
    return out


def atom_line(k, x_si, v_si, tname):
    """One atom of a #poly / #water / #matom section, '(I10,6E24.16,A3)'
    (wrsta.F90:89-96): positions [m], velocities [m/s], type right-justified."""
    return f"{k:10d}" + "".join(fortran_e(q) for q in (*x_si, *v_si)) + tname[:3].rjust(3)


def chain_lines(xlogs, vlogs_si, vlogv_si, pint_si, vboxg_si, pintt_si):
    """#nhc, #andersen, #andersen_aniso and #end (wrsta.F90:148-175)."""
    L = ["#nhc"]
    for i, (a, b) in enumerate(zip(xlogs, vlogs_si)):
        L.append(f"{i + 1:10d}" + fortran_e(a) + fortran_e(b))
    L += ["", "#andersen", f"{1:10d}" + fortran_e(vlogv_si) + fortran_e(pint_si), "", "#andersen_aniso",
          f"{1:10d}" + "".join(fortran_e(q) for q in vboxg_si) + "".join(fortran_e(q) for q in pintt_si),
          "", "#end"]
    return L


def write_sta(path, system, atmcor, atmvel, box, chain, nstep, mchain=3, npoly=None, nwater=None, nmatom=None):
    """Write a state record.  npoly / nwater / nmatom count the molecules of
    the three sections in topology order (poly first, then water, then
    monatomic, as the reference lays them out); by default trailing 1-atom
    molecules are monatomic and all others poly."""
    mols = _section_atoms(system, None)
    if npoly is None:
        nmatom = 0
        while nmatom < len(mols) and len(mols[len(mols) - 1 - nmatom]) == 1:
            nmatom += 1
        nwater = 0
        npoly = len(mols) - nmatom
    if npoly + nwater + nmatom != len(mols):
        raise ValueError("npoly + nwater + nmatom must equal the number of molecules")
    xref, vref, tref, pref = S.XREF, S.VREF, S.TIMEREF, S.PREF
    names = system.type_names
    L = header_lines(npoly, nwater, nmatom, system.natom, mchain, [q * xref for q in box], nstep)
    k = 0
    # section tags as wrsta.F90:79,102,125 write them: '(A6)', so the 5-letter '#poly' is right-justified
    bounds = ((" #poly", 0, npoly), ("#water", npoly, npoly + nwater), ("#matom", npoly + nwater, len(mols)))
    for tag, m0, m1 in bounds:
        L.append(tag)
        for m in range(m0, m1):
            for a in mols[m]:
                k += 1
                L.append(atom_line(k, atmcor[a] * xref, atmvel[a] * vref, names[system.atmindex[a] - 1]))
        L.append("")
    L += chain_lines([chain.xlogs[i] for i in range(mchain)], [chain.vlogs[i] / tref for i in range(mchain)],
                     chain.vlogv / tref, chain.pint * pref, [chain.vboxg[d] / tref for d in range(3)],
                     [chain.pintt[q] * pref for q in range(9)])
    with open(path, "w") as f:
        f.write("\n".join(L) + "\n")


def _num(s):
    s = s.strip().upper().replace("D", "E")
    if "E" not in s and ("+" in s[1:] or "-" in s[1:]):       # Fortran 3-digit exponent without E
        for i in range(len(s) - 1, 0, -1):
            if s[i] in "+-":
                s = s[:i] + "E" + s[i:]
                break
    return float(s)


def read_sta(path):
    """Parse a state record; returns a dict in reduced units."""
    xref, vref, tref, pref = S.XREF, S.VREF, S.TIMEREF, S.PREF
    out = {"cor": [], "vel": [], "typ": [], "xlogs": [], "vlogs": []}
    sec = None
    with open(path) as f:
        for line in f:
            fld = line.split()
            if not fld:
                sec = None
                continue
            key = fld[0]
            if key.startswith("#"):
                sec = None
                if key in ("#npoly", "#nwater", "#nmatom", "#natom", "#mchain", "#nstep"):
                    out[key[1:]] = int(fld[1])
                elif key in ("#xcel", "#ycel", "#zcel"):
                    out[key[1:]] = _num(fld[1]) / xref
                elif key in ("#poly", "#poly1", "#water", "#matom", "#nhc", "#andersen", "#andersen_aniso"):
                    sec = key
                continue
            if sec in ("#poly", "#poly1", "#water", "#matom"):
                out["cor"].append([_num(q) / xref for q in fld[1:4]])
                out["vel"].append([_num(q) / vref for q in fld[4:7]])
                out["typ"].append(fld[7] if len(fld) > 7 else "")
            elif sec == "#nhc":
                out["xlogs"].append(_num(fld[1]))
                out["vlogs"].append(_num(fld[2]) * tref)
            elif sec == "#andersen":
                out["vlogv"] = _num(fld[1]) * tref
                out["pint"] = _num(fld[2]) / pref
            elif sec == "#andersen_aniso":
                vals = [_num(q) for q in fld[1:]]
                out["vboxg"] = [q * tref for q in vals[:3]]
                out["pintt"] = [q / pref for q in vals[3:12]]
    out["cor"] = np.asarray(out["cor"], float)
    out["vel"] = np.asarray(out["vel"], float)
    out["box"] = np.array([out.get("xcel", 0.0), out.get("ycel", 0.0), out.get("zcel", 0.0)])
    return out


def chain_from(rec):
    """pgk_chain of a parsed record (xlogv and xboxh follow from the box)."""
    ch = abi.chain_init(rec["box"])
    for i, (a, b) in enumerate(zip(rec["xlogs"], rec["vlogs"])):
        ch.xlogs[i] = a
        ch.vlogs[i] = b
    ch.vlogv = rec.get("vlogv", 0.0)
    ch.pint = rec.get("pint", 0.0)
    for d, v in enumerate(rec.get("vboxg", [0.0] * 3)):
        ch.vboxg[d] = v
    for q, v in enumerate(rec.get("pintt", [0.0] * 9)):
        ch.pintt[q] = v
    return ch


def wrsta(engine, path, nstep, mchain=3, **sections):
    """Checkpoint the device state of a PgkEngine (download, then write_sta)."""
    cor, vel, box = engine.download_state()
    write_sta(path, engine.sys, cor, vel, box, engine.get_chain(), nstep, mchain=mchain, **sections)


def rdstarec(engine, path):
    """Restore a PgkEngine from a state record (read_sta, then upload); the atoms
    of the file are taken in topology order, as rdstarec.F90 numbers them."""
    rec = read_sta(path)
    order = [a for m in _section_atoms(engine.sys, None) for a in m]
    n = engine.sys.natom
    if rec["cor"].shape != (n, 3):
        raise ValueError(f"state record holds {len(rec['cor'])} atoms, the system {n}")
    cor = np.zeros((n, 3)); vel = np.zeros((n, 3))
    cor[order] = rec["cor"]
    vel[order] = rec["vel"]
    engine.upload_state(cor, vel, rec["box"])
    engine.set_chain(chain_from(rec))
    return rec
