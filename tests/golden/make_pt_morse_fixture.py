"""Build tests/golden/pt_morse_step1.npz from the reference's sample run.

The reference tree ships one recorded run of its Pt/Morse sample (10
1-propanol + 190 butane on a 3,584-atom Pt slab, peachgk.ini): the energies
of step 1 in out_ene.dat (output_data.F90 outene, SI units, E15.8) and the
positions of the same step in out_pos.dat (outpos, output_data.F90:345-394,
Fortran unformatted records, single precision unless -D_DOUBLE_OUTPOS).  This
script restates the reference's input processing for that system and stores
every array the oracle needs, in reduced units, beside the recorded energies
and the virials of the same step (out_pre.dat, outpre):

  * rdpara.F90:100-760     <ATOM>, <BOND>, <ANGLE>, <TORSION>, <TORSION_RB>,
                           <MORSE>, <VDW_SP> of para_bond.dat; para_vdw_s.dat;
                           unit conversions; LJ mixing (A/G flags, ifljari);
                           Morse type pairs and inter_inttyp (Morse pairs
                           carry no LJ)
  * rdtop.F90:62-440       topology sections, molecule copies, ring14 and
                           ring14_rb -- including the reference's reset of
                           ring14_rb(1:ntors) with the periodic-torsion count
                           (rdtop.F90:378), which leaves ring14_rb = 0 (the
                           initial value of the SAVEd array) for every RB
                           torsion past index ntors
  * linkbond.F90:27-200    exact-name parameter lookup (last match wins),
                           per-type mass and charge, the Morse atom list
  * prepmd.F90:220-247     degrees -> radians, q / sqrt(4 pi eps0)
  * main_md.F90:267,390-396, calbase.F90  the reference's unit bases

Run in a checkout that has the reference tree (not needed to run the tests):

    python tests/golden/make_pt_morse_fixture.py REFERENCE_DIR
"""
import math
import os
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "pt_morse_step1.npz")

# main_md.F90:267, 390-396 (qref as the reference writes it)
XREF = 1.0e-10
EREF = 6.9511042e-21
QREF = 1.602117733e-19
EPS0 = 8.854187817e-12
EPS0REF = QREF ** 2 / EREF / XREF              # calbase.F90:71
CHARGE_SCALE = 1.0 / math.sqrt(4.0 * math.pi * (EPS0 / EPS0REF))   # prepmd.F90:241

ENE_KEYS = ("ene_kin", "pot_tot", "pot_nonbon", "pot_bon", "pot_coul", "pot_vdw", "pot_elc", "pot_ewk", "pot_ewc",
            "pot_ewnq", "pot_vdw14", "pot_elc14", "pot_bond", "pot_angl", "pot_tors", "pot_torsrb", "pot_mor")


def fnum(s):
    """Fortran real literal (d exponent)."""
    return float(s.lower().replace("d", "e"))


def words(line):
    """rdfree-like split: blank-separated words, text after '!' dropped."""
    return line.split("!")[0].split()


def read_ini(path):
    """peachgk.ini: keyword -> list of value words (repeated keywords kept in order)."""
    kv = {}
    for line in open(path):
        w = words(line)
        if not w or w[0].startswith("#") or w[0] == "END":
            continue
        kv.setdefault(w[0], []).append(w[1:])
    return kv


def read_sections(path):
    """<SECTION> blocks of a parameter or topology file: name -> list of word lists
    (comment lines starting with '#' or ';' skipped)."""
    sec, cur = {}, None
    for line in open(path):
        w = line.split()
        if not w:
            continue
        if w[0].startswith("<"):
            cur = w[0].strip("<>")
            sec.setdefault(cur, [])
            continue
        if cur is None or w[0][0] in "#;":
            continue
        sec[cur].append(w)
    return sec


def lookup(table, name):
    """linkbond.F90: exact name match over a parameter section (rows: index,
    name, values...), last match wins."""
    hit = None
    for row in table:
        if row[1] == name:
            hit = row
    if hit is None:
        raise KeyError(name)
    return hit


def pair_match(kind, a, b):
    """rdpara.F90:680-760 two-letter pair names 'AA-BB' in either order."""
    return (kind[0:2] == a and kind[3:5] == b) or (kind[0:2] == b and kind[3:5] == a)


def read_records(path):
    """Fortran unformatted sequential records (4-byte little-endian markers)."""
    b = open(path, "rb").read()
    off, recs = 0, []
    while off < len(b):
        n = struct.unpack("<i", b[off:off + 4])[0]
        recs.append(b[off + 4:off + 4 + n])
        off += 8 + n
    return recs


def read_out_pos(path):
    """outpos / outvel (output_data.F90:381-385, :430-436): step, then
    (i, x, y, z, atmtyp) per atom, REAL*4 [m] or [m/s]."""
    recs = read_records(path)
    step = struct.unpack("<i", recs[0])[0]
    idx, xyz, typ = [], [], []
    for r in recs[1:]:
        if len(r) != 18:
            raise ValueError("expected single-precision outpos records of 18 bytes")
        i, x, y, z = struct.unpack("<ifff", r[:16])
        idx.append(i); xyz.append((x, y, z)); typ.append(r[16:18].decode())
    if idx != list(range(1, len(idx) + 1)):
        raise ValueError("atom records out of order")
    return step, np.array(xyz, np.float32), typ


def read_state_record(path):
    """wrsta (wrsta.F90:8-180) state record: '#nstep', and per atom in the
    #poly / #water / #matom sections: index, x y z [m], vx vy vz [m/s], type."""
    step, cor, vel, typ, sec = None, [], [], [], None
    for line in open(path):
        w = line.split()
        if not w:
            continue
        if w[0].startswith("#"):
            sec = w[0]
            if w[0] == "#nstep":
                step = int(w[1])
            continue
        if sec in ("#poly", "#water", "#matom"):
            cor.append([fnum(q) for q in w[1:4]])
            vel.append([fnum(q) for q in w[4:7]])
            typ.append(w[7])
    return step, np.array(cor), np.array(vel), typ


def read_out_ene(path):
    """outene: header line of names, then one line per output step [J]."""
    lines = [ln.split() for ln in open(path) if ln.strip()]
    names = lines[0]
    rows = [dict(zip(names, (float(v) for v in ln))) for ln in lines[1:]]
    return rows


def build(ref):
    ini = read_ini(os.path.join(ref, "peachgk.ini"))
    para = read_sections(os.path.join(ref, ini["iuparabondname"][0][0]))
    vdw = [w for w in (ln.split() for ln in open(os.path.join(ref, ini["iuparavdwname"][0][0])))
           if len(w) >= 5 and not w[0].startswith("#")]
    ifljari = ini["ifljari"][0][0].lower().startswith(".t")

    # ---- atoms, molecules and topology in the reference's order (rdtop.F90:62-370)
    atmtyp, mol_sizes = [], []
    bonds, angs, tors, rbs = [], [], [], []
    for row in ini["npolymoletyp"]:
        nmol, nat, corf, topf = int(row[1]), int(row[2]), row[3], row[4]
        cor_types = [w[1] for w in (ln.split() for ln in open(os.path.join(ref, corf)))
                     if len(w) >= 5 and w[0].isdigit()]
        assert len(cor_types) == nat, corf
        top = read_sections(os.path.join(ref, topf))
        base0 = len(atmtyp)
        for m in range(nmol):
            b = base0 + m * nat
            atmtyp.extend(cor_types)
            mol_sizes.append(nat)
            for w in top.get("BOND", []):
                bonds.append((b + int(w[1]) - 1, b + int(w[2]) - 1, w[3]))
            for w in top.get("ANGLE", []):
                angs.append((b + int(w[1]) - 1, b + int(w[2]) - 1, b + int(w[3]) - 1, w[4]))
            for w in top.get("TORSION", []):
                tors.append((b + int(w[1]) - 1, b + int(w[2]) - 1, b + int(w[3]) - 1, b + int(w[4]) - 1, w[5]))
            for w in top.get("TORSION_RB", []):
                rbs.append((b + int(w[1]) - 1, b + int(w[2]) - 1, b + int(w[3]) - 1, b + int(w[4]) - 1, w[5]))
    assert int(ini["nwater"][0][0]) == 0
    for row in ini["nmatomtyp"]:
        n, t = int(row[1]), row[2]
        atmtyp.extend([t] * n)
        mol_sizes.extend([1] * n)
    natom = len(atmtyp)

    # ---- per-type parameters (rdpara.F90, linkbond.F90:27-40)
    names = sorted(set(atmtyp), key=lambda t: int(lookup(para["ATOM"], t)[0]))
    ntyp = len(names)
    mass_t = np.array([fnum(lookup(para["ATOM"], t)[2]) for t in names])
    chrg_t = np.array([fnum(lookup(para["ATOM"], t)[3]) for t in names])
    eps_t, rad_t, comb_t = [], [], []
    for t in names:
        hit = [w for w in vdw if w[1][:2] == t[:2]]
        eps_t.append(fnum(hit[-1][2]) / EREF); rad_t.append(fnum(hit[-1][3]) / XREF); comb_t.append(hit[-1][4])
    welij = np.zeros((ntyp, ntyp)); radij = np.zeros((ntyp, ntyp))
    for i in range(ntyp):
        for j in range(ntyp):
            welij[i, j] = math.sqrt(eps_t[i] * eps_t[j])
            if comb_t[i] == "A" and comb_t[j] == "A":
                radij[i, j] = 0.5 * (rad_t[i] + rad_t[j])
            elif comb_t[i] == "G" and comb_t[j] == "G":
                radij[i, j] = math.sqrt(rad_t[i] * rad_t[j])
            else:
                radij[i, j] = 0.5 * (rad_t[i] + rad_t[j]) if ifljari else math.sqrt(rad_t[i] * rad_t[j])
            for w in para.get("VDW_SP", []):                       # rdpara.F90:742-760
                if pair_match(w[1], names[i][:2], names[j][:2]):
                    welij[i, j] = fnum(w[2]) / EREF; radij[i, j] = fnum(w[3]) / XREF
                    break
    inttyp = np.ones((ntyp, ntyp), np.int32)                        # INTTYPE_VDW
    welmor = np.zeros((ntyp, ntyp)); radmor = np.zeros((ntyp, ntyp)); almor = np.zeros((ntyp, ntyp))
    for i in range(ntyp):
        for j in range(ntyp):
            for w in para.get("MORSE", []):                        # rdpara.F90:700-720, 765-800
                if pair_match(w[1], names[i][:2], names[j][:2]):
                    inttyp[i, j] = 2                                # INTTYPE_MOR
                    welij[i, j] = 0.0; radij[i, j] = 0.0
                    welmor[i, j] = fnum(w[2]) / EREF
                    radmor[i, j] = fnum(w[3]) / XREF
                    almor[i, j] = fnum(w[4]) * XREF
                    break

    # ---- bonded terms: exact-name lookup (linkbond.F90:55-130), units (rdpara.F90:460-480,
    #      prepmd.F90:220-236)
    deg = math.pi / 180.0
    bpar = [lookup(para["BOND"], t) for *_, t in bonds]
    apar = [lookup(para["ANGLE"], t) for *_, t in angs]
    tpar = [lookup(para["TORSION"], t) for *_, t in tors]
    rpar = [lookup(para["TORSION_RB"], t) for *_, t in rbs]
    fix = dict(
        bonds=np.array([b[:2] for b in bonds], np.int32).reshape(-1, 2),
        bond_k=np.array([fnum(w[2]) / (EREF / XREF ** 2) for w in bpar]),
        bond_r0=np.array([fnum(w[3]) / XREF for w in bpar]),
        angles=np.array([a[:3] for a in angs], np.int32).reshape(-1, 3),
        angl_k=np.array([fnum(w[2]) / EREF for w in apar]),
        angl_t0=np.array([fnum(w[3]) * deg for w in apar]),
        tors=np.array([t[:4] for t in tors], np.int32).reshape(-1, 4),
        tors_divfac=np.array([int(w[2]) for w in tpar], np.int32),
        tors_barhig=np.array([fnum(w[3]) / EREF for w in tpar]),
        tors_phsang=np.array([fnum(w[4]) * deg for w in tpar]),
        tors_period=np.array([fnum(w[5]) for w in tpar]),
        tors_dvdw=np.array([fnum(w[6]) for w in tpar]),
        tors_delc=np.array([fnum(w[7]) for w in tpar]),
        torsrb=np.array([t[:4] for t in rbs], np.int32).reshape(-1, 4),
        torsrb_c=np.array([[fnum(x) / EREF for x in w[2:8]] for w in rpar]).reshape(-1, 6),
        torsrb_dvdw=np.array([fnum(w[8]) for w in rpar]),
        torsrb_delc=np.array([fnum(w[9]) for w in rpar]),
    )
    # rdpara.F90:1070-1090: no 1-4 pair when both divisors are ~0
    fix["tors_14"] = (~((np.abs(fix["tors_dvdw"]) < 1e-8) & (np.abs(fix["tors_delc"]) < 1e-8))).astype(np.int32)
    fix["torsrb_14"] = (~((np.abs(fix["torsrb_dvdw"]) < 1e-8) & (np.abs(fix["torsrb_delc"]) < 1e-8))).astype(np.int32)

    # ---- ring14 / ring14_rb (rdtop.F90:375-440), after all molecule copies
    ntors, ntorsrb = len(tors), len(rbs)
    b12 = {(min(i, j), max(i, j)) for i, j, _ in bonds}
    b13 = {(min(i, k), max(i, k)) for i, _, k, _ in angs}
    t14 = {}
    for n, (i, _, _, l, _) in enumerate(tors):
        t14.setdefault((min(i, l), max(i, l)), []).append(n)
    ring14 = np.ones(ntors)
    for n, (i, _, _, l, _) in enumerate(tors):
        key = (min(i, l), max(i, l))
        if key in b12 or key in b13:
            ring14[n] = 0.0
        if any(m != n for m in t14.get(key, [])):
            ring14[n] = 0.5
    # ring14_rb(1:ntors) = 1 resets only the first ntors entries; the rest keep
    # the zero initial value of the SAVEd array (md_global.inc:182)
    ring14_rb = np.zeros(ntorsrb)
    ring14_rb[:min(ntors, ntorsrb)] = 1.0
    for n, (i, _, _, l, _) in enumerate(rbs):
        key = (min(i, l), max(i, l))
        if key in b12 or key in b13:
            ring14_rb[n] = 0.0
        if t14.get(key):                    # a periodic torsion with the same ends (rdtop.F90:430-437)
            ring14_rb[n] = 0.5
    fix["tors_ring"] = ring14
    fix["torsrb_ring"] = ring14_rb
    return dict(ini=ini, atmtyp=atmtyp, mol_sizes=mol_sizes, names=names, mass_t=mass_t, chrg_t=chrg_t,
                welij=welij, radij=radij, inttyp=inttyp, welmor=welmor, radmor=radmor, almor=almor, fix=fix)


def main(ref):
    b = build(ref)
    ini = b["ini"]
    step, pos32, ptyp = read_out_pos(os.path.join(ref, "out_pos.dat"))
    if ptyp != b["atmtyp"]:
        raise ValueError("atom types of out_pos.dat differ from the topology order")
    vstep, vel32, vtyp = read_out_pos(os.path.join(ref, "out_vel.dat"))    # outvel: same record layout [m/s]
    if vstep != step or vtyp != ptyp:
        raise ValueError("out_vel.dat does not match out_pos.dat")
    # the state record of the same step holds the same configuration in
    # double precision (E24.16): use it, after checking it against the
    # single-precision outputs
    sta_path = os.path.join(ref, ini["iostarecname"][0][0])
    sstep, pos_m, vel_ms, styp = read_state_record(sta_path)
    # raw text of the record (wrsta.F90 formats): header, the first and last
    # atoms of each section and the chain sections, for the format tests
    raw = open(sta_path).read().split("\n")
    tags = [i for i, ln in enumerate(raw) if ln.strip().startswith("#")]
    keep = set(range(0, tags[tags.index(next(i for i in tags if raw[i].strip() == "#poly"))] + 1))
    for t in tags:
        if raw[t].strip() in ("#poly", "#water", "#matom"):
            keep.update(range(t, min(t + 13, len(raw))))
        if raw[t].strip() == "#nhc":
            keep.update(range(t - 13, len(raw)))
    sta_lines = [(i, raw[i]) for i in sorted(keep) if i < len(raw)]
    if sstep != step or styp != ptyp:
        raise ValueError("state record is not the out_pos.dat step")
    if np.abs(pos_m - pos32).max() > 1e-6 * np.abs(pos_m).max() or \
            np.abs(vel_ms - vel32).max() > 1e-6 * np.abs(vel_ms).max():
        raise ValueError("state record differs from out_pos.dat / out_vel.dat beyond single precision")
    ene = [r for r in read_out_ene(os.path.join(ref, "out_ene.dat")) if int(r["nstep"]) == step]
    if len(ene) != 1:
        raise ValueError("no out_ene.dat record for the out_pos.dat step")
    # outpre (same layout as outene): virials [J] and pressure tensors of the step
    pre = [r for r in read_out_ene(os.path.join(ref, "out_pre.dat")) if int(r["nstep"]) == step]
    if len(pre) != 1:
        raise ValueError("no out_pre.dat record for the out_pos.dat step")
    pre_keys = [k for k in pre[0] if k.startswith(("pot_viri", "atm_viri", "preatmt_vtot"))]
    g = lambda k: fnum(ini[k][0][0])
    an, mref = 6.0221367e23, 1.99431e-26                       # rdpara.F90:64, main_md.F90:395
    vref = math.sqrt(EREF / mref)                              # calbase.F90:66
    names = b["names"]
    tix = np.array([names.index(t) + 1 for t in b["atmtyp"]], np.int32)
    params = dict(xcel=g("xcel") / XREF, ycel=g("ycel") / XREF, zcel=g("zcel") / XREF,
                  alpha=g("alpha") * XREF, rrcut=g("rrcut") / XREF, rcut=g("rcut") / XREF,
                  rcut_book=g("rcut_book") / XREF, nfft1=int(g("nfft1")), nfft2=int(g("nfft2")),
                  nfft3=int(g("nfft3")), pme_order=int(g("pme_order")), nspltbl=int(g("nspltbl")),
                  rcutmor=g("rcutmor") / XREF, rcut_bookmor=g("rcut_bookmor") / XREF,
                  ifnetqcorrp=int(ini["ifnetqcorrp"][0][0].lower().startswith(".t")))
    np.savez_compressed(
        OUT, step=step, pos_m=pos_m, vel_ms=vel_ms, atmindex=tix, type_names=np.array(names),
        mass_t=b["mass_t"] * 1.0e-3 / an / mref, chrg_t=b["chrg_t"] * CHARGE_SCALE,
        vdw_welij=b["welij"], vdw_radij=b["radij"], inttyp=b["inttyp"],
        mor_wel=b["welmor"], mor_rad=b["radmor"], mor_alpha=b["almor"],
        mol_sizes=np.array(b["mol_sizes"], np.int32),
        params_keys=np.array(list(params)), params_vals=np.array(list(params.values()), float),
        ene_keys=np.array(ENE_KEYS), ene_joule=np.array([ene[0][k] for k in ENE_KEYS]), eref=EREF, xref=XREF, vref=vref,
        sta_line_no=np.array([i for i, _ in sta_lines]), sta_line_text=np.array([t for _, t in sta_lines]),
        pre_keys=np.array(pre_keys), pre_joule=np.array([pre[0][k] for k in pre_keys]),
        **b["fix"])
    print("wrote", OUT, "natom", len(tix), "step", step)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PEACHGK_MD_DIR")
    if not ref:
        sys.exit("usage: make_pt_morse_fixture.py REFERENCE_DIR (the peachgk-md directory of the reference "
                 "tree; or set PEACHGK_MD_DIR)")
    main(ref)
