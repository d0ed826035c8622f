"""Seeded synthetic systems in the reference's reduced units.

The reference reads its systems from peachgk.ini + *_cor.dat/*_top.dat +
para_*.dat and converts them to reduced units in calbase.F90:21-40
(xref = 1 A, eref = 6.9511e-21 J, mref = 1.9943e-26 kg, qref = e).  This
module builds the same arrays directly (no file round trip):

* atom arrays ``atmmass``, ``atmchrg`` (already x 1/sqrt(4 pi eps0),
  prepmd.F90:239-241), ``atmindex`` (1-based LJ type);
* the LJ pair tables ``vdw_radij``/``vdw_welij`` with the ifljari mixing rule
  (rdpara.F90:530-570: E_ij = sqrt(E_i E_j), R_ij = (R_i + R_j)/2);
* bonded terms with per-term parameters, the exclusion CSR exactly as
  mkexcl.F90 builds it (1-2, 1-3 and 1-4 partners, sorted, unique, j > i,
  0 sentinel), the 1-4 flags of calnon14.F90 and the RATTLE groups.

Configurations (shapes of the workloads the engine is measured on):
``water_box`` (512 rigid 3-site waters, 24.83 A), ``propanol_box``
(1000 flexible 1-propanol, 52 A), ``butane_box`` (14,286 flexible butane,
~130 A), ``slab`` (water slab with propanol faces, 50x50x150 A).
Parameters are OPLS-like values drawn within +-10 % from a seed; they are
synthetic stand-ins, not a published force field file.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

# ---- reduced units (calbase.F90:21-40) -------------------------------------
XREF = 1.0e-10
EREF = 6.9511e-21
MREF = 1.9943e-26
QREF = 1.60217733e-19
KB = 1.38066e-23
AMU = 1.6605402e-27
NA = 6.0221367e23
EPS0_SI = 8.854187817e-12
VREF = math.sqrt(EREF / MREF)
TIMEREF = XREF / VREF
TEMPREF = EREF / KB
PREF = EREF / XREF ** 3
EPS0 = EPS0_SI / (QREF ** 2 / EREF / XREF)
KCAL = 4184.0 / NA / EREF          # kcal/mol in reduced energy
CHARGE_SCALE = 1.0 / math.sqrt(4.0 * math.pi * EPS0)   # prepmd.F90:239-241

MTS_LONG, MTS_SHORT = 1, 3
PREC_FP64, PREC_MIXED = 0, 1


def fs_to_reduced(dt_fs: float) -> float:
    return dt_fs * 1.0e-15 / TIMEREF


def kelvin_to_reduced(t: float) -> float:
    return t / TEMPREF


def pa_to_reduced(p: float) -> float:
    return p / PREF


# ---- LJ atom types: (name, mass amu, sigma A, eps kcal/mol) ---------------
LJ_TYPES = {
    "OW": (15.999, 3.166, 0.1553),   # SPC/E-like water oxygen
    "HW": (1.008, None, 0.0),        # water hydrogen: E = 0, R = 1 A (para_vdw_s.dat HB)
    "CT": (12.011, 3.50, 0.066),
    "HC": (1.008, 2.50, 0.030),
    "OH": (15.999, 3.12, 0.170),
    "HO": (1.008, None, 0.0),
    "IP": (22.99, None, 0.0),        # bare ions of the Madelung known-answer lattice
    "IM": (35.45, None, 0.0),
}


@dataclasses.dataclass
class Molecule:
    """One molecule template: names, LJ types, charges, internal geometry."""
    name: str
    types: list
    charges: np.ndarray
    coords: np.ndarray              # (n,3) A, centred template geometry
    bonds: list                     # (i, j, k_red, r0)  0-based within molecule
    angles: list                    # (i, j, k, kang_red, theta0_rad)
    tors: list                      # periodic: (i,j,k,l, divfac, barhig, phsang, period)
    torsrb: list                    # RB: (i,j,k,l, c0..c5)
    constraints: list               # (i, j, d)
    axis: tuple                     # (a, b) atoms spanning the long axis


# ---- geometry helpers -------------------------------------------------------
def _place(a, b, c, bond, angle_deg, dihed_deg):
    """NeRF: position of D with |CD| = bond, angle BCD, dihedral ABCD."""
    ang = math.radians(angle_deg)
    dih = math.radians(dihed_deg)
    bc = c - b
    bc /= np.linalg.norm(bc)
    n = np.cross(b - a, bc)
    n /= np.linalg.norm(n)
    m = np.cross(n, bc)
    d2 = np.array([-bond * math.cos(ang),
                   bond * math.sin(ang) * math.cos(dih),
                   bond * math.sin(ang) * math.sin(dih)])
    return c + d2[0] * bc + d2[1] * m + d2[2] * n


def _rot_matrix(rng):
    """Uniform random rotation (quaternion method)."""
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _axis_rotation(axis, angle):
    axis = axis / np.linalg.norm(axis)
    k = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    return np.eye(3) + math.sin(angle) * k + (1 - math.cos(angle)) * (k @ k)


def _align(v_from, v_to):
    a = v_from / np.linalg.norm(v_from)
    b = v_to / np.linalg.norm(v_to)
    v = np.cross(a, b)
    c = float(a @ b)
    if np.linalg.norm(v) < 1e-12:
        return np.eye(3) if c > 0 else _axis_rotation(np.array([1.0, 0, 0]) if abs(a[0]) < 0.9
                                                      else np.array([0, 1.0, 0]), math.pi)
    k = np.array([[0, -v[2], v[1]], [v[2], 0, -v[0]], [-v[1], v[0], 0]])
    return np.eye(3) + k + k @ k * (1.0 / (1.0 + c))


def _jitter(rng, value, frac=0.10):
    return value * (1.0 + frac * (2.0 * rng.random() - 1.0))


# ---- molecule templates -----------------------------------------------------
def water_template() -> Molecule:
    """Rigid 3-site water: O, H, H; OH 1.0 A, HOH 109.47 deg (HH 1.633 A)."""
    r_oh = 1.0
    ang = math.radians(109.47)
    o = np.zeros(3)
    h1 = np.array([r_oh, 0.0, 0.0])
    h2 = np.array([r_oh * math.cos(ang), r_oh * math.sin(ang), 0.0])
    xyz = np.array([o, h1, h2])
    xyz -= xyz.mean(axis=0)
    d_hh = float(np.linalg.norm(h1 - h2))
    q = np.array([-0.8476, 0.4238, 0.4238])
    # k = 0 bonds/angle: they only define exclusions (H2O_topOB.dat, para_bond.dat:148-149,237)
    bonds = [(0, 1, 0.0, r_oh), (0, 2, 0.0, r_oh), (1, 2, 0.0, d_hh)]
    angles = [(1, 0, 2, 0.0, ang)]
    cons = [(0, 1, r_oh), (0, 2, r_oh), (1, 2, d_hh)]
    return Molecule("water", ["OW", "HW", "HW"], q, xyz, bonds, angles, [], [], cons, (1, 2))


def _alkyl_template(name, heavy, rng_par, alcohol):
    """Flexible united-chain alkane/alcohol with explicit hydrogens.

    heavy: number of carbons; alcohol=True appends O-H to the last carbon.
    X-H bonds are RATTLE constraints (their harmonic k is set to 0 so they
    only define exclusions, as constrained bonds do in the reference)."""
    r_cc = _jitter(rng_par, 1.53)
    r_co = _jitter(rng_par, 1.41)
    r_ch = _jitter(rng_par, 1.09)
    r_oh = _jitter(rng_par, 0.945)
    k_cc = _jitter(rng_par, 268.0) * KCAL
    k_co = _jitter(rng_par, 320.0) * KCAL
    a_ccc = math.radians(_jitter(rng_par, 112.7))
    a_cco = math.radians(_jitter(rng_par, 109.5))
    a_cch = math.radians(_jitter(rng_par, 110.7))
    a_hch = math.radians(_jitter(rng_par, 107.8))
    a_coh = math.radians(_jitter(rng_par, 108.5))
    k_ccc = _jitter(rng_par, 58.35) * KCAL
    k_cco = _jitter(rng_par, 50.0) * KCAL
    k_cch = _jitter(rng_par, 37.5) * KCAL
    k_hch = _jitter(rng_par, 33.0) * KCAL
    k_coh = _jitter(rng_par, 55.0) * KCAL
    # Ryckaert-Bellemans C0..C5 (kJ/mol -> kcal/mol), heavy-atom backbone
    rb = [c / 4.184 for c in (9.28, 12.16, -13.12, -3.06, 26.24, -31.5)]
    rb = [_jitter(rng_par, c) * KCAL for c in rb]
    v_hcch = _jitter(rng_par, 0.15) * KCAL      # periodic n=3, X-C-C-X with an H end
    v_ccoh = _jitter(rng_par, 0.35) * KCAL

    nbb = heavy + (1 if alcohol else 0)
    xyz = [np.zeros(3), np.array([r_cc, 0.0, 0.0])]
    xyz.append(_place(np.array([0.0, 1.0, 0.0]), xyz[0], xyz[1], r_cc, math.degrees(a_ccc), 180.0))
    for k in range(3, heavy):
        xyz.append(_place(xyz[k - 3], xyz[k - 2], xyz[k - 1], r_cc, math.degrees(a_ccc), 180.0))
    types = ["CT"] * heavy
    if alcohol:
        xyz.append(_place(xyz[heavy - 3], xyz[heavy - 2], xyz[heavy - 1], r_co, math.degrees(a_cco), 180.0))
        types.append("OH")
    bb = list(range(nbb))
    bonds, angles, tors, torsrb, cons = [], [], [], [], []
    for a in range(nbb - 1):
        if alcohol and a == nbb - 2:
            bonds.append((a, a + 1, k_co, r_co))
        else:
            bonds.append((a, a + 1, k_cc, r_cc))
    # hydrogens on carbons
    hs_of = {}
    for c in range(heavy):
        nh = 3 if (c == 0 or (c == heavy - 1 and not alcohol)) else 2
        ref_prev = xyz[c - 1] if c > 0 else xyz[1]
        ref_far = xyz[c - 2] if c > 1 else (xyz[2] if c == 0 else xyz[2])
        if c == 0:
            dihs = [60.0, 180.0, -60.0]
            a_, b_, c_ = xyz[2], xyz[1], xyz[0]
        elif nh == 3:
            dihs = [60.0, 180.0, -60.0]
            a_, b_, c_ = xyz[c - 2], xyz[c - 1], xyz[c]
        else:
            dihs = [121.5, -121.5]
            a_, b_, c_ = xyz[c + 1], xyz[c - 1], xyz[c]
        del ref_prev, ref_far
        hs = []
        for d in dihs:
            xyz.append(_place(a_, b_, c_, r_ch, math.degrees(a_cch), d))
            types.append("HC")
            hs.append(len(xyz) - 1)
            bonds.append((c, len(xyz) - 1, 0.0, r_ch))
            cons.append((c, len(xyz) - 1, r_ch))
        hs_of[c] = hs
    if alcohol:
        o = nbb - 1
        xyz.append(_place(xyz[o - 2], xyz[o - 1], xyz[o], r_oh, math.degrees(a_coh), 180.0))
        types.append("HO")
        hs_of[o] = [len(xyz) - 1]
        bonds.append((o, len(xyz) - 1, 0.0, r_oh))
        cons.append((o, len(xyz) - 1, r_oh))
    xyz = np.array(xyz)
    n = len(types)
    # adjacency -> angles / torsions
    adj = [[] for _ in range(n)]
    for (i, j, _, _) in bonds:
        adj[i].append(j)
        adj[j].append(i)
    for j in range(n):
        nb = sorted(adj[j])
        for x in range(len(nb)):
            for y in range(x + 1, len(nb)):
                i, k = nb[x], nb[y]
                ti, tk = types[i], types[k]
                if ti[0] == "H" and tk[0] == "H":
                    kk, th = k_hch, a_hch
                elif types[j] == "OH":
                    kk, th = k_coh, a_coh
                elif "OH" in (ti, tk):
                    kk, th = k_cco, a_cco
                elif ti[0] == "H" or tk[0] == "H":
                    kk, th = k_cch, a_cch
                else:
                    kk, th = k_ccc, a_ccc
                angles.append((i, j, k, kk, th))
    seen = set()
    for (j, k, _, _) in bonds:
        for i in adj[j]:
            if i == k:
                continue
            for l in adj[k]:
                if l == j or l == i:
                    continue
                key = (i, j, k, l) if i < l else (l, k, j, i)
                if key in seen:
                    continue
                seen.add(key)
                i2, j2, k2, l2 = key
                heavy_ends = types[i2][0] != "H" and types[l2][0] != "H"
                if heavy_ends:
                    torsrb.append((i2, j2, k2, l2, *rb))
                else:
                    v = v_ccoh if "OH" in (types[j2], types[k2]) else v_hcch
                    # barhig/divfac*(1+cos(3 phi - 0)), divfac 1
                    tors.append((i2, j2, k2, l2, 1, v, 0.0, 3.0))
    # OPLS-like charges, jittered, neutralised per molecule
    q = np.zeros(n)
    for a in range(n):
        t = types[a]
        if t == "CT":
            nh = len(hs_of.get(a, []))
            q[a] = -0.18 if nh == 3 else -0.12
            if alcohol and a == nbb - 2:
                q[a] = 0.145
        elif t == "HC":
            q[a] = 0.06
        elif t == "OH":
            q[a] = -0.683
        elif t == "HO":
            q[a] = 0.418
    q = np.array([_jitter(rng_par, v) for v in q])
    q = np.clip(q, -0.7, 0.45)
    q -= q.mean()
    xyz -= xyz.mean(axis=0)
    return Molecule(name, types, q, xyz, bonds, angles, tors, torsrb, cons, (0, nbb - 1))


def propanol_template(rng_par) -> Molecule:
    return _alkyl_template("propanol", 3, rng_par, alcohol=True)


def butane_template(rng_par) -> Molecule:
    return _alkyl_template("butane", 4, rng_par, alcohol=False)


# ---- the system container ---------------------------------------------------
@dataclasses.dataclass
class System:
    """All arrays of a system in the reference layout (0-based here where
    noted; ``abi.SystemStruct`` converts to the 1-based C ABI)."""
    name: str
    natom: int
    box: np.ndarray                  # (3,)
    atmcor: np.ndarray               # (natom,3)
    atmvel: np.ndarray               # (natom,3)
    atmmass: np.ndarray
    atmchrg: np.ndarray              # scaled
    atmindex: np.ndarray             # 1-based type
    type_names: list
    vdw_radij: np.ndarray            # (ntyp,ntyp)
    vdw_welij: np.ndarray
    molept_index: np.ndarray         # (nmole+1,) 0-based starts
    molept_list: np.ndarray          # 0-based atoms
    index_excl: np.ndarray           # (natom+1,) 1-based CSR starts (mkexcl)
    list_excl: np.ndarray            # 1-based partners, 0 sentinel
    bonds: np.ndarray                # (nb,2) 0-based
    bond_k: np.ndarray
    bond_r0: np.ndarray
    angles: np.ndarray               # (na,3)
    angl_k: np.ndarray
    angl_t0: np.ndarray
    tors: np.ndarray                 # (nt,4)
    tors_divfac: np.ndarray
    tors_barhig: np.ndarray
    tors_phsang: np.ndarray
    tors_period: np.ndarray
    tors_14: np.ndarray              # (nt,) int flag
    tors_dvdw: np.ndarray
    tors_delc: np.ndarray
    tors_ring: np.ndarray
    torsrb: np.ndarray               # (nrb,4)
    torsrb_c: np.ndarray             # (nrb,6)
    torsrb_14: np.ndarray
    torsrb_dvdw: np.ndarray
    torsrb_delc: np.ndarray
    torsrb_ring: np.ndarray
    const_index: np.ndarray          # (ngroups+1,) 0-based
    const_list: np.ndarray           # 0-based constraint ids
    const_ij: np.ndarray             # (nc,2) 0-based atoms
    const_d: np.ndarray
    degfree_all: int
    params: dict                     # peachgk.ini-like run parameters (reduced)
    regions: dict = dataclasses.field(default_factory=dict)
    inttyp: np.ndarray = None        # (ntyp,ntyp) inter_inttyp (1 LJ, 2 Morse); None = all LJ
    mor_wel: np.ndarray = None       # (ntyp,ntyp) Morse D, r0, alpha (rdpara.F90:680-720)
    mor_rad: np.ndarray = None
    mor_alpha: np.ndarray = None

    @property
    def nmole(self):
        return len(self.molept_index) - 1


def _mkexcl(natom, bonds, angles, tors, torsrb):
    """mkexcl.F90: partners = bond ends, angle ends (1-3), torsion ends (1-4);
    sorted + unique per atom; keep j > i; empty row -> single 0."""
    part = [set() for _ in range(natom)]
    for arr, a, b in ((bonds, 0, 1), (angles, 0, 2), (tors, 0, 3), (torsrb, 0, 3)):
        if len(arr) == 0:
            continue
        for row in arr:
            i, j = int(row[a]), int(row[b])
            part[i].add(j)
            part[j].add(i)
    index = np.zeros(natom + 1, dtype=np.int32)
    lst = []
    for i in range(natom):
        index[i] = len(lst) + 1
        js = sorted(j + 1 for j in part[i] if j > i)
        lst.extend(js if js else [0])
    index[natom] = len(lst) + 1
    return index, np.asarray(lst, dtype=np.int32)


def build_system(name, templates_and_counts, box, positions_fn, seed_vel, temp_k, params,
                 extra_regions=None):
    """Assemble molecules into one System.

    templates_and_counts: list of (Molecule, count); positions_fn(mol, idx)
    returns (n,3) coordinates for the idx-th molecule of that template."""
    names = []
    for mol, _ in templates_and_counts:
        for t in mol.types:
            if t not in names:
                names.append(t)
    ntyp = len(names)
    R = np.zeros(ntyp)
    E = np.zeros(ntyp)
    M = np.zeros(ntyp)
    for k, t in enumerate(names):
        mass, sig, eps = LJ_TYPES[t]
        M[k] = mass * AMU / MREF
        R[k] = 1.0 if sig is None else 2.0 ** (1.0 / 6.0) * sig
        E[k] = eps * KCAL
    welij = np.sqrt(np.outer(E, E))
    radij = 0.5 * (R[:, None] + R[None, :])

    cor, mass, chrg, idx, molidx, mollist = [], [], [], [], [0], []
    bonds, bk, br0, angs, ak, at0 = [], [], [], [], [], []
    tors, tdiv, tbar, tph, tper = [], [], [], [], []
    rbs, rbc = [], []
    cij, cd, cidx, clist = [], [], [0], []
    base = 0
    for mol, count in templates_and_counts:
        n = len(mol.types)
        tix = np.array([names.index(t) + 1 for t in mol.types], dtype=np.int32)
        for m in range(count):
            xyz = positions_fn(mol, m)
            cor.append(xyz)
            mass.append(M[tix - 1])
            chrg.append(mol.charges * CHARGE_SCALE)
            idx.append(tix)
            mollist.extend(range(base, base + n))
            molidx.append(molidx[-1] + n)
            for (i, j, k, r0) in mol.bonds:
                bonds.append((base + i, base + j)); bk.append(k); br0.append(r0)
            for (i, j, k, kk, th) in mol.angles:
                angs.append((base + i, base + j, base + k)); ak.append(kk); at0.append(th)
            for (i, j, k, l, dv, bh, ph, pe) in mol.tors:
                tors.append((base + i, base + j, base + k, base + l))
                tdiv.append(dv); tbar.append(bh); tph.append(ph); tper.append(pe)
            for t in mol.torsrb:
                rbs.append((base + t[0], base + t[1], base + t[2], base + t[3]))
                rbc.append(t[4:10])
            if mol.constraints:
                for (i, j, d) in mol.constraints:
                    clist.append(len(cij))
                    cij.append((base + i, base + j)); cd.append(d)
                cidx.append(len(clist))
            base += n
    natom = base
    atmcor = np.concatenate(cor).astype(np.float64)
    atmmass = np.concatenate(mass)
    bonds = np.asarray(bonds, dtype=np.int32).reshape(-1, 2)
    angs = np.asarray(angs, dtype=np.int32).reshape(-1, 3)
    tors = np.asarray(tors, dtype=np.int32).reshape(-1, 4)
    rbs = np.asarray(rbs, dtype=np.int32).reshape(-1, 4)
    iex, lex = _mkexcl(natom, bonds, angs, tors, rbs)
    rng = np.random.default_rng(seed_vel)
    vel = rng.normal(size=(natom, 3)) * np.sqrt(kelvin_to_reduced(temp_k) / atmmass)[:, None]
    vel -= (atmmass[:, None] * vel).sum(axis=0) / atmmass.sum()
    nt, nrb = len(tors), len(rbs)
    sysobj = System(
        name=name, natom=natom, box=np.asarray(box, dtype=np.float64),
        atmcor=atmcor, atmvel=vel, atmmass=atmmass,
        atmchrg=np.concatenate(chrg), atmindex=np.concatenate(idx), type_names=names,
        vdw_radij=radij, vdw_welij=welij,
        molept_index=np.asarray(molidx, dtype=np.int32), molept_list=np.asarray(mollist, dtype=np.int32),
        index_excl=iex, list_excl=lex,
        bonds=bonds, bond_k=np.asarray(bk, float), bond_r0=np.asarray(br0, float),
        angles=angs, angl_k=np.asarray(ak, float), angl_t0=np.asarray(at0, float),
        tors=tors, tors_divfac=np.asarray(tdiv, np.int32), tors_barhig=np.asarray(tbar, float),
        tors_phsang=np.asarray(tph, float), tors_period=np.asarray(tper, float),
        tors_14=np.ones(nt, np.int32), tors_dvdw=np.full(nt, 2.0), tors_delc=np.full(nt, 2.0),
        tors_ring=np.ones(nt),
        torsrb=rbs, torsrb_c=np.asarray(rbc, float).reshape(-1, 6),
        torsrb_14=np.ones(nrb, np.int32), torsrb_dvdw=np.full(nrb, 2.0), torsrb_delc=np.full(nrb, 2.0),
        torsrb_ring=np.ones(nrb),
        const_index=np.asarray(cidx, np.int32), const_list=np.asarray(clist, np.int32),
        const_ij=np.asarray(cij, np.int32).reshape(-1, 2), const_d=np.asarray(cd, float),
        degfree_all=3 * natom, params=dict(params), regions=extra_regions or {})
    return sysobj


def default_params(box, rcut, rrcut, alpha, nfft, pme_order, rcut_book=None, precision=PREC_FP64,
                   nstep_book=50):
    return dict(xcel=box[0], ycel=box[1], zcel=box[2], alpha=alpha, rrcut=rrcut, rcut=rcut,
                rcut_book=(rcut + 2.0) if rcut_book is None else rcut_book,
                nstep_book=nstep_book, list_mode=0, ifspme=1,
                nfft1=nfft[0], nfft2=nfft[1], nfft3=nfft[2], pme_order=pme_order,
                nspltbl=1100, precision=precision,
                mts_bond=MTS_LONG, mts_angl=MTS_LONG, mts_tors=MTS_LONG, mts_torsrb=MTS_LONG,
                mts_vdw=MTS_LONG, mts_ewk=MTS_LONG, mts_vdw14=MTS_LONG, mts_elc14=MTS_LONG,
                ifnetqcorrp=0, max_nbr=0)


def _lattice_positions(nside, spacing, origin=(0.0, 0.0, 0.0)):
    g = np.arange(nside) * spacing + 0.5 * spacing
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    return pts + np.asarray(origin)


def _chain_placer(sites, rng, axis=(1.0, 1.0, 1.0), tilt_deg=12.0):
    """Place a chain template on `sites`: long axis along `axis` with a
    random spin about it and a small random tilt (no overlaps at ~5 A spacing)."""
    axis = np.asarray(axis, float)
    axis /= np.linalg.norm(axis)
    cache = {}

    def fn(mol, m):
        if mol.name not in cache:
            a, b = mol.axis
            cache[mol.name] = _align(mol.coords[b] - mol.coords[a], axis)
        r0 = cache[mol.name]
        spin = _axis_rotation(axis, 2 * math.pi * rng.random())
        tilt_axis = np.cross(axis, rng.normal(size=3))
        tilt = _axis_rotation(tilt_axis, math.radians(tilt_deg) * rng.random())
        sign = 1.0 if rng.random() < 0.5 else -1.0
        flip = np.eye(3) if sign > 0 else _axis_rotation(np.cross(axis, [1.0, 0, 0]) if abs(axis[0]) < 0.9
                                                        else np.cross(axis, [0, 1.0, 0]), math.pi)
        rot = tilt @ spin @ flip @ r0
        return mol.coords @ rot.T + sites[m]
    return fn


def water_box(seed=555, nside=8, box=24.83, precision=PREC_FP64):
    """512 rigid waters on an 8^3 lattice in a 24.83 A cube, rc 10, alpha 0.32,
    SPME 32^3 order 4, list skin 2 A."""
    rng = np.random.default_rng(seed)
    wat = water_template()
    sites = _lattice_positions(nside, box / nside)
    rots = [_rot_matrix(rng) for _ in range(nside ** 3)]

    def fn(mol, m):
        return mol.coords @ rots[m].T + sites[m]
    p = default_params((box, box, box), rcut=10.0, rrcut=10.0, alpha=0.32, nfft=(32, 32, 32),
                       pme_order=4, precision=precision)
    return build_system("water_1536", [(wat, nside ** 3)], (box, box, box), fn, seed, 300.0, p)


def propanol_box(seed=2024, nside=10, box=52.0, precision=PREC_FP64, nmol=None):
    """1000 flexible 1-propanol on a 10^3 lattice in a 52 A cube, rc 12,
    SPME 64^3 order 4."""
    rng_par = np.random.default_rng(seed)
    mol = propanol_template(rng_par)
    rng = np.random.default_rng(seed + 1)
    sites = _lattice_positions(nside, box / nside)
    nmol = nside ** 3 if nmol is None else nmol
    p = default_params((box, box, box), rcut=12.0, rrcut=12.0, alpha=0.28, nfft=(64, 64, 64),
                       pme_order=4, precision=precision)
    return build_system("propanol_12000", [(mol, nmol)], (box, box, box),
                        _chain_placer(sites, rng), seed + 2, 300.0, p)


def butane_box(seed=4242, nmol=14286, nside=25, box=130.0, precision=PREC_MIXED):
    """14,286 flexible butane (200,004 atoms) on a 25^3 lattice (sites drawn
    without replacement) in a 130 A cube, rc 12, SPME 128^3 order 5."""
    rng_par = np.random.default_rng(seed)
    mol = butane_template(rng_par)
    rng = np.random.default_rng(seed + 1)
    sites = _lattice_positions(nside, box / nside)
    sites = sites[rng.permutation(len(sites))[:nmol]]
    p = default_params((box, box, box), rcut=12.0, rrcut=12.0, alpha=0.28, nfft=(128, 128, 128),
                       pme_order=5, precision=precision)
    return build_system(f"butane_{nmol * 14}", [(mol, nmol)], (box, box, box),
                        _chain_placer(sites, rng), seed + 2, 250.0, p)


def small_box(kind="propanol", nside=3, spacing=5.2, seed=7, precision=PREC_FP64, nfft=16, order=4,
              rcut=None):
    """Small test systems (a few hundred atoms) for oracle-speed parity cases."""
    box = nside * spacing
    rc = min(box / 2.0 - 2.2, 12.0) if rcut is None else rcut
    rng_par = np.random.default_rng(seed)
    if kind == "water":
        mol = water_template()
        rng = np.random.default_rng(seed + 1)
        sites = _lattice_positions(nside, spacing)
        rots = [_rot_matrix(rng) for _ in range(nside ** 3)]

        def fn(m_, m):
            return m_.coords @ rots[m].T + sites[m]
    else:
        mol = propanol_template(rng_par) if kind == "propanol" else butane_template(rng_par)
        fn = _chain_placer(_lattice_positions(nside, spacing), np.random.default_rng(seed + 1))
    p = default_params((box, box, box), rcut=rc, rrcut=rc, alpha=3.2 / rc, nfft=(nfft, nfft, nfft),
                       pme_order=order, precision=precision)
    return build_system(f"{kind}_small", [(mol, nside ** 3)], (box, box, box), fn, seed + 2, 300.0, p)


def slab_box(seed=99, nxy_w=16, nlay_w=32, nwater=8000, nxy_p=10, nlay_p=8, lxy=50.0, dz_w=3.1, dz_p=6.6,
             vacuum=15.0, rcut=12.0, nfft=(64, 64, 192), order=4, precision=PREC_MIXED, hf_width=10.0,
             t_hot=320.0, t_cold=280.0, damp_per_ps=1.0):
    """Two-sided alcohol/water interface slab: rigid waters in the centre,
    propanol (long axis along z, chain placer) on each face, vacuum above and
    below, periodic in x, y, z.  Water is laid on an nxy_w^2 x nlay_w lattice
    (first `nwater` sites), propanol on nxy_p^2 x nlay_p per face.  The box
    height follows from the layer stacks plus 2 x vacuum; the default makes
    8000 waters + 2 x 800 propanol (43,200 atoms) at liquid spacing, which
    needs Lz ~ 205 A (a 150 A box cannot hold that many molecules at liquid
    density).  Heat-flux regions: z slabs of `hf_width`; Langevin heat source
    and sink: 10 A water slabs at t_hot and t_cold, a quarter of the water
    stack from each end.  Water is molecule-based for the heat flux and the
    thermostat, propanol atom-based."""
    rng = np.random.default_rng(seed)
    wat = water_template()
    prop = propanol_template(np.random.default_rng(seed + 1))
    hw = nlay_w * dz_w
    hp = nlay_p * dz_p
    lz = hw + 2.0 * hp + 2.0 * vacuum
    z0w = vacuum + hp                                   # water stack start
    gw = (np.arange(nxy_w) + 0.5) * (lxy / nxy_w)
    wsites = np.array([(x, y, z0w + (k + 0.5) * dz_w) for k in range(nlay_w) for y in gw for x in gw])[:nwater]
    rots = [_rot_matrix(rng) for _ in range(len(wsites))]
    gp = (np.arange(nxy_p) + 0.5) * (lxy / nxy_p)
    psites = [(x, y, vacuum + (k + 0.5) * dz_p) for k in range(nlay_p) for y in gp for x in gp]
    psites += [(x, y, z0w + hw + (k + 0.5) * dz_p) for k in range(nlay_p) for y in gp for x in gp]
    psites = np.array(psites)
    placer = _chain_placer(psites, np.random.default_rng(seed + 2), axis=(0.0, 0.0, 1.0), tilt_deg=10.0)

    def fn(mol, m):
        if mol.name == wat.name:
            return mol.coords @ rots[m].T + wsites[m]
        return placer(mol, m)
    box = (lxy, lxy, lz)
    p = default_params(box, rcut=rcut, rrcut=rcut, alpha=3.4 / rcut, nfft=nfft, pme_order=order,
                       precision=precision)
    sysobj = build_system(f"slab_{nwater * 3 + len(psites) * 12}", [(wat, len(wsites)), (prop, len(psites))], box,
                          fn, seed + 3, 300.0, p)
    nw, npm = len(wsites), len(psites)
    hftyp = np.concatenate([np.full(3 * nw, 2, np.int32), np.ones(12 * npm, np.int32)])
    lt_mole = np.concatenate([np.ones(nw, np.int32), np.zeros(npm, np.int32)])
    nreg = max(1, int(lz // hf_width))
    regions = [(k * lz / nreg, (k + 1) * lz / nreg) for k in range(nreg)]
    zq = z0w + 0.25 * hw
    zq2 = z0w + 0.75 * hw
    gam = damp_per_ps * 1.0e12 * TIMEREF
    lang = [dict(box=((0.0, lxy), (0.0, lxy), (zq - 5.0, zq + 5.0)), temp=kelvin_to_reduced(t_hot), damp=gam),
            dict(box=((0.0, lxy), (0.0, lxy), (zq2 - 5.0, zq2 + 5.0)), temp=kelvin_to_reduced(t_cold), damp=gam)]
    sysobj.regions = dict(hf=dict(regions=regions, heatfinterval=1, hftyp=hftyp, langevin=lang, lt_mole=lt_mole,
                                  seed=seed, ifoutthc=1))
    return sysobj


def ion_template(sign):
    q = np.array([1.0 if sign > 0 else -1.0])
    return Molecule("ion+" if sign > 0 else "ion-", ["IP" if sign > 0 else "IM"], q, np.zeros((1, 3)),
                    [], [], [], [], [], (0, 0))


def nacl_lattice(nside=8, a=2.82, alpha=None, nfft=32, order=6, rcut=None, precision=PREC_FP64):
    """Rock-salt lattice of +-1 point charges (nearest-neighbour distance a);
    the Ewald energy per ion pair is -M q^2/a with the Madelung constant
    M = 1.747564594633 (known answer for the Ewald + SPME path)."""
    L = nside * a
    rc = L / 2.0 - 0.01 if rcut is None else rcut
    al = 3.6 / rc if alpha is None else alpha
    g = np.arange(nside)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    plus = pts[(pts.sum(axis=1) % 2) == 0] * a
    minus = pts[(pts.sum(axis=1) % 2) == 1] * a
    p = default_params((L, L, L), rcut=rc, rrcut=rc, alpha=al, nfft=(nfft, nfft, nfft), pme_order=order,
                       rcut_book=rc + 0.005, precision=precision)
    p["list_mode"] = 2
    sysobj = build_system("nacl", [(ion_template(+1), len(plus)), (ion_template(-1), len(minus))], (L, L, L),
                          lambda mol, m: (plus if mol.name == "ion+" else minus)[m][None, :] + 0.0,
                          1, 0.0, p)
    sysobj.atmvel[:] = 0.0
    return sysobj
