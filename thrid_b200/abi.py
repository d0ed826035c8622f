"""ctypes mirror of include/pgk_gpu.h (structs, constants) and the converter
from a :class:`thrid_b200.systems.System` to the 1-based C ABI arrays."""
from __future__ import annotations

import ctypes as C

import numpy as np

PGK_OK = 0
PGK_E_LIST_OVERFLOW = 1
PGK_E_CELL_OVERFLOW = 2
PGK_E_RATTLE_NOCONV = 3
PGK_E_BOX_TOO_SMALL = 4
PGK_E_DEVICE_TIMEOUT = 5
PGK_E_CUDA = 6
PGK_E_INVALID = 7
PGK_E_NOMEM = 8
PGK_E_UNSUPPORTED = 9
PGK_E_RATTLEV_NOCONV = 10
PGK_E_SCRATCH_LIMIT = 11

PREC_FP64, PREC_MIXED = 0, 1
MTS_LONG, MTS_SHORT, MTS_NONE = 1, 3, 0
PCONT_ISO, PCONT_ANISO, PCONT_X, PCONT_Y, PCONT_Z = 0, 1, 2, 3, 4
LIST_AUTO, LIST_CELL, LIST_ALLPAIR = 0, 1, 2

_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int32)


class SystemStruct(C.Structure):
    _fields_ = [
        ("natom", C.c_int32), ("atmmass", _pd), ("atmchrg", _pd), ("atmindex", _pi),
        ("ntyp", C.c_int32), ("vdw_radij", _pd), ("vdw_welij", _pd), ("inter_inttyp", _pi),
        ("nmole", C.c_int32), ("molept_index", _pi), ("molept_list", _pi),
        ("index_excl", _pi), ("list_excl", _pi),
        ("nbond", C.c_int32), ("ibond", _pi), ("jbond", _pi), ("para_cbond", _pd), ("para_eqbond", _pd),
        ("nangl", C.c_int32), ("iangl", _pi), ("jangl", _pi), ("kangl", _pi),
        ("para_cangl", _pd), ("para_eqangl", _pd),
        ("ntors", C.c_int32), ("itors", _pi), ("jtors", _pi), ("ktors", _pi), ("ltors", _pi),
        ("para_divfac", _pi), ("para_barhig", _pd), ("para_phsang", _pd), ("para_period", _pd),
        ("ifcalnonb14", _pi), ("para_divfac_vdw", _pd), ("para_divfac_elc", _pd), ("ring14", _pd),
        ("ntorsrb", C.c_int32), ("itorsrb", _pi), ("jtorsrb", _pi), ("ktorsrb", _pi), ("ltorsrb", _pi),
        ("para_barhigrb", _pd), ("ifcalnonb14_rb", _pi), ("para_divfac_vdwrb", _pd),
        ("para_divfac_elcrb", _pd), ("ring14_rb", _pd),
        ("nconst", C.c_int32), ("index_mconst", _pi), ("list_mconst", _pi),
        ("nconstraint", C.c_int32), ("iconst", _pi), ("jconst", _pi), ("dconst", _pd),
        ("degfree_all", C.c_int32),
        ("para_welmor", _pd), ("para_radmor", _pd), ("para_alphamor", _pd),
    ]


class ParamsStruct(C.Structure):
    _fields_ = [
        ("xcel", C.c_double), ("ycel", C.c_double), ("zcel", C.c_double),
        ("alpha", C.c_double), ("rrcut", C.c_double), ("rcut", C.c_double), ("rcut_book", C.c_double),
        ("nstep_book", C.c_int32), ("list_mode", C.c_int32), ("ifspme", C.c_int32),
        ("nfft1", C.c_int32), ("nfft2", C.c_int32), ("nfft3", C.c_int32), ("pme_order", C.c_int32),
        ("nspltbl", C.c_int32), ("precision", C.c_int32),
        ("mts_bond", C.c_int32), ("mts_angl", C.c_int32), ("mts_tors", C.c_int32), ("mts_torsrb", C.c_int32),
        ("mts_vdw", C.c_int32), ("mts_ewk", C.c_int32), ("mts_vdw14", C.c_int32), ("mts_elc14", C.c_int32),
        ("ifnetqcorrp", C.c_int32), ("max_nbr", C.c_int32),
        ("rcutmor", C.c_double), ("rcut_bookmor", C.c_double), ("mts_mor", C.c_int32), ("nstep_bookmor", C.c_int32),
    ]

# run-time parameters a system may leave out (no Morse pairs)
PARAM_DEFAULTS = {"rcutmor": 0.0, "rcut_bookmor": 0.0, "mts_mor": 0, "nstep_bookmor": 0}


class MdParamsStruct(C.Structure):
    _fields_ = [
        ("dt_long_cal", C.c_double), ("nstep_short", C.c_int32), ("mchain", C.c_int32),
        ("text", C.c_double), ("qmass", C.c_double * 8), ("vmass", C.c_double),
        ("next", C.c_int32), ("nyosh", C.c_int32), ("yscoeff", C.c_double * 8),
        ("pext", C.c_double), ("pcont_axis", C.c_int32), ("ifrattle", C.c_int32),
        ("eps_rattle", C.c_double), ("pressinterval", C.c_int32), ("outinterval", C.c_int32),
    ]


ENERGY_NAMES = ["pot_tot", "pot_nonbon", "pot_vdw", "pot_elc", "pot_ewk", "pot_ewc", "pot_ewnq",
                "pot_vdw14", "pot_elc14", "pot_bond", "pot_angl", "pot_tors", "pot_torsrb", "pot_mor"]


class EnergiesStruct(C.Structure):
    _fields_ = [(n, C.c_double) for n in ENERGY_NAMES]

    def as_dict(self):
        return {n: getattr(self, n) for n in ENERGY_NAMES}


class VirialsStruct(C.Structure):
    _fields_ = [
        ("pot_viri_coul", C.c_double), ("pot_viri_lj", C.c_double),
        ("pot_virit_coul", C.c_double * 9), ("pot_virit_lj", C.c_double * 9),
        ("atm_viri_bond", C.c_double), ("atm_viri_angl", C.c_double),
        ("atm_viri_tors", C.c_double), ("atm_viri_14", C.c_double),
        ("atm_virit_bond", C.c_double * 9), ("atm_virit_angl", C.c_double * 9),
        ("atm_virit_tors", C.c_double * 9), ("atm_virit_14", C.c_double * 9),
        ("pot_viri_mor", C.c_double), ("pot_virit_mor", C.c_double * 9),
    ]

    def as_dict(self):
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = np.array(v[:]) if not isinstance(v, float) else v
        return out


class ChainStruct(C.Structure):
    _fields_ = [
        ("xlogs", C.c_double * 8), ("vlogs", C.c_double * 8),
        ("xlogv", C.c_double), ("vlogv", C.c_double),
        ("xboxh", C.c_double * 3), ("vboxg", C.c_double * 3),
        ("pint", C.c_double), ("pintt", C.c_double * 9),
    ]


HF_MAX_REGIONS, LT_MAX_REGIONS, HF_NCOL = 32, 8, 18
HF_KSPACE_NONE, HF_KSPACE_EWK, HF_KSPACE_SPME = 0, 1, 2
HFTYP_ATOM, HFTYP_MOLE = 1, 2
HF_BO, HF_AN, HF_TO, HF_14, HF_ELIN, HF_LJIN, HF_ELC, HF_VDW = range(8)
HF_COLUMNS = ("hfkin", "hfpotbo", "hfpotan", "hfpotto", "hfpot14", "hfpotelin", "hfpotljin", "hfpotelc",
              "hfpotlj", "hfviribo", "hfvirian", "hfvirito", "hfviri14", "hfvirielin", "hfviriljin",
              "hfvirielc", "hfvirilj", "hftot")


class HfParamsStruct(C.Structure):
    _fields_ = [
        ("nhfregion", C.c_int32), ("ifhfvol", C.c_int32), ("heatfinterval", C.c_int32),
        ("nlangeregion", C.c_int32),
        ("hfzpos1", C.c_double * HF_MAX_REGIONS), ("hfzpos2", C.c_double * HF_MAX_REGIONS),
        ("hftyp_atm", _pi), ("lt_mole_based", _pi),
        ("ltxpos1", C.c_double * LT_MAX_REGIONS), ("ltxpos2", C.c_double * LT_MAX_REGIONS),
        ("ltypos1", C.c_double * LT_MAX_REGIONS), ("ltypos2", C.c_double * LT_MAX_REGIONS),
        ("ltzpos1", C.c_double * LT_MAX_REGIONS), ("ltzpos2", C.c_double * LT_MAX_REGIONS),
        ("r_ltemp", C.c_double * LT_MAX_REGIONS), ("r_ltdamp", C.c_double * LT_MAX_REGIONS),
        ("seed", C.c_uint64), ("ifoutthc", C.c_int32), ("_pad", C.c_int32),
    ]


class EwkHfStruct(C.Structure):
    """pgk_ewk_hf: scalars of ewaldkp_hf (ewaldk_hf.F90:8-304)."""
    _fields_ = [("pot_ewk", C.c_double), ("pot_ewk_cc", C.c_double), ("pot_virit_coul", C.c_double * 9),
                ("nwave", C.c_int32), ("_pad", C.c_int32)]


class CHfParams:
    """Owns the arrays behind an HfParamsStruct built from a dict:
    regions=[(z1, z2), ...], heatfinterval, hftyp (per-atom array or None),
    langevin=[dict(box=((x1,x2),(y1,y2),(z1,z2)), temp=T_reduced, damp=g_reduced)],
    lt_mole (per-molecule array or None), seed, ifoutthc."""

    def __init__(self, d):
        st = HfParamsStruct()
        regs = d.get("regions", [])
        st.nhfregion = len(regs)
        st.ifhfvol = int(d.get("ifhfvol", 1))
        st.heatfinterval = int(d.get("heatfinterval", 1))
        for k, (a, b) in enumerate(regs):
            st.hfzpos1[k] = a
            st.hfzpos2[k] = b
        keep = {}
        if d.get("hftyp") is not None:
            keep["t"] = np.ascontiguousarray(np.asarray(d["hftyp"], dtype=np.int32))
            st.hftyp_atm = _ptr(keep["t"], C.c_int32)
        else:
            st.hftyp_atm = _pi()
        if d.get("lt_mole") is not None:
            keep["m"] = np.ascontiguousarray(np.asarray(d["lt_mole"], dtype=np.int32))
            st.lt_mole_based = _ptr(keep["m"], C.c_int32)
        else:
            st.lt_mole_based = _pi()
        lts = d.get("langevin", [])
        st.nlangeregion = len(lts)
        for k, l in enumerate(lts):
            (x1, x2), (y1, y2), (z1, z2) = l["box"]
            st.ltxpos1[k], st.ltxpos2[k] = x1, x2
            st.ltypos1[k], st.ltypos2[k] = y1, y2
            st.ltzpos1[k], st.ltzpos2[k] = z1, z2
            st.r_ltemp[k] = l["temp"]
            st.r_ltdamp[k] = l["damp"]
        st.seed = int(d.get("seed", 12345))
        st.ifoutthc = int(d.get("ifoutthc", 0))
        self.struct = st
        self._keep = keep
        self.nreg = len(regs)
        self.nlt = len(lts)


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype)) if a is not None and a.size else C.POINTER(ctype)()


class CSystem:
    """Owns the 1-based int32/float64 arrays behind a SystemStruct."""

    def __init__(self, s):
        keep = {}

        def d(name, a):
            keep[name] = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())
            return _ptr(keep[name], C.c_double)

        def i(name, a, plus=0):
            keep[name] = np.ascontiguousarray(np.asarray(a, dtype=np.int64).ravel() + plus).astype(np.int32)
            return _ptr(keep[name], C.c_int32)

        st = SystemStruct()
        st.natom = s.natom
        st.atmmass = d("m", s.atmmass)
        st.atmchrg = d("q", s.atmchrg)
        st.atmindex = i("t", s.atmindex)
        ntyp = s.vdw_radij.shape[0]
        st.ntyp = ntyp
        st.vdw_radij = d("R", s.vdw_radij.T)      # column-major (i,j)
        st.vdw_welij = d("E", s.vdw_welij.T)
        inttyp = getattr(s, "inttyp", None)
        st.inter_inttyp = i("it", inttyp.T) if inttyp is not None else C.POINTER(C.c_int32)()
        st.nmole = s.nmole
        st.molept_index = i("mi", s.molept_index, 1)
        st.molept_list = i("ml", s.molept_list, 1)
        st.index_excl = i("ie", s.index_excl)
        st.list_excl = i("le", s.list_excl)
        st.nbond = len(s.bonds)
        st.ibond = i("bi", s.bonds[:, 0], 1); st.jbond = i("bj", s.bonds[:, 1], 1)
        st.para_cbond = d("bk", s.bond_k); st.para_eqbond = d("br", s.bond_r0)
        st.nangl = len(s.angles)
        st.iangl = i("ai", s.angles[:, 0], 1); st.jangl = i("aj", s.angles[:, 1], 1)
        st.kangl = i("ak", s.angles[:, 2], 1)
        st.para_cangl = d("akk", s.angl_k); st.para_eqangl = d("at", s.angl_t0)
        st.ntors = len(s.tors)
        st.itors = i("ti", s.tors[:, 0], 1); st.jtors = i("tj", s.tors[:, 1], 1)
        st.ktors = i("tk", s.tors[:, 2], 1); st.ltors = i("tl", s.tors[:, 3], 1)
        st.para_divfac = i("tdv", s.tors_divfac); st.para_barhig = d("tb", s.tors_barhig)
        st.para_phsang = d("tph", s.tors_phsang); st.para_period = d("tpe", s.tors_period)
        st.ifcalnonb14 = i("t14", s.tors_14); st.para_divfac_vdw = d("tdvv", s.tors_dvdw)
        st.para_divfac_elc = d("tdve", s.tors_delc); st.ring14 = d("tr", s.tors_ring)
        st.ntorsrb = len(s.torsrb)
        st.itorsrb = i("ri", s.torsrb[:, 0], 1); st.jtorsrb = i("rj", s.torsrb[:, 1], 1)
        st.ktorsrb = i("rk", s.torsrb[:, 2], 1); st.ltorsrb = i("rl", s.torsrb[:, 3], 1)
        st.para_barhigrb = d("rc", s.torsrb_c)
        st.ifcalnonb14_rb = i("r14", s.torsrb_14); st.para_divfac_vdwrb = d("rdv", s.torsrb_dvdw)
        st.para_divfac_elcrb = d("rde", s.torsrb_delc); st.ring14_rb = d("rr", s.torsrb_ring)
        st.nconst = len(s.const_index) - 1
        st.index_mconst = i("ci", s.const_index, 1)
        st.list_mconst = i("cl", s.const_list, 1)
        st.nconstraint = len(s.const_d)
        st.iconst = i("cii", s.const_ij[:, 0], 1); st.jconst = i("cjj", s.const_ij[:, 1], 1)
        st.dconst = d("cd", s.const_d)
        st.degfree_all = int(s.degfree_all)
        if getattr(s, "mor_wel", None) is not None:
            st.para_welmor = d("mw", s.mor_wel.T); st.para_radmor = d("mr", s.mor_rad.T)
            st.para_alphamor = d("ma", s.mor_alpha.T)
        self.struct = st
        self._keep = keep


def params_struct(p: dict) -> ParamsStruct:
    ps = ParamsStruct()
    for name, _ in ParamsStruct._fields_:
        setattr(ps, name, p[name] if name in p or name not in PARAM_DEFAULTS else PARAM_DEFAULTS[name])
    return ps


def md_struct(dt_long_cal, nstep_short=1, mchain=3, text=0.0, tfreq=None, vfreq=None, pext=0.0,
              pcont_axis=PCONT_ISO, degfree=1, next_=1, nyosh=3, ifrattle=1, eps_rattle=1e-7,
              pressinterval=1, outinterval=0) -> MdParamsStruct:
    """Integrator parameters incl. prepmd.F90:515-547 (Q/W masses, Yoshida-Suzuki)."""
    m = MdParamsStruct()
    m.dt_long_cal = dt_long_cal
    m.nstep_short = nstep_short
    m.mchain = mchain
    m.text = text
    if tfreq:
        m.qmass[0] = degfree * text / tfreq / tfreq
        for k in range(1, mchain):
            m.qmass[k] = text / tfreq / tfreq
    if vfreq:
        if pcont_axis == PCONT_ISO:
            m.vmass = (degfree + 3) * text / (vfreq * vfreq)
        else:
            m.vmass = (degfree + 3) * text / (3.0 * vfreq * vfreq)
    m.next = next_
    m.nyosh = nyosh
    if nyosh == 1:
        ys = [1.0]
    elif nyosh == 3:
        w = 1.0 / (2.0 - 2.0 ** (1.0 / 3.0))
        ys = [w, 1.0 - 2.0 * w, w]
    else:
        w = 1.0 / (4.0 - 4.0 ** (1.0 / 3.0))
        ys = [w, w, 1.0 - 4.0 * w, w, w]
    for k, v in enumerate(ys):
        m.yscoeff[k] = v
    m.pext = pext
    m.pcont_axis = pcont_axis
    m.ifrattle = ifrattle
    m.eps_rattle = eps_rattle
    m.pressinterval = pressinterval
    m.outinterval = outinterval
    return m


def chain_init(box, mchain=3):
    ch = ChainStruct()
    ch.xlogv = float(np.log(box[0] * box[1] * box[2]) / 3.0)
    for d in range(3):
        ch.xboxh[d] = box[d]
    return ch
