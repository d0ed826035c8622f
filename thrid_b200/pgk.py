"""Host-side mirror of the reference's operator interface over libpgkgpu.so.

The Fortran driver calls subroutines such as ``mklist_cell``, ``calforce``,
``ewaldr``, ``fft_pme``, ``rattle_c``, ``moldyn_nhc`` on module globals; this
class exposes the same operations on one device context through the C ABI of
include/pgk_gpu.h (names, argument meaning, STOP conditions turned into
:class:`PgkError`).  There is no CPU fallback: constructing an engine without
the built library or without a CUDA device raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpgkgpu.so")
HEADER = os.path.join(HERE, "..", "include", "pgk_gpu.h")

_lib = None


class PgkError(RuntimeError):
    def __init__(self, status, msg=""):
        super().__init__(f"pgk status {status}: {msg}")
        self.status = status


def header_symbols():
    """Entry points declared in include/pgk_gpu.h."""
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(pgk_[a-z0-9_]+)\s*\(", txt)))


def lib():
    """Load libpgkgpu.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise PgkError(abi.PGK_E_CUDA, f"{LIB_PATH} is not built (run thrid_b200/build.py)")
    L = C.CDLL(LIB_PATH)
    vp, pd, pi = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32)
    E, V = C.POINTER(abi.EnergiesStruct), C.POINTER(abi.VirialsStruct)
    L.pgk_version.restype = C.c_char_p
    L.pgk_status_string.restype = C.c_char_p
    L.pgk_status_string.argtypes = [C.c_int32]
    L.pgk_last_error.restype = C.c_char_p
    L.pgk_last_error.argtypes = [vp]
    L.pgk_init.argtypes = [C.POINTER(abi.SystemStruct), C.POINTER(abi.ParamsStruct), C.POINTER(vp)]
    L.pgk_free.argtypes = [vp]
    L.pgk_upload_state.argtypes = [vp, pd, pd, pd]
    L.pgk_download_state.argtypes = [vp, pd, pd, pd]
    L.pgk_set_chain.argtypes = [vp, C.POINTER(abi.ChainStruct)]
    L.pgk_get_chain.argtypes = [vp, C.POINTER(abi.ChainStruct)]
    L.pgk_transcor.argtypes = [vp]
    L.pgk_mklist_cell.argtypes = [vp, C.POINTER(C.c_int64)]
    L.pgk_get_nblist.argtypes = [vp, pi, pi, C.c_int64, C.POINTER(C.c_int64)]
    L.pgk_calforce.argtypes = [vp, C.c_int32, pd, E, V]
    for f in ("pgk_ewaldr", "pgk_fft_pme", "pgk_calbonded"):
        getattr(L, f).argtypes = [vp, pd, E, V]
    L.pgk_rattle_c.argtypes = [vp, pd, C.c_double, C.c_double]
    L.pgk_rattlep_v.argtypes = [vp, C.c_double]
    for f in ("pgk_moldyn_nve", "pgk_moldyn_nhc", "pgk_moldyn_mtk"):
        getattr(L, f).argtypes = [vp, C.c_int64, C.c_int64, C.POINTER(abi.MdParamsStruct), E]
    L.pgk_calpress.argtypes = [vp, pd, pd, pd]
    L.pgk_sync.argtypes = [vp]
    L.pgk_kernel_launches.restype = C.c_int64
    L.pgk_kernel_launches.argtypes = [vp]
    L.pgk_stream.restype = vp
    L.pgk_stream.argtypes = [vp]
    L.pgk_bench_kernel.argtypes = [vp, C.c_int32, C.c_int32, pd, pd, pd]
    L.pgk_set_hf.argtypes = [vp, C.POINTER(abi.HfParamsStruct)]
    L.pgk_set_output.argtypes = [vp, C.c_int64]
    L.pgk_get_output.argtypes = [vp, pd, C.c_int64, C.POINTER(C.c_int64)]
    L.pgk_moldyn_hf.argtypes = [vp, C.c_int64, C.c_int64, C.POINTER(abi.MdParamsStruct), E, pd, C.c_int64,
                                C.POINTER(C.c_int64)]
    L.pgk_calheatf.argtypes = [vp, pd]
    L.pgk_get_hf_atm.argtypes = [vp, pd, pd]
    L.pgk_langevin_dekin.argtypes = [vp, pd]
    L.pgk_ewaldkp_hf.argtypes = [vp, C.c_int32, pd, pd, pd, C.POINTER(abi.EwkHfStruct)]
    L.pgk_morsep.argtypes = [vp, pd, E, V]
    L.pgk_set_hf_kspace.argtypes = [vp, C.c_int32, C.c_int32]
    L.pgk_fft_pme_hf.argtypes = [vp, pd, pd]
    L.pgk_mklist_mor_cell.argtypes = [vp, C.POINTER(C.c_int64)]
    L.pgk_get_morlist.argtypes = [vp, pi, pi, pi, C.c_int64, C.POINTER(C.c_int64), pi]
    _lib = L
    return L


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def tuning_table():
    """Launch shapes the engine's autotuner chose in this process (one line
    per SPME grid shape and precision), as text."""
    L = lib()
    L.pgk_tuning_table.restype = C.c_int64
    L.pgk_tuning_table.argtypes = [C.c_char_p, C.c_int64]
    n = int(L.pgk_tuning_table(None, 0))
    buf = C.create_string_buffer(max(n, 1))
    L.pgk_tuning_table(buf, n)
    return buf.value.decode()


class PgkEngine:
    """One device context (the md_global state of one system)."""

    def __init__(self, system, params=None, upload=True):
        self.L = lib()
        self.sys = system
        self.csys = abi.CSystem(system)
        self.params = dict(params or system.params)
        self.prm = abi.params_struct(self.params)
        h = C.c_void_p()
        st = self.L.pgk_init(C.byref(self.csys.struct), C.byref(self.prm), C.byref(h))
        if st != abi.PGK_OK:
            raise PgkError(st, "pgk_init failed: " + self.L.pgk_status_string(st).decode())
        self.h = h
        if upload:
            self.upload_state(system.atmcor, system.atmvel, system.box)

    # -- lifetime ---------------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.L.pgk_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != abi.PGK_OK:
            msg = self.L.pgk_last_error(self.h)
            raise PgkError(st, (msg or b"").decode() or self.L.pgk_status_string(st).decode())

    # -- state --------------------------------------------------------------------
    def upload_state(self, atmcor, atmvel=None, box=None):
        cor = np.ascontiguousarray(atmcor, dtype=np.float64)
        vel = None if atmvel is None else np.ascontiguousarray(atmvel, dtype=np.float64)
        bx = None if box is None else np.ascontiguousarray(box, dtype=np.float64)
        self._check(self.L.pgk_upload_state(self.h, _p(cor), _p(vel) if vel is not None else None,
                                            _p(bx) if bx is not None else None))

    def download_state(self, cor=None, vel=None):
        """Positions, velocities (N,3) and box.  cor / vel: optional
        C-contiguous float64 (N,3) arrays to fill (e.g. pinned host memory)."""
        n = self.sys.natom
        for a in (cor, vel):
            if a is not None and (a.dtype != np.float64 or a.shape != (n, 3) or not a.flags.c_contiguous):
                raise ValueError("download_state: out arrays must be C-contiguous float64 (natom, 3)")
        cor = np.zeros((n, 3)) if cor is None else cor
        vel = np.zeros((n, 3)) if vel is None else vel
        box = np.zeros(3)
        self._check(self.L.pgk_download_state(self.h, _p(cor), _p(vel), _p(box)))
        return cor, vel, box

    def set_chain(self, ch):
        self._check(self.L.pgk_set_chain(self.h, C.byref(ch)))

    def get_chain(self):
        ch = abi.ChainStruct()
        self._check(self.L.pgk_get_chain(self.h, C.byref(ch)))
        return ch

    # -- reference-named operations ----------------------------------------------
    def transcor(self):
        self._check(self.L.pgk_transcor(self.h))

    def mklist_cell(self):
        nl = C.c_int64(0)
        self._check(self.L.pgk_mklist_cell(self.h, C.byref(nl)))
        return nl.value

    def get_nblist(self):
        n = self.sys.natom
        idx = np.zeros(n, np.int32)
        nl = C.c_int64(0)
        self._check(self.L.pgk_get_nblist(self.h, idx.ctypes.data_as(C.POINTER(C.c_int32)), None, 0, C.byref(nl)))
        lst = np.zeros(max(nl.value, 1), np.int32)
        self._check(self.L.pgk_get_nblist(self.h, idx.ctypes.data_as(C.POINTER(C.c_int32)),
                                          lst.ctypes.data_as(C.POINTER(C.c_int32)), nl.value, C.byref(nl)))
        return idx, lst[:nl.value]

    def mklist_mor_cell(self):
        nl = C.c_int64(0)
        self._check(self.L.pgk_mklist_mor_cell(self.h, C.byref(nl)))
        return nl.value

    def get_morlist(self):
        """(nmorselist, mor_indexall, mor_listall) of the last Morse list,
        1-based, in the reference layout."""
        nl = C.c_int64(0)
        nm = C.c_int32(0)
        self._check(self.L.pgk_get_morlist(self.h, None, None, None, 0, C.byref(nl), C.byref(nm)))
        atoms = np.zeros(max(nm.value, 1), np.int32)
        idx = np.zeros(max(nm.value, 1), np.int32)
        lst = np.zeros(max(nl.value, 1), np.int32)
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
        self._check(self.L.pgk_get_morlist(self.h, ip(atoms), ip(idx), ip(lst), nl.value, C.byref(nl),
                                           C.byref(nm)))
        return atoms[:nm.value], idx[:nm.value], lst[:nl.value]

    def morsep(self):
        return self._fev(self.L.pgk_morsep)

    def _fev(self, fn, *pre):
        f = np.zeros((self.sys.natom, 3))
        e = abi.EnergiesStruct()
        v = abi.VirialsStruct()
        self._check(fn(self.h, *pre, _p(f), C.byref(e), C.byref(v)))
        return f, e.as_dict(), v.as_dict()

    def calforce(self, mts_flag=abi.MTS_LONG):
        return self._fev(self.L.pgk_calforce, mts_flag)

    def ewaldr(self):
        return self._fev(self.L.pgk_ewaldr)

    def fft_pme(self):
        return self._fev(self.L.pgk_fft_pme)

    def calbonded(self):
        return self._fev(self.L.pgk_calbonded)

    def rattle_c(self, atmcor_old, eps_rattle, dt_short_cal):
        old = np.ascontiguousarray(atmcor_old, dtype=np.float64)
        self._check(self.L.pgk_rattle_c(self.h, _p(old), eps_rattle, dt_short_cal))

    def rattlep_v(self, eps_rattle):
        self._check(self.L.pgk_rattlep_v(self.h, eps_rattle))

    def calpress(self):
        k = C.c_double(); p = C.c_double(); t = np.zeros(9)
        self._check(self.L.pgk_calpress(self.h, C.byref(k), C.byref(p), _p(t)))
        return k.value, p.value, t.reshape(3, 3, order="F")

    def _md(self, fn, ini, end, md):
        e = abi.EnergiesStruct()
        self._check(fn(self.h, int(ini), int(end), C.byref(md), C.byref(e)))
        return e.as_dict()

    def moldyn_nve(self, ini, end, md):
        return self._md(self.L.pgk_moldyn_nve, ini, end, md)

    def moldyn_nhc(self, ini, end, md):
        return self._md(self.L.pgk_moldyn_nhc, ini, end, md)

    def moldyn_mtk(self, ini, end, md):
        return self._md(self.L.pgk_moldyn_mtk, ini, end, md)

    # ---- device-side output records (outene / outpre) ----
    OUT_COLUMNS = ("step",) + tuple(n for n, _ in abi.EnergiesStruct._fields_) + (
        "kint", "pint") + tuple(f"pintt{k}" for k in range(9)) + ("xcel", "ycel", "zcel")

    def set_output(self, cap_records):
        self._check(self.L.pgk_set_output(self.h, int(cap_records)))
        self._out_cap = int(cap_records)

    def get_output(self):
        cap = getattr(self, "_out_cap", 0)
        out = np.zeros((max(cap, 1), len(self.OUT_COLUMNS)))
        n = C.c_int64()
        self._check(self.L.pgk_get_output(self.h, _p(out), cap, C.byref(n)))
        return out[:min(n.value, cap)]

    # ---- heat flux + region Langevin (moldyn_hf.F90, calheatf.F90) ----
    def set_hf(self, hfd):
        """hfd: dict understood by abi.CHfParams (regions, heatfinterval,
        hftyp, langevin, lt_mole, seed, ifoutthc)."""
        self._hf = abi.CHfParams(hfd)
        self._check(self.L.pgk_set_hf(self.h, C.byref(self._hf.struct)))

    def calheatf(self):
        out = np.zeros((self._hf.nreg, abi.HF_NCOL))
        self._check(self.L.pgk_calheatf(self.h, _p(out)))
        return out

    def hf_atm(self):
        n = self.sys.natom
        pot = np.zeros((8, n)); W = np.zeros((8, max(self._hf.nreg, 1), 3, n))
        self._check(self.L.pgk_get_hf_atm(self.h, _p(pot), _p(W)))
        return pot, W[:, :self._hf.nreg]

    def moldyn_hf(self, ini, end, md, cap=100000):
        e = abi.EnergiesStruct()
        rec = np.zeros((max(cap, 1), max(self._hf.nreg, 1), abi.HF_NCOL))
        nr = C.c_int64(0)
        self._check(self.L.pgk_moldyn_hf(self.h, ini, end, C.byref(md), C.byref(e), _p(rec), cap, C.byref(nr)))
        return e.as_dict(), rec[:min(nr.value, cap), :self._hf.nreg]

    def ewaldkp_hf(self, kmax):
        """ewaldkp_hf (ewaldk_hf.F90:8-304) at the current positions: dict with
        force (N,3), pot_atm (N), viri_atm (N,3,3) with viri_atm[i, b, a] =
        virielct_atm(a,b,i,1), pot_ewk, pot_ewk_cc, pot_virit_coul (3,3) [b, a]
        and nwave."""
        n = self.sys.natom
        f = np.zeros((n, 3)); pot = np.zeros(n); vir = np.zeros((n, 3, 3))
        o = abi.EwkHfStruct()
        self._check(self.L.pgk_ewaldkp_hf(self.h, kmax, _p(f), _p(pot), _p(vir), C.byref(o)))
        return dict(force=f, pot_atm=pot, viri_atm=vir, pot_ewk=o.pot_ewk, pot_ewk_cc=o.pot_ewk_cc,
                    pot_virit_coul=np.array(o.pot_virit_coul[:]).reshape(3, 3), nwave=o.nwave)

    def set_hf_kspace(self, mode, kmax=0):
        """Per-atom reciprocal term of the heat flux: abi.HF_KSPACE_NONE,
        HF_KSPACE_EWK (ewaldkp_hf on heat-flux steps, waves up to kmax) or
        HF_KSPACE_SPME (the per-atom split of the SPME term)."""
        self._check(self.L.pgk_set_hf_kspace(self.h, int(mode), int(kmax)))

    def fft_pme_hf(self):
        """Per-atom split of fft_pmep: pot_atm (N) with the self term and
        viri_atm (N,3,3), viri_atm[i, b, a] = tensor(a,b) of atom i."""
        n = self.sys.natom
        pot = np.zeros(n); vir = np.zeros((n, 3, 3))
        self._check(self.L.pgk_fft_pme_hf(self.h, _p(pot), _p(vir)))
        return pot, vir

    def langevin_dekin(self):
        out = np.zeros(abi.LT_MAX_REGIONS)
        self._check(self.L.pgk_langevin_dekin(self.h, _p(out)))
        return out[:self._hf.nlt]

    def sync(self):
        self._check(self.L.pgk_sync(self.h))

    @property
    def kernel_launches(self):
        return int(self.L.pgk_kernel_launches(self.h))

    @property
    def stream(self):
        return self.L.pgk_stream(self.h)
