"""ctypes binding of the FP64 CPU oracle (oracle/liborc.so).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from thrid_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liborc.so")


def build(force=False):
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(
            os.path.join(HERE, "pgk_oracle.cpp")):
        subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        vp, pd, pi, i64p = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_longlong)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [C.POINTER(abi.SystemStruct), C.POINTER(abi.ParamsStruct)]
        L.orc_destroy.argtypes = [vp]
        L.orc_set_threads.argtypes = [vp, C.c_int]
        L.orc_set_state.argtypes = [vp, pd, pd, pd]
        L.orc_get_state.argtypes = [vp, pd, pd, pd]
        L.orc_set_chain.argtypes = [vp, C.POINTER(abi.ChainStruct)]
        L.orc_get_chain.argtypes = [vp, C.POINTER(abi.ChainStruct)]
        L.orc_transcor.argtypes = [vp]
        L.orc_mklist.argtypes = [vp, pi, pi, C.c_longlong, i64p]
        for f in ("orc_ewaldrp", "orc_fft_pmep", "orc_bonded"):
            getattr(L, f).argtypes = [vp, pd, C.POINTER(abi.EnergiesStruct), C.POINTER(abi.VirialsStruct)]
        L.orc_calforce.argtypes = [vp, C.c_int, pd, C.POINTER(abi.EnergiesStruct), C.POINTER(abi.VirialsStruct)]
        L.orc_rattle_c.argtypes = [vp, pd, C.c_double, C.c_double]
        L.orc_rattle_cmtk.argtypes = [vp, pd, C.c_double, C.c_double, pd]
        L.orc_rattlep_v.argtypes = [vp, C.c_double]
        for f in ("orc_nhcint", "orc_nhcpisoint", "orc_nhcpanisoint"):
            getattr(L, f).argtypes = [vp, C.POINTER(abi.MdParamsStruct)]
        L.orc_kint.restype = C.c_double
        L.orc_kint.argtypes = [vp]
        L.orc_calpress.argtypes = [vp, C.POINTER(abi.VirialsStruct), C.POINTER(abi.VirialsStruct), pd, pd]
        L.orc_rkcut.restype = C.c_double
        L.orc_rkcut.argtypes = [vp]
        L.orc_pot_ewc.restype = C.c_double
        L.orc_pot_ewc.argtypes = [vp]
        L.orc_spline.restype = C.c_double
        L.orc_spline.argtypes = [vp, C.c_int, C.c_double]
        L.orc_fill_bspline.argtypes = [C.c_double, C.c_int, pd, pd]
        L.orc_bsp_mod.argtypes = [vp, C.c_int, pd]
        L.orc_fft1d.argtypes = [pd, C.c_int, C.c_int]
        L.orc_moldyn.argtypes = [vp, C.c_int, C.c_longlong, C.c_longlong, C.POINTER(abi.MdParamsStruct),
                                 C.POINTER(abi.EnergiesStruct)]
        L.orc_set_hf.argtypes = [vp, C.POINTER(abi.HfParamsStruct)]
        L.orc_calheatf.argtypes = [vp, pd]
        L.orc_get_hf_atm.argtypes = [vp, pd, pd]
        L.orc_moldyn_hf.argtypes = [vp, C.c_longlong, C.c_longlong, C.POINTER(abi.MdParamsStruct),
                                    C.POINTER(abi.EnergiesStruct), pd, C.c_longlong, i64p]
        L.orc_langevin_dekin.argtypes = [vp, pd]
        L.orc_lt_regions.argtypes = [vp, pi]
        L.orc_philox.argtypes = [C.c_uint64, C.c_longlong, C.c_int, pd]
        L.orc_ewk_nvec.argtypes = [C.c_int, C.c_double, C.c_double, pi, C.c_int, pi]
        L.orc_ewaldkp_hf.argtypes = [vp, C.c_int, pd, pd, pd, pd, pi]
        L.orc_spme_hf_atm.argtypes = [vp, pd, pd]
        L.orc_set_hf_kspace.argtypes = [vp, C.c_int, C.c_int]
        L.orc_mor_list.argtypes = [vp, i64p]
        L.orc_get_mor_list.argtypes = [vp, pi, pi, pi, C.c_longlong, i64p, pi]
        L.orc_morsep.argtypes = [vp, pd, C.POINTER(abi.EnergiesStruct), C.POINTER(abi.VirialsStruct)]
        L.orc_morse_hf_atm.argtypes = [vp, pd, pd]
        _lib = L
    return _lib


def ewk_nvec(kmax, yratio=1.0, zratio=1.0):
    """prepewk.F90:100-135 wave-vector integers (nwave, 3), (0,0,0) first."""
    L = lib()
    nw = C.c_int(0)
    st = L.orc_ewk_nvec(kmax, yratio, zratio, None, 0, C.byref(nw))
    if st:
        raise RuntimeError(f"orc_ewk_nvec status {st}")
    out = np.zeros((nw.value, 3), np.int32)
    L.orc_ewk_nvec(kmax, yratio, zratio, out.ctypes.data_as(C.POINTER(C.c_int32)), nw.value, C.byref(nw))
    return out


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """FP64 restatement of the reference routines on one system."""

    def __init__(self, system, params=None, threads=1):
        self.L = lib()
        self.sys = system
        self.csys = abi.CSystem(system)
        self.prm = abi.params_struct(params or system.params)
        self.h = self.L.orc_create(C.byref(self.csys.struct), C.byref(self.prm))
        self.L.orc_set_threads(self.h, threads)
        self.set_state(system.atmcor, system.atmvel, system.box)

    def __del__(self):
        try:
            self.L.orc_destroy(self.h)
        except Exception:
            pass

    def set_threads(self, t):
        self.L.orc_set_threads(self.h, int(t))

    def set_state(self, cor, vel=None, box=None):
        cor = np.ascontiguousarray(cor, dtype=np.float64)
        vel = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64)
        box = None if box is None else np.ascontiguousarray(box, dtype=np.float64)
        self.L.orc_set_state(self.h, _p(cor), _p(vel) if vel is not None else None,
                             _p(box) if box is not None else None)

    def get_state(self):
        n = self.sys.natom
        cor = np.zeros((n, 3)); vel = np.zeros((n, 3)); box = np.zeros(3)
        self.L.orc_get_state(self.h, _p(cor), _p(vel), _p(box))
        return cor, vel, box

    def set_chain(self, ch):
        self.L.orc_set_chain(self.h, C.byref(ch))

    def get_chain(self):
        ch = abi.ChainStruct()
        self.L.orc_get_chain(self.h, C.byref(ch))
        return ch

    def transcor(self):
        self.L.orc_transcor(self.h)

    def mklist(self):
        n = self.sys.natom
        nl = C.c_longlong(0)
        idx = np.zeros(n, np.int32)
        mode = self.L.orc_mklist(self.h, idx.ctypes.data_as(C.POINTER(C.c_int32)), None, 0, C.byref(nl))
        lst = np.zeros(max(nl.value, 1), np.int32)
        self.L.orc_mklist(self.h, idx.ctypes.data_as(C.POINTER(C.c_int32)),
                          lst.ctypes.data_as(C.POINTER(C.c_int32)), nl.value, C.byref(nl))
        return mode, idx, lst[:nl.value]

    def _call3(self, fn, *pre):
        f = np.zeros((self.sys.natom, 3))
        e = abi.EnergiesStruct()
        v = abi.VirialsStruct()
        st = fn(self.h, *pre, _p(f), C.byref(e), C.byref(v))
        return f, e.as_dict(), v.as_dict(), st

    def ewaldrp(self):
        f, e, v, _ = self._call3(self.L.orc_ewaldrp)
        return f, e, v

    def fft_pmep(self):
        f, e, v, _ = self._call3(self.L.orc_fft_pmep)
        return f, e, v

    def bonded(self):
        f, e, v, st = self._call3(self.L.orc_bonded)
        return f, e, v

    def calforce(self, flag):
        f, e, v, st = self._call3(self.L.orc_calforce, flag)
        return f, e, v

    def rattle_c(self, old, eps, dt):
        old = np.ascontiguousarray(old, dtype=np.float64)
        return self.L.orc_rattle_c(self.h, _p(old), eps, dt)

    def rattlep_v(self, eps):
        return self.L.orc_rattlep_v(self.h, eps)

    def moldyn(self, kind, ini, end, md):
        e = abi.EnergiesStruct()
        st = self.L.orc_moldyn(self.h, kind, ini, end, C.byref(md), C.byref(e))
        return st, e.as_dict()

    # ---- heat flux + region Langevin ----
    def set_hf(self, hfd):
        self._hf = abi.CHfParams(hfd)
        st = self.L.orc_set_hf(self.h, C.byref(self._hf.struct))
        if st:
            raise RuntimeError(f"orc_set_hf status {st}")

    def calheatf(self):
        out = np.zeros((self._hf.nreg, abi.HF_NCOL))
        st = self.L.orc_calheatf(self.h, _p(out))
        if st:
            raise RuntimeError(f"orc_calheatf status {st}")
        return out

    def hf_atm(self):
        n = self.sys.natom
        pot = np.zeros((8, n)); W = np.zeros((8, self._hf.nreg, 3, n))
        self.L.orc_get_hf_atm(self.h, _p(pot), _p(W))
        return pot, W

    def moldyn_hf(self, ini, end, md, cap=100000):
        e = abi.EnergiesStruct()
        rec = np.zeros((max(cap, 1), max(self._hf.nreg, 1), abi.HF_NCOL))
        nr = C.c_longlong(0)
        st = self.L.orc_moldyn_hf(self.h, ini, end, C.byref(md), C.byref(e), _p(rec), cap, C.byref(nr))
        return st, e.as_dict(), rec[:min(nr.value, cap)]

    def ewaldkp_hf(self, kmax):
        """ewaldkp_hf (ewaldk_hf.F90:8-304): dict with force (N,3), pot_atm (N),
        viri_atm (N,3,3) with viri_atm[i, b, a] = virielct_atm(a,b,i,1), the
        scalars pot_ewk, pot_ewk_cc, pot_virit_coul (3,3) [b, a] and nwave."""
        n = self.sys.natom
        f = np.zeros((n, 3)); pot = np.zeros(n); vir = np.zeros((n, 3, 3)); sc = np.zeros(11)
        nw = C.c_int(0)
        st = self.L.orc_ewaldkp_hf(self.h, kmax, _p(f), _p(pot), _p(vir), _p(sc), C.byref(nw))
        if st:
            raise RuntimeError(f"orc_ewaldkp_hf status {st}")
        return dict(force=f, pot_atm=pot, viri_atm=vir, pot_ewk=sc[0], pot_ewk_cc=sc[1],
                    pot_virit_coul=sc[2:].reshape(3, 3), nwave=nw.value)

    def morse_hf_atm(self):
        """morsep_hf: per-atom Morse energy (N) and virial W (nreg,3,N) with
        W[r, a, i] = virimort_atm(a,3,i,r); needs set_hf."""
        n = self.sys.natom
        pot = np.zeros(n); W = np.zeros((self._hf.nreg, 3, n))
        st = self.L.orc_morse_hf_atm(self.h, _p(pot), _p(W))
        if st:
            raise RuntimeError(f"orc_morse_hf_atm status {st}")
        return pot, W

    def mor_list(self):
        """(PGK_LIST_* order, pair count) of the Morse list of the last mklist."""
        n = C.c_longlong(0)
        mode = self.L.orc_mor_list(self.h, C.byref(n))
        return mode, n.value

    def get_mor_list(self):
        """(nmorselist, mor_indexall, mor_listall) of the last Morse list,
        1-based, in the reference layout."""
        nl = C.c_longlong(0)
        nm = C.c_int32(0)
        self.L.orc_get_mor_list(self.h, None, None, None, 0, C.byref(nl), C.byref(nm))
        atoms = np.zeros(max(nm.value, 1), np.int32)
        idx = np.zeros(max(nm.value, 1), np.int32)
        lst = np.zeros(max(nl.value, 1), np.int32)
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
        self.L.orc_get_mor_list(self.h, ip(atoms), ip(idx), ip(lst), nl.value, C.byref(nl), C.byref(nm))
        return atoms[:nm.value], idx[:nm.value], lst[:nl.value]

    def morsep(self):
        f, e, v, _ = self._call3(self.L.orc_morsep)
        return f, e, v

    def set_hf_kspace(self, mode, kmax=0):
        st = self.L.orc_set_hf_kspace(self.h, int(mode), int(kmax))
        if st:
            raise RuntimeError(f"orc_set_hf_kspace status {st}")

    def spme_hf_atm(self):
        """Per-atom split of fft_pmep: pot_atm (N) with the self term and
        viri_atm (N,3,3), viri_atm[i, b, a] = tensor(a,b) of atom i."""
        n = self.sys.natom
        pot = np.zeros(n); vir = np.zeros((n, 3, 3))
        st = self.L.orc_spme_hf_atm(self.h, _p(pot), _p(vir))
        if st:
            raise RuntimeError(f"orc_spme_hf_atm status {st}")
        return pot, vir

    def langevin_dekin(self):
        out = np.zeros(abi.LT_MAX_REGIONS)
        self.L.orc_langevin_dekin(self.h, _p(out))
        return out[:self._hf.nlt]

    def lt_regions(self):
        out = np.zeros(self.sys.natom, np.int32)
        self.L.orc_lt_regions(self.h, out.ctypes.data_as(C.POINTER(C.c_int32)))
        return out

    def spline(self, k, x):
        return self.L.orc_spline(self.h, k, x)

    def bsp_mod(self, dim, n):
        out = np.zeros(n)
        self.L.orc_bsp_mod(self.h, dim, _p(out))
        return out

    def kint(self):
        return self.L.orc_kint(self.h)

    @property
    def rkcut(self):
        return self.L.orc_rkcut(self.h)

    @property
    def pot_ewc(self):
        return self.L.orc_pot_ewc(self.h)


def fill_bspline(w, order):
    a = np.zeros(order); d = np.zeros(order)
    lib().orc_fill_bspline(w, order, _p(a), _p(d))
    return a, d


def philox_uniforms(seed, step, atom):
    u = np.zeros(4)
    lib().orc_philox(seed, step, atom, _p(u))
    return u


def fft1d(x, sign):
    a = np.ascontiguousarray(np.asarray(x, dtype=np.complex128))
    buf = a.view(np.float64).copy()
    lib().orc_fft1d(_p(buf), len(a), sign)
    return buf.view(np.complex128)
