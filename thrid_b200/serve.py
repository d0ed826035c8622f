"""Replica server (continuous batching of independent systems) over the C ABI
(`pgk_server_*` in include/pgk_gpu.h).

    srv = ReplicaServer(max_slots=4)
    rid = srv.submit(system, md, kind=0, nsteps=1000)
    x, v, box, ene, rec, times = srv.result(rid)      # blocks until done

Requests are admitted while earlier ones run, as slots and the device-memory
budget allow; each replica runs in its own context and CUDA stream.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

# Every replica context drives two CUDA streams; with the default eight
# hardware work queues per device, more than four concurrent replicas would
# share queues and serialise each other's kernels.  The setting only takes
# effect before the process initialises CUDA, so it is made on import unless
# the caller chose a value.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

from thrid_b200 import abi
from thrid_b200.pgk import PgkError, lib as _pgk_lib


class RequestStruct(C.Structure):
    _fields_ = [
        ("sys", C.POINTER(abi.SystemStruct)), ("prm", C.POINTER(abi.ParamsStruct)),
        ("md", C.POINTER(abi.MdParamsStruct)), ("kind", C.c_int32), ("_pad", C.c_int32),
        ("hf", C.POINTER(abi.HfParamsStruct)),
        ("atmcor", C.POINTER(C.c_double)), ("atmvel", C.POINTER(C.c_double)), ("box", C.POINTER(C.c_double)),
        ("chain", C.POINTER(abi.ChainStruct)), ("nsteps", C.c_int64),
    ]


def _lib():
    L = _pgk_lib()
    if not getattr(L, "_serve_bound", False):
        vp, pd = C.c_void_p, C.POINTER(C.c_double)
        L.pgk_estimate_bytes.restype = C.c_int64
        L.pgk_estimate_bytes.argtypes = [C.POINTER(abi.SystemStruct), C.POINTER(abi.ParamsStruct)]
        L.pgk_server_create.argtypes = [C.c_int32, C.c_int64, C.POINTER(vp)]
        L.pgk_server_submit.argtypes = [vp, C.POINTER(RequestStruct), C.POINTER(C.c_int64)]
        L.pgk_server_poll.argtypes = [vp, C.c_int64, C.POINTER(C.c_int32)]
        L.pgk_server_wait.argtypes = [vp, C.c_int64]
        L.pgk_server_result.argtypes = [vp, C.c_int64, pd, pd, pd, C.POINTER(abi.EnergiesStruct), pd, C.c_int64,
                                        C.POINTER(C.c_int64), pd]
        L.pgk_server_release.argtypes = [vp, C.c_int64]
        L.pgk_server_error.restype = C.c_char_p
        L.pgk_server_error.argtypes = [vp, C.c_int64]
        L.pgk_server_free.argtypes = [vp]
        L._serve_bound = True
    return L


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def estimate_bytes(system, params=None):
    L = _lib()
    cs = abi.CSystem(system)
    pr = abi.params_struct(dict(params or system.params))
    return int(L.pgk_estimate_bytes(C.byref(cs.struct), C.byref(pr)))


class ReplicaServer:
    def __init__(self, max_slots=4, hbm_budget_bytes=0):
        self.L = _lib()
        h = C.c_void_p()
        st = self.L.pgk_server_create(int(max_slots), int(hbm_budget_bytes), C.byref(h))
        if st:
            raise PgkError(st, "pgk_server_create failed")
        self.h = h
        self._meta = {}

    def submit(self, system, md, kind=0, nsteps=100, params=None, hf=None, chain=None, atmcor=None, atmvel=None):
        """Queue one replica; returns its id.  kind: 0 NVE, 1 NHC, 2 MTK, 3 heat flux (hf dict)."""
        cs = abi.CSystem(system)
        pr = abi.params_struct(dict(params or system.params))
        x = np.ascontiguousarray(system.atmcor if atmcor is None else atmcor, dtype=np.float64)
        v = np.ascontiguousarray(system.atmvel if atmvel is None else atmvel, dtype=np.float64)
        box = np.ascontiguousarray(system.box, dtype=np.float64)
        req = RequestStruct()
        req.sys = C.pointer(cs.struct)
        req.prm = C.pointer(pr)
        req.md = C.pointer(md)
        req.kind = int(kind)
        chf = abi.CHfParams(hf) if hf is not None else None
        req.hf = C.pointer(chf.struct) if chf else C.POINTER(abi.HfParamsStruct)()
        req.atmcor, req.atmvel, req.box = _p(x), _p(v), _p(box)
        req.chain = C.pointer(chain) if chain is not None else C.POINTER(abi.ChainStruct)()
        req.nsteps = int(nsteps)
        rid = C.c_int64()
        st = self.L.pgk_server_submit(self.h, C.byref(req), C.byref(rid))   # copies every input
        if st:
            raise PgkError(st, "pgk_server_submit failed")
        nreg = chf.nreg if chf else 0
        self._meta[rid.value] = (system.natom, nreg, int(nsteps), kind)
        return rid.value

    def done(self, rid):
        d = C.c_int32()
        self.L.pgk_server_poll(self.h, rid, C.byref(d))
        return bool(d.value)

    def result(self, rid, release=True):
        """Blocks until the replica is done; returns (x, v, box, energies, hf_records, times)
        with times = (submit, start, done) in seconds of a steady clock."""
        self.L.pgk_server_wait(self.h, rid)
        n, nreg, nsteps, kind = self._meta[rid]
        x = np.zeros((n, 3)); v = np.zeros((n, 3)); box = np.zeros(3)
        e = abi.EnergiesStruct()
        cap = nsteps if (kind == 3 and nreg) else 0
        rec = np.zeros((max(cap, 1), max(nreg, 1), abi.HF_NCOL))
        nr = C.c_int64()
        t = np.zeros(3)
        st = self.L.pgk_server_result(self.h, rid, _p(x), _p(v), _p(box), C.byref(e), _p(rec), cap, C.byref(nr),
                                      _p(t))
        if st:
            msg = (self.L.pgk_server_error(self.h, rid) or b"").decode()
            raise PgkError(st, f"replica {rid} failed: {msg}")
        if release:
            self.L.pgk_server_release(self.h, rid)
            del self._meta[rid]
        return x, v, box, e.as_dict(), rec[:min(nr.value, cap), :nreg], tuple(t)

    def close(self):
        if getattr(self, "h", None):
            self.L.pgk_server_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
