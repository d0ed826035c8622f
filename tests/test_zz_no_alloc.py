"""The allocation-free SPME entry point (pgk_fft_pme_noalloc) against the
context-based one (pgk_fft_pme), through the C ABI.

Callers that reserve all device memory up front (a host driver or replica
server whose pool owns the HBM) cannot let the engine call cudaMalloc in the
middle of a run; this entry point works on their device buffers and keeps its
temporaries in one static device array.  The test allocates its own input and
output buffers (as such a caller would) and checks two calls in a row, so the
second call proves the shared scratch is cleared between calls.  It lives in a
file of its own that pytest collects last.
"""
import ctypes as C

import numpy as np
import pytest

from tests.conftest import rel_rms
from thrid_b200 import abi
from thrid_b200 import systems as S
from thrid_b200.pgk import PgkEngine, lib

pytestmark = pytest.mark.gpu

TOL_FORCE = 1e-12       # FP64 path: force RMS relative error
TOL_ENERGY = 1e-10


def _noalloc(L):
    f = L.pgk_fft_pme_noalloc
    pd = C.POINTER(C.c_double)
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, pd, C.c_double, C.c_int32, C.c_int32, C.c_int32,
                  C.c_int32, C.c_void_p, pd, C.c_void_p]
    f.restype = C.c_int32
    return f


def test_noalloc_spme_matches_context_entry_point(oracle_mod):
    import torch
    s = S.water_box()
    p = dict(s.params)
    p["precision"] = abi.PREC_FP64
    eng = PgkEngine(s, p)
    ref, ene, _ = eng.fft_pme()
    eng.close()
    # the oracle's fft_pmep (fft_pme.F90:144-270) on the same state
    o = oracle_mod.Oracle(s, p)
    oref, oene, _ = o.fft_pmep()
    assert rel_rms(ref, oref) < TOL_FORCE

    dev = torch.device("cuda:0")
    pos = torch.tensor(s.atmcor.ravel(), dtype=torch.float64, device=dev)
    chg = torch.tensor(s.atmchrg, dtype=torch.float64, device=dev)
    force = torch.zeros(3 * s.natom, dtype=torch.float64, device=dev)
    box = (C.c_double * 3)(*s.box)
    fn = _noalloc(lib())
    for call in range(2):
        force.zero_()
        e = C.c_double(0.0)
        torch.cuda.synchronize()
        st = fn(pos.data_ptr(), chg.data_ptr(), s.natom, box, p["alpha"], p["nfft1"], p["nfft2"], p["nfft3"],
                p["pme_order"], force.data_ptr(), C.byref(e), None)
        assert st == abi.PGK_OK, (call, st)
        torch.cuda.synchronize()
        got = force.cpu().numpy().reshape(-1, 3)
        assert rel_rms(got, ref) < TOL_FORCE, call
        assert rel_rms(got, oref) < TOL_FORCE, call
        assert abs(e.value - ene["pot_ewk"]) < TOL_ENERGY * max(1.0, abs(ene["pot_ewk"])), call
        assert abs(e.value - oene["pot_ewk"]) < TOL_ENERGY * max(1.0, abs(oene["pot_ewk"])), call


def test_noalloc_rejects_grids_beyond_its_static_scratch():
    import torch
    s = S.water_box()
    dev = torch.device("cuda:0")
    pos = torch.tensor(s.atmcor.ravel(), dtype=torch.float64, device=dev)
    chg = torch.tensor(s.atmchrg, dtype=torch.float64, device=dev)
    force = torch.zeros(3 * s.natom, dtype=torch.float64, device=dev)
    box = (C.c_double * 3)(*s.box)
    fn = _noalloc(lib())
    st = fn(pos.data_ptr(), chg.data_ptr(), s.natom, box, 0.32, 128, 128, 128, 4, force.data_ptr(), None, None)
    assert st == abi.PGK_E_SCRATCH_LIMIT
    assert lib().pgk_status_string(st).startswith(b"size exceeds")
    st = fn(pos.data_ptr(), chg.data_ptr(), s.natom, box, 0.32, 32, 32, 4, 6, force.data_ptr(), None, None)
    assert st == abi.PGK_E_INVALID      # an axis shorter than the B-spline order
    assert float(force.abs().max()) == 0.0
