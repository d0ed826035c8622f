"""The C ABI library builds, loads and exports every entry point that
include/pgk_gpu.h declares (no GPU needed: nothing here computes)."""
import ctypes
import os
import subprocess

import pytest

from thrid_b200 import abi, build, pgk


def test_header_declares_the_reference_operations():
    syms = pgk.header_symbols()
    for name in ("pgk_init", "pgk_free", "pgk_upload_state", "pgk_download_state", "pgk_mklist_cell",
                 "pgk_get_nblist", "pgk_calforce", "pgk_ewaldr", "pgk_fft_pme", "pgk_calbonded",
                 "pgk_rattle_c", "pgk_rattlep_v", "pgk_moldyn_nve", "pgk_moldyn_nhc", "pgk_moldyn_mtk",
                 "pgk_calpress", "pgk_transcor"):
        assert name in syms


def test_library_exports_every_declared_symbol():
    lib = build.build()
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in pgk.header_symbols() if s not in exported]
    assert not missing, missing


def test_library_loads_and_reports_version():
    L = pgk.lib()
    assert b"sm_100a" in L.pgk_version()
    assert L.pgk_status_string(abi.PGK_E_RATTLE_NOCONV).startswith(b"ERROR: RATTLE(C)")


def test_struct_sizes_match_the_header():
    # compile a tiny C probe of the header's struct sizes with gcc
    here = os.path.dirname(os.path.abspath(__file__))
    inc = os.path.join(here, "..", "include")
    src = ('#include "pgk_gpu.h"\n#include <stdio.h>\nint main(){printf("%zu %zu %zu %zu %zu %zu %zu %zu\\n",'
           'sizeof(pgk_system),sizeof(pgk_params),sizeof(pgk_mdparams),sizeof(pgk_energies),'
           'sizeof(pgk_virials),sizeof(pgk_chain),sizeof(pgk_hfparams),sizeof(pgk_ewk_hf));return 0;}\n')
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "p.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "p")
        subprocess.check_call(["gcc", "-I", inc, c, "-o", exe])
        sizes = [int(x) for x in subprocess.check_output([exe]).split()]
    want = [ctypes.sizeof(t) for t in (abi.SystemStruct, abi.ParamsStruct, abi.MdParamsStruct,
                                       abi.EnergiesStruct, abi.VirialsStruct, abi.ChainStruct,
                                       abi.HfParamsStruct, abi.EwkHfStruct)]
    assert sizes == want


def _header_define(name):
    import re
    txt = open(pgk.HEADER).read()
    m = re.search(r"#define\s+%s\s+(\d+)" % name, txt)
    assert m, name
    return int(m.group(1))


def test_output_record_columns_match_the_header():
    """The host mirror reads device output records with the header's width:
    a change of pgk_energies must change both together."""
    ncol = _header_define("PGK_OUT_NCOL")
    cols = pgk.PgkEngine.OUT_COLUMNS
    assert len(cols) == ncol
    assert cols[1:1 + len(abi.ENERGY_NAMES)] == tuple(abi.ENERGY_NAMES)
    assert cols[-3:] == ("xcel", "ycel", "zcel")


def test_noalloc_rejects_bad_grids_before_any_cuda_call():
    """pgk_fft_pme_noalloc checks its sizes before it touches the device: a
    grid axis shorter than the B-spline order (spread and gather wrap an index
    only once) is invalid, an axis that does not factor into 2, 3 and 5 is
    unsupported, and sizes beyond the static scratch are refused.  Runs
    without a GPU: the dummy pointers are never dereferenced."""
    L = pgk.lib()
    f = L.pgk_fft_pme_noalloc
    pd = ctypes.POINTER(ctypes.c_double)
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, pd, ctypes.c_double, ctypes.c_int32,
                  ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, pd, ctypes.c_void_p]
    f.restype = ctypes.c_int32
    box = (ctypes.c_double * 3)(20.0, 20.0, 20.0)
    dummy = ctypes.c_void_p(16)

    def call(k1, k2, k3, order):
        return f(dummy, dummy, 10, box, 0.3, k1, k2, k3, order, dummy, None, None)

    assert call(4, 32, 32, 8) == abi.PGK_E_INVALID
    assert call(32, 32, 5, 6) == abi.PGK_E_INVALID
    assert call(32, 32, 14, 4) == abi.PGK_E_UNSUPPORTED      # 14 = 2 * 7
    assert call(128, 128, 128, 4) == abi.PGK_E_SCRATCH_LIMIT
    assert call(32, 32, 32, 9) == abi.PGK_E_SCRATCH_LIMIT
    assert L.pgk_status_string(abi.PGK_E_UNSUPPORTED) == b"unsupported option"
