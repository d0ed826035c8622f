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
