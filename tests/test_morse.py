"""Morse pairs on the device (morse.F90:206-414 morsep, mklist_mor_cell.F90 /
mklist_mor.F90 lists) against the oracle, through the C ABI.

The system is the reference's recorded Pt/Morse sample (10 1-propanol + 190
butane on a 3,584-atom Pt slab; tests/golden/pt_morse_step1.npz), whose
oracle energies tests/test_golden_pt_morse.py pins to the printed values.
  * Morse list: bit-exact in the reference layout (nmorselist, mor_indexall
    with 0 sentinels, mor_listall), in the all-pairs order (2 x 2 x 9 cells
    at rcut_bookmor 14 A, the recorded run) and in the 27-cell order (3 x 3 x
    10 cells at 12 A).
  * morsep and calforce with Morse: FP64 forces within 1e-12 RMS relative,
    energies and virials within 1e-10; mixed precision within 1e-5.
  * MD with Morse (NVE, XO-RESPA with the bonded terms in the short group):
    FP64 positions within 1e-9 A of the oracle after 4 outer steps.
"""
import os

import numpy as np
import pytest

from tests.conftest import rel_rms
from tests.test_golden_pt_morse import load_pt_morse
from thrid_b200 import abi
from thrid_b200 import systems as S

pytestmark = pytest.mark.gpu

TOL_F64 = 1e-12
TOL_E64 = 1e-10
TOL_MIXED = 1e-5


def _pair(oracle_mod, precision=abi.PREC_FP64, **prm):
    from thrid_b200.pgk import PgkEngine
    s, want = load_pt_morse(precision)
    s.params.update(prm)
    o = oracle_mod.Oracle(s, threads=os.cpu_count() or 1)
    e = PgkEngine(s)
    return s, want, o, e


@pytest.mark.parametrize("rbook,mode", [(None, abi.LIST_ALLPAIR), (12.0, abi.LIST_CELL)])
def test_morse_list_is_bit_exact(oracle_mod, rbook, mode):
    prm = {} if rbook is None else {"rcut_bookmor": rbook}
    s, _, o, e = _pair(oracle_mod, **prm)
    o.mklist()
    assert o.mor_list()[0] == mode
    nl = e.mklist_mor_cell()
    ga, gi, gl = e.get_morlist()
    oa, oi, ol = o.get_mor_list()
    assert len(ga) == 3584 and np.array_equal(ga, oa)
    assert nl == len(ol)
    assert np.array_equal(gi, oi)
    assert np.array_equal(gl, ol)
    e.close()


def test_morsep_fp64_matches_oracle(oracle_mod):
    s, _, o, e = _pair(oracle_mod)
    o.mklist()
    of, oe, ov = o.morsep()
    gf, ge, gv = e.morsep()
    assert rel_rms(gf, of) < TOL_F64
    assert abs(ge["pot_mor"] - oe["pot_mor"]) <= TOL_E64 * abs(oe["pot_mor"])
    assert abs(gv["pot_viri_mor"] - ov["pot_viri_mor"]) <= TOL_E64 * abs(ov["pot_viri_mor"])
    t, ot = np.asarray(gv["pot_virit_mor"]), np.asarray(ov["pot_virit_mor"])
    assert np.abs(t - ot).max() <= TOL_E64 * np.abs(ot).max()
    e.close()


def test_morsep_mixed_matches_oracle(oracle_mod):
    s, _, o, e = _pair(oracle_mod, precision=abi.PREC_MIXED)
    o.mklist()
    of, oe, ov = o.morsep()
    gf, ge, gv = e.morsep()
    assert rel_rms(gf, of) < TOL_MIXED
    assert abs(ge["pot_mor"] - oe["pot_mor"]) <= TOL_MIXED * abs(oe["pot_mor"])
    assert abs(gv["pot_viri_mor"] - ov["pot_viri_mor"]) <= TOL_MIXED * abs(ov["pot_viri_mor"])
    e.close()


@pytest.mark.parametrize("precision,tol", [(abi.PREC_FP64, TOL_F64), (abi.PREC_MIXED, TOL_MIXED)])
def test_calforce_with_morse_matches_oracle(oracle_mod, precision, tol):
    """Both MTS groups of calforce on the recorded state (Morse in the long
    group, as in the recorded run): forces, every energy term, the virials."""
    s, _, o, e = _pair(oracle_mod, precision=precision)
    o.mklist()
    e.mklist_cell()
    for flag in (abi.MTS_LONG, abi.MTS_SHORT):
        of, oe, ov = o.calforce(flag)
        gf, ge, gv = e.calforce(flag)
        err = rel_rms(gf, of)
        print(f"group {flag} precision {precision}: force RMS relative error {err:.2e}")
        assert err < tol, (flag, err)
        etol = TOL_E64 if precision == abi.PREC_FP64 else TOL_MIXED
        for k in ("pot_mor", "pot_tot", "pot_vdw", "pot_elc", "pot_bond"):
            if oe[k] != 0.0:
                assert abs(ge[k] - oe[k]) <= etol * max(abs(oe[k]), 1.0), (flag, k, ge[k], oe[k])
        for k in ("pot_viri_mor", "pot_viri_lj"):
            if ov[k] != 0.0:
                assert abs(gv[k] - ov[k]) <= etol * abs(ov[k]), (flag, k)
    e.close()


def test_md_with_morse_fp64_matches_oracle(oracle_mod):
    """4 outer NVE steps (2 short steps each; bonded terms short, nonbonded and
    Morse long) from the recorded state: positions within 1e-9 A."""
    s, _, o, e = _pair(oracle_mod)
    md = abi.md_struct(S.fs_to_reduced(1.0), nstep_short=2, ifrattle=0, outinterval=0)
    st, _ = o.moldyn(0, 0, 4, md)
    assert st == 0
    e.moldyn_nve(0, 4, md)
    ox, ov, _ = o.get_state()
    gx, gv, _ = e.download_state()
    assert np.abs(gx - ox).max() < 1e-9
    assert rel_rms(gv, ov) < 1e-9
    e.close()
