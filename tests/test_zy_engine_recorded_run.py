"""Device engine against the reference's recorded Pt/Morse step.

The engine has no Morse kernel yet, so it runs the recorded state with Morse
switched off (mts_mor = none: the Pt-Pt pairs carry neither Morse nor LJ) and
every other printed term of the step is compared with the device result
(tests/golden/pt_morse_step1.npz, loaded by tests/test_golden_pt_morse.py,
whose CPU tests pin the oracle to the same values).
"""
import math

import numpy as np
import pytest

from tests.test_golden_pt_morse import load_pt_morse, printed
from thrid_b200 import abi

NON_MORSE = ("pot_vdw", "pot_elc", "pot_ewk", "pot_ewc", "pot_vdw14", "pot_elc14", "pot_bond", "pot_angl",
             "pot_tors", "pot_torsrb")


def _engine_terms(precision):
    """The device engine on the recorded state with Morse switched off
    (mts_mor = none: Pt-Pt pairs carry neither Morse nor LJ), both MTS
    groups summed."""
    from thrid_b200.pgk import PgkEngine
    s, want = load_pt_morse(precision)
    p = dict(s.params)
    p["mts_mor"] = 0
    eng = PgkEngine(s, p)
    eng.mklist_cell()
    _, el, vl = eng.calforce(abi.MTS_LONG)
    _, es, vs = eng.calforce(abi.MTS_SHORT)
    e = {k: el[k] + es[k] for k in el}
    v = {k: np.asarray(vl[k]) + np.asarray(vs[k]) for k in vl}
    return want, e, v


@pytest.mark.gpu
def test_engine_fp64_matches_recorded_run():
    """FP64 device path against the reference's printed step-1 values: every
    energy term but Morse, and the LJ, Coulomb, bond and 1-4 virials, within
    half a unit of the 8th printed digit (slack 2 for the device sum order)."""
    want, e, v = _engine_terms(abi.PREC_FP64)
    assert e["pot_mor"] == 0.0
    for k in NON_MORSE:
        assert printed(want[k], e[k], want["eref"], slack=2.0), (k, e[k] * want["eref"], want[k])
    # pot_tot less the Morse term: a difference of two printed values, so the
    # bound is the sum of their half-units
    hu = lambda x: 0.5 * 10.0 ** (math.floor(math.log10(abs(x))) + 1 - 8)
    assert abs(e["pot_tot"] * want["eref"] - (want["pot_tot"] - want["pot_mor"])) <= \
        2.0 * (hu(want["pot_tot"]) + hu(want["pot_mor"]))
    assert printed(want["pot_virilj_all"], float(v["pot_viri_lj"]), want["eref"], slack=2.0)
    assert printed(want["pot_viric_all"], float(v["pot_viri_coul"]) + e["pot_ewc"] + e["pot_ewnq"],
                   want["eref"], slack=2.0)
    assert printed(want["atm_viribo_all"], float(v["atm_viri_bond"]), want["eref"], slack=2.0)
    assert printed(want["atm_viri14_all"], float(v["atm_viri_14"]), want["eref"], slack=2.0)


@pytest.mark.gpu
def test_engine_mixed_tracks_recorded_run():
    """Mixed-precision device path against the same printed values, each
    energy term within 1e-4 of itself (FP32 pair and bonded arithmetic)."""
    want, e, _ = _engine_terms(abi.PREC_MIXED)
    for k in NON_MORSE:
        w = want[k] / want["eref"]
        assert abs(e[k] - w) <= 1e-4 * abs(w), (k, e[k], w)
