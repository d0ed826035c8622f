"""Device engine against the reference's recorded Pt/Morse step.

The engine evaluates the recorded state (tests/golden/pt_morse_step1.npz,
loaded by tests/test_golden_pt_morse.py, whose CPU tests pin the oracle to the
same values) with both MTS groups, Morse pairs included (k_morse.cu), and
every printed energy term, the total, the virials and the virial tensor of
the step are compared with the device result directly.
"""
import numpy as np
import pytest

from tests.conftest import rel_rms
from tests.test_golden_pt_morse import load_pt_morse, printed
from thrid_b200 import abi

TERMS = ("pot_mor", "pot_vdw", "pot_elc", "pot_ewk", "pot_ewc", "pot_vdw14", "pot_elc14", "pot_bond", "pot_angl",
         "pot_tors", "pot_torsrb", "pot_tot")


def _engine_terms(precision):
    """The device engine on the recorded state, both MTS groups summed
    (forces, energies, virials)."""
    from thrid_b200.pgk import PgkEngine
    s, want = load_pt_morse(precision)
    eng = PgkEngine(s)
    eng.mklist_cell()
    fl, el, vl = eng.calforce(abi.MTS_LONG)
    fs, es, vs = eng.calforce(abi.MTS_SHORT)
    eng.close()
    e = {k: el[k] + es[k] for k in el}
    v = {k: np.asarray(vl[k]) + np.asarray(vs[k]) for k in vl}
    return s, want, fl + fs, e, v


@pytest.mark.gpu
def test_engine_fp64_matches_recorded_run():
    """FP64 device path against the reference's printed step-1 values: every
    energy term (Morse included) and the total, the LJ, Morse, Coulomb, bond
    and 1-4 virials and the nine entries of the virial tensor, within half a
    unit of the 8th printed digit (slack 2 for the device sum order)."""
    _, want, _, e, v = _engine_terms(abi.PREC_FP64)
    for k in TERMS:
        assert printed(want[k], e[k], want["eref"], slack=2.0), (k, e[k] * want["eref"], want[k])
    assert printed(want["pot_virilj_all"], float(v["pot_viri_lj"]), want["eref"], slack=2.0)
    assert printed(want["pot_virimor_all"], float(v["pot_viri_mor"]), want["eref"], slack=2.0)
    assert printed(want["pot_viric_all"], float(v["pot_viri_coul"]) + e["pot_ewc"] + e["pot_ewnq"],
                   want["eref"], slack=2.0)
    assert printed(want["atm_viribo_all"], float(v["atm_viri_bond"]), want["eref"], slack=2.0)
    assert printed(want["atm_viri14_all"], float(v["atm_viri_14"]), want["eref"], slack=2.0)
    tens = sum(v[k] for k in ("pot_virit_coul", "pot_virit_lj", "pot_virit_mor", "atm_virit_bond",
                              "atm_virit_angl", "atm_virit_tors", "atm_virit_14")).reshape(3, 3).T
    for i in range(3):
        for j in range(3):
            assert printed(want[f"preatmt_vtot{i + 1}{j + 1}"], tens[i, j], want["eref"], slack=2.0), (i, j)


@pytest.mark.gpu
def test_engine_mixed_tracks_recorded_run(oracle_mod):
    """Mixed-precision device path on the recorded state: force RMS relative
    error within 1e-5 of the FP64 oracle (whose energies reproduce the
    printed ones), every printed energy term within 1e-5 of the largest
    energy term and within 1e-4 of itself."""
    from tests.test_golden_pt_morse import oracle_energies
    s, want, f, e, _ = _engine_terms(abi.PREC_MIXED)
    o = oracle_mod.Oracle(s, threads=8)
    o.mklist()
    of = o.calforce(abi.MTS_LONG)[0] + o.calforce(abi.MTS_SHORT)[0]
    err = rel_rms(f, of)
    print(f"mixed force RMS relative error on the recorded state: {err:.2e}")
    assert err < 1e-5
    scale = max(abs(want[k]) for k in TERMS) / want["eref"]
    for k in TERMS:
        w = want[k] / want["eref"]
        print(f"{k}: mixed {e[k]:.10e} recorded {w:.10e} rel {abs(e[k] - w) / abs(w):.2e}")
        assert abs(e[k] - w) <= 1e-5 * scale and abs(e[k] - w) <= 1e-4 * abs(w), (k, e[k], w)
