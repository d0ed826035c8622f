"""NVE energy drift of the mixed-precision path against the FP64 device path
(the mixed path's bound: its drift within 2x the FP64 drift).

Total energy E = pot_tot + sum(m v^2)/2 is sampled every 100 steps of a
rigid-water NVE run (RATTLE, 1 fs, 2 ps); the drift is the slope of a
least-squares line through the samples, in units of the mean kinetic energy
per ps, with the slope's standard error.  Both drifts and their errors are
recorded as test properties (pytest --junitxml keeps them).  The bound is
statistical instead of a fixed floor: the mixed drift may exceed twice the
FP64 drift by no more than three combined standard errors of the two fits.
"""
import numpy as np
import pytest

from thrid_b200 import abi
from thrid_b200 import systems as S

pytestmark = pytest.mark.gpu


def _drift(prec, nchunk=20, chunk=100):
    from thrid_b200.pgk import PgkEngine
    s = S.water_box()
    eng = PgkEngine(s, dict(s.params, precision=prec))
    md = abi.md_struct(S.fs_to_reduced(1.0), ifrattle=1, outinterval=0)
    eng.moldyn_nve(0, 0, md)
    t, E, K = [], [], []
    for k in range(nchunk):
        e = eng.moldyn_nve(k * chunk + 1, (k + 1) * chunk, md)
        kint, _, _ = eng.calpress()
        t.append((k + 1) * chunk * 1e-3)          # ps
        E.append(e["pot_tot"] + 0.5 * kint)
        K.append(0.5 * kint)
    eng.close()
    (slope, _), cov = np.polyfit(np.asarray(t), np.asarray(E), 1, cov=True)
    ke = np.mean(K)
    return slope / ke, float(np.sqrt(cov[0, 0])) / ke


def test_mixed_nve_drift_within_twice_fp64(record_property):
    d64, se64 = _drift(abi.PREC_FP64)
    dmx, semx = _drift(abi.PREC_MIXED)
    for k, v in (("drift_fp64_ke_per_ps", d64), ("drift_fp64_stderr", se64),
                 ("drift_mixed_ke_per_ps", dmx), ("drift_mixed_stderr", semx)):
        record_property(k, v)
    print(f"NVE drift per ps (units of <KE>): fp64 {d64:.3e} +- {se64:.1e}  mixed {dmx:.3e} +- {semx:.1e}")
    assert abs(dmx) <= 2.0 * abs(d64) + 3.0 * np.hypot(semx, 2.0 * se64)
