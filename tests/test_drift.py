"""NVE energy drift of the mixed-precision path against the FP64 device path
(mixed drift within 2x the FP64 drift).

Total energy E = pot_tot + sum(m v^2)/2 is sampled every 100 steps of a
rigid-water NVE run (RATTLE, 1 fs); the drift is the slope of a least-squares
line through the samples, in units of the mean kinetic energy per ps.  The
bound allows 2x the FP64 drift plus a floor of 2e-3 KE/ps (the cutoff noise
both paths share makes tiny drifts statistically indistinguishable).
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
    slope = np.polyfit(np.asarray(t), np.asarray(E), 1)[0]
    return slope / np.mean(K)


def test_mixed_nve_drift_within_twice_fp64():
    d64 = _drift(abi.PREC_FP64)
    dmx = _drift(abi.PREC_MIXED)
    print(f"NVE drift per ps (units of <KE>): fp64 {d64:.3e}  mixed {dmx:.3e}")
    assert abs(dmx) <= 2.0 * abs(d64) + 2e-3
