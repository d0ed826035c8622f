"""Device-side output records (outene / outpre values without a host sync per
output step) agree with the host read-back of the same steps."""
import numpy as np
import pytest

from thrid_b200 import abi
from thrid_b200 import systems as S

pytestmark = pytest.mark.gpu


def test_output_records_match_host_readback():
    from thrid_b200.pgk import PgkEngine
    s = S.small_box("propanol", nside=3, spacing=5.6, precision=abi.PREC_MIXED)
    md = abi.md_struct(S.fs_to_reduced(1.0), ifrattle=1, outinterval=10)
    a = PgkEngine(s)
    a.set_output(8)
    ea = a.moldyn_nve(0, 30, md)
    rec = a.get_output()
    assert rec.shape[0] == 4 and list(rec[:, 0]) == [0, 10, 20, 30]
    b = PgkEngine(s)
    host = []
    for lo, hi in ((0, 0), (1, 10), (11, 20), (21, 30)):
        host.append(b.moldyn_nve(lo, hi, md))
        kint, _, _ = b.calpress()
        host[-1]["kint"] = kint
    cols = PgkEngine.OUT_COLUMNS
    for r, h in zip(rec, host):
        for name in ("pot_tot", "pot_vdw", "pot_elc", "pot_ewk", "pot_bond", "pot_angl", "pot_torsrb"):
            assert r[cols.index(name)] == pytest.approx(h[name], rel=1e-12, abs=1e-12)
        assert r[cols.index("kint")] == pytest.approx(h["kint"], rel=1e-12)
    assert ea["pot_tot"] == pytest.approx(rec[-1][cols.index("pot_tot")], rel=1e-15)
    np.testing.assert_allclose(rec[:, cols.index("xcel")], s.box[0])
