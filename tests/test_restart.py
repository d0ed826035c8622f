"""State record files in the reference format (wrsta.F90 / rdstarec.F90)."""
import numpy as np
import pytest

from thrid_b200 import abi
from thrid_b200 import restart as R
from thrid_b200 import systems as S


def test_fortran_e_format():
    assert R.fortran_e(1.0) == "  0.1000000000000000E+01"
    assert R.fortran_e(-2.5e-10) == " -0.2500000000000000E-09"
    assert R.fortran_e(0.0) == "  0.0000000000000000E+00"
    assert len(R.fortran_e(123456.789)) == 24
    assert R._num(R.fortran_e(3.141592653589793)) == pytest.approx(3.141592653589793, rel=1e-15)
    assert R._num("0.1234567890123456+100") == pytest.approx(0.1234567890123456e100)


def test_round_trip_of_a_state_record(tmp_path):
    s = S.small_box("propanol", nside=3, spacing=5.6)
    ch = abi.chain_init(s.box)
    for i in range(3):
        ch.xlogs[i] = 0.1 * (i + 1)
        ch.vlogs[i] = -0.01 * (i + 1)
    ch.vlogv, ch.pint = 1e-4, 2.5e-3
    for d in range(3):
        ch.vboxg[d] = 1e-5 * (d + 1)
    for q in range(9):
        ch.pintt[q] = 1e-3 * q
    p = tmp_path / "sta.dat"
    R.write_sta(p, s, s.atmcor, s.atmvel, s.box, ch, nstep=1234, mchain=3)
    text = p.read_text().splitlines()
    assert text[0] == "#npoly" + f"{s.nmole:8d}" and "#end" in text[-1]
    atom_lines = [l for l in text if l[:10].strip().isdigit() and len(l) == 10 + 6 * 24 + 3]
    assert len(atom_lines) == s.natom
    rec = R.read_sta(p)
    assert rec["natom"] == s.natom and rec["nstep"] == 1234 and rec["mchain"] == 3
    np.testing.assert_allclose(rec["cor"], s.atmcor, rtol=2e-15, atol=1e-14)
    np.testing.assert_allclose(rec["vel"], s.atmvel, rtol=2e-15, atol=1e-20)
    np.testing.assert_allclose(rec["box"], s.box, rtol=2e-15)
    c2 = R.chain_from(rec)
    np.testing.assert_allclose(list(c2.xlogs[:3]), [0.1, 0.2, 0.3], rtol=1e-15)
    np.testing.assert_allclose(list(c2.vlogs[:3]), [-0.01, -0.02, -0.03], rtol=2e-15)
    assert c2.vlogv == pytest.approx(1e-4, rel=2e-15) and c2.pint == pytest.approx(2.5e-3, rel=2e-15)
    np.testing.assert_allclose(list(c2.pintt), [1e-3 * q for q in range(9)], rtol=2e-15, atol=1e-30)


@pytest.mark.gpu
def test_device_checkpoint_restart(tmp_path):
    from thrid_b200.pgk import PgkEngine
    s = S.small_box("propanol", nside=3, spacing=5.6, precision=abi.PREC_MIXED)
    md = abi.md_struct(S.fs_to_reduced(1.0), ifrattle=1, outinterval=0)
    a = PgkEngine(s)
    a.moldyn_nve(0, 20, md)
    p = tmp_path / "sta.dat"
    R.wrsta(a, p, nstep=20)
    x, v, box = a.download_state()
    b = PgkEngine(s, upload=False)
    R.rdstarec(b, p)
    xb, vb, boxb = b.download_state()
    np.testing.assert_allclose(xb, x, rtol=2e-15, atol=1e-13)
    np.testing.assert_allclose(vb, v, rtol=2e-15, atol=1e-18)
