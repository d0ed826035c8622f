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


def test_reference_state_record_lines_reproduced():
    """Lines of the reference's own state record (sta_peachgk-2.0.dat of its
    Pt/Morse sample, kept in tests/golden/pt_morse_step1.npz) rendered again
    from their values by the writer's line functions: byte-identical header,
    section tags, atom lines ('(I10,6E24.16,A3)') and chain sections."""
    import os
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "pt_morse_step1.npz"))
    lines = dict(zip((int(i) for i in z["sta_line_no"]), (str(t) for t in z["sta_line_text"])))
    num = R._num
    box = [num(lines[k].split()[1]) for k in (10, 12, 14)]
    hdr = R.header_lines(int(lines[0].split()[1]), int(lines[2].split()[1]), int(lines[4].split()[1]),
                         int(lines[6].split()[1]), int(lines[8].split()[1]), box, int(lines[16].split()[1]))
    assert hdr == [lines[k] for k in range(18)]
    tags = {t for t in lines.values() if t.strip() in ("#poly", "#water", "#matom")}
    assert tags <= {" #poly", "#water", "#matom"} and " #poly" in tags
    natom_lines = 0
    for k, t in lines.items():
        f = t.split()
        if len(f) == 8 and f[0].isdigit():
            x = [num(q) for q in f[1:4]]
            v = [num(q) for q in f[4:7]]
            assert R.atom_line(int(f[0]), x, v, f[7]) == t
            natom_lines += 1
    assert natom_lines >= 20
    k0 = next(k for k, t in lines.items() if t == "#nhc")
    nhc = [lines[k].split() for k in range(k0 + 1, k0 + 4)]
    ander = lines[k0 + 6].split()
    aniso = lines[k0 + 9].split()
    got = R.chain_lines([num(a[1]) for a in nhc], [num(a[2]) for a in nhc], num(ander[1]), num(ander[2]),
                        [num(q) for q in aniso[1:4]], [num(q) for q in aniso[4:13]])
    assert got == [lines[k] for k in range(k0, k0 + len(got))]
