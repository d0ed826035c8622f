"""ewaldkp_hf (ewaldk_hf.F90:8-304): standard-Ewald k-space force, energy and
virial with the per-atom split of the bulk heat flux (-D_HF_BULK_EWK).

CPU tests pin the oracle's restatement:
  * the prepewk.F90:100-135 wave set (count, order, anint of the box ratios);
  * the Madelung constant of rock salt from ewaldrp + ewaldkp_hf + self term;
  * an independent vectorised numpy restatement (all outputs, net-charge
    correction included);
  * forces as the finite-difference gradient of pot_ewk;
  * agreement with the oracle's SPME (fft_pmep) on a fine grid;
  * per-atom energies summing to pot_ewk, per-atom tensors to the total;
  * the oracle's SPME per-atom split (spme_hf_atm) summing to fft_pmep and
    converging to ewaldkp_hf's per-atom terms on a fine grid.
GPU tests compare the engine (through the C ABI) with the oracle: every
output within 1e-10 of the largest entry of its kind, run-to-run identical.
"""
import math

import numpy as np
import pytest

from tests.conftest import rel_rms
from thrid_b200 import abi
from thrid_b200 import systems as S

EWK_TOL = 1e-10


def ewk_numpy(pos, q, box, alpha, nv, cc=False):
    """Vectorised restatement of ewaldk_hf.F90:130-299 (sums in numpy order)."""
    box = np.asarray(box, float)
    K = nv / box
    k2 = (K ** 2).sum(axis=1)
    aw = np.zeros(len(nv))
    aw[1:] = np.exp(-(math.pi / alpha) ** 2 * k2[1:]) / k2[1:]
    vol = box.prod()
    pf = 0.5 / math.pi / vol
    th = 2.0 * math.pi * (pos @ K.T)
    s, c = np.sin(th), np.cos(th)
    bsk, bck = q @ s, q @ c
    poti = pf * aw * (bsk ** 2 + bck ** 2)
    t1 = s * bsk + c * bck                       # (N, nwave)
    pot_atm = pf * q * (t1 @ aw) - alpha / math.sqrt(math.pi) * q ** 2
    force = (2.0 * q / vol)[:, None] * (((s * bck - c * bsk) * aw) @ K)
    fac_vir = 2.0 * math.pi ** 2 / alpha ** 2
    g = np.zeros(len(nv)); g[1:] = 2.0 / k2[1:] + fac_vir
    M = np.eye(3)[None] - g[:, None, None] * K[:, :, None] * K[:, None, :]
    M[0] = 0.0
    fac3 = pf * aw * (q.sum() ** 2) if cc else np.zeros(len(nv))
    e = pf * aw * q[:, None] * t1 - fac3[None, :]
    viri = np.einsum("ik,kab->iab", e, M)
    virit = np.einsum("k,kab->ab", poti - fac3, M)
    cc_sum = float((fac3[1:] * (-1.0 + fac_vir * k2[1:])).sum())
    return dict(force=force, pot_atm=pot_atm, viri_atm=viri, pot_ewk=float(poti.sum()), pot_ewk_cc=cc_sum,
                pot_virit_coul=virit)


def _charged_water(cc=True):
    s = S.small_box("water", nside=3, spacing=6.0)
    s.atmchrg[0] += 0.25 * S.CHARGE_SCALE    # net charge
    s.params["ifnetqcorrp"] = 1 if cc else 0
    return s


def _close(a, b, tol=EWK_TOL):
    a = np.asarray(a, float); b = np.asarray(b, float)
    return np.abs(a - b).max() <= tol * max(np.abs(b).max(), 1e-300)


# ------------------------------------------------------------------ CPU ----
def test_wave_set(oracle_mod):
    nv = oracle_mod.ewk_nvec(1)
    assert nv.tolist() == [[0, 0, 0], [-1, 0, 0], [0, -1, 0], [0, 0, -1], [0, 0, 1], [0, 1, 0], [1, 0, 0]]
    # integer points of the radius-2 ball: 1 + 6 + 12 + 8 + 6
    assert len(oracle_mod.ewk_nvec(2)) == 33
    for kmax, yr, zr in [(4, 1.0, 1.0), (3, 2.0, 1.0), (2, 1.0, 2.6), (3, 2.5, 1.4)]:
        nv = oracle_mod.ewk_nvec(kmax, yr, zr)
        ny0 = math.floor(yr + 0.5); nz0 = math.floor(zr + 0.5)     # anint (round half away)
        g = np.array([(x, y, z) for x in range(-kmax, kmax + 1) for y in range(-kmax * ny0, kmax * ny0 + 1)
                      for z in range(-kmax * nz0, kmax * nz0 + 1)
                      if (x, y, z) != (0, 0, 0) and x * x + y * y / ny0 ** 2 + z * z / nz0 ** 2 <= kmax ** 2])
        assert (nv[0] == 0).all()
        assert np.array_equal(nv[1:], g)                              # the reference's loop order


def test_madelung_constant_standard_ewald(oracle_mod):
    s = S.nacl_lattice()
    o = oracle_mod.Oracle(s)
    o.mklist()
    f1, e1, _ = o.ewaldrp()
    r = o.ewaldkp_hf(10)
    E = e1["pot_elc"] + r["pot_ewk"] + o.pot_ewc
    M = -E / (s.natom / 2) * 2.82 / S.CHARGE_SCALE ** 2
    assert abs(M - 1.747564594633) < 2e-6
    assert np.abs(f1 + r["force"]).max() < 1e-10
    # per-atom energies: every ion of a perfect lattice carries the same share
    pa = r["pot_atm"] + (o.pot_ewc / s.natom)
    assert np.abs(pa - pa.mean()).max() < 1e-9 * abs(pa.mean())


@pytest.mark.parametrize("cc", [False, True])
def test_matches_numpy_restatement(oracle_mod, cc):
    s = _charged_water(cc) if cc else S.small_box("water", nside=3, spacing=6.0)
    o = oracle_mod.Oracle(s)
    r = o.ewaldkp_hf(5)
    nv = oracle_mod.ewk_nvec(5).astype(float)
    w = ewk_numpy(s.atmcor, s.atmchrg, s.box, s.params["alpha"], nv, cc)
    assert r["nwave"] == len(nv)
    for k in ("force", "pot_atm", "viri_atm", "pot_virit_coul"):
        assert _close(r[k], w[k], 1e-11), k
    assert abs(r["pot_ewk"] - w["pot_ewk"]) <= 1e-12 * abs(w["pot_ewk"])
    if cc:
        assert r["pot_ewk_cc"] != 0.0
        assert abs(r["pot_ewk_cc"] - w["pot_ewk_cc"]) <= 1e-11 * abs(w["pot_ewk_cc"])
    else:
        assert r["pot_ewk_cc"] == 0.0


def test_force_is_energy_gradient(oracle_mod):
    s = S.small_box("water", nside=3, spacing=6.0)
    o = oracle_mod.Oracle(s)
    r = o.ewaldkp_hf(6)
    h = 1e-5
    for i in (0, 7, 40):
        for d in range(3):
            xs = []
            for sgn in (+1, -1):
                x = s.atmcor.copy(); x[i, d] += sgn * h
                o.set_state(x)
                xs.append(o.ewaldkp_hf(6)["pot_ewk"])
            fd = -(xs[0] - xs[1]) / (2 * h)
            assert abs(fd - r["force"][i, d]) <= 1e-6 * max(1.0, abs(r["force"][i, d]))
    o.set_state(s.atmcor)


def test_matches_spme_on_a_fine_grid(oracle_mod):
    s = S.water_box()
    s.params.update(nfft1=64, nfft2=64, nfft3=64, pme_order=8)
    o = oracle_mod.Oracle(s)
    f2, e2, v2 = o.fft_pmep()
    r = o.ewaldkp_hf(12)
    assert rel_rms(r["force"], f2) < 1e-7                            # measured 1.4e-9
    assert abs(r["pot_ewk"] - e2["pot_ewk"]) < 1e-8 * abs(e2["pot_ewk"])   # 4.6e-10
    assert _close(r["pot_virit_coul"], np.asarray(v2["pot_virit_coul"]).reshape(3, 3), 1e-6)   # 2.0e-8


def test_per_atom_sums(oracle_mod):
    s = S.small_box("propanol", nside=3, spacing=5.2)
    o = oracle_mod.Oracle(s)
    r = o.ewaldkp_hf(6)
    self_e = -s.params["alpha"] / math.sqrt(math.pi) * s.atmchrg ** 2
    assert abs((r["pot_atm"] - self_e).sum() - r["pot_ewk"]) <= 1e-12 * abs(r["pot_ewk"])
    assert _close(r["viri_atm"].sum(axis=0), r["pot_virit_coul"], 1e-12)
    assert abs(r["force"].sum(axis=0)).max() < 1e-10 * np.abs(r["force"]).max()


def test_net_charge_tensor_offset(oracle_mod):
    """With ifnetqcorrp every atom carries -fac_vir3 per wave (ewaldk_hf.F90:
    257-272): the atom tensors exceed the total by (N-1) sum_k fac_vir3 M_k."""
    s = _charged_water(True)
    o = oracle_mod.Oracle(s)
    r = o.ewaldkp_hf(4)
    s0 = _charged_water(True)
    q = s0.atmchrg
    nv = oracle_mod.ewk_nvec(4).astype(float)
    box = np.asarray(s0.box, float)
    K = nv[1:] / box
    k2 = (K ** 2).sum(axis=1)
    alpha = s0.params["alpha"]
    fac3 = 0.5 / math.pi / box.prod() * np.exp(-(math.pi / alpha) ** 2 * k2) / k2 * q.sum() ** 2
    g = 2.0 / k2 + 2.0 * math.pi ** 2 / alpha ** 2
    C = np.einsum("k,kab->ab", fac3, np.eye(3)[None] - g[:, None, None] * K[:, :, None] * K[:, None, :])
    n = len(q)
    assert _close(r["viri_atm"].sum(axis=0) - r["pot_virit_coul"], -(n - 1) * C, 1e-9)


def test_spme_per_atom_split_sums_to_fft_pmep(oracle_mod):
    """SPME per-atom split (oracle spme_hf_atm): the atoms' energies less the
    self term sum to fft_pmep's pot_ewk, their tensors to its tensor."""
    s = S.water_box()
    o = oracle_mod.Oracle(s)
    _, e, v = o.fft_pmep()
    pot, vir = o.spme_hf_atm()
    self_e = -s.params["alpha"] / math.sqrt(math.pi) * s.atmchrg ** 2
    assert abs((pot - self_e).sum() - e["pot_ewk"]) <= 1e-12 * abs(e["pot_ewk"])
    assert _close(vir.sum(axis=0), np.asarray(v["pot_virit_coul"]).reshape(3, 3), 1e-12)


def test_spme_per_atom_split_matches_standard_ewald(oracle_mod):
    """On a fine grid the SPME per-atom energies and tensors equal ewaldkp_hf's
    (measured 6.7e-11 and 1.6e-9 of the largest entry)."""
    s = S.water_box()
    s.params.update(nfft1=64, nfft2=64, nfft3=64, pme_order=8)
    o = oracle_mod.Oracle(s)
    pot, vir = o.spme_hf_atm()
    r = o.ewaldkp_hf(12)
    assert _close(pot, r["pot_atm"], 1e-9)
    assert _close(vir, r["viri_atm"], 1e-8)


# ------------------------------------------------------------------ GPU ----
def _engine(s, prec=abi.PREC_FP64):
    from thrid_b200.pgk import PgkEngine
    p = dict(s.params)
    p["precision"] = prec
    return PgkEngine(s, p)


def _check(got, want, force_abs=None):
    assert got["nwave"] == want["nwave"]
    for k in ("pot_atm", "viri_atm", "pot_virit_coul"):
        assert _close(got[k], want[k]), k
    if force_abs is None:
        assert _close(got["force"], want["force"])
    else:                                                             # forces that cancel to rounding
        assert np.abs(got["force"]).max() < force_abs and np.abs(want["force"]).max() < force_abs
    assert abs(got["pot_ewk"] - want["pot_ewk"]) <= EWK_TOL * abs(want["pot_ewk"])
    assert abs(got["pot_ewk_cc"] - want["pot_ewk_cc"]) <= EWK_TOL * max(abs(want["pot_ewk_cc"]), 1e-300)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_gpu_water_matches_oracle(oracle_mod, prec):
    s = S.water_box()
    want = oracle_mod.Oracle(s).ewaldkp_hf(8)
    eng = _engine(s, prec)
    got = eng.ewaldkp_hf(8)
    _check(got, want)
    again = eng.ewaldkp_hf(8)
    for k in ("force", "pot_atm", "viri_atm"):
        assert np.array_equal(again[k], got[k])                       # run-to-run identical
    assert again["pot_ewk"] == got["pot_ewk"]


@pytest.mark.gpu
def test_gpu_slab_box_ratios(oracle_mod):
    """Tall slab: anint(zcel/xcel) > 1 widens the z wave range."""
    s = S.slab_box(nxy_w=6, nlay_w=6, nwater=216, nxy_p=3, nlay_p=1, lxy=18.6, rcut=7.0, nfft=(16, 16, 64),
                   vacuum=8.0, hf_width=5.0, precision=abi.PREC_FP64)
    assert round(s.params["zcel"] / s.params["xcel"]) > 1
    want = oracle_mod.Oracle(s).ewaldkp_hf(6)
    _check(_engine(s).ewaldkp_hf(6), want)


@pytest.mark.gpu
def test_gpu_net_charge_and_kmax_change(oracle_mod):
    s = _charged_water(True)
    o = oracle_mod.Oracle(s)
    eng = _engine(s)
    for kmax in (3, 7, 3):                                            # rebuilds the wave set
        _check(eng.ewaldkp_hf(kmax), o.ewaldkp_hf(kmax))


@pytest.mark.gpu
def test_gpu_madelung_and_rejects_oversize(oracle_mod):
    s = S.nacl_lattice()
    eng = _engine(s)
    want = oracle_mod.Oracle(s).ewaldkp_hf(10)
    _check(eng.ewaldkp_hf(10), want, force_abs=1e-10)                # perfect lattice: no net force
    with pytest.raises(Exception):
        eng.ewaldkp_hf(84)                                            # 3*84 + 3 rows > 253
    with pytest.raises(Exception):
        eng.ewaldkp_hf(0)
    _check(eng.ewaldkp_hf(10), want, force_abs=1e-10)                # context still usable
