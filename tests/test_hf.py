"""Heat flux (calvirihf / *_hf / calheatf) and region Langevin thermostat.

CPU tests pin the oracle's restatement with known answers:
  * Philox4x32-10 against the published known-answer vectors of Salmon et
    al. (SC 2011, Random123 kat_vectors);
  * the calvirihf fragment rule for a hand-placed two-atom pair;
  * per-atom energy shares summing to the term energies (bond, angle,
    torsion, 1-4, LJ);
  * the z column of the per-atom LJ and bond virial summing to the pressure
    tensor column when one region covers the box and no pair crosses z;
  * Box-Muller deviates with unit variance.
GPU tests compare the engine (through the C ABI) with the oracle:
  FP64 path: heat-flux records and per-atom arrays within 1e-9 relative
  (of the largest entry), MD with Langevin + heat flux within 1e-9 A;
  mixed path: records within 2e-4 of the largest entry.
"""
import ctypes as C

import numpy as np
import pytest

from thrid_b200 import abi
from thrid_b200 import systems as S

HF_FP64 = 1e-9
HF_MIXED = 2e-4


def small_slab(prec=abi.PREC_FP64, **kw):
    args = dict(nxy_w=6, nlay_w=6, nwater=216, nxy_p=3, nlay_p=1, lxy=18.6, rcut=7.0, nfft=(16, 16, 64),
                vacuum=8.0, hf_width=5.0, precision=prec)
    args.update(kw)
    return S.slab_box(**args)


def test_philox_known_answers(oracle_mod):
    L = oracle_mod.lib()

    def raw(ctr, key):
        c = np.array(ctr, np.uint32); k = np.array(key, np.uint32); o = np.zeros(4, np.uint32)
        L.orc_philox_raw(c.ctypes.data_as(C.c_void_p), k.ctypes.data_as(C.c_void_p), o.ctypes.data_as(C.c_void_p))
        return [int(x) for x in o]
    assert raw([0, 0, 0, 0], [0, 0]) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert raw([0xffffffff] * 4, [0xffffffff] * 2) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert raw([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0]) == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_box_muller_moments(oracle_mod):
    u = np.array([oracle_mod.philox_uniforms(7, 3, i) for i in range(20000)])
    assert u.min() > 0.0 and u.max() <= 1.0
    g = np.concatenate([np.sqrt(-2 * np.log(u[:, 0])) * np.cos(2 * np.pi * u[:, 1]),
                        np.sqrt(-2 * np.log(u[:, 0])) * np.sin(2 * np.pi * u[:, 1]),
                        np.sqrt(-2 * np.log(u[:, 2])) * np.cos(2 * np.pi * u[:, 3])])
    assert abs(g.mean()) < 0.02 and abs(g.var() - 1.0) < 0.03


def _two_body(z_i, z_j, regions, lz=40.0):
    """Two LJ atoms (different molecules) on the z axis of a tall box."""
    mol = S.ion_template(1)
    p = S.default_params((20.0, 20.0, lz), rcut=8.0, rrcut=8.0, alpha=0.3, nfft=(16, 16, 32), pme_order=4)
    sysobj = S.build_system("pair", [(mol, 2)], (20.0, 20.0, lz),
                            lambda m, k: np.array([[10.0, 10.0, (z_i, z_j)[k]]]), 1, 300.0, p)
    sysobj.vdw_radij[:] = 3.0
    sysobj.vdw_welij[:] = 0.5
    sysobj.atmchrg[:] = 0.0
    return sysobj


def test_calvirihf_fragment_rule(oracle_mod):
    # i at z=12, j at z=16: slabs [10,14] (one crossing: frag 2), [13,15]
    # (two crossings: frag 2), [11,20] (both inside: frag 4), [0,5] (none)
    regs = [(10.0, 14.0), (13.0, 15.0), (11.0, 20.0), (0.0, 5.0)]
    s = _two_body(12.0, 16.0, regs)
    o = oracle_mod.Oracle(s)
    o.set_hf(dict(regions=regs))
    o.mklist()
    o.calheatf()
    pot, W = o.hf_atm()
    f, e, v = o.ewaldrp()
    fz = f[0, 2]                     # force on atom 0 (LJ, along z)
    # reference rule: viri(:,3,i) += fi * sign(zi-zj) * frag / 2, same for j
    for r, frag in enumerate([2.0, 2.0, 4.0, 0.0]):
        want = -frag * 0.5 * fz       # zi - zj < 0
        np.testing.assert_allclose(W[abi.HF_VDW, r, 2, 0], want, rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(W[abi.HF_VDW, r, 2, 1], want, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(pot[abi.HF_VDW].sum(), e["pot_vdw"], rtol=1e-12)


def test_energy_shares_sum_to_terms(oracle_mod):
    s = small_slab()
    o = oracle_mod.Oracle(s)
    o.set_hf(s.regions["hf"])
    o.mklist()
    o.calheatf()
    pot, W = o.hf_atm()
    _, eb, _ = o.bonded()
    _, ep, _ = o.ewaldrp()
    np.testing.assert_allclose(pot[abi.HF_BO].sum(), eb["pot_bond"], rtol=1e-10, atol=1e-10)
    np.testing.assert_allclose(pot[abi.HF_AN].sum(), eb["pot_angl"], rtol=1e-10, atol=1e-10)
    np.testing.assert_allclose(pot[abi.HF_TO].sum(), eb["pot_tors"] + eb["pot_torsrb"], rtol=1e-10, atol=1e-10)
    np.testing.assert_allclose(pot[abi.HF_14].sum(), eb["pot_elc14"] + eb["pot_vdw14"], rtol=1e-10)
    np.testing.assert_allclose(pot[abi.HF_LJIN].sum() + pot[abi.HF_VDW].sum(), ep["pot_vdw"], rtol=1e-10)


def test_virial_column_identity(oracle_mod):
    # one region over the whole box, all atoms atom-based, vacuum wider than
    # the cutoff: sum_i viri(a,3,i) = sum_pairs f_a z_ij = pressure tensor (a, z)
    s = small_slab(vacuum=9.0)
    o = oracle_mod.Oracle(s)
    d = dict(s.regions["hf"])
    d["regions"] = [(0.0, s.box[2])]
    d["hftyp"] = None
    o.set_hf(d)
    o.mklist()
    o.calheatf()
    pot, W = o.hf_atm()
    _, _, vp = o.ewaldrp()
    _, _, vb = o.bonded()
    lj = W[abi.HF_LJIN, 0].sum(axis=1) + W[abi.HF_VDW, 0].sum(axis=1)
    np.testing.assert_allclose(lj, np.asarray(vp["pot_virit_lj"])[6:9], rtol=1e-9, atol=1e-9)
    bo = W[abi.HF_BO, 0].sum(axis=1)
    np.testing.assert_allclose(bo, np.asarray(vb["atm_virit_bond"])[6:9], rtol=1e-9, atol=1e-9)


def test_hf_steps_and_records_oracle(oracle_mod):
    s = small_slab()
    o = oracle_mod.Oracle(s)
    d = dict(s.regions["hf"])
    d["heatfinterval"] = 2
    o.set_hf(d)
    md = abi.md_struct(S.fs_to_reduced(1.0), ifrattle=1, outinterval=0)
    st, e, rec = o.moldyn_hf(0, 5, md)
    assert st == 0
    assert rec.shape[0] == 3                                   # steps 1, 3, 5
    np.testing.assert_allclose(rec[..., 17], rec[..., :17].sum(axis=-1), rtol=1e-12, atol=1e-14)


# ------------------------------------------------------------------ GPU ----
def _gpu_engine(s, prec):
    from thrid_b200.pgk import PgkEngine
    p = dict(s.params)
    p["precision"] = prec
    return PgkEngine(s, p)


@pytest.mark.gpu
def test_calheatf_fp64_parity(oracle_mod):
    s = small_slab()
    o = oracle_mod.Oracle(s)
    o.set_hf(s.regions["hf"])
    o.mklist()
    want = o.calheatf()
    pw, Ww = o.hf_atm()
    eng = _gpu_engine(s, abi.PREC_FP64)
    eng.set_hf(s.regions["hf"])
    eng.mklist_cell()
    got = eng.calheatf()
    pg, Wg = eng.hf_atm()
    scale = np.abs(want).max()
    assert np.abs(got - want).max() <= HF_FP64 * scale
    assert np.abs(pg - pw).max() <= HF_FP64 * np.abs(pw).max()
    assert np.abs(Wg - Ww).max() <= HF_FP64 * np.abs(Ww).max()


@pytest.mark.gpu
def test_calheatf_mixed_parity(oracle_mod):
    s = small_slab()
    o = oracle_mod.Oracle(s)
    o.set_hf(s.regions["hf"])
    o.mklist()
    want = o.calheatf()
    eng = _gpu_engine(s, abi.PREC_MIXED)
    eng.set_hf(s.regions["hf"])
    eng.mklist_cell()
    got = eng.calheatf()
    assert np.abs(got - want).max() <= HF_MIXED * np.abs(want).max()


@pytest.mark.gpu
def test_moldyn_hf_fp64_parity(oracle_mod):
    s = small_slab()
    md = abi.md_struct(S.fs_to_reduced(1.0), ifrattle=1, outinterval=0)
    o = oracle_mod.Oracle(s)
    o.set_hf(s.regions["hf"])
    st, eo, rec_o = o.moldyn_hf(0, 6, md)
    assert st == 0
    eng = _gpu_engine(s, abi.PREC_FP64)
    eng.set_hf(s.regions["hf"])
    eg, rec_g = eng.moldyn_hf(0, 6, md)
    xo, vo, _ = o.get_state()
    xg, vg, _ = eng.download_state()
    assert np.abs(xg - xo).max() < 1e-9
    assert np.abs(vg - vo).max() < 1e-9 * max(1.0, np.abs(vo).max())
    assert rec_g.shape == rec_o.shape
    assert np.abs(rec_g - rec_o).max() <= 1e-7 * np.abs(rec_o).max()
    np.testing.assert_allclose(eng.langevin_dekin(), o.langevin_dekin(), rtol=1e-8, atol=1e-10)


@pytest.mark.gpu
def test_moldyn_hf_mixed_tracks_fp64(oracle_mod):
    s = small_slab()
    md = abi.md_struct(S.fs_to_reduced(1.0), ifrattle=1, outinterval=0)
    o = oracle_mod.Oracle(s)
    o.set_hf(s.regions["hf"])
    o.moldyn_hf(0, 4, md)
    eng = _gpu_engine(s, abi.PREC_MIXED)
    eng.set_hf(s.regions["hf"])
    eng.moldyn_hf(0, 4, md)
    xo, _, _ = o.get_state()
    xg, _, _ = eng.download_state()
    assert np.abs(xg - xo).max() < 1e-4


@pytest.mark.gpu
def test_langevin_region_temperature():
    """Non-interacting atoms inside a Langevin region relax to its temperature."""
    n_side = 6
    mol = S.ion_template(1)
    L = 30.0
    g = (np.arange(n_side) + 0.5) * (L / n_side)
    sites = np.array([(x, y, z) for z in g for y in g for x in g])
    p = S.default_params((L, L, L), rcut=6.0, rrcut=6.0, alpha=0.5, nfft=(16, 16, 16), pme_order=4)
    s = S.build_system("gas", [(mol, len(sites))], (L, L, L), lambda m, k: sites[k][None, :], 5, 50.0, p)
    s.atmchrg[:] = 0.0
    s.vdw_welij[:] = 0.0
    T = S.kelvin_to_reduced(300.0)
    gam = 5.0e12 * S.TIMEREF
    hf = dict(regions=[], langevin=[dict(box=((0, L), (0, L), (0, L)), temp=T, damp=gam)], seed=3)
    eng = _gpu_engine(s, abi.PREC_FP64)
    eng.set_hf(hf)
    md = abi.md_struct(S.fs_to_reduced(2.0), ifrattle=0, outinterval=0)
    eng.moldyn_hf(0, 3000, md, cap=0)
    _, v, _ = eng.download_state()
    tk = (s.atmmass[:, None] * v ** 2).sum() / (3 * len(v))
    assert abs(tk / T - 1.0) < 0.12
