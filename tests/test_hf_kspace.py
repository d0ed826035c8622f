"""Per-atom reciprocal term of the bulk heat flux on the device.

  * pgk_fft_pme_hf, the per-atom split of fft_pmep's reciprocal energy and
    tensor (the SPME form of ewaldkp_hf's per-atom terms, ewaldk_hf.F90:
    165-230), against the oracle's spme_hf_atm: FP64 in both precisions,
    within 1e-9 of the largest entry.
  * The two heat-flux options of pgk_set_hf_kspace, through calheatf and
    moldyn_hf, against the oracle's restatement of the same options:
      EWK  (-D_HF_BULK_EWK, calforce_hf.F90:1046-1062): on heat-flux steps
           ewaldkp_hf replaces the SPME term and adds its per-atom terms;
      SPME: the SPME force stays and its per-atom split is added.
    FP64 heat-flux records within 1e-9 (calheatf) / 1e-7 (6 MD steps) of the
    largest entry, positions within 1e-9 A.
  * A CPU test of the option's host checks.
"""
import numpy as np
import pytest

from tests.test_hf import small_slab
from thrid_b200 import abi
from thrid_b200 import systems as S

KMAX = 5


def _engine(s, prec):
    from thrid_b200.pgk import PgkEngine
    return PgkEngine(s, dict(s.params, precision=prec))


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_spme_split_matches_oracle(oracle_mod, prec):
    s = S.water_box()
    o = oracle_mod.Oracle(s)
    pw, vw = o.spme_hf_atm()
    e = _engine(s, prec)
    pg, vg = e.fft_pme_hf()
    e.close()
    assert np.abs(pg - pw).max() <= 1e-9 * np.abs(pw).max()
    assert np.abs(vg - vw).max() <= 1e-9 * np.abs(vw).max()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [abi.HF_KSPACE_SPME, abi.HF_KSPACE_EWK])
def test_calheatf_with_kspace_matches_oracle(oracle_mod, mode):
    s = small_slab()
    o = oracle_mod.Oracle(s)
    o.set_hf(s.regions["hf"])
    o.set_hf_kspace(mode, KMAX)
    o.mklist()
    want = o.calheatf()
    pw, Ww = o.hf_atm()
    e = _engine(s, abi.PREC_FP64)
    e.set_hf(s.regions["hf"])
    e.set_hf_kspace(mode, KMAX)
    e.mklist_cell()
    got = e.calheatf()
    pg, Wg = e.hf_atm()
    e.close()
    assert np.abs(got - want).max() <= 1e-9 * np.abs(want).max()
    assert np.abs(pg - pw).max() <= 1e-9 * np.abs(pw).max()
    assert np.abs(Wg - Ww).max() <= 1e-9 * np.abs(Ww).max()
    # the reciprocal term is there: the Coulomb category differs from the default
    o2 = oracle_mod.Oracle(s)
    o2.set_hf(s.regions["hf"])
    o2.mklist()
    o2.calheatf()
    p0, _ = o2.hf_atm()
    assert np.abs(pw[abi.HF_ELC] - p0[abi.HF_ELC]).max() > 1e-3 * np.abs(p0[abi.HF_ELC]).max()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [abi.HF_KSPACE_SPME, abi.HF_KSPACE_EWK])
def test_moldyn_hf_with_kspace_matches_oracle(oracle_mod, mode):
    s = small_slab()
    md = abi.md_struct(S.fs_to_reduced(1.0), ifrattle=1, outinterval=0)
    o = oracle_mod.Oracle(s)
    o.set_hf(s.regions["hf"])
    o.set_hf_kspace(mode, KMAX)
    st, eo, rec_o = o.moldyn_hf(0, 6, md)
    assert st == 0
    e = _engine(s, abi.PREC_FP64)
    e.set_hf(s.regions["hf"])
    e.set_hf_kspace(mode, KMAX)
    eg, rec_g = e.moldyn_hf(0, 6, md)
    xo, vo, _ = o.get_state()
    xg, vg, _ = e.download_state()
    e.close()
    assert np.abs(xg - xo).max() < 1e-9
    assert rec_g.shape == rec_o.shape
    assert np.abs(rec_g - rec_o).max() <= 1e-7 * np.abs(rec_o).max()
    assert abs(eg["pot_ewk"] - eo["pot_ewk"]) <= 1e-9 * max(1.0, abs(eo["pot_ewk"]))


def test_kspace_option_host_checks(oracle_mod):
    s = small_slab()
    o = oracle_mod.Oracle(s)
    with pytest.raises(RuntimeError):
        o.set_hf_kspace(abi.HF_KSPACE_EWK, 0)          # the standard-Ewald option needs waves
    with pytest.raises(RuntimeError):
        o.set_hf_kspace(7, 3)
    o.set_hf_kspace(abi.HF_KSPACE_NONE)
