"""Parity with the FP64 oracle at the sizes of the named workloads, through
the C ABI (the other GPU parity tests use boxes of a few hundred to ~16k
atoms).  Collected after the smaller GPU tests: each case builds the oracle's
list and forces on all host cores (a few seconds each).

  C4  butane 200,004 atoms, 130 A box, rc 12 A, rcut_book 14 A (mklist_cell
      over 9^3 cells), SPME 128^3 order 5, aniso MTK + NHC:
        pair list bit-exact (nb_indexall, nb_listall, nlistnball);
        FP64 forces of both MTS groups <= 1e-12 RMS relative, energies and
        virials <= 1e-10; mixed forces <= 1e-5;
        one FP64 MTK step (RATTLE on the X-H bonds) within 1e-9 A.
  C2  propanol 12,000 atoms in 52 A, SPME 64^3 order 4 (3^3 = 27 cells:
      the mklist2a fallback of rdscript.F90:1595-1610), NHC:
        pair list bit-exact in the all-pairs order; FP64 forces <= 1e-12;
        mixed <= 1e-5; one FP64 NHC step within 1e-9 A.
  C3  alcohol/water slab, 43,200 atoms, 64 x 64 x 192, per-atom heat flux
      in 23 z regions:
        calheatf records and per-atom arrays (FP64) within 1e-9 of the
        largest entry; mixed within 2e-4.
"""
import os

import numpy as np
import pytest

from tests.conftest import rel_rms
from thrid_b200 import abi
from thrid_b200 import systems as S

pytestmark = pytest.mark.gpu

FP64_FORCE = 1e-12
FP64_ENERGY = 1e-10
MIXED_FORCE = 1e-5
HF_FP64 = 1e-9
HF_MIXED = 2e-4
THREADS = os.cpu_count() or 1


def _engine(s, prec, **over):
    from thrid_b200.pgk import PgkEngine
    return PgkEngine(s, dict(s.params, precision=prec, **over))


def _both_groups(x):
    fl, el, vl = x.calforce(abi.MTS_LONG)
    fs, es, vs = x.calforce(abi.MTS_SHORT)
    return fl + fs, {k: el[k] + es[k] for k in el}, {k: np.asarray(vl[k]) + np.asarray(vs[k]) for k in vl}


def _check_list_and_forces(oracle_mod, s, mode):
    o = oracle_mod.Oracle(s, threads=THREADS)
    omode, oidx, olst = o.mklist()
    assert omode == mode
    of, oe, ov = _both_groups(o)
    e = _engine(s, abi.PREC_FP64)
    nl = e.mklist_cell()
    idx, lst = e.get_nblist()
    assert nl == len(olst)
    assert np.array_equal(idx, oidx)
    assert np.array_equal(lst, olst)
    gf, ge, gv = _both_groups(e)
    err = rel_rms(gf, of)
    print(f"{s.name}: FP64 force RMS relative error {err:.2e}")
    assert err < FP64_FORCE
    for k in ("pot_tot", "pot_vdw", "pot_elc", "pot_ewk", "pot_bond", "pot_angl", "pot_torsrb", "pot_vdw14",
              "pot_elc14"):
        assert abs(ge[k] - oe[k]) <= FP64_ENERGY * max(1.0, abs(oe[k])), (k, ge[k], oe[k])
    for k in ("pot_viri_coul", "pot_viri_lj", "atm_viri_bond"):
        assert abs(float(gv[k]) - float(ov[k])) <= FP64_ENERGY * max(1.0, abs(float(ov[k]))), k
    e.close()
    m = _engine(s, abi.PREC_MIXED)
    m.mklist_cell()
    mf, _, _ = _both_groups(m)
    m.close()
    errm = rel_rms(mf, of)
    print(f"{s.name}: mixed force RMS relative error {errm:.2e}")
    assert errm < MIXED_FORCE
    return o


def test_c4_butane_200k(oracle_mod):
    s = S.butane_box(precision=abi.PREC_FP64)
    assert s.natom == 200004
    o = _check_list_and_forces(oracle_mod, s, abi.LIST_CELL)
    md = abi.md_struct(S.fs_to_reduced(1.0), mchain=3, text=S.kelvin_to_reduced(250.0), tfreq=1.0e13 * S.TIMEREF,
                       vfreq=0.2e12 * S.TIMEREF, pext=S.pa_to_reduced(1.01325e5), pcont_axis=abi.PCONT_ANISO,
                       degfree=s.degfree_all, ifrattle=1, eps_rattle=1e-7, outinterval=0)
    o.set_state(s.atmcor, s.atmvel, s.box)
    o.set_chain(abi.chain_init(s.box))
    st, _ = o.moldyn(2, 0, 1, md)
    assert st == 0
    e = _engine(s, abi.PREC_FP64)
    e.set_chain(abi.chain_init(s.box))
    e.moldyn_mtk(0, 1, md)
    ox, ov, ob = o.get_state()
    gx, gv, gb = e.download_state()
    e.close()
    print(f"C4 one MTK step: max |dx| {np.abs(gx - ox).max():.2e} A, box {np.abs(gb - ob).max():.2e}")
    assert np.abs(gx - ox).max() < 1e-9
    assert np.abs(gb - ob).max() < 1e-12 * ob.max()


def test_c2_propanol_12000_as_configured(oracle_mod):
    s = S.propanol_box(precision=abi.PREC_FP64)
    assert s.natom == 12000 and tuple(s.box) == (52.0, 52.0, 52.0)
    o = _check_list_and_forces(oracle_mod, s, abi.LIST_ALLPAIR)
    md = abi.md_struct(S.fs_to_reduced(1.0), mchain=3, text=S.kelvin_to_reduced(300.0), tfreq=1.0e13 * S.TIMEREF,
                       degfree=s.degfree_all, ifrattle=1, outinterval=0)
    o.set_state(s.atmcor, s.atmvel, s.box)
    o.set_chain(abi.chain_init(s.box))
    st, _ = o.moldyn(1, 0, 1, md)
    assert st == 0
    e = _engine(s, abi.PREC_FP64)
    e.set_chain(abi.chain_init(s.box))
    e.moldyn_nhc(0, 1, md)
    ox, _, _ = o.get_state()
    gx, _, _ = e.download_state()
    e.close()
    assert np.abs(gx - ox).max() < 1e-9


@pytest.mark.parametrize("prec,tol", [(abi.PREC_FP64, HF_FP64), (abi.PREC_MIXED, HF_MIXED)])
def test_c3_slab_43200_heat_flux(oracle_mod, prec, tol):
    s = S.slab_box(precision=abi.PREC_FP64)
    assert s.natom == 43200
    o = oracle_mod.Oracle(s, threads=THREADS)
    o.set_hf(s.regions["hf"])
    o.mklist()
    want = o.calheatf()
    pw, Ww = o.hf_atm()
    e = _engine(s, prec)
    e.set_hf(s.regions["hf"])
    e.mklist_cell()
    got = e.calheatf()
    pg, Wg = e.hf_atm()
    e.close()
    d = np.abs(got - want).max() / np.abs(want).max()
    print(f"C3 heat-flux records, precision {prec}: max deviation {d:.2e} of the largest entry")
    assert d <= tol
    if prec == abi.PREC_FP64:
        assert np.abs(pg - pw).max() <= tol * np.abs(pw).max()
        assert np.abs(Wg - Ww).max() <= tol * np.abs(Ww).max()
