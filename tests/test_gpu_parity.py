"""Parity of the sm_100a engine (through the C ABI) with the FP64 oracle.

Bars (written here, per result):
  pair list          bit-exact: identical nb_indexall / nb_listall / nlistnball
  FP64 device path   force RMS relative error <= 1e-12, energies <= 1e-10 relative
  mixed precision    force RMS relative error <= 1e-5 (the mixed path's accuracy bound)
  MD trajectories    FP64 positions within 1e-9 A of the oracle after the steps run
"""
import numpy as np
import pytest

from tests.conftest import rel_rms
from thrid_b200 import abi
from thrid_b200 import systems as S
from thrid_b200.pgk import PgkEngine, PgkError

pytestmark = pytest.mark.gpu

FP64_FORCE = 1e-12
FP64_ENERGY = 1e-10
MIXED_FORCE = 1e-5
MIXED_ENERGY = 1e-5

_cache = {}


def case(name):
    if name not in _cache:
        _cache[name] = {
            "water": lambda: S.water_box(),                                   # mklist2a fallback, 2^3 cells
            "propanol_small": lambda: S.small_box("propanol", nside=4, spacing=5.6),
            "propanol_cells": lambda: S.propanol_box(nside=11, box=57.2),    # mklist_cell, 4^3 cells
            "butane_small": lambda: S.small_box("butane", nside=5, spacing=5.4, nfft=24, order=5),
            "nacl": lambda: _jittered(S.nacl_lattice()),
            "propanol_scattered": lambda: _scattered(S.small_box("propanol", nside=4, spacing=5.6)),
        }[name]()
    return _cache[name]


def _jittered(s, amp=0.05, seed=11):
    """Perfect lattices have ~0 net force; displace ions so forces are O(1)."""
    s.atmcor = s.atmcor + np.random.default_rng(seed).normal(0.0, amp, s.atmcor.shape)
    return s


def _scattered(s):
    """The same system with the atoms of its second half of molecules
    interleaved (atom k of molecule m -> far from atom k+1): their bonded
    terms span hundreds of atom indices, the first half's stay compact, so
    both bonded paths (per-block and per-type) run."""
    import dataclasses
    nm = s.nmole
    mols = [list(s.molept_list[s.molept_index[m]:s.molept_index[m + 1]]) for m in range(nm)]
    order = [a for m in mols[:nm // 2] for a in m]
    rest = mols[nm // 2:]
    for k in range(max(len(m) for m in rest)):
        order += [m[k] for m in rest if k < len(m)]
    new_of = np.empty(s.natom, dtype=np.int64)
    new_of[np.asarray(order)] = np.arange(s.natom)
    old = np.asarray(order)
    mp = lambda a: new_of[np.asarray(a, dtype=np.int64)] if len(a) else np.asarray(a)
    bonds, angles, tors, torsrb = mp(s.bonds), mp(s.angles), mp(s.tors), mp(s.torsrb)
    index_excl, list_excl = S._mkexcl(s.natom, bonds, angles, tors, torsrb)
    return dataclasses.replace(
        s, name=s.name + "_scattered", atmcor=s.atmcor[old].copy(), atmvel=s.atmvel[old].copy(),
        atmmass=s.atmmass[old].copy(), atmchrg=s.atmchrg[old].copy(), atmindex=s.atmindex[old].copy(),
        molept_list=mp(s.molept_list).astype(s.molept_list.dtype), index_excl=index_excl, list_excl=list_excl,
        bonds=bonds.astype(s.bonds.dtype), angles=angles.astype(s.angles.dtype), tors=tors.astype(s.tors.dtype),
        torsrb=torsrb.astype(s.torsrb.dtype) if len(s.torsrb) else s.torsrb,
        const_ij=mp(s.const_ij).astype(s.const_ij.dtype) if len(s.const_ij) else s.const_ij)


def engine(s, prec, **over):
    p = dict(s.params)
    p["precision"] = prec
    p.update(over)
    return PgkEngine(s, p)


def oracle_for(oracle_mod, s, **over):
    p = dict(s.params)
    p.update(over)
    return oracle_mod.Oracle(s, p)


def erel(a, b):
    return abs(a - b) / max(1.0, abs(b))


# ---------------------------------------------------------------- pair list ---
@pytest.mark.parametrize("name", ["water", "propanol_small", "propanol_cells", "nacl"])
def test_pair_list_is_bit_exact(oracle_mod, name):
    s = case(name)
    o = oracle_for(oracle_mod, s)
    mode, oidx, olst = o.mklist()
    e = engine(s, abi.PREC_FP64)
    nl = e.mklist_cell()
    idx, lst = e.get_nblist()
    assert nl == len(olst)
    assert np.array_equal(idx, oidx)
    assert np.array_equal(lst, olst)


def test_pair_list_regrows_rows_on_overflow(oracle_mod):
    s = case("propanol_small")
    o = oracle_for(oracle_mod, s)
    _, oidx, olst = o.mklist()
    e = engine(s, abi.PREC_MIXED, max_nbr=32)     # far too small: the engine regrows and rebuilds
    e.mklist_cell()
    idx, lst = e.get_nblist()
    assert np.array_equal(idx, oidx) and np.array_equal(lst, olst)


def test_cell_mode_order_matches_mklist_cell(oracle_mod):
    s = case("propanol_cells")
    o = oracle_for(oracle_mod, s, list_mode=abi.LIST_CELL)
    mode, oidx, olst = o.mklist()
    assert mode == abi.LIST_CELL
    e = engine(s, abi.PREC_FP64, list_mode=abi.LIST_CELL)
    e.mklist_cell()
    idx, lst = e.get_nblist()
    assert np.array_equal(idx, oidx) and np.array_equal(lst, olst)


def test_transcor_matches(oracle_mod):
    s = case("propanol_small")
    x = s.atmcor + np.array([30.0, -25.0, 0.5])      # push molecules out of the box
    o = oracle_for(oracle_mod, s)
    o.set_state(x)
    o.transcor()
    ox, _, _ = o.get_state()
    e = engine(s, abi.PREC_FP64)
    e.upload_state(x)
    e.transcor()
    gx, _, _ = e.download_state()
    assert np.array_equal(gx, ox)


# ------------------------------------------------------------------- forces ---
def _ref_terms(oracle_mod, s):
    o = oracle_for(oracle_mod, s)
    o.mklist()
    return o, o.ewaldrp(), o.fft_pmep(), o.bonded()


@pytest.mark.parametrize("name", ["water", "propanol_small", "butane_small", "nacl", "propanol_scattered"])
def test_fp64_forces_energies_virials(oracle_mod, name):
    s = case(name)
    o, (rf, re, rv), (kf, ke, kv), (bf, be, bv) = _ref_terms(oracle_mod, s)
    e = engine(s, abi.PREC_FP64)
    e.mklist_cell()
    f, en, vi = e.ewaldr()
    assert rel_rms(f, rf) < FP64_FORCE
    assert erel(en["pot_vdw"], re["pot_vdw"]) < FP64_ENERGY
    assert erel(en["pot_elc"], re["pot_elc"]) < FP64_ENERGY
    assert erel(vi["pot_viri_lj"], rv["pot_viri_lj"]) < FP64_ENERGY
    assert np.abs(vi["pot_virit_coul"] - rv["pot_virit_coul"]).max() < 1e-9 * max(1, np.abs(rv["pot_virit_coul"]).max())
    assert np.abs(vi["pot_virit_lj"] - rv["pot_virit_lj"]).max() < 1e-9 * max(1, np.abs(rv["pot_virit_lj"]).max())
    f, en, vi = e.fft_pme()
    assert rel_rms(f, kf) < FP64_FORCE
    assert erel(en["pot_ewk"], ke["pot_ewk"]) < FP64_ENERGY
    assert np.abs(vi["pot_virit_coul"] - kv["pot_virit_coul"]).max() < 1e-9 * max(1, np.abs(kv["pot_virit_coul"]).max())
    if np.abs(bf).max() > 0:
        f, en, vi = e.calbonded()
        assert rel_rms(f, bf) < FP64_FORCE
        for k in ("pot_bond", "pot_angl", "pot_tors", "pot_torsrb", "pot_elc14", "pot_vdw14"):
            assert erel(en[k], be[k]) < FP64_ENERGY, k
        for k in ("atm_viri_angl", "atm_viri_tors", "atm_viri_14"):
            assert erel(vi[k], bv[k]) < 1e-9, k


@pytest.mark.parametrize("name", ["water", "propanol_small", "butane_small", "nacl", "propanol_scattered"])
def test_mixed_forces_within_1e5(oracle_mod, name):
    s = case(name)
    o, (rf, re, rv), (kf, ke, kv), (bf, be, bv) = _ref_terms(oracle_mod, s)
    e = engine(s, abi.PREC_MIXED)
    e.mklist_cell()
    f1, en, _ = e.ewaldr()
    assert rel_rms(f1, rf) < MIXED_FORCE
    assert erel(en["pot_elc"], re["pot_elc"]) < MIXED_ENERGY * max(1, abs(re["pot_elc"]))
    f2, en, _ = e.fft_pme()
    assert rel_rms(f2, kf) < MIXED_FORCE
    f3, en, _ = e.calbonded()
    if np.abs(bf).max() > 0:
        assert rel_rms(f3, bf) < MIXED_FORCE
    assert rel_rms(f1 + f2 + f3, rf + kf + bf) < MIXED_FORCE


@pytest.mark.parametrize("nfft", [(20, 16, 24), (15, 16, 16)])
def test_spme_real_transform_matches_complex(oracle_mod, monkeypatch, nfft):
    """The SPME convolution with the real-to-complex x transform (half
    spectrum, mirrored points counted twice in the energy and virial) equals
    the complex transform of the full grid and the oracle's fft_pmep, in FP64
    (<= 1e-12) and in mixed precision (<= 1e-5); an odd K1 (15) runs the
    complex transform whatever the switch says."""
    s = S.small_box("propanol", nside=4, spacing=5.6)
    s.params.update(nfft1=nfft[0], nfft2=nfft[1], nfft3=nfft[2])
    o = oracle_for(oracle_mod, s)
    o.mklist()
    kf, ke, kv = o.fft_pmep()
    res = {}
    for prec in (abi.PREC_FP64, abi.PREC_MIXED):
        for r2c in ("1", "0"):
            monkeypatch.setenv("PGK_SPME_R2C", r2c)
            e = engine(s, prec)
            e.mklist_cell()
            res[(prec, r2c)] = e.fft_pme()
            e.close()
    for prec, tol in ((abi.PREC_FP64, FP64_FORCE), (abi.PREC_MIXED, MIXED_FORCE)):
        (f1, e1, v1), (f0, e0, v0) = res[(prec, "1")], res[(prec, "0")]
        assert rel_rms(f1, kf) < tol and rel_rms(f0, kf) < tol
        assert rel_rms(f1, f0) < tol
        assert erel(e1["pot_ewk"], ke["pot_ewk"]) < (FP64_ENERGY if prec == abi.PREC_FP64 else MIXED_ENERGY)
        vt = np.abs(kv["pot_virit_coul"]).max()
        assert np.abs(v1["pot_virit_coul"] - kv["pot_virit_coul"]).max() < (1e-9 if prec == abi.PREC_FP64 else 1e-5) * vt
        assert np.abs(v1["pot_virit_coul"] - v0["pot_virit_coul"]).max() < (1e-9 if prec == abi.PREC_FP64 else 1e-5) * vt


def test_calforce_mts_groups(oracle_mod):
    s = case("propanol_small")
    over = dict(mts_bond=abi.MTS_SHORT, mts_angl=abi.MTS_SHORT, mts_tors=abi.MTS_SHORT,
                mts_torsrb=abi.MTS_SHORT)
    o = oracle_for(oracle_mod, s, **over)
    o.mklist()
    e = engine(s, abi.PREC_FP64, **over)
    e.mklist_cell()
    for flag in (abi.MTS_SHORT, abi.MTS_LONG):
        rf, re, rv = o.calforce(flag)
        f, en, vi = e.calforce(flag)
        assert rel_rms(f, rf) < FP64_FORCE
        for k in ("pot_tot", "pot_nonbon", "pot_ewc", "pot_ewnq"):
            assert erel(en[k], re[k]) < FP64_ENERGY, (flag, k)
        assert erel(vi["pot_viri_coul"], rv["pot_viri_coul"]) < 1e-9


def test_mixed_is_deterministic():
    """Run-to-run reproducibility: two engines taking the same steps give
    bit-identical forces and energies (integer force sums, fixed work
    assignment).  A repeated evaluation on one engine reads the pruned rows
    the first one wrote (another summation order in FP32): equal to 1e-6."""
    s = case("propanol_small")
    out = []
    for _ in range(2):
        e = engine(s, abi.PREC_MIXED)
        e.mklist_cell()
        a, ea, _ = e.calforce(abi.MTS_LONG)
        b, eb, _ = e.calforce(abi.MTS_LONG)
        out.append((a, ea, b, eb))
        e.close()
    (a1, ea1, b1, eb1), (a2, ea2, b2, eb2) = out
    assert np.array_equal(a1, a2) and np.array_equal(b1, b2)
    assert ea1 == ea2 and eb1 == eb2
    assert rel_rms(b1, a1) < 1e-6


# ------------------------------------------------------------------ RATTLE ---
def test_rattle_matches_oracle(oracle_mod):
    s = case("water")
    dt = S.fs_to_reduced(1.0)
    old = s.atmcor.copy()
    new = old + dt * s.atmvel
    o = oracle_for(oracle_mod, s)
    o.set_state(new, s.atmvel)
    assert o.rattle_c(old, 1e-7, dt) == 0
    assert o.rattlep_v(1e-7) == 0
    ox, ov, _ = o.get_state()
    e = engine(s, abi.PREC_FP64)
    e.upload_state(new, s.atmvel)
    e.rattle_c(old, 1e-7, dt)
    e.rattlep_v(1e-7)
    gx, gv, _ = e.download_state()
    assert np.abs(gx - ox).max() < 1e-12
    assert np.abs(gv - ov).max() < 1e-10


def test_rattle_nonconvergence_is_a_status_not_a_fault():
    s = case("water")
    dt = S.fs_to_reduced(1.0)
    old = s.atmcor.copy()
    e = engine(s, abi.PREC_FP64)
    e.upload_state(old + dt * s.atmvel, s.atmvel)
    with pytest.raises(PgkError) as ex:
        e.rattle_c(old, 0.0, dt)       # tolerance 0 cannot be met: bounded loop gives up
    assert ex.value.status == abi.PGK_E_RATTLE_NOCONV
    e.rattle_c(old, 1e-7, dt)          # context still usable afterwards


# -------------------------------------------------------------- MD drivers ---
def _md(s, dt_fs=1.0, kind="nve", nstep_short=1, T=300.0, pext_pa=0.0, axis=abi.PCONT_ISO, outinterval=0):
    Tr = S.kelvin_to_reduced(T)
    return abi.md_struct(S.fs_to_reduced(dt_fs), nstep_short=nstep_short, mchain=3, text=Tr,
                         tfreq=1.0e13 * S.TIMEREF, vfreq=0.2e12 * S.TIMEREF, pext=S.pa_to_reduced(pext_pa),
                         pcont_axis=axis, degfree=s.degfree_all, ifrattle=1, eps_rattle=1e-7,
                         outinterval=outinterval)


def _run_pair(oracle_mod, s, kind, md, steps, prec=abi.PREC_FP64, **over):
    o = oracle_for(oracle_mod, s, **over)
    o.set_chain(abi.chain_init(s.box))
    st, oe = o.moldyn({"nve": 0, "nhc": 1, "mtk": 2}[kind], 0, steps, md)
    assert st == 0
    e = engine(s, prec, **over)
    e.set_chain(abi.chain_init(s.box))
    ge = getattr(e, "moldyn_" + kind)(0, steps, md)
    return o, e, oe, ge


@pytest.mark.parametrize("kind,name", [("nve", "water"), ("nhc", "propanol_small"), ("mtk", "propanol_small")])
def test_fp64_md_matches_oracle(oracle_mod, kind, name):
    s = case(name)
    md = _md(s, kind=kind, pext_pa=1.0e5)
    o, e, oe, ge = _run_pair(oracle_mod, s, kind, md, 8)
    ox, ov, ob = o.get_state()
    gx, gv, gb = e.download_state()
    assert np.abs(gx - ox).max() < 1e-9
    assert np.abs(gv - ov).max() < 1e-8
    assert np.abs(gb - ob).max() < 1e-12
    assert erel(ge["pot_tot"], oe["pot_tot"]) < 1e-8
    if kind != "nve":
        oc, gc = o.get_chain(), e.get_chain()
        assert np.abs(np.array(gc.vlogs[:3]) - np.array(oc.vlogs[:3])).max() < 1e-9
    if kind == "mtk":
        assert abs(gc.vlogv - oc.vlogv) < 1e-9 * max(1.0, abs(oc.vlogv))
        assert abs(gc.pint - oc.pint) < 1e-8 * max(1.0, abs(oc.pint))


def test_fp64_mtk_aniso_matches_oracle(oracle_mod):
    s = case("propanol_small")
    md = _md(s, kind="mtk", pext_pa=1.0e5, axis=abi.PCONT_ANISO)
    o, e, oe, ge = _run_pair(oracle_mod, s, "mtk", md, 6)
    ox, _, ob = o.get_state()
    gx, _, gb = e.download_state()
    assert np.abs(gx - ox).max() < 1e-9
    assert np.abs(gb - ob).max() < 1e-12
    oc, gc = o.get_chain(), e.get_chain()
    assert np.abs(np.array(gc.vboxg[:]) - np.array(oc.vboxg[:])).max() < 1e-9


def test_fp64_respa_matches_oracle(oracle_mod):
    s = case("propanol_small")
    over = dict(mts_bond=abi.MTS_SHORT, mts_angl=abi.MTS_SHORT, mts_tors=abi.MTS_SHORT, mts_torsrb=abi.MTS_SHORT)
    md = _md(s, dt_fs=2.0, kind="nhc", nstep_short=4)
    o, e, oe, ge = _run_pair(oracle_mod, s, "nhc", md, 5, **over)
    ox, _, _ = o.get_state()
    gx, _, _ = e.download_state()
    assert np.abs(gx - ox).max() < 1e-9


def test_mixed_md_tracks_fp64(oracle_mod):
    s = case("propanol_small")
    md = _md(s, kind="nhc")
    o, e, oe, ge = _run_pair(oracle_mod, s, "nhc", md, 10, prec=abi.PREC_MIXED)
    ox, _, _ = o.get_state()
    gx, _, _ = e.download_state()
    assert np.abs(gx - ox).max() < 1e-4
    assert erel(ge["pot_tot"], oe["pot_tot"]) < 1e-4 * max(1.0, abs(oe["pot_tot"]))


def test_mixed_mtk_aniso_tracks_fp64(oracle_mod):
    """Anisotropic MTK in mixed precision: the steps without output read only
    the total virial tensor (tensor-only pair and bonded kernels); the
    pressure tensor, box and positions track the FP64 oracle."""
    s = case("propanol_small")
    md = _md(s, kind="mtk", pext_pa=1.0e5, axis=abi.PCONT_ANISO)
    o, e, oe, ge = _run_pair(oracle_mod, s, "mtk", md, 6, prec=abi.PREC_MIXED)
    ox, _, ob = o.get_state()
    gx, _, gb = e.download_state()
    assert np.abs(gx - ox).max() < 1e-4
    assert np.abs(gb - ob).max() < 1e-6 * np.abs(ob).max()
    oc, gc = o.get_chain(), e.get_chain()
    op, gp = np.array(oc.pintt[:]), np.array(gc.pintt[:])
    assert np.abs(gp - op).max() < 1e-4 * np.abs(op).max()


def test_list_rebuild_inside_md_run(oracle_mod):
    s = case("water")
    md = _md(s, kind="nve")
    over = dict(nstep_book=3)
    o, e, oe, ge = _run_pair(oracle_mod, s, "nve", md, 7, **over)
    ox, _, _ = o.get_state()
    gx, _, _ = e.download_state()
    assert np.abs(gx - ox).max() < 1e-9


# ------------------------------------------------------- pruned pair list ---
def test_mixed_pruned_list_keeps_every_pair(monkeypatch):
    """The mixed pair kernel reads a pruned copy of the book list (pairs
    inside cutoff + buffer, re-pruned when atoms have moved half the buffer).
    With a thin buffer it re-prunes every few steps; after an MD run its
    forces must equal those of an engine whose list was just built at the
    same positions (every pair inside the cutoff present in both)."""
    s = case("propanol_cells")
    md = _md(s, kind="nve")
    monkeypatch.setenv("PGK_PRUNE_BUFFER", "0.3")
    e1 = engine(s, abi.PREC_MIXED)
    e1.moldyn_nve(0, 40, md)
    x, v, _ = e1.download_state()
    f1, en1, _ = e1.calforce(abi.MTS_LONG)
    monkeypatch.setenv("PGK_PRUNE_BUFFER", "0")
    e2 = engine(s, abi.PREC_MIXED)
    e2.upload_state(x, v)
    e2.mklist_cell()
    f2, en2, _ = e2.calforce(abi.MTS_LONG)
    assert rel_rms(f1, f2) < 1e-6
    assert erel(en1["pot_nonbon"], en2["pot_nonbon"]) < 1e-6


# ------------------------------------------------------------ cluster frame ---
def test_mixed_cluster_frame_matches_per_pair_image(monkeypatch):
    """Boxes wide enough for the cluster frame (here 93.6 A, 70k atoms): the
    pair kernel takes displacements as FP32 offsets from each cluster's first
    atom and the tensor-only virial from the atom forces.  Anisotropic MTK
    steps (tensor-only between outputs) must match the per-pair minimum-image
    kernel to FP32 rounding and track the FP64 device path."""
    s = S.propanol_box(nside=18, box=93.6)
    md = _md(s, kind="mtk", pext_pa=1.0e5, axis=abi.PCONT_ANISO)
    res = {}
    for tag, prec, frame in (("frame", abi.PREC_MIXED, "1"), ("pair", abi.PREC_MIXED, "0"), ("fp64", abi.PREC_FP64, "1")):
        monkeypatch.setenv("PGK_PAIR_FRAME", frame)
        e = engine(s, prec)
        e.set_chain(abi.chain_init(s.box))
        en = e.moldyn_mtk(0, 4, md)
        x, _, b = e.download_state()
        res[tag] = (x, b, en["pot_tot"], np.array(e.get_chain().vboxg[:]))
        e.close()
    xf, bf, pf, vf = res["frame"]
    xp, bp, pp, vp = res["pair"]
    x6, b6, p6, v6 = res["fp64"]
    assert np.abs(xf - xp).max() < 1e-5
    assert np.abs(bf - bp).max() < 1e-9 * np.abs(bp).max()
    assert erel(pf, pp) < 1e-6 * max(1.0, abs(pp))
    assert np.abs(vf - vp).max() < 1e-2 * max(np.abs(v6).max(), 1e-12)      # barostat velocity: the virial
    assert np.abs(xf - x6).max() < 1e-4
    assert erel(pf, p6) < 1e-5 * max(1.0, abs(p6))
