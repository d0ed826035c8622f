"""Parity of the oracle against the reference's own recorded run.

tests/golden/pt_morse_step1.npz holds the reference's Pt/Morse sample (10
1-propanol + 190 butane on a 3,584-atom Pt slab, 6,364 atoms, peachgk.ini):
its topology and parameters as the reference's input processing produces
them, the step-1 positions and velocities of its state record
(sta_peachgk-2.0.dat, E24.16; the same configuration as its single-precision
out_pos.dat / out_vel.dat), and what it printed for that step: every energy
term (out_ene.dat) and every virial and the virial tensor (out_pre.dat), in
E15.8.  The script beside the fixture (make_pt_morse_fixture.py) made it from
the reference tree.

The oracle evaluates both MTS groups (calforce.F90) at the recorded state and
each term must equal the printed value to within half a unit of its 8th
printed digit -- the whole precision the record carries.
"""
import math
import os

import numpy as np
import pytest

from thrid_b200 import abi
from thrid_b200 import systems as S

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "pt_morse_step1.npz")

TERMS = ("pot_mor", "pot_vdw", "pot_elc", "pot_ewk", "pot_ewc", "pot_vdw14", "pot_elc14", "pot_bond",
         "pot_angl", "pot_tors", "pot_torsrb", "pot_tot")


def printed(rec_joule, got_reduced, eref, slack=1.2):
    """True when got (reduced) matches a value printed as E15.8 [J] to within
    half a unit of its 8th digit (slack covers the oracle's own summation order)."""
    e = math.floor(math.log10(abs(rec_joule))) + 1          # 0.dddddddd x 10^e
    return abs(got_reduced * eref - rec_joule) <= slack * 0.5 * 10.0 ** (e - 8)


def load_pt_morse(precision=abi.PREC_FP64):
    z = np.load(FIX)
    p = dict(zip((str(k) for k in z["params_keys"]), (float(v) for v in z["params_vals"])))
    box = np.array([p["xcel"], p["ycel"], p["zcel"]])
    params = S.default_params(box, p["rcut"], p["rrcut"], p["alpha"],
                              (int(p["nfft1"]), int(p["nfft2"]), int(p["nfft3"])), int(p["pme_order"]),
                              rcut_book=p["rcut_book"], precision=precision)
    params.update(nspltbl=int(p["nspltbl"]), ifnetqcorrp=int(p["ifnetqcorrp"]), rcutmor=p["rcutmor"],
                  rcut_bookmor=p["rcut_bookmor"], mts_mor=S.MTS_LONG,
                  mts_bond=S.MTS_SHORT, mts_angl=S.MTS_SHORT, mts_tors=S.MTS_SHORT, mts_torsrb=S.MTS_SHORT)
    tix = z["atmindex"]
    natom = len(tix)
    sizes = z["mol_sizes"]
    molidx = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    iex, lex = S._mkexcl(natom, z["bonds"], z["angles"], z["tors"], z["torsrb"])
    s = S.System(
        name="pt_morse_6364", natom=natom, box=box,
        atmcor=z["pos_m"].astype(np.float64) / float(z["xref"]),
        atmvel=z["vel_ms"].astype(np.float64) / float(z["vref"]),
        atmmass=z["mass_t"][tix - 1], atmchrg=z["chrg_t"][tix - 1], atmindex=tix,
        type_names=[str(t) for t in z["type_names"]],
        vdw_radij=z["vdw_radij"], vdw_welij=z["vdw_welij"],
        molept_index=molidx, molept_list=np.arange(natom, dtype=np.int32),
        index_excl=iex, list_excl=lex,
        bonds=z["bonds"], bond_k=z["bond_k"], bond_r0=z["bond_r0"],
        angles=z["angles"], angl_k=z["angl_k"], angl_t0=z["angl_t0"],
        tors=z["tors"], tors_divfac=z["tors_divfac"], tors_barhig=z["tors_barhig"],
        tors_phsang=z["tors_phsang"], tors_period=z["tors_period"], tors_14=z["tors_14"],
        tors_dvdw=z["tors_dvdw"], tors_delc=z["tors_delc"], tors_ring=z["tors_ring"],
        torsrb=z["torsrb"], torsrb_c=z["torsrb_c"], torsrb_14=z["torsrb_14"],
        torsrb_dvdw=z["torsrb_dvdw"], torsrb_delc=z["torsrb_delc"], torsrb_ring=z["torsrb_ring"],
        const_index=np.zeros(1, np.int32), const_list=np.zeros(0, np.int32),
        const_ij=np.zeros((0, 2), np.int32), const_d=np.zeros(0),
        degfree_all=3 * natom, params=params,
        inttyp=z["inttyp"], mor_wel=z["mor_wel"], mor_rad=z["mor_rad"], mor_alpha=z["mor_alpha"])
    want = {str(k): float(v) for k, v in zip(z["ene_keys"], z["ene_joule"])}           # [J], as printed
    want.update({str(k): float(v) for k, v in zip(z["pre_keys"], z["pre_joule"])})
    want["eref"] = float(z["eref"])
    return s, want


def oracle_energies(oracle_mod, s, virials=False):
    o = oracle_mod.Oracle(s, threads=os.cpu_count() or 1)
    o.mklist()
    _, el, vl = o.calforce(abi.MTS_LONG)
    _, es, vs = o.calforce(abi.MTS_SHORT)
    e = {k: el[k] + es[k] for k in el}
    if not virials:
        return e
    return e, {k: np.asarray(vl[k]) + np.asarray(vs[k]) for k in vl}


@pytest.fixture(scope="module")
def pt_morse(oracle_mod):
    s, want = load_pt_morse()
    e, v = oracle_energies(oracle_mod, s, virials=True)
    return s, want, e, v


def test_fixture_shape(pt_morse):
    s, want, _, _ = pt_morse
    assert s.natom == 6364 and len(s.bonds) == 2580 and len(s.angles) == 4750
    assert len(s.tors) == 210 and len(s.torsrb) == 5130
    # the reference's ring14_rb reset covers only the first ntors RB torsions
    assert s.torsrb_ring[:210].min() == 1.0 and s.torsrb_ring[210:].max() == 0.0


@pytest.mark.parametrize("term", TERMS)
def test_oracle_matches_recorded_energy(pt_morse, term):
    _, want, got, _ = pt_morse
    assert printed(want[term], got[term], want["eref"]), (term, got[term] * want["eref"], want[term])


# recorded virial (calpress.F90 outputs) -> the oracle's terms
VIR = {"pot_virilj_all": ("pot_viri_lj",), "pot_virimor_all": ("pot_viri_mor",),
       "atm_viribo_all": ("atm_viri_bond",), "atm_viri14_all": ("atm_viri_14",)}


@pytest.mark.parametrize("term", sorted(VIR))
def test_oracle_matches_recorded_virial(pt_morse, term):
    _, want, _, vir = pt_morse
    g = sum(float(vir[k]) for k in VIR[term])
    assert printed(want[term], g, want["eref"]), (term, g * want["eref"], want[term])


def test_oracle_matches_recorded_coulomb_virial_and_tensor(pt_morse):
    _, want, e, vir = pt_morse
    # pot_viric_all: real-space + SPME virial with the self and net-charge terms
    g = float(vir["pot_viri_coul"]) + e["pot_ewc"] + e["pot_ewnq"]
    assert printed(want["pot_viric_all"], g, want["eref"])
    # angle and torsion forces carry no scalar virial (recorded ~1e-32 J)
    assert abs(float(vir["atm_viri_angl"])) * want["eref"] < 1e-30
    assert abs(float(vir["atm_viri_tors"])) * want["eref"] < 1e-30
    # preatmt_vtot: the virial tensor of every term, entry by entry
    tens = sum(vir[k] for k in ("pot_virit_coul", "pot_virit_lj", "pot_virit_mor", "atm_virit_bond",
                                "atm_virit_angl", "atm_virit_tors", "atm_virit_14")).reshape(3, 3).T
    for i in range(3):
        for j in range(3):
            assert printed(want[f"preatmt_vtot{i + 1}{j + 1}"], tens[i, j], want["eref"]), (i, j)


def test_oracle_kinetic_energy_matches_recorded(oracle_mod):
    """ene_kin of out_ene.dat = half the oracle's sum m v^2 (calkin) over the
    recorded velocities: pins the mass and velocity units (rdpara.F90:461,
    calbase.F90:66)."""
    s, want = load_pt_morse()
    o = oracle_mod.Oracle(s)
    assert printed(want["ene_kin"], 0.5 * o.kint(), want["eref"])


def test_ring14_rb_reset_is_what_the_reference_ran(oracle_mod):
    """With every ring14_rb = 1 the 1-4 energies miss the recorded ones by
    factors of 9 (vdW) and 6 (Coulomb): the recorded run used the partial
    reset of rdtop.F90:378."""
    s, want = load_pt_morse()
    s.torsrb_ring = np.ones_like(s.torsrb_ring)
    got = oracle_energies(oracle_mod, s)
    for k in ("pot_vdw14", "pot_elc14"):
        assert abs(got[k] * want["eref"] - want[k]) > 5.0 * abs(want[k])


def test_engine_accepts_morse_pair_types():
    """Morse type pairs (inter_inttyp 2) pass pgk_init's input checks (the
    device evaluates them, k_morse.cu); a Morse pair type without Morse
    parameters is invalid.  Without a GPU the call ends at the device check."""
    import ctypes as C
    from thrid_b200 import pgk
    L = pgk.lib()

    def init(s):
        cs = abi.CSystem(s)
        ps = abi.params_struct(s.params)
        h = C.c_void_p()
        st = L.pgk_init(C.byref(cs.struct), C.byref(ps), C.byref(h))
        if h.value:
            L.pgk_free(h)
        return st
    s, _ = load_pt_morse()
    assert init(s) in (abi.PGK_OK, abi.PGK_E_CUDA)
    s.mor_wel = None
    assert init(s) == abi.PGK_E_INVALID


def test_engine_input_checks_for_pair_types():
    """Morse switched off (mts_mor = none) is accepted up to the device check;
    pair potentials the engine does not build are refused before any device
    call; an out-of-range type code is invalid."""
    import ctypes as C
    from thrid_b200 import pgk
    L = pgk.lib()

    def init(s):
        cs = abi.CSystem(s)
        ps = abi.params_struct(s.params)
        h = C.c_void_p()
        st = L.pgk_init(C.byref(cs.struct), C.byref(ps), C.byref(h))
        if h.value:
            L.pgk_free(h)
        return st
    s, _ = load_pt_morse()
    for code, want in ((3, abi.PGK_E_UNSUPPORTED), (10, abi.PGK_E_UNSUPPORTED), (11, abi.PGK_E_INVALID)):
        s.inttyp = s.inttyp.copy()
        s.inttyp[0, 1] = s.inttyp[1, 0] = code
        assert init(s) == want
    s, _ = load_pt_morse()
    s.params["mts_mor"] = 0                                        # PGK_MTS_NONE: Morse switched off
    assert init(s) not in (abi.PGK_E_UNSUPPORTED, abi.PGK_E_INVALID)   # passes the pair-type checks


def test_morse_cell_list_matches_all_pairs(oracle_mod):
    """mklist_mor_cell and mklist2a_mor give the same Morse pairs: with
    rcut_bookmor 12 A the slab has 3 x 3 x 10 cells, so the cell scan runs
    (rdscript.F90:1616-1632); forcing the all-pairs order changes only the
    summation order.  The recorded run itself used all pairs (2 x 2 x 9
    cells at 14 A)."""
    s, want = load_pt_morse()
    o = oracle_mod.Oracle(s)
    o.mklist()
    assert o.mor_list()[0] == abi.LIST_ALLPAIR
    out = {}
    for mode in (abi.LIST_AUTO, abi.LIST_ALLPAIR):
        s2, _ = load_pt_morse()
        s2.params.update(rcut_bookmor=12.0, list_mode=mode)
        o = oracle_mod.Oracle(s2)
        o.mklist()
        _, e, _ = o.calforce(abi.MTS_LONG)
        out[mode] = (o.mor_list(), e["pot_mor"])
    (m_cell, n_cell), e_cell = out[abi.LIST_AUTO]
    (m_all, n_all), e_all = out[abi.LIST_ALLPAIR]
    assert m_cell == abi.LIST_CELL and m_all == abi.LIST_ALLPAIR and n_cell == n_all
    assert abs(e_cell - e_all) <= 1e-12 * abs(e_all)
    assert printed(want["pot_mor"], e_cell, want["eref"])


def test_morse_heat_flux_shares(pt_morse, oracle_mod):
    """morsep_hf (morse_hf.F90): half of each pair energy to either atom, so
    the shares sum to pot_mor; with one region over the whole box and every
    atom atom-based, the per-atom z column of the Morse virial sums to the
    (a, z) column of the Morse virial tensor (no Morse pair crosses the
    vacuum gap in z)."""
    s, want, e, vir = pt_morse
    o = oracle_mod.Oracle(s, threads=os.cpu_count() or 1)
    o.set_hf({"regions": [(0.0, s.box[2])], "hftyp": None})
    o.mklist()
    pot, W = o.morse_hf_atm()
    assert abs(pot.sum() - e["pot_mor"]) <= 1e-12 * abs(e["pot_mor"])
    assert printed(want["pot_mor"], pot.sum(), want["eref"])
    col = np.asarray(vir["pot_virit_mor"])[6:9]          # t[a + 3*2]: f_a z_ij
    np.testing.assert_allclose(W[0].sum(axis=1), col, rtol=1e-10, atol=1e-8 * np.abs(col).max())
