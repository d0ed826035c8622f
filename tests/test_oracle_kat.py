"""Known-answer checks that pin the FP64 CPU oracle (no GPU).

The reference has no tests and its Fortran cannot be compiled here.  Its
recorded Pt/Morse run pins every energy and virial term
(tests/test_golden_pt_morse.py); these analytical answers pin what a recorded
energy cannot show: FFT vs a direct DFT, B-spline partition of unity, spline
tables vs erfc/erf, the Madelung constant of rock salt, LJ two-body values,
finite-difference forces, constraint residuals and energy conservation.
"""
import math

import numpy as np
import pytest

from tests.conftest import rel_rms
from thrid_b200 import abi
from thrid_b200 import systems as S


@pytest.mark.parametrize("n", [8, 12, 30, 32, 45, 64, 128, 192, 240])
def test_fft_matches_direct_dft(oracle_mod, n):
    rng = np.random.default_rng(n)
    x = rng.normal(size=n) + 1j * rng.normal(size=n)
    k = np.arange(n)
    W = np.exp(-2j * np.pi * np.outer(k, k) / n)
    assert np.abs(oracle_mod.fft1d(x, -1) - W @ x).max() < 1e-11 * n
    assert np.abs(oracle_mod.fft1d(x, +1) - np.conj(W) @ x).max() < 1e-11 * n


@pytest.mark.parametrize("order", [3, 4, 5, 6, 7, 8])
def test_bspline_partition_of_unity(oracle_mod, order):
    for w in np.linspace(0.0, 0.999, 37):
        th, dth = oracle_mod.fill_bspline(w, order)
        assert abs(th.sum() - 1.0) < 1e-14
        assert abs(dth.sum()) < 1e-14
        assert (th >= -1e-16).all()
    # derivative consistency: d theta / dw by central difference
    h = 1e-6
    a, da = oracle_mod.fill_bspline(0.37, order)
    p, _ = oracle_mod.fill_bspline(0.37 + h, order)
    m, _ = oracle_mod.fill_bspline(0.37 - h, order)
    assert np.abs((p - m) / (2 * h) - da).max() < 1e-8


def test_spline_tables_match_erfc(oracle_mod):
    s = S.water_box()
    o = oracle_mod.Oracle(s)
    a = s.params["alpha"]
    pe = 2 * a / math.sqrt(math.pi)
    for r in np.linspace(1.0, s.params["rrcut"], 400):
        ec = math.erfc(a * r)
        assert abs(o.spline(1, r) - ec / r) < 2e-9
        assert abs(o.spline(0, r) - (pe * math.exp(-a * a * r * r) / r + ec / r / r) / r) < 2e-8
        assert abs(o.spline(3, r) - (1 - ec) / r) < 2e-9
        assert abs(o.spline(2, r) - (-pe * math.exp(-a * a * r * r) / r + (1 - ec) / r / r) / r) < 2e-8
    # beyond the table the reference returns 0 (spline_interp.F90:218)
    assert o.spline(1, 1e3) == 0.0


def test_madelung_constant_rock_salt(oracle_mod):
    s = S.nacl_lattice()
    o = oracle_mod.Oracle(s)
    o.mklist()
    f1, e1, _ = o.ewaldrp()
    f2, e2, _ = o.fft_pmep()
    E = e1["pot_elc"] + e2["pot_ewk"] + o.pot_ewc
    M = -E / (s.natom / 2) * 2.82 / S.CHARGE_SCALE ** 2
    assert abs(M - 1.747564594633) < 2e-5
    assert np.abs(f1 + f2).max() < 1e-8          # perfect lattice: no net force


def test_lj_two_body(oracle_mod):
    s = S.small_box("water", nside=2, spacing=9.0)
    # keep two oxygens only interacting: zero all charges
    s.atmchrg[:] = 0.0
    o = oracle_mod.Oracle(s)
    cor = s.atmcor.copy()
    o.mklist()
    f, e, v = o.ewaldrp()
    # direct double loop over O-O pairs with min image, cutoff rcut
    R = s.vdw_radij[0, 0]
    E = s.vdw_welij[0, 0]
    oxy = np.where(s.atmindex == 1)[0]
    L = s.box
    tot = 0.0
    for a in range(len(oxy)):
        for b in range(a + 1, len(oxy)):
            d = cor[oxy[a]] - cor[oxy[b]]
            d -= L * np.round(d / L)
            r = np.linalg.norm(d)
            if r * r <= s.params["rcut"] ** 2:
                tot += E * ((R / r) ** 12 - 2 * (R / r) ** 6)
    assert abs(e["pot_vdw"] - tot) < 1e-10 * max(1.0, abs(tot))


def _etot(o, x):
    o.set_state(x)
    f, e, v = o.calforce(abi.MTS_LONG)
    return e["pot_tot"], f


def test_finite_difference_forces(oracle_mod):
    s = S.small_box("propanol", nside=3, spacing=5.6)
    p = dict(s.params)
    o = oracle_mod.Oracle(s, p)
    o.mklist()
    x0 = s.atmcor.copy()
    E0, F = _etot(o, x0)
    h = 1e-5
    rng = np.random.default_rng(3)
    worst = 0.0
    for a in rng.choice(s.natom, 8, replace=False):
        for d in range(3):
            xp = x0.copy(); xp[a, d] += h
            xm = x0.copy(); xm[a, d] -= h
            Ep, _ = _etot(o, xp)
            Em, _ = _etot(o, xm)
            fd = -(Ep - Em) / (2 * h)
            worst = max(worst, abs(fd - F[a, d]) / max(1.0, abs(F[a, d])))
    assert worst < 2e-4


def test_cell_and_allpair_lists_share_the_pair_set(oracle_mod):
    s = S.propanol_box(nside=11, box=57.2)
    p = dict(s.params)
    sets = []
    for mode in (abi.LIST_CELL, abi.LIST_ALLPAIR):
        p["list_mode"] = mode
        o = oracle_mod.Oracle(s, p)
        m, idx, lst = o.mklist()
        assert m == mode
        pairs = set()
        for i in range(s.natom - 1):
            row = lst[idx[i] - 1: idx[i + 1] - 1]
            pairs.update((i + 1, int(j)) for j in row if j)
        sets.append(pairs)
    assert sets[0] == sets[1]
    assert len(sets[0]) > 1_000_000


def test_rattle_satisfies_constraints(oracle_mod):
    s = S.water_box()
    o = oracle_mod.Oracle(s)
    dt = S.fs_to_reduced(1.0)
    old = s.atmcor.copy()
    new = old + dt * s.atmvel
    o.set_state(new, s.atmvel)
    assert o.rattle_c(old, 1e-7, dt) == 0
    cor, vel, _ = o.get_state()
    ij = s.const_ij
    r2 = ((cor[ij[:, 0]] - cor[ij[:, 1]]) ** 2).sum(1)
    assert (np.abs(r2 - s.const_d ** 2) / s.const_d ** 2).max() < 1e-7
    assert o.rattlep_v(1e-7) == 0
    cor, vel, _ = o.get_state()
    rv = ((cor[ij[:, 0]] - cor[ij[:, 1]]) * (vel[ij[:, 0]] - vel[ij[:, 1]])).sum(1)
    assert np.abs(rv).max() < 1e-5


def test_rattle_reports_nonconvergence(oracle_mod):
    s = S.water_box()
    o = oracle_mod.Oracle(s)
    dt = S.fs_to_reduced(1.0)
    old = s.atmcor.copy()
    o.set_state(old + dt * s.atmvel, s.atmvel)
    # eps = 0 can never be met: the bounded loop must give up with a status
    assert o.rattle_c(old, 0.0, dt) == abi.PGK_E_RATTLE_NOCONV


def _md(dt_fs, nstep_short=1, **kw):
    return abi.md_struct(S.fs_to_reduced(dt_fs), nstep_short=nstep_short, **kw)


def test_nve_energy_conservation_water(oracle_mod):
    s = S.water_box()
    o = oracle_mod.Oracle(s)
    md = _md(1.0, ifrattle=1, eps_rattle=1e-9, outinterval=1)
    # the lattice start's velocities are projected onto the constraints by the
    # first RATTLE(V); measure from step 2 on
    st, e0 = o.moldyn(0, 0, 2, md)
    assert st == 0
    k0 = 0.5 * o.kint()
    h0 = k0 + e0["pot_tot"]
    st, e1 = o.moldyn(0, 3, 60, md)
    assert st == 0
    h1 = 0.5 * o.kint() + e1["pot_tot"]
    # rigid water at 1 fs from a lattice start: drift well under 1 % of KE
    assert abs(h1 - h0) < 0.01 * k0


def test_nhc_extended_energy_is_conserved(oracle_mod):
    s = S.small_box("propanol", nside=3, spacing=5.6)
    o = oracle_mod.Oracle(s)
    T = S.kelvin_to_reduced(300.0)
    tfreq = 1.0e13 * S.TIMEREF
    md = _md(0.5, mchain=3, text=T, tfreq=tfreq, degfree=s.degfree_all, ifrattle=1, eps_rattle=1e-10,
             outinterval=1)

    def H(e):
        ch = o.get_chain()
        q = md.qmass
        ext = sum(0.5 * q[i] * ch.vlogs[i] ** 2 for i in range(md.mchain))
        ext += s.degfree_all * T * ch.xlogs[0] + T * sum(ch.xlogs[i] for i in range(1, md.mchain))
        return 0.5 * o.kint() + e["pot_tot"] + ext

    st, e0 = o.moldyn(1, 0, 2, md)
    assert st == 0
    h0 = H(e0)
    st, e1 = o.moldyn(1, 3, 40, md)
    assert st == 0
    ch = o.get_chain()
    assert abs(ch.vlogs[0]) > 0          # the thermostat is active
    assert abs(H(e1) - h0) < 0.02 * 0.5 * o.kint()
