"""CPU checks of the FP64 oracle (known-answer and invariance tests restated
from the reference's test strategy) and of the committed golden vectors."""

import os

import numpy as np
import pytest
import scipy.sparse as sp

from gpusim2grid_b200.synthetic import build_ybus, n1_branches
from oracle import nr_oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden", "case118_golden.npz")


def test_jacobian_matches_finite_differences(g118):
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    pvpq, pq_, d = O.j_layout(g118.n_bus, pv, pq)
    rng = np.random.default_rng(0)
    V = np.abs(V0) * (1 + 0.02 * rng.standard_normal(g118.n_bus)) * np.exp(1j * 0.05 * rng.standard_normal(g118.n_bus))
    J = O.jacobian(Y, V, pvpq, pq_).toarray()
    F0 = O.mismatch(Y, V, S, pvpq, pq_)
    h = 1e-7
    for col in rng.choice(d, 12, replace=False):
        dx = np.zeros(d)
        dx[col] = h
        F1 = O.mismatch(Y, O.update_v(V, dx, pvpq, pq_), S, pvpq, pq_)
        # F = -mismatch, so dF/dx = -J
        np.testing.assert_allclose(-(F1 - F0) / h, J[:, col], atol=2e-4 * max(1, np.abs(J[:, col]).max()))


def test_branch_trip_equals_rebuilt_ybus(g118):
    rows = n1_branches(g118)[:5]
    for b in rows:
        Yt = O.trip_branches(g118.Ybus, [b, b], g118.branch_from, g118.branch_to,
                             g118.yff, g118.yft, g118.ytf, g118.ytt)
        keep = np.ones(g118.n_branch, dtype=bool)
        keep[b] = False
        *_, Yr = build_ybus(g118.n_bus, g118.branch_from[keep], g118.branch_to[keep], g118.r[keep],
                            g118.x[keep], g118.b[keep], g118.tap[keep])
        np.testing.assert_allclose((Yt - Yr).toarray(), 0, atol=1e-9)


def test_base_solve_power_balance(g118):
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    V, st, it, res = O.nr_solve(Y, V0, S, pv, pq, 10, 1e-8)
    assert st == O.CONVERGED and 2 <= it <= 10 and res < 1e-8
    Sc = V * np.conj(Y @ V)   # independent recompute of the injections
    mism = Sc - S
    assert np.abs(mism.real[np.concatenate([pv, pq])]).max() < 1e-8
    assert np.abs(mism.imag[pq]).max() < 1e-8
    # one iteration is not converged (reference test_base_case.py:52-107)
    _, st1, _, _ = O.nr_solve(Y, V0, S, pv, pq, 1, 1e-8)
    assert st1 == O.MAX_ITER


def test_nan_injection_diverges(g118):
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    S = S.copy()
    S[pq[0]] = np.nan
    _, st, _, res = O.nr_solve(Y, V0, S, pv, pq, 10, 1e-8)
    assert st == O.DIVERGED and np.isnan(res)


def test_islanding_detected(g118):
    bridges = np.setdiff1d(np.arange(g118.n_branch), n1_branches(g118))
    assert bridges.size > 0
    assert O.islands(g118.n_bus, g118.branch_from, g118.branch_to, [int(bridges[0])])
    assert not O.islands(g118.n_bus, g118.branch_from, g118.branch_to, [int(n1_branches(g118)[0])])


def test_golden_vectors_reproduce(g118):
    gd = np.load(GOLD)
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    Vb, st, it, _ = O.nr_solve(Y, V0, S, pv, pq, 10, 1e-8, mode="single")
    np.testing.assert_allclose(Vb, gd["V_base"], atol=1e-12)
    assert it == int(gd["base_iters"])
    ptr, ids = gd["ctg_ptr"], gd["ctg_ids"]
    ctg = [list(ids[ptr[r]:ptr[r + 1]]) for r in range(len(ptr) - 1)]
    Vc, sc, ic, _ = O.contingency_sweep(Y, V0, S, pv, pq, ctg[:6] + ctg[-2:], g118.branch_from,
                                        g118.branch_to, g118.yff, g118.yft, g118.ytf, g118.ytt, 10, 1e-8)
    sel = list(range(6)) + [len(ctg) - 2, len(ctg) - 1]
    np.testing.assert_allclose(np.nan_to_num(Vc), np.nan_to_num(gd["V_ctg"][sel]), atol=1e-12)
    np.testing.assert_array_equal(sc, gd["status_ctg"][sel])
    np.testing.assert_array_equal(ic, gd["iters_ctg"][sel])
    assert gd["status_ctg"][-2] == O.NOT_SIMULATED


def test_fixed_mode_runs_exact_steps(g118):
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    Vb, _, _, _ = O.nr_solve(Y, V0, S, pv, pq, 10, 1e-8)
    V, st, it, res = O.nr_solve(Y, Vb, S, pv, pq, 4, 1e-8, mode="fixed")
    assert it == 4 and st == O.CONVERGED and res < 1e-8


def test_branch_flows_balance_every_bus(g118):
    """At a converged solution the flows leaving every bus through its
    branches add up to the bus injection V conj(Y V) (the branches' pi models
    are the whole Ybus of the synthetic grids)."""
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    V, st, _, _ = O.nr_solve(Y, V0, S, pv, pq, 10, 1e-10)
    assert st == O.CONVERGED
    Sf, St = O.branch_flows(V, g118.branch_from, g118.branch_to, g118.yff, g118.yft, g118.ytf, g118.ytt)
    out = np.zeros(g118.n_bus, dtype=np.complex128)
    np.add.at(out, g118.branch_from, Sf)
    np.add.at(out, g118.branch_to, St)
    np.testing.assert_allclose(out, V * np.conj(Y @ V), atol=1e-10)
    # loading: unlimited and tripped branches load 0
    rate = np.abs(Sf) * 2
    rate[:3] = 0
    ld = O.branch_loading(V, g118.branch_from, g118.branch_to, g118.yff, g118.yft, g118.ytf, g118.ytt, rate,
                          tripped=[5])
    assert np.all(ld[:3] == 0) and ld[5] == 0
    np.testing.assert_allclose(ld[6:], np.maximum(np.abs(Sf), np.abs(St))[6:] / rate[6:])


def test_schedules_count_steps_as_the_reference(g118):
    """The three schedules on one solve: the single-solve order takes one
    step past the first passing test (acpf_nr.cu:505-561); rounds of k steps
    end on a multiple of k (batch_pf_driver.cu:2691-2724); a row that starts
    converged still runs its first round."""
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    Vc, st_c, it_c, _ = O.nr_solve(Y, V0, S, pv, pq, 10, 1e-8)
    Vs, st_s, it_s, res_s = O.nr_solve(Y, V0, S, pv, pq, 10, 1e-8, mode="single")
    assert st_c == st_s == O.CONVERGED and it_s == it_c + 1 and res_s < 1e-8
    pvpq, pq_, _ = O.j_layout(g118.n_bus, pv, pq)
    # the single solve's V is the continuous one's plus one more Newton step
    V1 = O.newton_step(Y, Vc, O.mismatch(Y, Vc, S, pvpq, pq_), pvpq, pq_)
    np.testing.assert_allclose(Vs, V1, atol=1e-13)
    for k in (2, 3, 4):
        _, st, it, res = O.nr_solve(Y, V0, S, pv, pq, 10, 1e-8, k=k)
        assert st == O.CONVERGED and it % k == 0 and it - k < it_c <= it and res < 1e-8
    # budget: MAX_ITER at the first round end at or past max_iter
    _, st, it, _ = O.nr_solve(Y, V0, S, pv, pq, 2, 1e-8, k=3)
    assert st == O.MAX_ITER and it == 3
    # a converged start still runs one round
    _, st, it, _ = O.nr_solve(Y, Vc, S, pv, pq, 10, 1e-8, k=2)
    assert st == O.CONVERGED and it == 2
    # NaN injections: DIVERGED at the end of the first round
    Sn = S.copy()
    Sn[pq[0]] = np.nan
    _, st, it, _ = O.nr_solve(Y, V0, Sn, pv, pq, 10, 1e-8, k=3)
    assert st == O.DIVERGED and it == 3
    _, st, it, _ = O.nr_solve(Y, V0, Sn, pv, pq, 4, 1e-8, mode="fixed")
    assert st == O.DIVERGED and it == 4
    _, st, it, _ = O.nr_solve(Y, V0, Sn, pv, pq, 4, 1e-8, mode="single")
    assert st == O.DIVERGED and it == 4


def test_half_open_branch_trips_only_its_live_end(g118):
    """A branch whose to-end is open (endpoint -1) contributes only its
    from-end self term; tripping it removes that term alone and joins no two
    buses in the islanding test (contingency_analysis_helper.cpp:53-75)."""
    from gpusim2grid_b200.synthetic import half_open_variant
    h = half_open_variant(g118, n_open=2, seed=0)
    l = int(h.open_branches[0])
    assert h.branch_to[l] == -1 and h.branch_from[l] >= 0
    Y, V0, S, _, _, pv, pq = h.as_tuple()
    Yt = O.trip_branches(Y, [l], h.branch_from, h.branch_to, h.yff, h.yft, h.ytf, h.ytt)
    d = (Y - Yt).tocoo()
    nz = np.abs(d.data) > 0
    assert list(zip(d.row[nz], d.col[nz])) == [(h.branch_from[l], h.branch_from[l])]
    np.testing.assert_allclose(d.data[nz], [h.yff[l]])
    assert not O.islands(h.n_bus, h.branch_from, h.branch_to, [l])
    # flows: the open end carries nothing, the live end its charging
    V, st, _, _ = O.nr_solve(Y, V0, S, pv, pq, 10, 1e-10)
    assert st == O.CONVERGED
    Sf, St = O.branch_flows(V, h.branch_from, h.branch_to, h.yff, h.yft, h.ytf, h.ytt)
    assert St[l] == 0
    f = h.branch_from[l]
    np.testing.assert_allclose(Sf[l], V[f] * np.conj(h.yff[l] * V[f]))


def test_disconnected_rows_solve_their_largest_component(g118):
    """handle_disconnected: a bridge outage solves the main component (power
    balance holds on its buses), masks the rest as NaN, and a split that
    strands the slack stays NOT_SIMULATED."""
    bridges = np.setdiff1d(np.arange(g118.n_branch), n1_branches(g118))
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    rows = [[int(b)] for b in bridges]
    V, st, it, res = O.contingency_sweep(Y, V0, S, pv, pq, rows, g118.branch_from, g118.branch_to, g118.yff,
                                         g118.yft, g118.ytf, g118.ytt, 10, 1e-8, handle_disconnected=True)
    solved = st == O.CONVERGED
    assert solved.sum() >= 1
    for r in np.flatnonzero(solved):
        live = O.main_component(g118.n_bus, g118.branch_from, g118.branch_to, rows[r])
        assert g118.slack in np.flatnonzero(live) and live.sum() >= g118.n_bus / 2
        assert np.all(np.isnan(V[r][~live])) and np.all(np.isfinite(V[r][live]))
        Yr = O.trip_branches(Y, rows[r], g118.branch_from, g118.branch_to, g118.yff, g118.yft, g118.ytf, g118.ytt)
        Vz = np.where(live, V[r], 0)
        mis = Vz * np.conj(Yr @ Vz) - S
        pvpq = np.concatenate([pv, pq])
        assert np.abs(mis.real[pvpq[live[pvpq]]]).max() < 1e-8 and np.abs(mis.imag[pq[live[pq]]]).max() < 1e-8
    for r in np.flatnonzero(~solved):
        live = O.main_component(g118.n_bus, g118.branch_from, g118.branch_to, rows[r])
        assert not live[g118.slack] and st[r] == O.NOT_SIMULATED


def test_step_scaling_restates_max_voltage_change(g118):
    """The MaxVoltageChange scaling (acpf_nr_kernels.cu:677-726): the whole
    step times min(1, max_dVa / max|dtheta|, max_dVm / max|dVm|), applied only
    when a bound is exceeded; damped solves reach the same solution in more
    steps."""
    dx = np.array([0.3, -0.05, 0.02, -0.2])  # two angles, then two magnitudes
    np.testing.assert_array_equal(O.step_scale(dx, 2, 0.5, 0.25), dx)
    np.testing.assert_allclose(O.step_scale(dx, 2, 0.1, 0.25), dx * (0.1 / 0.3))
    np.testing.assert_allclose(O.step_scale(dx, 2, 0.5, 0.05), dx * (0.05 / 0.2))
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    V1, st1, it1, _ = O.nr_solve(Y, V0, S, pv, pq, 20, 1e-10)
    V2, st2, it2, _ = O.nr_solve(Y, V0, S, pv, pq, 20, 1e-10, scaling=(0.1, 0.03))
    assert st1 == st2 == O.CONVERGED and it2 > it1
    assert np.abs(V1 - V2).max() < 1e-9
