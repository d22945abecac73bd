"""GPU parity: the CUDA path (through the C-ABI, via the facades) against the
FP64 oracle and the committed golden vectors."""

import os

import numpy as np
import pytest

from conftest import TOL_V_FP64, TOL_V_MIXED
from gpusim2grid_b200 import (AcPfGPU, ContingencyAnalysisGPU, InjectionSweepGPU, RowStatus, ScenarioSweepGPU,
                              acpf_nr_gpu)
from gpusim2grid_b200.synthetic import injection_scenarios, n1_branches, scenario_outages
from oracle import nr_oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "case118_golden.npz")


@pytest.mark.parametrize("precision,tol_v", [("fp64", TOL_V_FP64), ("mixed", TOL_V_MIXED)])
def test_single_solve_vs_golden(g118, precision, tol_v):
    gd = np.load(GOLD)
    out = np.zeros(g118.n_bus, dtype=np.complex128)
    Y, V0, S, sl, w, pv, pq = g118.as_tuple()
    t = acpf_nr_gpu(out, Y, V0, S, sl, w, pv, pq, 10, 1e-8, 1, precision=precision)
    assert t.converged and t.residual < 1e-8
    assert t.nb_iter == int(gd["base_iters"])
    assert np.abs(out - gd["V_base"]).max() < tol_v
    ac = AcPfGPU(g118.as_tuple(), precision=precision, init_from_n_powerflow=False)
    assert np.abs(ac.solve() - gd["V_base"]).max() < tol_v
    # a second identical call is reproducible (reference test_base_case.py:23)
    t2 = ac.resolve(V0)
    assert t2.converged and np.abs(ac.solve() - gd["V_base"]).max() < tol_v


def test_init_from_n_powerflow_validates(g118):
    gd = np.load(GOLD)
    Y, V0, S, sl, w, pv, pq = g118.as_tuple()
    ac = AcPfGPU((Y, gd["V_base"], S, sl, w, pv, pq))
    np.testing.assert_array_equal(ac.solve(), gd["V_base"])
    with pytest.raises(RuntimeError):
        AcPfGPU(g118.as_tuple())  # the flat start is not a solution


@pytest.mark.parametrize("precision,tol_v", [("fp64", TOL_V_FP64), ("mixed", TOL_V_MIXED)])
def test_contingency_continuous_vs_golden(g118, precision, tol_v):
    gd = np.load(GOLD)
    ca = ContingencyAnalysisGPU(g118.as_tuple(), init_from_n_powerflow=False, precision=precision,
                                nb_iter=10, scheduling="continuous", tol=1e-8, start="flat")
    ca.set_branch_data(*g118.branch_data())
    ptr, ids = gd["ctg_ptr"], gd["ctg_ids"]
    ca.add_contingencies_by_branch_id([list(ids[ptr[r]:ptr[r + 1]]) for r in range(len(ptr) - 1)])
    cap = ca.compute()
    assert cap is not None
    V = ca.V_results
    st = ca.get_row_status()
    np.testing.assert_array_equal(st, gd["status_ctg"])
    np.testing.assert_array_equal(ca.get_row_iterations(), gd["iters_ctg"])
    ok = st != RowStatus.NOT_SIMULATED
    assert np.abs(V[ok] - gd["V_ctg"][ok]).max() < tol_v
    assert np.all(np.isnan(V[~ok]))
    assert np.all(ca.last_residuals()[ok] < 1e-8)


def test_contingency_chunked_vs_golden(g118):
    """The reference's default: every row runs exactly nb_iter=4 steps from
    the converged base case, then the residual is evaluated."""
    gd = np.load(GOLD)
    Y, V0, S, sl, w, pv, pq = g118.as_tuple()
    ca = ContingencyAnalysisGPU((Y, gd["V_base"], S, sl, w, pv, pq), nb_iter=4)
    ca.set_branch_data(*g118.branch_data())
    ptr, ids = gd["ctg_ptr"], gd["ctg_ids"]
    ca.add_contingencies_by_branch_id([list(ids[ptr[r]:ptr[r + 1]]) for r in range(len(ptr) - 1)])
    ca.compute()
    st = ca.get_row_status()
    np.testing.assert_array_equal(st, gd["status_chunked"])
    ok = st != RowStatus.NOT_SIMULATED
    assert np.abs(ca.V_results[ok] - gd["V_chunked"][ok]).max() < TOL_V_FP64
    assert np.all(ca.get_row_iterations()[ok] == 4)


@pytest.mark.parametrize("precision,tol_v", [("fp64", TOL_V_FP64), ("mixed", TOL_V_MIXED)])
def test_injection_sweep_vs_golden(g118, precision, tol_v):
    gd = np.load(GOLD)
    sw = InjectionSweepGPU(g118.as_tuple(), init_from_n_powerflow=False, precision=precision, nb_iter=10,
                           scheduling="continuous", start="flat")
    sw.set_injections(gd["p_mw"], gd["q_mvar"], g118.sn_mva)
    sw.compute()
    np.testing.assert_array_equal(sw.get_row_status(), gd["status_inj"])
    np.testing.assert_array_equal(sw.get_row_iterations(), gd["iters_inj"])
    assert np.abs(sw.V_results - gd["V_inj"]).max() < tol_v


def test_n1_sweep_2000_vs_oracle(g2000):
    """Full 2000-bus N-1 sweep on the GPU; a sample of rows against the oracle."""
    rows = n1_branches(g2000)
    ca = ContingencyAnalysisGPU(g2000.as_tuple(), init_from_n_powerflow=False, nb_iter=10,
                                scheduling="continuous", start="flat")
    ca.set_branch_data(*g2000.branch_data())
    ca.add_contingencies_by_branch_id([[int(b)] for b in rows])
    ca.compute()
    st, it, V = ca.get_row_status(), ca.get_row_iterations(), ca.V_results
    assert np.all(st == RowStatus.CONVERGED)
    sample = np.random.default_rng(0).choice(len(rows), 12, replace=False)
    Y, V0, S, _, _, pv, pq = g2000.as_tuple()
    Vo, so, io, _ = O.contingency_sweep(Y, V0, S, pv, pq, [[int(rows[r])] for r in sample], g2000.branch_from,
                                        g2000.branch_to, g2000.yff, g2000.yft, g2000.ytf, g2000.ytt, 10, 1e-8)
    np.testing.assert_array_equal(st[sample], so)
    np.testing.assert_array_equal(it[sample], io)
    assert np.abs(V[sample] - Vo).max() < TOL_V_FP64


def test_scenario_sweep_vs_oracle(g118):
    p, q = injection_scenarios(g118, 12, seed=7)
    topo = scenario_outages(g118, 12, max_trips=2, seed=8)
    sw = ScenarioSweepGPU(g118.as_tuple(), init_from_n_powerflow=False, nb_iter=10, scheduling="continuous",
                          start="flat")
    sw.set_branch_data(*g118.branch_data())
    sw.set_injections(p, q, g118.sn_mva)
    sw.set_topology(topo)
    sw.compute()
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    for r in range(12):
        Yr = O.trip_branches(Y, topo[r], g118.branch_from, g118.branch_to, g118.yff, g118.yft, g118.ytf, g118.ytt)
        Vo, so, io, _ = O.nr_solve(Yr, V0, (p[r] + 1j * q[r]) / g118.sn_mva, pv, pq, 10, 1e-8)
        assert sw.get_row_status()[r] == so and sw.get_row_iterations()[r] == io
        assert np.abs(sw.V_results[r] - Vo).max() < TOL_V_FP64
    assert not sw.get_disconnected().any()


@pytest.mark.parametrize("precision,tol_v", [("fp64", TOL_V_FP64), ("mixed", TOL_V_MIXED)])
def test_rounds_of_k_steps_vs_golden(g118, precision, tol_v):
    """nb_iter_per_round = 3: rows are tested every third step only, so every
    row runs a multiple of 3 steps (reference batch_pf_driver.cu:2691-2724)."""
    gd = np.load(GOLD)
    ca = ContingencyAnalysisGPU(g118.as_tuple(), init_from_n_powerflow=False, precision=precision,
                                nb_iter=10, scheduling="continuous", nb_iter_per_round=3, tol=1e-8, start="flat")
    ca.set_branch_data(*g118.branch_data())
    ptr, ids = gd["ctg_ptr"], gd["ctg_ids"]
    ca.add_contingencies_by_branch_id([list(ids[ptr[r]:ptr[r + 1]]) for r in range(len(ptr) - 1)])
    ca.compute()
    st = ca.get_row_status()
    np.testing.assert_array_equal(st, gd["status_k3"])
    np.testing.assert_array_equal(ca.get_row_iterations(), gd["iters_k3"])
    ok = st != RowStatus.NOT_SIMULATED
    assert np.all(ca.get_row_iterations()[ok] % 3 == 0)
    assert np.abs(ca.V_results[ok] - gd["V_k3"][ok]).max() < tol_v
    with pytest.raises(ValueError):
        ca.nb_iter_per_round = 0


@pytest.mark.parametrize("strategy", ["refactor_every", "base_chord"])
@pytest.mark.parametrize("precision,tol_v", [("fp64", TOL_V_FP64), ("mixed", TOL_V_MIXED)])
def test_rows_from_the_base_case_vs_golden(g118, precision, tol_v, strategy):
    """Rows started from the converged base case, the first tripping nothing:
    that row starts converged and still runs its first round (1 step), as
    every loaded row does in the reference's continuous schedule."""
    gd = np.load(GOLD)
    ca = ContingencyAnalysisGPU(g118.as_tuple(), init_from_n_powerflow=False, precision=precision,
                                nb_iter=10, scheduling="continuous", tol=1e-8, start="base", strategy=strategy)
    ca.set_branch_data(*g118.branch_data())
    ptr, ids = gd["ctg_ptr"], gd["ctg_ids"]
    ca.add_contingencies_by_branch_id([[]] + [list(ids[ptr[r]:ptr[r + 1]]) for r in range(8)])
    ca.compute()
    np.testing.assert_array_equal(ca.get_row_status(), gd["status_base_start"])
    it = ca.get_row_iterations()
    assert it[0] == 1
    if strategy == "refactor_every":
        np.testing.assert_array_equal(it, gd["iters_base_start"])
    assert np.abs(ca.V_results - gd["V_base_start"]).max() < tol_v
    assert np.all(ca.last_residuals() < 1e-8)


@pytest.mark.parametrize("strategy", ["refactor_every", "base_chord"])
def test_half_open_branches_vs_oracle(g118, strategy):
    """Two branches open at their to-end (endpoint -1): tripping one removes
    only its live end's self term and never islands the grid; its flow at the
    open end is 0 (reference contingency_analysis_helper.cpp:53-75,
    acpf_nr_kernels.cu:87-183)."""
    from gpusim2grid_b200.synthetic import half_open_variant
    h = half_open_variant(g118, n_open=2, seed=0)
    lo = [int(l) for l in h.open_branches]
    other = [int(l) for l in n1_branches(h)[:6] if int(l) not in lo]
    rows = [[lo[0]], [lo[1]], lo, [lo[0], other[0]]] + [[l] for l in other[1:5]]
    ca = ContingencyAnalysisGPU(h.as_tuple(), init_from_n_powerflow=False, nb_iter=10, scheduling="continuous",
                                tol=1e-8, start="flat", strategy=strategy)
    ca.set_branch_data(*h.branch_data())
    rate = np.full(h.n_branch, 200.0)
    ca.set_branch_limits(rate)
    ca.add_contingencies_by_branch_id(rows)
    ca.compute()
    Y, V0, S, _, _, pv, pq = h.as_tuple()
    Vo, so, io, _ = O.contingency_sweep(Y, V0, S, pv, pq, rows, h.branch_from, h.branch_to, h.yff, h.yft, h.ytf,
                                        h.ytt, 10, 1e-8)
    np.testing.assert_array_equal(ca.get_row_status(), so)
    assert np.all(so == RowStatus.CONVERGED)
    if strategy == "refactor_every":
        # plain Newton: the oracle's iterates, so its iteration counts and voltages to rounding
        np.testing.assert_array_equal(ca.get_row_iterations(), io)
        assert np.abs(ca.V_results - Vo).max() < TOL_V_FP64
    else:
        # chord / Broyden steps converge to the same solution along other iterates
        assert np.abs(ca.V_results - Vo).max() < TOL_V_MIXED
    loading, _, _ = ca.branch_loading()
    for r in range(len(rows)):
        ref = O.branch_loading(Vo[r], h.branch_from, h.branch_to, h.yff, h.yft, h.ytf, h.ytt, rate / h.sn_mva,
                               tripped=rows[r])
        np.testing.assert_allclose(loading[r], ref, rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("precision,tol_v", [("fp64", 1e-10), ("mixed", TOL_V_MIXED)])
def test_solutions_equal_the_references_own_dense_nr(g118, precision, tol_v):
    """The engine against voltages the reference's own Python wrote
    (tests/golden/make_reference_golden.py: the dense Newton-Raphson of its
    test_injection_batch.py, to 1e-10): load-scaled base cases through the
    injection sweep, N-1 rows through the contingency sweep, and the grid with
    half-open branches through a single solve."""
    ref = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_golden.npz"))
    Y, V0, S, sl, w, pv, pq = g118.as_tuple()
    sc = ref["scales"]
    P = np.outer(sc, S.real) * g118.sn_mva
    Q = np.outer(sc, S.imag) * g118.sn_mva
    sw = InjectionSweepGPU(g118.as_tuple(), init_from_n_powerflow=False, precision=precision, nb_iter=20,
                           scheduling="continuous", tol=1e-10, start="flat")
    sw.set_injections(P, Q, g118.sn_mva)
    sw.compute()
    assert np.all(sw.get_row_status() == RowStatus.CONVERGED)
    assert np.abs(sw.V_results - ref["V_scaled"]).max() < tol_v
    ca = ContingencyAnalysisGPU(g118.as_tuple(), init_from_n_powerflow=False, precision=precision, nb_iter=20,
                                scheduling="continuous", tol=1e-10, start="flat")
    ca.set_branch_data(*g118.branch_data())
    ca.add_contingencies_by_branch_id([[int(l)] for l in ref["n1_rows"]])
    ca.compute()
    assert np.all(ca.get_row_status() == RowStatus.CONVERGED)
    assert np.abs(ca.V_results - ref["V_n1"]).max() < tol_v
    from gpusim2grid_b200.synthetic import half_open_variant
    h = half_open_variant(g118, n_open=2, seed=0)
    out = np.zeros(h.n_bus, dtype=np.complex128)
    Yh, V0h, Sh, slh, wh, pvh, pqh = h.as_tuple()
    t = acpf_nr_gpu(out, Yh, V0h, Sh, slh, wh, pvh, pqh, 20, 1e-10, 1, precision=precision)
    assert t.converged and np.abs(out - ref["V_half"]).max() < tol_v


def test_single_solve_takes_the_step_after_the_test(g118):
    """acpf_nr_gpu / AcPfGPU follow the reference's single-solve order: a
    step, then the test of the mismatch before it (acpf_nr.cu:505-561), so a
    solve reports one step more than a continuous-schedule row and returns
    the voltage after that step; a budget that ends before the test passes is
    not converged."""
    Y, V0, S, sl, w, pv, pq = g118.as_tuple()
    Vo, so, io, _ = O.nr_solve(Y, V0, S, pv, pq, 10, 1e-8, mode="single")
    _, _, ic, _ = O.nr_solve(Y, V0, S, pv, pq, 10, 1e-8)
    assert io == ic + 1
    ac = AcPfGPU(g118.as_tuple(), init_from_n_powerflow=False, max_iter=10, tol=1e-8)
    assert ac.timings.converged and ac.timings.nb_iter == io
    assert np.abs(ac.solve() - Vo).max() < TOL_V_FP64
    t = ac.resolve(V0, max_iter=ic)
    assert not t.converged and t.nb_iter == ic
