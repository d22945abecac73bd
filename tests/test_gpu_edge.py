"""GPU edge cases: islanding, NaN rows, invariances, determinism, full-size
properties (restated from the reference's test families)."""

import numpy as np
import pytest

from gpusim2grid_b200 import ContingencyAnalysisGPU, InjectionSweepGPU, RowStatus, ScenarioSweepGPU
from gpusim2grid_b200.synthetic import injection_scenarios, n1_branches
from oracle import nr_oracle as O

pytestmark = pytest.mark.gpu


def _ca(g, **kw):
    kw.setdefault("init_from_n_powerflow", False)
    kw.setdefault("nb_iter", 10)
    kw.setdefault("scheduling", "continuous")
    kw.setdefault("start", "flat")
    ca = ContingencyAnalysisGPU(g.as_tuple(), **kw)
    ca.set_branch_data(*g.branch_data())
    return ca


def test_islanded_row_is_nan_and_neighbours_unaffected(g118):
    rows = n1_branches(g118)
    bridge = int(np.setdiff1d(np.arange(g118.n_branch), rows)[0])
    ca = _ca(g118)
    ca.add_contingencies_by_branch_id([[int(rows[0])], [bridge], [int(rows[1])]])
    ca.compute()
    st = ca.get_row_status()
    assert list(st) == [RowStatus.CONVERGED, RowStatus.NOT_SIMULATED, RowStatus.CONVERGED]
    assert np.all(np.isnan(ca.V_results[1])) and np.isnan(ca.last_residuals()[1])
    ca2 = _ca(g118)
    ca2.add_contingencies_by_branch_id([[int(rows[0])], [int(rows[1])]])
    ca2.compute()
    np.testing.assert_array_equal(ca2.V_results, ca.V_results[[0, 2]])


def test_nan_scenario_diverges_alone(g118):
    p, q = injection_scenarios(g118, 4, seed=3)
    p[2, g118.pq[0]] = np.nan
    sw = InjectionSweepGPU(g118.as_tuple(), init_from_n_powerflow=False, nb_iter=10, scheduling="continuous",
                           start="flat")
    sw.set_injections(p, q, g118.sn_mva)
    sw.compute()
    st = sw.get_row_status()
    assert st[2] == RowStatus.DIVERGED and np.isnan(sw.last_residuals()[2])
    assert np.all(st[[0, 1, 3]] == RowStatus.CONVERGED)


def test_batch_size_and_order_invariance(g118):
    rows = [[int(b)] for b in n1_branches(g118)[:40]]
    ca = _ca(g118)
    ca.add_contingencies_by_branch_id(rows)
    ca.compute(batch_size=512)
    V_full = ca.V_results.copy()
    ca.compute(batch_size=3)
    np.testing.assert_array_equal(ca.V_results, V_full)  # bitwise: a row's arithmetic is independent of its CTA
    perm = np.random.default_rng(1).permutation(len(rows))
    ca.add_contingencies_by_branch_id([rows[i] for i in perm])
    ca.compute()
    np.testing.assert_array_equal(ca.V_results, V_full[perm])


def test_duplicate_branch_ids_trip_once(g118):
    b = int(n1_branches(g118)[3])
    ca = _ca(g118)
    ca.add_contingencies_by_branch_id([[b], [b, b]])
    ca.compute()
    np.testing.assert_array_equal(ca.V_results[0], ca.V_results[1])


def test_unit_scale_injection_reproduces_base(g118):
    """Injection rows equal to the base injections reproduce the base case
    (reference test_injection_batch.py:169)."""
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    Vb, *_ = O.nr_solve(Y, V0, S, pv, pq, 10, 1e-8)
    P = np.tile(S.real * g118.sn_mva, (3, 1))
    Q = np.tile(S.imag * g118.sn_mva, (3, 1))
    sw = InjectionSweepGPU(g118.as_tuple(), init_from_n_powerflow=False, nb_iter=10, scheduling="continuous",
                           start="flat")
    sw.set_injections(P, Q, g118.sn_mva)
    sw.compute()
    assert np.abs(sw.V_results - Vb[None]).max() < 1e-9


def test_out_of_range_branch_is_runtime_error(g118):
    """build_contingency_from_branch_ids throws std::runtime_error
    (reference contingency_analysis_helper.cpp:46-48): RuntimeError."""
    ca = _ca(g118)
    with pytest.raises(RuntimeError, match="out of range"):
        ca.add_contingencies_by_branch_id([[g118.n_branch + 3]])
    with pytest.raises(RuntimeError, match="out of range"):
        ca.add_contingencies_by_branch_id([[0], [-1]])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_injection_6500_full_size_properties(g6500, precision):
    """Full-size 6500-bus injection sweep: every row converges and the
    reported residual equals a host recompute of the mismatch."""
    n = 256
    p, q = injection_scenarios(g6500, n, seed=11)
    sw = InjectionSweepGPU(g6500.as_tuple(), init_from_n_powerflow=False, precision=precision, nb_iter=10,
                           scheduling="continuous", start="flat")
    sw.set_injections(p, q, g6500.sn_mva)
    sw.compute()
    st = sw.get_row_status()
    assert np.all(st == RowStatus.CONVERGED)
    Y, V0, S, _, _, pv, pq = g6500.as_tuple()
    pvpq, pq_, _ = O.j_layout(g6500.n_bus, pv, pq)
    for r in (0, 77, n - 1):
        F = O.mismatch(Y, sw.V_results[r], (p[r] + 1j * q[r]) / g6500.sn_mva, pvpq, pq_)
        assert abs(np.abs(F).max() - sw.last_residuals()[r]) < 1e-10
        assert np.abs(F).max() < 1e-8


def test_islanding_flags_every_single_and_some_double_outages(g118):
    """Single outages are flagged from the bridges of the branch graph,
    multi-branch outages by a connectivity check: both must agree with the
    oracle's connectivity check for every single-branch row and for double
    outages that include non-bridge pairs."""
    m = g118.n_branch
    rows = [[b] for b in range(m)]
    rng = np.random.default_rng(7)
    for _ in range(64):
        rows.append(sorted(int(v) for v in rng.choice(m, 2, replace=False)))
    ca = ContingencyAnalysisGPU(g118.as_tuple(), init_from_n_powerflow=False, nb_iter=10, scheduling="continuous",
                                start="flat")
    ca.set_branch_data(*g118.branch_data())
    ca.add_contingencies_by_branch_id(rows)
    ca.compute()
    st = ca.get_row_status()
    for r, ids in enumerate(rows):
        islanded = bool(O.islands(g118.n_bus, g118.branch_from, g118.branch_to, ids))
        assert (st[r] == RowStatus.NOT_SIMULATED) == islanded, (r, ids)


@pytest.mark.parametrize("grid", ["g118", "g2000"])
def test_islanding_flags_of_cut_pairs_and_triples(grid, request):
    """Rows that trip two or three branches are pre-checked by the branches'
    cycle-space labels (independent labels: connected for certain) and, when
    the labels are dependent, by the exact connectivity check.  Cut pairs (the
    two branches of a bus of degree 2), triples holding such a pair, random
    pairs and triples: the flags must equal the oracle's connectivity check."""
    g = request.getfixturevalue(grid)
    m = g.n_branch
    deg = np.bincount(np.concatenate([g.branch_from, g.branch_to]), minlength=g.n_bus)
    rng = np.random.default_rng(17)
    rows = []
    for b in np.flatnonzero(deg == 2)[:40]:
        pair = sorted(int(l) for l in np.flatnonzero((g.branch_from == b) | (g.branch_to == b)))
        rows.append(pair)
        rows.append(sorted(set(pair) | {int(rng.integers(m))}))
    for _ in range(120):
        rows.append(sorted(int(v) for v in rng.choice(m, 2, replace=False)))
        rows.append(sorted(int(v) for v in rng.choice(m, 3, replace=False)))
    ca = ContingencyAnalysisGPU(g.as_tuple(), init_from_n_powerflow=False, nb_iter=10, scheduling="continuous",
                                start="flat", precision="mixed", strategy="base_chord")
    ca.set_branch_data(*g.branch_data())
    ca.add_contingencies_by_branch_id(rows)
    ca.compute()
    st = ca.get_row_status()
    islanded = np.array([bool(O.islands(g.n_bus, g.branch_from, g.branch_to, ids)) for ids in rows])
    assert islanded.sum() >= 20 and (~islanded).sum() >= 100
    np.testing.assert_array_equal(st == RowStatus.NOT_SIMULATED, islanded)


def test_set_injections_from_elements_needs_a_grid_object(g118):
    """Array-tuple mode has no loads or generators to map: RuntimeError, as in
    the reference (``injection_sweep/gpu_facade.py:394``)."""
    sw = InjectionSweepGPU(g118.as_tuple(), init_from_n_powerflow=False)
    with pytest.raises(RuntimeError, match="lightsim2grid grid"):
        sw.set_injections_from_elements(np.zeros((1, 3)), np.zeros((1, 3)), np.zeros((1, 2)))


def test_results_view_equals_the_owned_copies(g118):
    """results_view(): the same results as the owned host copies, from the
    session's page-locked buffer (valid until the next compute())."""
    ca = _ca(g118)
    ca.add_contingencies_by_branch_id([[int(b)] for b in n1_branches(g118)[:20]])
    ca.compute()
    V, res, st, it = ca.results_view()
    np.testing.assert_array_equal(V, ca.V_results)
    np.testing.assert_array_equal(res, ca.last_residuals())
    np.testing.assert_array_equal(st, ca.get_row_status())
    np.testing.assert_array_equal(it, ca.get_row_iterations())
    assert V.shape == (20, g118.n_bus) and not V.flags.owndata


@pytest.mark.parametrize("precision,strategy", [("fp64", "refactor_every"), ("mixed", "base_chord")])
def test_results_to_host_mirror_equals_the_device_results(g118, precision, strategy):
    """results_to_host: the kernels write each row's final V into the
    page-locked buffer as it leaves; equal, NaNs included, to the device
    results, for islanded rows (NaN), split rows (masked NaN buses) and
    solved rows, over batches of changing size and after switching off."""
    m = g118.n_branch
    bridges = np.setdiff1d(np.arange(m), n1_branches(g118))
    rows = [[int(b)] for b in n1_branches(g118)[:30]] + [[int(b)] for b in bridges[:4]]
    ca = _ca(g118, precision=precision, strategy=strategy)
    ca.results_to_host = True
    for hd, rr in ((False, rows), (True, rows[:7] + rows[-3:]), (True, rows)):
        ca.handle_disconnected_grid = hd
        ca.add_contingencies_by_branch_id(rr)
        ca.compute()
        V, res, st, it = ca.results_view()
        np.testing.assert_array_equal(V, ca.V_results)
        np.testing.assert_array_equal(st, ca.get_row_status())
        np.testing.assert_array_equal(res, ca.last_residuals())
        np.testing.assert_array_equal(it, ca.get_row_iterations())
        assert np.isnan(V[-1]).any()
    ca.results_to_host = False
    ca.add_contingencies_by_branch_id(rows[:5])
    ca.compute()
    np.testing.assert_array_equal(ca.results_view()[0], ca.V_results)


@pytest.mark.parametrize("precision,strategy,tol_v", [("fp64", "refactor_every", 1e-9),
                                                      ("mixed", "base_chord", 1e-6)])
def test_handle_disconnected_grid_vs_oracle(g118, precision, strategy, tol_v):
    """handle_disconnected_grid: rows whose trips split the grid solve the
    largest component, with NaN voltages at the other buses, or stay
    NOT_SIMULATED when the split strands the slack; flows of branches at a
    masked bus are NaN and left out of the row's count and maximum."""
    m = g118.n_branch
    rows = [[b] for b in range(m)]
    rng = np.random.default_rng(11)
    for _ in range(48):
        rows.append(sorted(int(v) for v in rng.choice(m, 2, replace=False)))
    ca = _ca(g118, precision=precision, strategy=strategy, handle_disconnected_grid=True)
    rate = np.full(m, 150.0)
    ca.set_branch_limits(rate)
    ca.add_contingencies_by_branch_id(rows)
    ca.compute()
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    Vo, so, io, ro = O.contingency_sweep(Y, V0, S, pv, pq, rows, g118.branch_from, g118.branch_to, g118.yff,
                                         g118.yft, g118.ytf, g118.ytt, 10, 1e-8, handle_disconnected=True)
    st = ca.get_row_status()
    np.testing.assert_array_equal(st, so)
    split = np.array([O.islands(g118.n_bus, g118.branch_from, g118.branch_to, r) for r in rows])
    assert (split & (so == RowStatus.CONVERGED)).sum() > 0  # some splits were solved
    V = ca.V_results
    np.testing.assert_array_equal(np.isnan(V), np.isnan(Vo))
    ok = so == RowStatus.CONVERGED
    assert np.nanmax(np.abs(V[ok] - Vo[ok])) < tol_v
    assert np.all(ca.last_residuals()[ok] < 1e-8)
    if strategy == "refactor_every":
        np.testing.assert_array_equal(ca.get_row_iterations(), io)
    loading, nviol, mx = ca.branch_loading()
    for r in np.flatnonzero(ok & split):
        ref = O.branch_loading(np.nan_to_num(Vo[r]), g118.branch_from, g118.branch_to, g118.yff, g118.yft,
                               g118.ytf, g118.ytt, rate / g118.sn_mva, tripped=rows[r])
        dead = np.isnan(Vo[r][g118.branch_from]) | np.isnan(Vo[r][g118.branch_to])
        assert np.all(np.isnan(loading[r][dead & ~np.isin(np.arange(m), rows[r])]))
        live = ~dead
        np.testing.assert_allclose(loading[r][live], ref[live], rtol=1e-5, atol=1e-6)
        assert np.isfinite(mx[r]) and nviol[r] == int((ref[live] > 1).sum())
    # off: every split is NOT_SIMULATED
    ca.handle_disconnected_grid = False
    ca.compute()
    assert np.all((ca.get_row_status() == RowStatus.NOT_SIMULATED) == split)
