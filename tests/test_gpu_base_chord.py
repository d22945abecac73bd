"""Strategy base_chord: rows start their chord steps on the base case's
factor (computed once, shared by every row) and factor their own Jacobian
only when a step stops contracting.  The answers must be the same solutions
(1e-6 pu bar against plain FP64) with fewer factorizations."""

import numpy as np
import pytest

from conftest import TOL_V_MIXED
from gpusim2grid_b200 import ContingencyAnalysisGPU, InjectionSweepGPU, RowStatus, ScenarioSweepGPU
from gpusim2grid_b200.synthetic import injection_scenarios, n1_branches

pytestmark = pytest.mark.gpu


def _ca(g, precision, strategy, start):
    ca = ContingencyAnalysisGPU(g.as_tuple(), init_from_n_powerflow=False, precision=precision, nb_iter=10,
                                scheduling="continuous", tol=1e-8, start=start, strategy=strategy)
    ca.set_branch_data(*g.branch_data())
    ca.add_contingencies_by_branch_id([[int(b)] for b in n1_branches(g)])
    ca.compute()
    return ca


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_base_chord_n1(g118, precision):
    ref = _ca(g118, "fp64", "refactor_every", "flat")
    ad = _ca(g118, precision, "adaptive", "base")
    bc = _ca(g118, precision, "base_chord", "base")
    ok = ref.get_row_status() == RowStatus.CONVERGED
    np.testing.assert_array_equal(bc.get_row_status(), ref.get_row_status())
    assert np.abs(bc.V_results[ok] - ref.V_results[ok]).max() < TOL_V_MIXED
    assert bc.get_row_factorizations().sum() < ad.get_row_factorizations().sum()


def test_base_chord_injections(g118):
    p, q = injection_scenarios(g118, 64, seed=5)
    out = []
    for strategy in ("refactor_every", "base_chord"):
        sw = InjectionSweepGPU(g118.as_tuple(), init_from_n_powerflow=False, precision="mixed", nb_iter=10,
                               scheduling="continuous", start="base", strategy=strategy)
        sw.set_injections(p, q, g118.sn_mva)
        sw.compute()
        out.append(sw)
    a, b = out
    np.testing.assert_array_equal(b.get_row_status(), a.get_row_status())
    ok = a.get_row_status() == RowStatus.CONVERGED
    assert np.abs(a.V_results[ok] - b.V_results[ok]).max() < TOL_V_MIXED


def test_device_rows_match_host_definitions(g118):
    """gs2g_get_device_rows hands out the session's device copies of the
    rows: Sbus = (p + jq) / sn_mva (uploaded through the pinned staging
    chunks, several of them at this size) and the trip CSR."""
    import torch
    from gpusim2grid_b200 import ScenarioSweepGPU
    n = 2 * (8 << 20) // (16 * g118.n_bus) + 7  # more than two 8 MiB chunks of complex rows
    p, q = injection_scenarios(g118, n, seed=3)
    trips = [[int(b)] if r % 3 else [] for r, b in enumerate(np.resize(n1_branches(g118), n))]
    sw = ScenarioSweepGPU(g118.as_tuple(), init_from_n_powerflow=False, precision="mixed", nb_iter=10,
                          scheduling="continuous", tol=1e-8)
    sw.set_branch_data(*g118.branch_data())
    sw.set_injections(p, q, g118.sn_mva)
    sw.set_topology(trips)
    sbus, (ptr, ids), nr = sw._device_row_defs()
    assert nr == n and sbus.shape == (n, g118.n_bus)
    np.testing.assert_array_equal(sbus.cpu().numpy(), (p + 1j * q) / g118.sn_mva)
    np.testing.assert_array_equal(ptr.cpu().numpy(), np.cumsum([0] + [len(t) for t in trips]))
    np.testing.assert_array_equal(ids.cpu().numpy(), [b for t in trips for b in t])
    assert isinstance(sbus, torch.Tensor) and sbus.is_cuda


@pytest.mark.parametrize("name,kind,precision", [("case2000_synth", "n1", "mixed"), ("case2000_synth", "heavy", "mixed"),
                                                 ("case6500_synth", "heavy", "mixed"), ("case2000_synth", "n1", "fp64"),
                                                 ("case2000_synth", "heavy", "fp64")])
def test_cluster_handoffs_equal_one_cta_handoffs(name, kind, precision):
    """The chord sweep's hand-offs (rows that factor their own Jacobian) run
    on a cluster of CTAs per row when every such row can have a cluster (the
    N-1 sweep: about a dozen rows), all CTAs of the cluster sharing each
    Schur update and dense tail LU (FP32 or FP64); with more hand-offs than
    clusters (heavily loaded scenarios) every CTA takes rows of its own.  The
    shared factorization is bit-identical to the one-CTA one, so every output
    must be too."""
    from gpusim2grid_b200.synthetic import grid_by_name, scenario_outages
    g = grid_by_name(name, 0)
    out = []
    for cluster in (0, 1):
        kw = dict(init_from_n_powerflow=False, precision=precision, nb_iter=10, scheduling="continuous", tol=1e-8,
                  start="base", strategy="base_chord")
        if kind == "n1":
            sw = ContingencyAnalysisGPU(g.as_tuple(), **kw)
            sw.set_branch_data(*g.branch_data())
            sw.add_contingencies_by_branch_id([[int(b)] for b in n1_branches(g)])
        else:
            n = 512
            p, q = injection_scenarios(g, n, seed=31)
            sw = ScenarioSweepGPU(g.as_tuple(), **kw)
            sw.set_branch_data(*g.branch_data())
            # heavier loading than the sweeps' scenarios, so that many rows leave the chord
            sw.set_injections(1.25 * p, 1.25 * q, g.sn_mva)
            sw.set_topology(scenario_outages(g, n, max_trips=2, seed=32))
        sw.session.set_handoff(cluster)
        sw.compute()
        out.append((sw.V_results, sw.get_row_status(), sw.get_row_iterations(), sw.get_row_factorizations()))
    (V0, s0, i0, f0), (V1, s1, i1, f1) = out
    assert f0.sum() > 0  # some rows were handed off and factored their own Jacobian
    np.testing.assert_array_equal(s0, s1)
    np.testing.assert_array_equal(i0, i1)
    np.testing.assert_array_equal(f0, f1)
    np.testing.assert_array_equal(V0, V1)


@pytest.mark.parametrize("name", ["case2000_synth", "case6500_synth"])
def test_fp64_subset_on_clusters_equals_one_cta(name):
    """A small FP64 re-solve (gs2g_run_subset with at most one row per 8 CTAs:
    the fallback of rows a mixed sweep did not converge) runs each row on a
    cluster of 8 CTAs sharing its Schur updates and dense LUs; bit-identical
    to the one-CTA rows and to the same rows of a full FP64 run."""
    from gpusim2grid_b200._native import lib
    from gpusim2grid_b200.synthetic import grid_by_name
    g = grid_by_name(name, 0)
    rows = [[int(b)] for b in n1_branches(g)[:24]]
    sub = np.array([1, 5, 11, 17, 23], dtype=np.int32)
    ca = ContingencyAnalysisGPU(g.as_tuple(), init_from_n_powerflow=False, precision="fp64", nb_iter=10,
                                scheduling="continuous", tol=1e-8, start="flat")
    ca.set_branch_data(*g.branch_data())
    ca.add_contingencies_by_branch_id(rows)
    ca.compute()
    full = ca.V_results, ca.get_row_status(), ca.get_row_iterations()
    s = ca.session
    out = []
    for cluster in (0, 1):
        s.set_handoff(cluster)
        s.run(10, 1e-8, False, lib.PREC_FP64, lib.START_VINIT, refactor=lib.REFACTOR_EVERY)
        s.run_subset(sub, 10, 1e-8, False, lib.PREC_FP64, lib.START_VINIT, refactor=lib.REFACTOR_EVERY)
        V, res, st, it = s.results()
        out.append((V[sub], st[sub], it[sub]))
    for k in range(3):
        np.testing.assert_array_equal(out[0][k], out[1][k])
        np.testing.assert_array_equal(out[1][k], full[k][sub])
    assert np.all(out[1][1] == 0)


@pytest.mark.parametrize("kind", ["n1", "scenario"])
def test_row_order_leaves_results_unchanged(kind):
    """The sweeps take the rows largest difficulty estimate first (distance
    from the base injections, base flow of the tripped branches); a row's
    results do not depend on when it runs, so they equal the in-order run
    bit for bit, hand-offs, islanded rows and the FP64 fallback included."""
    from gpusim2grid_b200.synthetic import grid_by_name, scenario_outages
    g = grid_by_name("case2000_synth", 0)
    kw = dict(init_from_n_powerflow=False, precision="mixed", nb_iter=10, scheduling="continuous", tol=1e-8,
              start="base", strategy="base_chord")
    if kind == "n1":
        sw = ContingencyAnalysisGPU(g.as_tuple(), **kw)
        sw.set_branch_data(*g.branch_data())
        bridges = np.setdiff1d(np.arange(g.n_branch), n1_branches(g))[:3]
        sw.add_contingencies_by_branch_id([[int(b)] for b in n1_branches(g)] + [[int(b)] for b in bridges])
    else:
        n = 1024
        p, q = injection_scenarios(g, n, seed=41)
        sw = ScenarioSweepGPU(g.as_tuple(), **kw)
        sw.set_branch_data(*g.branch_data())
        sw.set_injections(1.2 * p, 1.2 * q, g.sn_mva)
        sw.set_topology(scenario_outages(g, n, max_trips=2, seed=42))
    out = []
    for order in (0, 1):
        sw.session.set_row_order(order)
        sw.compute()
        out.append((sw.V_results, sw.get_row_status(), sw.get_row_iterations(), sw.get_row_factorizations()))
    for a, b in zip(*out):
        np.testing.assert_array_equal(a, b)
    assert out[0][3].sum() > 0


@pytest.mark.parametrize("kind", ["n1", "scenario"])
def test_start_switch_equals_base_start(kind):
    """A row whose own start has the larger mismatch starts from the base V
    instead (start selection).  The chord sweep then writes the row's F at
    the base V from the base case's Ybus product (summed as the sweep's
    mismatch sums), corrected at the row's edited Ybus rows, instead of a
    sparse product.  Rows that all start flat (every one switches) must give
    the base-start results bit for bit."""
    from gpusim2grid_b200.synthetic import grid_by_name, scenario_outages
    g = grid_by_name("case2000_synth", 0)
    kw = dict(init_from_n_powerflow=False, precision="mixed", nb_iter=10, scheduling="continuous", tol=1e-8,
              start="base", strategy="base_chord")
    if kind == "n1":
        sw = ContingencyAnalysisGPU(g.as_tuple(), **kw)
        sw.set_branch_data(*g.branch_data())
        sw.add_contingencies_by_branch_id([[int(b)] for b in n1_branches(g)])
        n = len(n1_branches(g))
    else:
        n = 1024
        p, q = injection_scenarios(g, n, seed=51)
        sw = ScenarioSweepGPU(g.as_tuple(), **kw)
        sw.set_branch_data(*g.branch_data())
        sw.set_injections(p, q, g.sn_mva)
        sw.set_topology(scenario_outages(g, n, max_trips=2, seed=52))
    sw.compute()
    base = (sw.V_results.copy(), sw.get_row_status().copy(), sw.get_row_iterations().copy(),
            sw.get_row_factorizations().copy())
    sw.set_start_voltages(np.tile(np.asarray(g.vinit(), dtype=np.complex128), (n, 1)))
    sw.compute()
    switched = sw.V_results, sw.get_row_status(), sw.get_row_iterations(), sw.get_row_factorizations()
    # (equal results also show that every row switched: a flat start takes other steps)
    for a, b in zip(base, switched):
        np.testing.assert_array_equal(a, b)


def test_compensation_records_and_in_sweep_setup_reach_fp64_solutions():
    """Rows tripping up to four branches: a row touching at most 8 Jacobian
    positions takes its outage compensation from the records set up ahead of
    the chord sweep, a larger one sets it up in the sweep, and beyond 16
    positions a row steps uncompensated until it leaves the chord.  Every
    row must reach the plain FP64 flat-start solution."""
    from gpusim2grid_b200.synthetic import grid_by_name, scenario_outages
    g = grid_by_name("case2000_synth", 0)
    n = 512
    p, q = injection_scenarios(g, n, seed=61)
    trips = scenario_outages(g, n, max_trips=4, seed=62)
    assert max(len(t) for t in trips) == 4
    out = []
    for precision, strategy, start in (("fp64", "refactor_every", "flat"), ("mixed", "base_chord", "base")):
        sw = ScenarioSweepGPU(g.as_tuple(), init_from_n_powerflow=False, precision=precision, nb_iter=10,
                              scheduling="continuous", tol=1e-8, start=start, strategy=strategy)
        sw.set_branch_data(*g.branch_data())
        sw.set_injections(p, q, g.sn_mva)
        sw.set_topology(trips)
        sw.compute()
        out.append(sw)
    ref, bc = out
    np.testing.assert_array_equal(bc.get_row_status(), ref.get_row_status())
    ok = ref.get_row_status() == RowStatus.CONVERGED
    assert ok.sum() > 0.9 * n
    assert np.abs(bc.V_results[ok] - ref.V_results[ok]).max() < TOL_V_MIXED
