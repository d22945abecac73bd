"""Branch flows and the limit check done by the sweep kernel as each row
leaves the GPU, against the oracle's flow formulas on the GPU's own
voltages, in one-grid and heterogeneous launches."""

import numpy as np
import pytest

from gpusim2grid_b200 import RowStatus, ScenarioSweepGPU, compute_many
from gpusim2grid_b200.synthetic import grid_by_name, injection_scenarios, scenario_outages
from oracle import nr_oracle as O

pytestmark = pytest.mark.gpu


def _limits(g, rng):
    """MVA limits near the base-case flows, so that some rows overload."""
    Y, V0, S, _, _, pv, pq = g.as_tuple()
    V, st, _, _ = O.nr_solve(Y, V0, S, pv, pq, 20, 1e-10)
    Sf, St = O.branch_flows(V, g.branch_from, g.branch_to, g.yff, g.yft, g.ytf, g.ytt)
    rate = np.maximum(np.abs(Sf), np.abs(St)) * g.sn_mva * rng.uniform(1.0, 1.4, g.n_branch)
    rate[rng.random(g.n_branch) < 0.1] = 0.0  # some unlimited branches
    return rate


def _sweep(g, n, seed, rate):
    sw = ScenarioSweepGPU(g.as_tuple(), init_from_n_powerflow=False, precision="mixed", nb_iter=10,
                          scheduling="continuous", start="flat", strategy="adaptive")
    sw.set_branch_data(*g.branch_data())
    p, q = injection_scenarios(g, n, seed=seed)
    sw.set_injections(p, q, g.sn_mva)
    sw.set_topology(scenario_outages(g, n, max_trips=2, seed=seed + 1))
    sw.set_branch_limits(rate, g.sn_mva)
    return sw


def _check(sw, g, rate):
    ld, nv, mx = sw.branch_loading()
    st = sw.get_row_status()
    V = sw.V_results
    topo = sw.get_topology() if hasattr(sw, "get_topology") else sw._topo
    assert ld.shape == (len(st), g.n_branch)
    assert (st == RowStatus.CONVERGED).sum() > 0.8 * len(st)
    seen_violation = False
    for r in range(len(st)):
        if st[r] != RowStatus.CONVERGED:
            assert np.all(np.isnan(ld[r])) and nv[r] == -1
            continue
        ref = O.branch_loading(V[r], g.branch_from, g.branch_to, g.yff, g.yft, g.ytf, g.ytt, rate / g.sn_mva,
                               tripped=topo[r])
        np.testing.assert_allclose(ld[r], ref, rtol=1e-5, atol=1e-6)
        near = np.abs(ref - 1.0) < 1e-5
        assert abs(int(nv[r]) - int((ref > 1.0).sum())) <= int(near.sum())
        assert abs(mx[r] - ref.max()) <= 1e-5 * max(1.0, ref.max())
        seen_violation |= nv[r] > 0
    return seen_violation


def test_flows_and_limits_one_grid():
    g = grid_by_name("case118_synth", 0)
    rate = _limits(g, np.random.default_rng(0))
    sw = _sweep(g, 96, 31, rate)
    sw.compute()
    assert _check(sw, g, rate)
    # not simulated (islanded) rows carry NaN loadings as well
    sw.set_topology([[0, 1, 2, 3, 4, 5, 6, 7]] + [[]] * 95)
    sw.compute()
    ld, nv, _ = sw.branch_loading()
    if sw.get_row_status()[0] == RowStatus.NOT_SIMULATED:
        assert np.all(np.isnan(ld[0])) and nv[0] == -1


def test_flows_and_limits_in_a_heterogeneous_launch():
    parts = []
    for i, name in enumerate(["case118_synth", "case2000_synth"]):
        g = grid_by_name(name, 0)
        rate = _limits(g, np.random.default_rng(i))
        parts.append((g, rate, _sweep(g, 32, 40 + i, rate)))
    compute_many([sw for _, _, sw in parts])
    for g, rate, sw in parts:
        _check(sw, g, rate)
