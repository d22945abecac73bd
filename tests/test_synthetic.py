"""The seeded synthetic grid generator."""

import numpy as np
import scipy.sparse as sp
from scipy.sparse.csgraph import connected_components

from gpusim2grid_b200.synthetic import (GRID_SPECS, grid_by_name, injection_scenarios, n1_branches,
                                        scenario_outages)


def test_specs_and_determinism():
    for name, (n, nbr, npv, nld, _, _) in GRID_SPECS.items():
        if n > 2000:
            continue
        a = grid_by_name(name, 3)
        b = grid_by_name(name, 3)
        assert a.n_bus == n and a.n_branch == nbr and a.pv.size == npv and a.load_bus.size == nld
        assert a.pq.size == n - npv - 1
        np.testing.assert_array_equal(a.branch_from, b.branch_from)
        np.testing.assert_array_equal(a.Ybus.data, b.Ybus.data)
        A = sp.coo_matrix((np.ones(a.n_branch), (a.branch_from, a.branch_to)), shape=(n, n))
        assert connected_components(A, directed=False)[0] == 1
        assert abs(a.gen_p.sum() - 1.02 * a.load_p.sum()) < 1e-9
        assert a.Ybus.has_sorted_indices


def test_n1_branches_match_bruteforce(g118):
    rows = set(n1_branches(g118).tolist())
    n = g118.n_bus
    for l in range(g118.n_branch):
        keep = np.arange(g118.n_branch) != l
        A = sp.coo_matrix((np.ones(keep.sum()), (g118.branch_from[keep], g118.branch_to[keep])), shape=(n, n))
        assert (connected_components(A, directed=False)[0] == 1) == (l in rows)


def test_injection_scenarios_balance(g118):
    p, q = injection_scenarios(g118, 16, seed=5)
    assert p.shape == (16, g118.n_bus) and q.shape == p.shape
    # generation stays 1.02 x load in every scenario
    load = -p.copy()
    load[:, g118.gen_bus] = 0
    # bus-level check of totals: sum(p) = gen - load = 0.02 load
    lp = (q.sum(axis=1))
    assert np.all(np.isfinite(p)) and np.all(lp < 0)


def test_scenario_outages_connected(g118):
    rows = scenario_outages(g118, 30, max_trips=2, seed=4)
    assert len(rows) == 30 and all(len(r) <= 2 for r in rows)
