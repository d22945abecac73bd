"""Parity of the measured configurations against the FP64 oracle.

* cfg 1 as the bench runs it: the 2000-bus N-1 sweep, every row (plus bridge
  outages, which island the grid), learned start + mixed precision +
  ``base_chord`` (Broyden steps on the shared base factor) + the FP64
  fallback, compared row by row with the oracle's flat-start FP64 Newton:
  same convergence and islanding flags, |dV| <= 1e-6 pu, residual < 1e-8.
* cfg 2: the 6500-bus injection sweep (4096 scenarios) under the same
  strategy: every row's status against the engine's plain FP64 arm, and a
  sample of 128 rows against the oracle.
* the 10000-bus grid (cfg 4's largest): 64 scenario rows with 0-2 tripped
  branches; 32 of them against the oracle.

The oracle runs in spawned processes (tests/_oracle_pool.py).  The learned
starts are trained on fewer rows than the bench uses: the start only decides
where each row begins, the answers are the converged solutions either way.
"""

import numpy as np
import pytest

from _oracle_pool import oracle_rows
from conftest import TOL_V_MIXED
from gpusim2grid_b200 import ContingencyAnalysisGPU, InjectionSweepGPU, RowStatus, ScenarioSweepGPU
from gpusim2grid_b200.synthetic import grid_by_name, injection_scenarios, n1_branches, scenario_outages

pytestmark = pytest.mark.gpu


def _check(V, st, res, Vo, so, tol_v=TOL_V_MIXED):
    np.testing.assert_array_equal(st, so)
    ok = so == RowStatus.CONVERGED
    assert np.abs(V[ok] - Vo[ok]).max() <= tol_v
    assert np.all(res[ok] < 1e-8)
    assert np.all(np.isnan(V[so == RowStatus.NOT_SIMULATED]))


def test_cfg1_benched_path_every_row_vs_oracle(g2000):
    from gpusim2grid_b200.warmstart import LearnedStart
    rows = [[int(b)] for b in n1_branches(g2000)]
    bridges = np.setdiff1d(np.arange(g2000.n_branch), n1_branches(g2000))[:3]
    rows += [[int(b)] for b in bridges]
    ls = LearnedStart(g2000, hidden=1024, layers=2, seed=0)
    ls.train(n_rows=20000, epochs=10, batch=1024, lr=1e-3, lr_decay=0.8, seed=7, broad=0.5)
    ca = ContingencyAnalysisGPU(g2000.as_tuple(), init_from_n_powerflow=False, precision="mixed", nb_iter=10,
                                scheduling="continuous", tol=1e-8, start="flat", strategy="base_chord")
    ca.set_branch_data(*g2000.branch_data())
    ca.add_contingencies_by_branch_id(rows)
    ca.set_learned_start(ls)
    ca.results_to_host = True
    ca.compute()
    Vo, so, _, _ = oracle_rows(g2000, trips=rows)
    _check(ca.V_results, ca.get_row_status(), ca.last_residuals(), Vo, so)
    # the kernels' host copy of V (chord rows, hand-offs, fallback) equals the device results
    np.testing.assert_array_equal(ca.results_view()[0], ca.V_results)
    assert int((so == RowStatus.NOT_SIMULATED).sum()) == len(bridges)
    # the path the bench measures: nearly every step on the shared base factor
    assert ca.session.timings()["chord_steps"] > 0.9 * ca.get_row_iterations().sum()


def test_cfg2_injection_sweep_vs_fp64_arm_and_oracle(g6500):
    from gpusim2grid_b200.warmstart import LearnedStart
    p, q = injection_scenarios(g6500, 4096, seed=1)
    ls = LearnedStart(g6500, hidden=1024, layers=2, seed=0)
    ls.train(n_rows=8192, epochs=10, batch=1024, lr=1e-3, lr_decay=0.8, seed=7, broad=1.0, p_outage=0.0)
    out = {}
    for arm in ("mixed", "fp64"):
        sw = InjectionSweepGPU(g6500.as_tuple(), init_from_n_powerflow=False, precision=arm, nb_iter=10,
                               scheduling="continuous", tol=1e-8, start="flat",
                               strategy="base_chord" if arm == "mixed" else "refactor_every")
        sw.set_injections(p, q, g6500.sn_mva)
        if arm == "mixed":
            sw.set_learned_start(ls)
        sw.compute()
        out[arm] = (sw.V_results, sw.get_row_status(), sw.last_residuals())
    V, st, res = out["mixed"]
    np.testing.assert_array_equal(st, out["fp64"][1])
    ok = st == RowStatus.CONVERGED
    assert ok.mean() > 0.99 and np.all(res[ok] < 1e-8)
    assert np.abs(V[ok] - out["fp64"][0][ok]).max() <= TOL_V_MIXED
    sample = np.random.default_rng(5).choice(p.shape[0], 128, replace=False)
    Vo, so, _, _ = oracle_rows(g6500, sbus_rows=(p + 1j * q) / g6500.sn_mva, idx=sample)
    _check(V[sample], st[sample], res[sample], Vo, so)


def test_10000_bus_scenarios_vs_oracle():
    g = grid_by_name("case10000_synth", 0)
    n = 64
    p, q = injection_scenarios(g, n, seed=21)
    topo = scenario_outages(g, n, max_trips=2, seed=22)
    sw = ScenarioSweepGPU(g.as_tuple(), init_from_n_powerflow=False, precision="mixed", nb_iter=10,
                          scheduling="continuous", tol=1e-8, start="base", strategy="base_chord")
    sw.set_branch_data(*g.branch_data())
    sw.set_injections(p, q, g.sn_mva)
    sw.set_topology(topo)
    sw.compute()
    sample = np.arange(0, n, 2)
    Vo, so, _, _ = oracle_rows(g, trips=topo, sbus_rows=(p + 1j * q) / g.sn_mva, idx=sample)
    _check(sw.V_results[sample], sw.get_row_status()[sample], sw.last_residuals()[sample], Vo, so)
