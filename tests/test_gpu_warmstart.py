"""Learned warm start end to end on the GPU: train the MLP on GPU-solved
operating points of the 118-bus grid, then run the N-1 sweep from its
predictions.  The answers must equal the flat-start FP64 answers within the
mixed-precision bar, and the learned start must take fewer Newton steps and
LU factorizations than a flat start.  A start that fails is restarted from
Vinit inside the same launch."""

import numpy as np
import pytest

from conftest import TOL_V_MIXED
from gpusim2grid_b200 import ContingencyAnalysisGPU, InjectionSweepGPU, RowStatus
from gpusim2grid_b200.synthetic import injection_scenarios, n1_branches
from oracle import nr_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def learned118(g118):
    from gpusim2grid_b200.warmstart import LearnedStart
    ls = LearnedStart(g118, hidden=256, layers=2, seed=0)
    rep = ls.train(n_rows=16384, epochs=30, batch=512, lr=1e-3, lr_decay=0.9, seed=1)
    # random operating points past a feasibility limit do not converge and
    # are left out of the training set
    assert rep["n_unconverged"] < 0.01 * rep["n_rows"]
    assert rep["loss"][-1] < 0.1 * rep["loss"][0]
    return ls


def _sweep(g, precision, start, learned=None):
    ca = ContingencyAnalysisGPU(g.as_tuple(), init_from_n_powerflow=False, precision=precision, nb_iter=10,
                                scheduling="continuous", tol=1e-8, start="flat", strategy="adaptive")
    ca.set_branch_data(*g.branch_data())
    ca.add_contingencies_by_branch_id([[int(b)] for b in n1_branches(g)])
    if learned is not None:
        ca.set_learned_start(learned)
    ca.start = start
    ca.compute()
    return ca


def test_learned_start_n1_parity_and_fewer_steps(g118, learned118):
    ref = _sweep(g118, "fp64", "flat")
    flat = _sweep(g118, "mixed", "flat")
    warm = _sweep(g118, "mixed", "learned", learned118)
    assert np.all(ref.get_row_status() == RowStatus.CONVERGED)
    assert np.all(warm.get_row_status() == RowStatus.CONVERGED)
    assert np.all(warm.last_residuals() < 1e-8)
    assert np.abs(warm.V_results - ref.V_results).max() < TOL_V_MIXED
    assert warm.get_row_iterations().sum() < flat.get_row_iterations().sum()
    assert warm.get_row_factorizations().sum() < flat.get_row_factorizations().sum()
    assert warm.warm_report["n_rescued"] == 0
    # a sample against the FP64 oracle as well
    rows = n1_branches(g118)
    sample = np.random.default_rng(3).choice(len(rows), 8, replace=False)
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    Vo, so, _, _ = O.contingency_sweep(Y, V0, S, pv, pq, [[int(rows[r])] for r in sample], g118.branch_from,
                                       g118.branch_to, g118.yff, g118.yft, g118.ytf, g118.ytt, 10, 1e-8)
    assert np.all(so == O.CONVERGED)
    assert np.abs(warm.V_results[sample] - Vo).max() < TOL_V_MIXED


def test_learned_start_injection_rows(g118, learned118):
    p, q = injection_scenarios(g118, 512, seed=11)
    out = []
    for start in ("flat", "learned"):
        sw = InjectionSweepGPU(g118.as_tuple(), init_from_n_powerflow=False, precision="mixed", nb_iter=10,
                               scheduling="continuous", start="flat", strategy="adaptive")
        sw.set_injections(p, q, g118.sn_mva)
        if start == "learned":
            sw.set_learned_start(learned118)
        sw.compute()
        out.append(sw)
    flat, warm = out
    assert np.all(warm.get_row_status() == RowStatus.CONVERGED)
    assert np.abs(warm.V_results - flat.V_results).max() < TOL_V_MIXED
    assert warm.get_row_iterations().sum() < flat.get_row_iterations().sum()


def test_failed_start_rows_are_rescued(g118):
    """Half the rows get a NaN start, the others Vinit.  (1) With a (solved)
    base case every row begins from the base V instead -- its mismatch is
    below both -- and runs exactly as a base-start row.  (2) On a session
    without a base case the NaN rows end DIVERGED at step 0 and restart from
    Vinit in the same launch, matching the flat-start run."""
    from gpusim2grid_b200._common import grid_arrays, make_session
    from gpusim2grid_b200._native import lib
    p, q = injection_scenarios(g118, 64, seed=4)
    V0 = np.tile(g118.vinit(), (64, 1))
    V0[::2] = np.nan
    kw = dict(init_from_n_powerflow=False, precision="mixed", nb_iter=10, scheduling="continuous")
    base = InjectionSweepGPU(g118.as_tuple(), start="base", **kw)
    base.set_injections(p, q, g118.sn_mva)
    base.compute()
    sw = InjectionSweepGPU(g118.as_tuple(), start="flat", **kw)
    sw.set_injections(p, q, g118.sn_mva)
    sw.set_start_voltages(V0)
    sw.compute()
    t = sw.session.timings()
    assert t["n_base_start"] == 64 and t["n_rescued"] == 0
    assert np.all(sw.get_row_status() == RowStatus.CONVERGED)
    np.testing.assert_array_equal(sw.get_row_iterations(), base.get_row_iterations())
    assert np.abs(sw.V_results - base.V_results).max() < TOL_V_MIXED

    s = make_session(grid_arrays(g118.as_tuple()), None)
    s.set_injections(p, q, g118.sn_mva)
    s.run(10, 1e-8, False, lib.PREC_MIXED, lib.START_VINIT, 0.0, 0, False, lib.REFACTOR_EVERY, 0.3, 3, False)
    Vf, _, stf, itf = s.results()
    assert np.all(stf == RowStatus.CONVERGED)
    s.set_start_rows(V0)
    s.run(10, 1e-8, False, lib.PREC_MIXED, lib.START_ROWS, 0.0, 0, False, lib.REFACTOR_EVERY, 0.3, 3, True)
    t = s.timings()
    assert t["n_rescued"] == 32 and t["n_base_start"] == 0
    V, _, st, it = s.results()
    assert np.all(st == RowStatus.CONVERGED)
    np.testing.assert_array_equal(it, itf)
    assert np.abs(V - Vf).max() < TOL_V_MIXED


def test_given_start_worse_than_base_begins_from_base(g118):
    """With a base case, a row whose given start has a larger mismatch than
    the base V begins from the base V (and then runs exactly as a base-start
    row); a better given start stands."""
    p, q = injection_scenarios(g118, 64, seed=6)
    kw = dict(init_from_n_powerflow=False, precision="mixed", nb_iter=10, scheduling="continuous",
              strategy="base_chord")
    base = InjectionSweepGPU(g118.as_tuple(), start="base", **kw)
    base.set_injections(p, q, g118.sn_mva)
    base.compute()
    assert np.all(base.get_row_status() == RowStatus.CONVERGED)
    sw = InjectionSweepGPU(g118.as_tuple(), start="flat", **kw)
    sw.set_injections(p, q, g118.sn_mva)
    V0 = base.V_results.copy()       # the solutions themselves: better than the base V
    V0[::2] = 0.7 * g118.vinit()     # far worse than the base V
    sw.set_start_voltages(V0)
    sw.compute()
    t = sw.session.timings()
    assert t["n_base_start"] == 32 and t["n_rescued"] == 0
    assert np.all(sw.get_row_status() == RowStatus.CONVERGED)
    np.testing.assert_array_equal(sw.get_row_iterations()[::2], base.get_row_iterations()[::2])
    assert np.all(sw.get_row_iterations()[1::2] <= 1)
    assert np.abs(sw.V_results - base.V_results).max() < TOL_V_MIXED


def test_sparse_first_layer_equals_the_gemm(g118, learned118):
    """Rows without injection part (outage rows at the base injections) take
    the network's first layer from the few input columns their tripped
    branches reach.  Its pre-activations must equal the GEMM of the full
    standardised inputs up to fp32 summation order: rows with one trip,
    rows with three, an empty row, and a row with more contributions than
    the kernel's shared list holds (the full dot product in the CTA).  The
    start voltages then agree to the bf16 activations' precision."""
    ls = learned118
    net = ls.net
    rng = np.random.default_rng(7)
    trips = ([[int(b)] for b in n1_branches(g118)[:40]]
             + [sorted(int(b) for b in rng.choice(g118.n_branch, 3, replace=False)) for _ in range(20)]
             + [list(range(70)), []])
    n = len(trips)
    X, _ = ls.inputs(None, trips, n)
    net.predict(X)
    dense = net._buffers(X.shape[0], False)["pre"][0][:n].clone()
    tp, ti = ls._device_trips(trips)
    net.predict_trips(tp, ti, ls._br_cols32, ls._br_vals32, n)
    sparse = net._buffers(X.shape[0], False)["pre"][0][:n].clone()
    assert float((sparse - dense).abs().max()) <= 1e-3 * float(dense.abs().max())
    ls.sparse_first_layer = False
    v_dense = ls.start_voltages(None, trips, n).cpu().numpy()
    ls.sparse_first_layer = True
    v_sparse = ls.start_voltages(None, trips, n).cpu().numpy()
    assert np.abs(v_sparse - v_dense).max() < 1e-2
