"""MaxVoltageChange step scaling (the reference's scaling_max_voltage_change,
reduce_step_norms_kernel / apply_step_scale_kernel in
src/_cpp/acpf_nr_kernels.cu:677-726) against the oracle's restatement: every
Newton step multiplied by min(1, max_dVa / max|dtheta|, max_dVm / max|dVm|).
The bounds are set low enough that the flat-start steps of the 118-bus grid
are scaled."""

import numpy as np
import pytest

from conftest import TOL_V_FP64, TOL_V_MIXED
from gpusim2grid_b200 import AcPfGPU, ContingencyAnalysisGPU, RowStatus
from gpusim2grid_b200.synthetic import n1_branches
from oracle import nr_oracle as O

pytestmark = pytest.mark.gpu

BOUNDS = (0.1, 0.03)  # rad, pu: the first flat-start steps reach 0.26 rad and 0.07 pu


def _rows(g):
    return [[int(b)] for b in n1_branches(g)[:24]]


def test_fp64_rows_scaled_as_the_oracle(g118):
    """FP64, plain Newton, continuous schedule from flat: the same statuses,
    the same step counts (6-8 instead of 4-5 unscaled) and the same voltages
    as the oracle's scaled Newton."""
    rows = _rows(g118)
    ca = ContingencyAnalysisGPU(g118.as_tuple(), init_from_n_powerflow=False, precision="fp64", nb_iter=10,
                                scheduling="continuous", tol=1e-8, start="flat", scaling_max_voltage_change=True,
                                max_dVa=BOUNDS[0], max_dVm=BOUNDS[1])
    ca.set_branch_data(*g118.branch_data())
    ca.add_contingencies_by_branch_id(rows)
    ca.compute()
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    Vo, so, io, _ = O.contingency_sweep(Y, V0, S, pv, pq, rows, g118.branch_from, g118.branch_to, g118.yff,
                                        g118.yft, g118.ytf, g118.ytt, 10, 1e-8, scaling=BOUNDS)
    np.testing.assert_array_equal(ca.get_row_status(), so)
    np.testing.assert_array_equal(ca.get_row_iterations(), io)
    assert io.min() > 5  # the steps were scaled
    ok = so == RowStatus.CONVERGED
    assert ok.all() and np.abs(ca.V_results - Vo).max() <= TOL_V_FP64


def test_single_solve_scaled_as_the_oracle(g118):
    """AcPfGPU (the single-solve order: step, then test the mismatch before
    it) with the scaling: the oracle's iteration count and voltage."""
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    ac = AcPfGPU(g118.as_tuple(), precision="fp64", max_iter=10, tol=1e-8, init_from_n_powerflow=False,
                 scaling_max_voltage_change=True, max_dVa=BOUNDS[0], max_dVm=BOUNDS[1])
    t = ac.timings
    Vo, so, io, _ = O.nr_solve(Y, V0, S, pv, pq, 10, 1e-8, mode="single", scaling=BOUNDS)
    assert t.converged and so == O.CONVERGED and t.nb_iter == io
    assert np.abs(ac.solve() - Vo).max() <= TOL_V_FP64


def test_base_chord_rows_with_scaled_steps_leave_the_chord(g118):
    """Mixed precision on the shared base factor: a row whose chord step would
    be scaled leaves the chord for its own factor, where its steps are scaled.
    With bounds of 0.05 rad / 0.01 pu the rows whose first step from the base
    case is larger (about a fifth of them) do so; every row converges to the
    unscaled oracle's solution."""
    rows = _rows(g118)
    out = {}
    for scaled in (False, True):
        ca = ContingencyAnalysisGPU(g118.as_tuple(), init_from_n_powerflow=False, precision="mixed", nb_iter=30,
                                    scheduling="continuous", tol=1e-8, start="base", strategy="base_chord",
                                    scaling_max_voltage_change=scaled, max_dVa=0.05, max_dVm=0.01)
        ca.set_branch_data(*g118.branch_data())
        ca.add_contingencies_by_branch_id(rows)
        ca.compute()
        out[scaled] = (ca.V_results, ca.get_row_status(), ca.get_row_factorizations())
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    Vo, so, _, _ = O.contingency_sweep(Y, V0, S, pv, pq, rows, g118.branch_from, g118.branch_to, g118.yff,
                                       g118.yft, g118.ytf, g118.ytt, 10, 1e-8)
    for scaled, (V, st, fac) in out.items():
        np.testing.assert_array_equal(st, so)
        assert np.abs(V - Vo).max() <= TOL_V_MIXED
    assert out[True][2].sum() > out[False][2].sum()  # scaled rows factor their own Jacobian
