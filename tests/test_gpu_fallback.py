"""FP64 fallback of mixed-precision sweeps: rows a mixed run leaves
MAX_ITER or DIVERGED are re-solved in plain FP64 from Vinit
(gs2g_run_subset) and that verdict stands.  With a 3-step budget most rows
need it, so the final statuses must equal a pure FP64 run's and the
re-solved rows must be bit-identical to it."""

import numpy as np
import pytest

from gpusim2grid_b200 import InjectionSweepGPU, RowStatus
from gpusim2grid_b200.synthetic import injection_scenarios

pytestmark = pytest.mark.gpu


def _sweep(g, p, q, precision, fallback):
    sw = InjectionSweepGPU(g.as_tuple(), init_from_n_powerflow=False, precision=precision, nb_iter=3,
                           scheduling="continuous", start="flat", strategy="refactor_every")
    sw.fallback = fallback
    sw.set_injections(p, q, g.sn_mva)
    sw.compute()
    return sw


def test_fp64_fallback_decides_rows_mixed_leaves_unconverged(g118):
    p, q = injection_scenarios(g118, 128, seed=12)
    ref = _sweep(g118, p, q, "fp64", None)
    raw = _sweep(g118, p, q, "mixed", None)
    fb = _sweep(g118, p, q, "mixed", "fp64")
    st_raw = raw.get_row_status()
    redo = (st_raw == RowStatus.MAX_ITER) | (st_raw == RowStatus.DIVERGED)
    assert redo.sum() > 0 and fb.fallback_rows == int(redo.sum())
    np.testing.assert_array_equal(fb.get_row_status(), ref.get_row_status())
    np.testing.assert_array_equal(fb.V_results[redo], ref.V_results[redo])
    np.testing.assert_array_equal(fb.get_row_iterations()[redo], ref.get_row_iterations()[redo])
    # rows mixed precision converged keep their own result
    np.testing.assert_array_equal(fb.V_results[~redo], raw.V_results[~redo])


def test_no_fallback_in_fp64_or_chunked(g118):
    p, q = injection_scenarios(g118, 16, seed=13)
    sw = _sweep(g118, p, q, "fp64", "fp64")
    assert sw.fallback_rows == 0
    ch = InjectionSweepGPU(g118.as_tuple(), init_from_n_powerflow=False, precision="mixed", nb_iter=2,
                           start="flat")  # chunked: exactly nb_iter steps, no fallback
    ch.set_injections(p, q, g118.sn_mva)
    ch.compute()
    assert ch.fallback_rows == 0
