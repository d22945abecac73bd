"""The per-unit algorithmic bytes behind the bench's roofline, checked on the
CPU against the per-row-iteration formula they restate (shared structure
amortised to zero), with the planner's own counts for the 2000-bus grid."""

import os
import sys

import numpy as np

from gpusim2grid_b200._native import lib

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def _info(g):
    Y = g.Ybus
    return lib.plan_info(g.n_bus, Y.indptr.astype(np.int32), Y.indices.astype(np.int32), g.pv, g.pq, 1)


def test_bytes_per_lu_and_per_step(g2000):
    a = _info(g2000)
    n, d, nJ, nLU = a["n_bus"], a["dim_j"], a["nnz_j"], a["nnz_lu"]
    for w in (4, 8):
        per_factor, per_iter = bench.algorithmic_bytes(a, w)
        # one factorization: J write + J read by the LU + factor write
        assert per_factor == w * nJ + w * nJ + w * nLU
        # one Newton step: V read, outage edits, F write, factor read by the
        # solves, rhs/x, dx read, V read-modify-write
        assert per_iter == 16 * n + 16 * 4 + 8 * d + w * nLU + 2 * 8 * d + 8 * d + 32 * n
    # FP64, one factorization plus one step of a 2000-bus row: about 5.7 MB,
    # most of it the factor written and read back
    f64 = sum(bench.algorithmic_bytes(a, 8))
    assert 5.0e6 < f64 < 6.5e6
    assert 2 * 8 * nLU > 0.8 * f64


def test_shared_factor_step_reads_no_factor(g2000):
    """A step on the shared base factor reads that factor from L2 once per
    four rows; as shared structure it counts zero per row."""
    a = _info(g2000)
    _, per_iter = bench.algorithmic_bytes(a, 4)
    shared = per_iter - 4 * a["nnz_lu"]
    assert 0 < shared < per_iter / 5
