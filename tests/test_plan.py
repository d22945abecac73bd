"""The host symbolic planner, through the C-ABI's GPU-free gs2g_plan_info."""

import numpy as np
import pytest

from gpusim2grid_b200._native import lib


def _info(g, policy=1):
    Y = g.Ybus
    return lib.plan_info(g.n_bus, Y.indptr.astype(np.int32), Y.indices.astype(np.int32), g.pv, g.pq, policy)


def test_plan_dimensions(g118, g2000):
    for g in (g118, g2000):
        a = _info(g)
        assert a["dim_j"] == a["n_pvpq"] + a["n_pq"] == (g.n_bus - 1) + g.pq.size
        assert a["nnz_j"] == 4 * 0 + a["nnz_j"]  # reported
        assert a["head_dim"] + a["tail_dim"] == a["dim_j"]
        assert a["tail_dim"] >= a["tail_dim_exact"] > 0
        assert a["nnz_lu"] >= a["nnz_j"]
        e = _info(g, 0)
        assert e["tail_dim"] == e["tail_dim_exact"]
        # the exact tail is a clique: every dense madd is counted once
        assert e["dense_madds"] == sum((e["tail_dim"] - 1 - k) ** 2 for k in range(e["tail_dim"]))


def test_plan_is_deterministic(g2000):
    a, b = _info(g2000), _info(g2000)
    a.pop("plan_ms"); b.pop("plan_ms")
    assert a == b


def test_plan_fill_matches_scipy_mmd_order_of_magnitude(g2000):
    import scipy.sparse.linalg as spla
    from oracle.nr_oracle import j_layout, jacobian
    Y, V0, *_ = g2000.as_tuple()
    pvpq, pq, d = j_layout(g2000.n_bus, g2000.pv, g2000.pq)
    J = jacobian(Y, V0, pvpq, pq)
    lu = spla.splu(J, permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.0, options=dict(SymmetricMode=True))
    ref = lu.L.nnz + lu.U.nnz - d
    # our minimum-degree order is at least as good as SuperLU's MMD here, and
    # the dense-tail extension adds at most ~25 % explicit zeros
    assert _info(g2000, 0)["nnz_lu"] <= 1.05 * ref
    assert _info(g2000, 1)["nnz_lu"] <= 1.25 * ref


def test_plan_rejects_bad_input(g118):
    Y = g118.Ybus
    ip, ix = Y.indptr.astype(np.int32), Y.indices.astype(np.int32)
    with pytest.raises(ValueError):
        lib.plan_info(g118.n_bus, ip, ix, g118.pv, np.concatenate([g118.pq, g118.pv[:1]]), 1)
    with pytest.raises(ValueError):
        bad = ix.copy(); bad[0] = g118.n_bus + 5
        lib.plan_info(g118.n_bus, ip, bad, g118.pv, g118.pq, 1)
