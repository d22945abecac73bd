"""Batched adjoint (gs2g_solve_jt) and the differentiable sweep built on it.

* solve_JT against scipy's spsolve(J^T, b) with J the oracle's Jacobian at
  each row's converged voltage (the reference's test_batch_power_flow.py
  ``test_solve_JT_batch_matches_spsolve``): N-1 rows, an islanded row (0), a
  split row solved on its largest component, non-finite right-hand sides.
* gradients of a loss of the voltages w.r.t. the injections, through
  BatchPowerFlowFunction, against central differences of the engine's own
  solves.
"""

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from gpusim2grid_b200 import ContingencyAnalysisGPU, InjectionSweepGPU, RowStatus
from gpusim2grid_b200.synthetic import injection_scenarios, n1_branches
from oracle import nr_oracle as O

pytestmark = pytest.mark.gpu


def test_solve_jt_matches_spsolve(g118):
    rows = [[int(b)] for b in n1_branches(g118)[:6]]
    bridges = np.setdiff1d(np.arange(g118.n_branch), n1_branches(g118))
    rows += [[int(bridges[0])], [int(bridges[1]), int(n1_branches(g118)[7])]]
    ca = ContingencyAnalysisGPU(g118.as_tuple(), init_from_n_powerflow=False, nb_iter=20, scheduling="continuous",
                                tol=1e-12, start="flat", handle_disconnected_grid=True)
    ca.set_branch_data(*g118.branch_data())
    ca.add_contingencies_by_branch_id(rows)
    ca.compute()
    st = ca.get_row_status()
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    pvpq, pq_, dim = O.j_layout(g118.n_bus, pv, pq)
    assert ca.dim_J == dim
    rng = np.random.default_rng(0)
    rhs = rng.standard_normal((len(rows), dim))
    rhs[0, 3] = np.nan  # non-finite entries count as 0
    lam = ca.solve_JT(rhs)
    V = ca.V_results
    for r, ids in enumerate(rows):
        if st[r] != RowStatus.CONVERGED:
            assert np.all(lam[r] == 0)
            continue
        Yr = O.trip_branches(Y, ids, g118.branch_from, g118.branch_to, g118.yff, g118.yft, g118.ytf, g118.ytt)
        live = ~np.isnan(V[r])
        if live.all():
            J = O.jacobian(Yr, V[r], pvpq, pq_)
            exp = spla.spsolve(J.T.tocsc(), np.nan_to_num(rhs[r]))
            np.testing.assert_allclose(lam[r], exp, rtol=1e-8, atol=1e-8 * np.abs(exp).max())
        else:
            # a split row: the live block's Jacobian; the masked entries are 0
            lp = pvpq[live[pvpq]]
            lq = pq_[live[pq_]]
            J = O.jacobian(Yr, np.where(live, V[r], 0), lp, lq)
            sel = np.concatenate([np.flatnonzero(live[pvpq]), pvpq.size + np.flatnonzero(live[pq_])])
            exp = spla.spsolve(J.T.tocsc(), rhs[r][sel])
            np.testing.assert_allclose(lam[r][sel], exp, rtol=1e-8, atol=1e-8 * np.abs(exp).max())
            dead = np.setdiff1d(np.arange(dim), sel)
            assert dead.size > 0 and np.all(lam[r][dead] == 0)


def test_gradients_match_central_differences(g118):
    import torch
    from gpusim2grid_b200.differentiable import batch_power_flow
    p, q = injection_scenarios(g118, 3, seed=13)
    sw = InjectionSweepGPU(g118.as_tuple(), init_from_n_powerflow=False, nb_iter=30, scheduling="continuous",
                           tol=1e-12, start="flat")
    rng = np.random.default_rng(2)
    wm = torch.as_tensor(rng.standard_normal((3, g118.n_bus)), device="cuda")
    wa = torch.as_tensor(rng.standard_normal((3, g118.n_bus)), device="cuda")

    def loss_of(P, Q):
        V = batch_power_flow(P, Q, sw, g118.sn_mva)
        return (wm * V.abs()).sum() + (wa * torch.angle(V)).sum()

    P = torch.as_tensor(p, device="cuda").requires_grad_(True)
    Q = torch.as_tensor(q, device="cuda").requires_grad_(True)
    L = loss_of(P, Q)
    L.backward()
    gP, gQ = P.grad.cpu().numpy(), Q.grad.cpu().numpy()
    # P at the slack and Q at pv / slack buses do not move the solution
    assert np.all(gP[:, g118.slack] == 0) and np.all(gQ[:, g118.pv] == 0)
    eps = 1e-3
    checks = [(0, "p", int(g118.pq[5])), (1, "p", int(g118.pv[3])), (2, "q", int(g118.pq[11])), (0, "q", int(g118.pq[0]))]
    for r, kind, b in checks:
        out = []
        for sgn in (1, -1):
            P2, Q2 = p.copy(), q.copy()
            (P2 if kind == "p" else Q2)[r, b] += sgn * eps
            with torch.no_grad():
                out.append(float(loss_of(torch.as_tensor(P2, device="cuda"), torch.as_tensor(Q2, device="cuda"))))
        fd = (out[0] - out[1]) / (2 * eps)
        g = (gP if kind == "p" else gQ)[r, b]
        assert abs(g - fd) <= 1e-5 * max(1.0, abs(fd)), (r, kind, b, g, fd)
