"""CPU oracle for the batched Newton–Raphson AC power flow (FP64, numpy/scipy).

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import this
module, and only as the checker or the timed CPU baseline.  The product path
(``gpusim2grid_b200``) never imports it and has no CPU fallback.

It restates, in plain numpy + scipy ``splu``, the algorithm of the reference's
bare ``[pvpq | pq]`` Newton–Raphson path:

* J layout: P/θ rows+cols on ``sorted(pv ∪ pq)`` at ``[0, n_pvpq)``, Q/Vm on
  ``pq`` in input order at ``[n_pvpq, dim_J)`` (``src/_cpp/acpf_nr.cu:130-236``,
  ``:645-685``).
* Mismatch ``F = -[Re, Im](V∘conj(Y V) − Sbus)`` at those rows
  (``src/_cpp/acpf_nr_kernels.cu:493-557``).
* Jacobian from MATPOWER's dS/dVa, dS/dVm (``src/_cpp/acpf_nr_kernels.cu:559-650``,
  ``tests/python/_jacobian_ref.py:15-44``).
* Update Va on pvpq, then Vm on pq, in polar form
  (``src/_cpp/acpf_nr_kernels.cu:728-790``).
* Convergence ``‖F‖∞ < tol``, NaN-sticky (``src/_cpp/acpf_nr.cu:520-561``;
  ``src/_cpp/contingency/row_status.hpp:33-50``).
* Branch-trip Ybus deltas (``src/_cpp/contingency_analysis_helper.cpp:23-84``).
* Sbus ``(p + j q) / sn_mva`` (``src/_cpp/injection_sweep_session.cu:239-245``).

The lightsim2grid KLU oracle the reference tests against is not installable
here; parity of this restatement is pinned by the known-answer and invariance
tests of ``tests/test_oracle.py`` (power balance recomputed independently,
Jacobian against finite differences, branch-trip deltas against a Ybus rebuilt
without the branch) and by the committed golden vectors in ``tests/golden/``.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

CONVERGED, MAX_ITER, DIVERGED, NOT_SIMULATED = 0, 1, 2, 3


def j_layout(n_bus, pv, pq):
    """(pvpq, pq, dim_J): the reference's J row/col ordering."""
    pvpq = np.sort(np.concatenate([np.asarray(pv), np.asarray(pq)])).astype(np.int64)
    pq = np.asarray(pq, dtype=np.int64)
    return pvpq, pq, pvpq.size + pq.size


def mismatch(Y, V, Sbus, pvpq, pq):
    """F = -[ΔP(pvpq), ΔQ(pq)] (acpf_nr_kernels.cu:493-557)."""
    I = Y @ V
    S = V * np.conj(I) - Sbus
    return -np.concatenate([S.real[pvpq], S.imag[pq]])


def dS_dV(Y, V):
    """MATPOWER dS/dVa, dS/dVm (tests/python/_jacobian_ref.py:15-44)."""
    I = Y @ V
    n = V.size
    diagV = sp.diags(V)
    diagI = sp.diags(I)
    Vnorm = V / np.abs(V)
    diagVnorm = sp.diags(Vnorm)
    dS_dVa = 1j * diagV @ np.conj(diagI - Y @ diagV)
    dS_dVm = diagV @ np.conj(Y @ diagVnorm) + np.conj(diagI) @ diagVnorm
    return sp.csr_matrix(dS_dVa), sp.csr_matrix(dS_dVm)


def jacobian(Y, V, pvpq, pq):
    """J = [[Re dSdVa[pvpq,pvpq], Re dSdVm[pvpq,pq]], [Im dSdVa[pq,pvpq], Im dSdVm[pq,pq]]]."""
    dVa, dVm = dS_dV(Y, V)
    J11 = dVa[pvpq][:, pvpq].real
    J12 = dVm[pvpq][:, pq].real
    J21 = dVa[pq][:, pvpq].imag
    J22 = dVm[pq][:, pq].imag
    return sp.bmat([[J11, J12], [J21, J22]], format="csc")


def update_v(V, dx, pvpq, pq):
    """Va += dx[θ] on pvpq, then Vm += dx[vm] on pq (polar; acpf_nr_kernels.cu:728-790)."""
    V = V.copy()
    n_pvpq = pvpq.size
    vm = np.abs(V[pvpq])
    va = np.angle(V[pvpq]) + dx[:n_pvpq]
    V[pvpq] = vm * np.exp(1j * va)
    vm = np.abs(V[pq]) + dx[n_pvpq:]
    va = np.angle(V[pq])
    V[pq] = vm * np.exp(1j * va)
    return V


def nan_inf_norm(F):
    """‖F‖∞ that returns NaN as soon as any entry is NaN (acpf_nr.cu:116-125)."""
    if F.size == 0:
        return 0.0
    if np.isnan(F).any():
        return float("nan")
    return float(np.max(np.abs(F)))


def nr_solve(Y, V0, Sbus, pv, pq, max_iter=10, tol=1e-8, mode="converge"):
    """One NR solve.

    mode="converge": evaluate F(V_k); stop with CONVERGED once ‖F‖∞ < tol (no
    further step); otherwise step.  ``iters`` counts Newton steps taken.
    mode="fixed": take exactly ``max_iter`` steps without checking, then report
    the residual of the final V (the reference's chunked schedule,
    ``src/_cpp/contingency/driver.cuh:136-259`` + the residual pass).

    Returns (V, status, iters, residual).
    """
    Y = sp.csr_matrix(Y)
    pvpq, pq_, _ = j_layout(Y.shape[0], pv, pq)
    V = np.asarray(V0, dtype=np.complex128).copy()
    it = 0
    while True:
        F = mismatch(Y, V, Sbus, pvpq, pq_)
        nrm = nan_inf_norm(F)
        if mode == "converge":
            if not np.isfinite(nrm):
                return V, DIVERGED, it, nrm
            if nrm < tol:
                return V, CONVERGED, it, nrm
        if it >= max_iter:
            if not np.isfinite(nrm):
                return V, DIVERGED, it, nrm
            return V, (CONVERGED if nrm < tol else MAX_ITER), it, nrm
        J = jacobian(Y, V, pvpq, pq_)
        try:
            dx = spla.splu(J, permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.1,
                            options=dict(SymmetricMode=True)).solve(F)
        except RuntimeError:
            return V, DIVERGED, it, float("nan")
        V = update_v(V, dx, pvpq, pq_)
        it += 1


def trip_branches(Y, branch_ids, f, t, yff, yft, ytf, ytt):
    """Ybus with the given branches' π-model admittances subtracted, pattern
    kept (contingency_analysis_helper.cpp:23-84: Yff at (f,f), Ytt at (t,t),
    Yft at (f,t), Ytf at (t,f); a branch named twice is tripped once)."""
    Y = sp.csr_matrix(Y, copy=True)
    Y.sort_indices()
    seen = []
    for l in branch_ids:
        l = int(l)
        if l in seen:
            continue
        seen.append(l)
        i, j = int(f[l]), int(t[l])
        for (r, c, v) in ((i, i, yff[l]), (j, j, ytt[l]), (i, j, yft[l]), (j, i, ytf[l])):
            lo, hi = Y.indptr[r], Y.indptr[r + 1]
            k = lo + int(np.searchsorted(Y.indices[lo:hi], c))
            assert k < hi and Y.indices[k] == c
            Y.data[k] -= v
    return Y


def islands(n_bus, f, t, branch_ids):
    """True when removing ``branch_ids`` disconnects the branch graph."""
    from scipy.sparse.csgraph import connected_components
    keep = np.ones(len(f), dtype=bool)
    keep[list(branch_ids)] = False
    A = sp.coo_matrix((np.ones(keep.sum()), (np.asarray(f)[keep], np.asarray(t)[keep])),
                      shape=(n_bus, n_bus))
    ncomp, _ = connected_components(A, directed=False)
    return ncomp > 1


def contingency_sweep(Y, V0, Sbus, pv, pq, branch_rows, f, t, yff, yft, ytf, ytt,
                      max_iter=10, tol=1e-8, mode="converge"):
    """Solve every row (a list of tripped-branch lists).  Islanding rows are
    NOT_SIMULATED with NaN voltages (contingency_analysis_helper.cpp:634-651)."""
    n = Y.shape[0]
    out_V = np.full((len(branch_rows), n), np.nan + 0j)
    status = np.full(len(branch_rows), NOT_SIMULATED, dtype=np.int32)
    iters = np.zeros(len(branch_rows), dtype=np.int32)
    res = np.full(len(branch_rows), np.nan)
    for r, ids in enumerate(branch_rows):
        if islands(n, f, t, ids):
            continue
        Yr = trip_branches(Y, ids, f, t, yff, yft, ytf, ytt)
        V, st, it, nrm = nr_solve(Yr, V0, Sbus, pv, pq, max_iter, tol, mode)
        out_V[r], status[r], iters[r], res[r] = V, st, it, nrm
    return out_V, status, iters, res


def injection_sweep(Y, V0, Sbus_rows, pv, pq, max_iter=10, tol=1e-8, mode="converge"):
    """Solve one row per Sbus row."""
    B, n = Sbus_rows.shape
    out_V = np.empty((B, n), dtype=np.complex128)
    status = np.empty(B, dtype=np.int32)
    iters = np.empty(B, dtype=np.int32)
    res = np.empty(B)
    for r in range(B):
        V, st, it, nrm = nr_solve(Y, V0, Sbus_rows[r], pv, pq, max_iter, tol, mode)
        out_V[r], status[r], iters[r], res[r] = V, st, it, nrm
    return out_V, status, iters, res


def branch_flows(V, f, t, yff, yft, ytf, ytt):
    """Complex power entering every branch at its from and to ends, the
    reference's formulas (``src/_cpp/acpf_nr_kernels.cu:87-183``):
    S_from = V_f conj(yff V_f + yft V_t), S_to = V_t conj(ytf V_f + ytt V_t)."""
    V = np.asarray(V)
    f = np.asarray(f)
    t = np.asarray(t)
    return V[f] * np.conj(yff * V[f] + yft * V[t]), V[t] * np.conj(ytf * V[f] + ytt * V[t])


def branch_loading(V, f, t, yff, yft, ytf, ytt, rate_pu, tripped=()):
    """Per-branch loading max(|S_from|, |S_to|) / rate (0 for tripped or
    unlimited branches), the reference's limit check
    (``contingency/violation_kernels.cu:297``)."""
    Sf, St = branch_flows(V, f, t, yff, yft, ytf, ytt)
    smax = np.maximum(np.abs(Sf), np.abs(St))
    rate = np.asarray(rate_pu, dtype=np.float64)
    out = np.where(rate > 0, smax / np.where(rate > 0, rate, 1.0), 0.0)
    if len(tripped):
        out[list(tripped)] = 0.0
    return out
