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


def step_scale(dx, n_pvpq, max_dva, max_dvm):
    """The MaxVoltageChange step scaling (reduce_step_norms_kernel +
    apply_step_scale_kernel, ``src/_cpp/acpf_nr_kernels.cu:677-726``): the
    whole step times alpha = min(1, max_dVa / max|dtheta|, max_dVm / max|dVm|),
    applied only when a maximum exceeds its bound."""
    dth, dvm = np.abs(dx[:n_pvpq]), np.abs(dx[n_pvpq:])
    mdt = float(dth.max()) if dth.size else 0.0
    mdv = float(dvm.max()) if dvm.size else 0.0
    alpha = 1.0
    if mdt > max_dva:
        alpha = min(alpha, max_dva / mdt)
    if mdv > max_dvm:
        alpha = min(alpha, max_dvm / mdv)
    return dx if alpha == 1.0 else dx * alpha


def newton_step(Y, V, F, pvpq, pq, scaling=None):
    """One full Newton step from V with mismatch F: J at V, dx = J^-1 F, then
    the polar update (acpf_nr.cu nr_iter_step: SpMV, fill F, fill J,
    factorize, solve, update V).  A step that cannot be taken (a non-finite
    mismatch or a singular J) leaves every unknown NaN, as NaN propagates
    through the reference's solve.  ``scaling`` = (max_dVa, max_dVm) turns on
    the MaxVoltageChange step scaling (``step_scale``)."""
    if np.all(np.isfinite(F)):
        J = jacobian(Y, V, pvpq, pq)
        try:
            dx = spla.splu(J, permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.1,
                           options=dict(SymmetricMode=True)).solve(F)
        except RuntimeError:
            dx = np.full(F.size, np.nan)
    else:
        dx = np.full(F.size, np.nan)
    if scaling is not None and np.all(np.isfinite(dx)):
        dx = step_scale(dx, pvpq.size, *scaling)
    return update_v(V, dx, pvpq, pq)


def nr_solve(Y, V0, Sbus, pv, pq, max_iter=10, tol=1e-8, mode="continuous", k=1, scaling=None):
    """One NR solve under one of the reference's three schedules.

    mode="continuous" (``src/_cpp/contingency/batch_pf_driver.cu:2691-2724``):
    rounds of ``k`` steps (``nb_iter_per_round``); after each round the
    residual of the current V decides: not finite -> DIVERGED, < tol ->
    CONVERGED, steps >= max_iter -> MAX_ITER, else another round.  A row
    always runs its first round, also when it starts converged, so ``iters``
    is a positive multiple of k.
    mode="fixed" (the chunked schedule, ``src/_cpp/contingency/driver.cuh:136-259``
    + the residual pass ``batch_pf_driver.cu:2019-2061``): exactly ``max_iter``
    steps, then the residual of the final V decides.
    mode="single" (``src/_cpp/acpf_nr.cu:505-561``): each iteration takes a
    full step, then tests the mismatch evaluated BEFORE it; a converged
    solve reports the step that followed the passing test and returns the V
    after it; no pass within ``max_iter`` steps is MAX_ITER (DIVERGED when the
    last mismatch is not finite).  ``residual`` is the last mismatch
    evaluated (for a converged single solve: the one that passed).
    "converge" is an alias of "continuous".  ``scaling`` = (max_dVa, max_dVm)
    scales every step (``step_scale``).

    Returns (V, status, iters, residual).
    """
    Y = sp.csr_matrix(Y)
    pvpq, pq_, _ = j_layout(Y.shape[0], pv, pq)
    V = np.asarray(V0, dtype=np.complex128).copy()
    k = max(int(k), 1)
    if mode == "converge":
        mode = "continuous"
    if mode not in ("continuous", "fixed", "single"):
        raise ValueError(f"unknown mode {mode!r}")
    it = 0
    while True:
        F = mismatch(Y, V, Sbus, pvpq, pq_)
        nrm = nan_inf_norm(F)
        finite = np.isfinite(nrm)
        if mode == "fixed":
            if it >= max_iter:
                return V, (DIVERGED if not finite else CONVERGED if nrm < tol else MAX_ITER), it, nrm
        elif mode == "single":
            if it >= max_iter:
                return V, (DIVERGED if not finite else MAX_ITER), it, nrm
        elif it > 0 and it % k == 0:
            if not finite:
                return V, DIVERGED, it, nrm
            if nrm < tol:
                return V, CONVERGED, it, nrm
            if it >= max_iter:
                return V, MAX_ITER, it, nrm
        V = newton_step(Y, V, F, pvpq, pq_, scaling)
        it += 1
        if mode == "single" and nrm < tol:
            return V, CONVERGED, it, nrm


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
            if r < 0 or c < 0:
                continue  # an open endpoint has no Ybus row or column (:53-75)
            lo, hi = Y.indptr[r], Y.indptr[r + 1]
            k = lo + int(np.searchsorted(Y.indices[lo:hi], c))
            assert k < hi and Y.indices[k] == c
            Y.data[k] -= v
    return Y


def islands(n_bus, f, t, branch_ids):
    """True when removing ``branch_ids`` disconnects the branch graph."""
    from scipy.sparse.csgraph import connected_components
    f, t = np.asarray(f), np.asarray(t)
    keep = (f >= 0) & (t >= 0)  # a branch open at one end joins no two buses
    keep[list(branch_ids)] = False
    A = sp.coo_matrix((np.ones(keep.sum()), (f[keep], t[keep])), shape=(n_bus, n_bus))
    ncomp, _ = connected_components(A, directed=False)
    return ncomp > 1


def main_component(n_bus, f, t, branch_ids):
    """Boolean mask of the buses of the largest connected component once
    ``branch_ids`` are out: the most buses, on a tie the component holding
    the lowest bus (compute_component_masks,
    contingency_analysis_helper.cpp:657-700: components labelled from bus 0
    upwards, the first largest wins)."""
    from scipy.sparse.csgraph import connected_components
    f, t = np.asarray(f), np.asarray(t)
    keep = (f >= 0) & (t >= 0)
    keep[list(branch_ids)] = False
    A = sp.coo_matrix((np.ones(keep.sum()), (f[keep], t[keep])), shape=(n_bus, n_bus))
    _, lab = connected_components(A, directed=False)
    # scipy labels components in order of their lowest bus, as the reference
    counts = np.bincount(lab)
    return lab == int(np.argmax(counts))


def contingency_sweep(Y, V0, Sbus, pv, pq, branch_rows, f, t, yff, yft, ytf, ytt,
                      max_iter=10, tol=1e-8, mode="continuous", k=1, handle_disconnected=False, scaling=None):
    """Solve every row (a list of tripped-branch lists).  Islanding rows are
    NOT_SIMULATED with NaN voltages (contingency_analysis_helper.cpp:634-651),
    or, with ``handle_disconnected``, solved on their largest component with
    the other buses masked (identity rows, zero mismatch:
    acpf_nr_kernels.cu:219; NaN voltages in the result) unless that masks a
    slack bus (then NOT_SIMULATED).  Masking a decoupled part is the same as
    leaving its buses out of the unknowns and the mismatch, which is how it
    is restated here."""
    n = Y.shape[0]
    pv, pq = np.asarray(pv), np.asarray(pq)
    slack = np.ones(n, dtype=bool)
    slack[pv] = False
    slack[pq] = False
    out_V = np.full((len(branch_rows), n), np.nan + 0j)
    status = np.full(len(branch_rows), NOT_SIMULATED, dtype=np.int32)
    iters = np.zeros(len(branch_rows), dtype=np.int32)
    res = np.full(len(branch_rows), np.nan)
    for r, ids in enumerate(branch_rows):
        live = None
        if islands(n, f, t, ids):
            if not handle_disconnected:
                continue
            live = main_component(n, f, t, ids)
            if slack[~live].any():
                continue
        Yr = trip_branches(Y, ids, f, t, yff, yft, ytf, ytt)
        if live is None:
            V, st, it, nrm = nr_solve(Yr, V0, Sbus, pv, pq, max_iter, tol, mode, k, scaling)
        else:
            V, st, it, nrm = nr_solve(Yr, V0, Sbus, pv[live[pv]], pq[live[pq]], max_iter, tol, mode, k, scaling)
            V = np.where(live, V, np.nan + 0j)
        out_V[r], status[r], iters[r], res[r] = V, st, it, nrm
    return out_V, status, iters, res


def injection_sweep(Y, V0, Sbus_rows, pv, pq, max_iter=10, tol=1e-8, mode="continuous", k=1, scaling=None):
    """Solve one row per Sbus row."""
    B, n = Sbus_rows.shape
    out_V = np.empty((B, n), dtype=np.complex128)
    status = np.empty(B, dtype=np.int32)
    iters = np.empty(B, dtype=np.int32)
    res = np.empty(B)
    for r in range(B):
        V, st, it, nrm = nr_solve(Y, V0, Sbus_rows[r], pv, pq, max_iter, tol, mode, k, scaling)
        out_V[r], status[r], iters[r], res[r] = V, st, it, nrm
    return out_V, status, iters, res


def branch_flows(V, f, t, yff, yft, ytf, ytt):
    """Complex power entering every branch at its from and to ends, the
    reference's formulas (``src/_cpp/acpf_nr_kernels.cu:87-183``):
    S_from = V_f conj(yff V_f + yft V_t), S_to = V_t conj(ytf V_f + ytt V_t)."""
    V = np.asarray(V)
    f = np.asarray(f)
    t = np.asarray(t)
    # an open end (negative endpoint) has V = 0 and carries no power
    hf, ht = f >= 0, t >= 0
    Vf = np.where(hf, V[np.where(hf, f, 0)], 0)
    Vt = np.where(ht, V[np.where(ht, t, 0)], 0)
    return (np.where(hf, Vf * np.conj(yff * Vf + yft * Vt), 0),
            np.where(ht, Vt * np.conj(ytf * Vf + ytt * Vt), 0))


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


def branch_currents_amps(V, f, t, yff, yft, ytf, ytt, bus_vn_kv, sn_mva):
    """Branch terminal current magnitudes in amperes (the reference's host
    check, ``src/gpusim2grid/acpf_nr/_branch_flows.py``, same formulas as its
    ``compute_branch_flows_kernel``): I_or = yff V_f + yft V_t at the from end,
    I_ex = ytf V_f + ytt V_t at the to end, each scaled by its own bus's base
    current sn_mva / (sqrt(3) vn_kv) kA.  An open end (negative endpoint) has
    V = 0, carries 0 A, and its base falls back to the other end's."""
    V = np.asarray(V)
    f = np.asarray(f)
    t = np.asarray(t)
    vn = np.asarray(bus_vn_kv, dtype=np.float64)
    hf, ht = f >= 0, t >= 0
    fz, tz = np.where(hf, f, 0), np.where(ht, t, 0)
    Vf = np.where(hf, V[fz], 0)
    Vt = np.where(ht, V[tz], 0)
    i_or = np.where(hf, np.abs(yff * Vf + yft * Vt), 0.0)
    i_ex = np.where(ht, np.abs(ytf * Vf + ytt * Vt), 0.0)
    vf = np.where(hf, vn[fz], np.where(ht, vn[tz], 1.0))
    vt = np.where(ht, vn[tz], vf)
    base = lambda kv: sn_mva * 1e6 / (np.sqrt(3.0) * kv * 1e3)
    return i_or * base(vf), i_ex * base(vt)
