"""Run the FP64 CPU oracle over many rows in a pool of spawned processes
(test helper, not a test module).  Spawned workers start clean, so the pool
is safe to use next to a CUDA context in the parent."""

from __future__ import annotations

import multiprocessing as mp
import os

import numpy as np


def _solve_chunk(payload):
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    from oracle import nr_oracle as O
    (Y, V0, S, pv, pq, f, t, yff, yft, ytf, ytt, rows, max_iter, tol) = payload
    out = []
    for r, trips, sb in rows:
        if trips and O.islands(Y.shape[0], f, t, trips):
            out.append((r, np.full(Y.shape[0], np.nan + 0j), O.NOT_SIMULATED, 0, np.nan))
            continue
        Yr = O.trip_branches(Y, trips, f, t, yff, yft, ytf, ytt) if trips else Y
        V, st, it, res = O.nr_solve(Yr, V0, S if sb is None else sb, pv, pq, max_iter, tol)
        out.append((r, V, st, it, res))
    return out


def oracle_rows(g, trips=None, sbus_rows=None, idx=None, max_iter=10, tol=1e-8, workers=None):
    """FP64 flat-start NR (continuous schedule) of the selected rows of a
    workload: ``trips`` a list of tripped-branch lists, ``sbus_rows`` a
    (rows, n_bus) complex per-unit array, either may be None.  Returns
    (V, status, iters, residual) for the rows ``idx`` (default: all)."""
    Y, V0, S, _, _, pv, pq = g.as_tuple()
    n = len(trips) if trips is not None else sbus_rows.shape[0]
    idx = np.arange(n) if idx is None else np.asarray(idx)
    rows = [(int(k), list(trips[k]) if trips is not None else [], None if sbus_rows is None else sbus_rows[k])
            for k in idx]
    workers = max(1, min(workers or os.cpu_count() or 1, len(rows)))
    chunks = [rows[i::workers] for i in range(workers)]
    payload = [(Y, V0, S, pv, pq, g.branch_from, g.branch_to, g.yff, g.yft, g.ytf, g.ytt, c, max_iter, tol)
               for c in chunks if c]
    with mp.get_context("spawn").Pool(len(payload)) as pool:
        parts = pool.map(_solve_chunk, payload)
    got = {r: (V, st, it, res) for part in parts for (r, V, st, it, res) in part}
    V = np.stack([got[int(k)][0] for k in idx])
    st = np.array([got[int(k)][1] for k in idx], dtype=np.int32)
    it = np.array([got[int(k)][2] for k in idx], dtype=np.int32)
    res = np.array([got[int(k)][3] for k in idx])
    return V, st, it, res
