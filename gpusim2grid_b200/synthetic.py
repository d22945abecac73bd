"""Seeded synthetic transmission grids and the batch rows run on them.

The grids follow one recipe at every size: a random spanning tree plus extra
random edges, π-model branches with r ~ U(0.005, 0.05) pu, x = r·U(3, 10),
total charging b ~ U(0, 0.05) pu, a fixed fraction of branches made
transformers with an off-nominal tap ~ U(0.95, 1.05), one slack bus plus PV
buses with V set-points ~ U(0.98, 1.05), loads with P ~ U(0, 1.5) pu and Q from a
power factor ~ U(0.9, 0.98), and generation summing to 1.02 × load split in
proportion to U(0.5, 1.5) weights.  Base power 100 MVA.

The Ybus convention is MATPOWER's π model (the one the reference's array-tuple
mode expects from its caller, ``contingency_analysis_helper.cpp:23-84`` takes
the same four per-branch admittances to trip a branch):

    yff = (ys + j b/2) / |tap|²,  yft = -ys / conj(tap),
    ytf = -ys / tap,              ytt = ys + j b/2,      ys = 1 / (r + j x).

Everything is numpy; nothing here runs on the GPU.  The generator is data, not
solver: the engine and the oracle both consume what it produces.
"""

from __future__ import annotations

import dataclasses
from typing import Optional

import numpy as np
import scipy.sparse as sp

__all__ = [
    "Grid",
    "GRID_SPECS",
    "make_grid",
    "grid_by_name",
    "build_ybus",
    "n1_branches",
    "injection_scenarios",
    "scenario_outages",
    "half_open_variant",
]


@dataclasses.dataclass
class Grid:
    """A synthetic grid in the array-tuple form the facades take.

    ``as_tuple()`` gives ``(Ybus, Vinit, Sbus, slack_ids, slack_weights, pv,
    pq)``, the explicit-array tuple of the reference's facades
    (``acpf_nr/gpu_facade.py:165``).  Vinit is the flat start: 1 pu at PQ
    buses, the set-point magnitude at PV/slack buses, angle 0.
    """

    name: str
    n_bus: int
    branch_from: np.ndarray  # int32 [n_branch]
    branch_to: np.ndarray  # int32 [n_branch]
    r: np.ndarray
    x: np.ndarray
    b: np.ndarray
    tap: np.ndarray  # 1.0 for lines
    is_trafo: np.ndarray  # bool
    slack: int
    pv: np.ndarray  # int32, sorted
    pq: np.ndarray  # int32, sorted
    vset: np.ndarray  # float64 [n_bus]; 1.0 where not a generator bus
    load_bus: np.ndarray  # int32 [n_load]
    load_p: np.ndarray  # pu
    load_q: np.ndarray  # pu
    gen_bus: np.ndarray  # int32 [n_gen]; gen 0 is the slack
    gen_p: np.ndarray  # pu
    sn_mva: float = 100.0
    seed: int = 0

    # derived
    yff: np.ndarray = None
    yft: np.ndarray = None
    ytf: np.ndarray = None
    ytt: np.ndarray = None
    Ybus: sp.csr_matrix = None
    # branches open at their to-end (branch_to = -1), see half_open_variant
    open_branches: Optional[np.ndarray] = None

    @property
    def n_branch(self) -> int:
        return int(self.branch_from.shape[0])

    def sbus(self, load_p=None, load_q=None, gen_p=None) -> np.ndarray:
        """Complex per-unit bus injections, generation minus load."""
        lp = self.load_p if load_p is None else load_p
        lq = self.load_q if load_q is None else load_q
        gp = self.gen_p if gen_p is None else gen_p
        s = np.zeros(self.n_bus, dtype=np.complex128)
        np.add.at(s, self.gen_bus, gp.astype(np.complex128))
        np.subtract.at(s, self.load_bus, lp + 1j * lq)
        return s

    def vinit(self) -> np.ndarray:
        """Flat start."""
        return self.vset.astype(np.complex128).copy()

    def as_tuple(self):
        w = np.zeros(self.n_bus)
        w[self.slack] = 1.0
        return (
            self.Ybus,
            self.vinit(),
            self.sbus(),
            np.array([self.slack], dtype=np.int32),
            w,
            self.pv.astype(np.int32),
            self.pq.astype(np.int32),
        )

    def branch_data(self):
        """Arguments of ``set_branch_data`` (``gpu_facade.py:569``)."""
        vn = np.full(self.n_bus, 138.0)
        return (self.branch_from.astype(np.int32), self.branch_to.astype(np.int32),
                self.yff, self.yft, self.ytf, self.ytt, vn, float(self.sn_mva))


# name -> (n_bus, n_branch, n_pv, n_load, n_trafo or None for the 20/186 fraction,
#          load_scale)
#
# load_scale: the recipe's loads (P ~ U(0, 1.5) pu on 100 MVA) exceed the
# loadability limit of these networks -- Newton-Raphson from a flat start
# diverges for every seed tried, and a load-scaling continuation puts the nose
# of the P-V curve near 0.45-0.6 (118 buses), 0.35-0.45 (2000), 0.15-0.25
# (6500) and 0.12-0.18 (10000).  Every load (and so the generation, which
# follows the load) is multiplied by load_scale, which puts each base case at
# roughly half of its nose, where flat-start NR converges in 4-6 iterations.
GRID_SPECS = {
    "case118_synth": (118, 186, 53, 99, 20, 0.3),
    "case2000_synth": (2000, 3200, 400, 1500, None, 0.2),
    "case6500_synth": (6500, 9000, 1300, 4800, None, 0.08),
    "case10000_synth": (10000, 13500, 2000, 7400, None, 0.07),
}
_TRAFO_FRACTION = 20.0 / 186.0


def build_ybus(n_bus, f, t, r, x, b, tap):
    """π-model branch admittances and the CSR Ybus (sorted column indices,
    explicit entries for every branch even where values cancel)."""
    ys = 1.0 / (r + 1j * x)
    tapc = tap.astype(np.complex128)
    ytt = ys + 0.5j * b
    yff = ytt / (np.abs(tapc) ** 2)
    yft = -ys / np.conj(tapc)
    ytf = -ys / tapc
    rows = np.concatenate([f, t, f, t])
    cols = np.concatenate([f, t, t, f])
    vals = np.concatenate([yff, ytt, yft, ytf])
    Y = sp.coo_matrix((vals, (rows, cols)), shape=(n_bus, n_bus)).tocsr()
    Y.sum_duplicates()
    Y.sort_indices()
    # every bus gets a diagonal entry even if isolated by construction
    diag = Y.diagonal()
    missing = np.flatnonzero(diag == 0)
    if missing.size:
        Y = Y + sp.csr_matrix((np.full(missing.size, 0j), (missing, missing)), shape=Y.shape)
        Y.sort_indices()
    return yff, yft, ytf, ytt, Y.astype(np.complex128)


def make_grid(n_bus, n_branch, n_pv, n_load, n_trafo=None, seed=0, name=None,
              load_scale=1.0) -> Grid:
    """Generate one grid.  Deterministic in ``seed``.  ``load_scale``
    multiplies every load after sampling (see ``GRID_SPECS``)."""
    if n_branch < n_bus - 1:
        raise ValueError("need at least n_bus - 1 branches for a spanning tree")
    rng = np.random.default_rng(seed)
    # random recursive spanning tree over a random bus order
    order = rng.permutation(n_bus)
    f_list = []
    t_list = []
    edges = set()
    for i in range(1, n_bus):
        j = int(rng.integers(0, i))
        a, c = int(order[i]), int(order[j])
        f_list.append(a)
        t_list.append(c)
        edges.add((min(a, c), max(a, c)))
    while len(f_list) < n_branch:
        a, c = (int(v) for v in rng.integers(0, n_bus, size=2))
        if a == c:
            continue
        key = (min(a, c), max(a, c))
        if key in edges:
            continue
        edges.add(key)
        f_list.append(a)
        t_list.append(c)
    f = np.array(f_list, dtype=np.int32)
    t = np.array(t_list, dtype=np.int32)
    # shuffle branch order so tree edges are not all first
    perm = rng.permutation(n_branch)
    f, t = f[perm], t[perm]

    r = rng.uniform(0.005, 0.05, n_branch)
    x = r * rng.uniform(3.0, 10.0, n_branch)
    b = rng.uniform(0.0, 0.05, n_branch)
    if n_trafo is None:
        n_trafo = int(round(_TRAFO_FRACTION * n_branch))
    is_trafo = np.zeros(n_branch, dtype=bool)
    is_trafo[rng.choice(n_branch, size=n_trafo, replace=False)] = True
    tap = np.ones(n_branch)
    tap[is_trafo] = rng.uniform(0.95, 1.05, n_trafo)

    gens = rng.choice(n_bus, size=n_pv + 1, replace=False)
    slack = int(gens[0])
    pv = np.sort(gens[1:]).astype(np.int32)
    is_gen = np.zeros(n_bus, dtype=bool)
    is_gen[gens] = True
    pq = np.flatnonzero(~is_gen).astype(np.int32)
    vset = np.ones(n_bus)
    vset[gens] = rng.uniform(0.98, 1.05, n_pv + 1)

    load_bus = np.sort(rng.choice(n_bus, size=n_load, replace=False)).astype(np.int32)
    load_p = rng.uniform(0.0, 1.5, n_load)
    pf = rng.uniform(0.9, 0.98, n_load)
    load_q = load_p * np.tan(np.arccos(pf))
    load_p = load_p * load_scale
    load_q = load_q * load_scale

    w = rng.uniform(0.5, 1.5, n_pv + 1)
    gen_p = 1.02 * load_p.sum() * w / w.sum()
    gen_bus = gens.astype(np.int32)

    yff, yft, ytf, ytt, Y = build_ybus(n_bus, f, t, r, x, b, tap)
    return Grid(
        name=name or f"synth{n_bus}", n_bus=n_bus, branch_from=f, branch_to=t,
        r=r, x=x, b=b, tap=tap, is_trafo=is_trafo, slack=slack, pv=pv, pq=pq,
        vset=vset, load_bus=load_bus, load_p=load_p, load_q=load_q,
        gen_bus=gen_bus, gen_p=gen_p, seed=seed,
        yff=yff, yft=yft, ytf=ytf, ytt=ytt, Ybus=Y)


def grid_by_name(name: str, seed: int = 0) -> Grid:
    n_bus, n_branch, n_pv, n_load, n_trafo, scale = GRID_SPECS[name]
    return make_grid(n_bus, n_branch, n_pv, n_load, n_trafo, seed=seed, name=name,
                     load_scale=scale)


def _bridges(n_bus, f, t):
    """Bridge edges (branch ids whose removal disconnects the graph), by an
    iterative Tarjan low-link DFS.  A branch open at one end (a negative
    endpoint) is no edge and never a bridge."""
    f = np.asarray(f)
    t = np.asarray(t)
    edge = (f >= 0) & (t >= 0)
    adj_ptr = np.zeros(n_bus + 1, dtype=np.int64)
    np.add.at(adj_ptr, f[edge] + 1, 1)
    np.add.at(adj_ptr, t[edge] + 1, 1)
    adj_ptr = np.cumsum(adj_ptr)
    adj_to = np.empty(adj_ptr[-1], dtype=np.int64)
    adj_e = np.empty(adj_ptr[-1], dtype=np.int64)
    head = adj_ptr[:-1].copy()
    for e, (a, c) in enumerate(zip(f, t)):
        if a < 0 or c < 0:
            continue
        adj_to[head[a]] = c; adj_e[head[a]] = e; head[a] += 1
        adj_to[head[c]] = a; adj_e[head[c]] = e; head[c] += 1
    disc = -np.ones(n_bus, dtype=np.int64)
    low = np.zeros(n_bus, dtype=np.int64)
    is_bridge = np.zeros(len(f), dtype=bool)
    timer = 0
    for root in range(n_bus):
        if disc[root] >= 0:
            continue
        stack = [(root, -1, adj_ptr[root])]
        disc[root] = low[root] = timer; timer += 1
        while stack:
            v, pe, it = stack[-1]
            if it < adj_ptr[v + 1]:
                stack[-1] = (v, pe, it + 1)
                w, e = adj_to[it], adj_e[it]
                if e == pe:
                    continue
                if disc[w] < 0:
                    disc[w] = low[w] = timer; timer += 1
                    stack.append((w, e, adj_ptr[w]))
                else:
                    low[v] = min(low[v], disc[w])
            else:
                stack.pop()
                if stack:
                    u = stack[-1][0]
                    low[u] = min(low[u], low[v])
                    if low[v] > disc[u]:
                        is_bridge[pe] = True
    return is_bridge


def n1_branches(grid: Grid) -> np.ndarray:
    """Every branch whose single outage keeps the grid connected."""
    return np.flatnonzero(~_bridges(grid.n_bus, grid.branch_from, grid.branch_to)).astype(np.int32)


def injection_scenarios(grid: Grid, n_scenarios: int, seed: int = 1):
    """Load scaling scenarios: every load × a global U(0.8, 1.2) factor × a
    per-bus lognormal(0, 0.1) factor; generators rescaled so generation stays
    1.02 × load.  Returns (p_mw, q_mvar) as dense (n_scenarios, n_bus) arrays
    in MW / MVAr, the form ``set_injections`` takes
    (``injection_sweep/gpu_facade.py:378``)."""
    rng = np.random.default_rng(seed)
    g = rng.uniform(0.8, 1.2, size=(n_scenarios, 1))
    per_bus = rng.lognormal(0.0, 0.1, size=(n_scenarios, grid.load_bus.size))
    scale = g * per_bus
    lp = grid.load_p[None, :] * scale
    lq = grid.load_q[None, :] * scale
    gp = grid.gen_p[None, :] * (lp.sum(axis=1, keepdims=True) / grid.load_p.sum())
    p = np.zeros((n_scenarios, grid.n_bus))
    q = np.zeros((n_scenarios, grid.n_bus))
    np.add.at(p, (slice(None), grid.gen_bus), gp)
    np.subtract.at(p, (slice(None), grid.load_bus), lp)
    np.subtract.at(q, (slice(None), grid.load_bus), lq)
    return p * grid.sn_mva, q * grid.sn_mva


def scenario_outages(grid: Grid, n_rows: int, max_trips: int = 2, seed: int = 2,
                     candidates: Optional[np.ndarray] = None):
    """0..max_trips tripped branches per row, drawn among single-outage-safe
    branches; a double trip that islands the grid is redrawn."""
    rng = np.random.default_rng(seed)
    cand = n1_branches(grid) if candidates is None else candidates
    out = []
    for _ in range(n_rows):
        k = int(rng.integers(0, max_trips + 1))
        while True:
            ids = sorted(set(int(v) for v in rng.choice(cand, size=k, replace=False))) if k else []
            if len(ids) < 2 or _connected_without(grid, ids):
                break
        out.append(ids)
    return out


def _connected_without(grid: Grid, ids) -> bool:
    keep = (grid.branch_from >= 0) & (grid.branch_to >= 0)
    keep[list(ids)] = False
    f, t = grid.branch_from[keep], grid.branch_to[keep]
    A = sp.coo_matrix((np.ones(f.size), (f, t)), shape=(grid.n_bus, grid.n_bus))
    from scipy.sparse.csgraph import connected_components
    ncomp, _ = connected_components(A, directed=False)
    return ncomp == 1


def half_open_variant(grid: Grid, n_open: int = 2, seed: int = 0) -> Grid:
    """The grid with ``n_open`` branches open at their to-end: their
    ``branch_to`` is -1 (a side with no bus in the solved system, as the
    reference's bus relabelling gives the open end of a half-open line,
    ``contingency_analysis_helper.cpp:53-64``) and Ybus keeps only their
    from-end self term yff (the line's charging seen from the live end).  The
    branches are chosen among those whose loss keeps the grid connected, so
    the variant stays connected."""
    rng = np.random.default_rng(seed)
    cand = [int(l) for l in rng.permutation(n1_branches(grid))]
    chosen = []
    for l in cand:
        if len(chosen) == n_open:
            break
        if _connected_without(grid, chosen + [l]):
            chosen.append(l)
    ids = np.array(sorted(chosen), dtype=np.int32)
    f = grid.branch_from.astype(np.int64)
    t = grid.branch_to.astype(np.int64)
    live = np.ones(grid.n_branch, dtype=bool)
    live[ids] = False
    rows = np.concatenate([f, t[live], f[live], t[live]])
    cols = np.concatenate([f, t[live], t[live], f[live]])
    vals = np.concatenate([grid.yff, grid.ytt[live], grid.yft[live], grid.ytf[live]])
    Y = sp.coo_matrix((vals, (rows, cols)), shape=(grid.n_bus, grid.n_bus)).tocsr()
    Y.sum_duplicates()
    Y.sort_indices()
    to = grid.branch_to.copy()
    to[ids] = -1
    return dataclasses.replace(grid, name=grid.name + "_half_open", branch_to=to, Ybus=Y.astype(np.complex128),
                               open_branches=ids)
