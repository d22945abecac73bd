"""Batched sweeps on the GPU: ``ContingencyAnalysisGPU``, ``InjectionSweepGPU``
and ``ScenarioSweepGPU`` (array-tuple mode).

Facade signatures follow the reference:
``src/gpusim2grid/contingency_analysis/gpu_facade.py:347-782`` (constructor,
``set_branch_data`` :569, ``add_contingencies_by_branch_id`` :595, ``compute`` :762,
``last_residuals`` :1025), ``src/gpusim2grid/injection_sweep/gpu_facade.py:220-546``
(``set_injections`` :378, ``compute`` :515) and
``src/gpusim2grid/scenario_sweep/gpu_facade.py:215-838`` (``set_topology`` :690,
``get_disconnected`` :838).  Scheduling names and row statuses:
``src/gpusim2grid/contingency_analysis/_scheduling.py:61-170``.

Every row runs on the persistent kernel: a row is one CTA's whole Newton loop,
and it leaves the GPU as soon as it is done (``scheduling='continuous'``) or
after exactly ``nb_iter`` steps (``scheduling='chunked'``, the reference's
default).  Rows start from the converged base case as the reference's batch
sources do (``start='base'``), or from ``Vinit`` (``start='flat'``), or from
per-row voltages (``set_start_voltages``), or from voltages a trained
network predicts for each row (``set_learned_start``, ``start='learned'``;
see ``warmstart.py``).  A row given a start of their own begins from the
base case instead when that has the smaller mismatch, and a row that fails
from its start restarts once from the base case (``Vinit`` without one)
inside the same launch.
"""

from __future__ import annotations

import itertools
import time

import numpy as np

from ._common import (BatchTimings, RowStatus, default_tol, grid_arrays, make_session, resolve_precision,
                      resolve_scheduling)
from ._native import lib

__all__ = ["ContingencyAnalysisGPU", "InjectionSweepGPU", "ScenarioSweepGPU", "compute_many"]

_START = {"base": lib.START_BASE, "flat": lib.START_VINIT, "rows": lib.START_ROWS, "learned": lib.START_ROWS}
_STRATEGY = {"refactor_every": lib.REFACTOR_EVERY, "adaptive": lib.REFACTOR_ADAPTIVE,
             "base_chord": lib.REFACTOR_BASE_CHORD}


def _rows_csr(branch_ids_per_row):
    """(rows, ptr, ids) of branch-id lists, each row's duplicates dropped
    (first occurrence kept).  Rows of one id each (the N-1 case), given as
    lists or as an integer array, take a vectorised path (rows None: the
    CSR is the only copy)."""
    if isinstance(branch_ids_per_row, np.ndarray) and branch_ids_per_row.ndim == 2 and \
            branch_ids_per_row.shape[1] == 1:
        flat = np.ascontiguousarray(branch_ids_per_row[:, 0], dtype=np.int32)
    elif len(branch_ids_per_row) and all(len(r) == 1 for r in branch_ids_per_row):
        flat = np.fromiter((int(r[0]) for r in branch_ids_per_row), dtype=np.int32, count=len(branch_ids_per_row))
    else:
        try:
            ptr, ids = _dedup_csr(branch_ids_per_row)
        except (TypeError, ValueError, OverflowError):
            rows = [list(dict.fromkeys(int(v) for v in ids)) for ids in branch_ids_per_row]
            ptr, ids = _ids_csr(rows)
            return rows, ptr, ids
        return None, ptr, ids
    ptr = np.arange(flat.size + 1, dtype=np.int32)
    return None, ptr, flat


def _dedup_csr(branch_ids_per_row):
    """(ptr, ids) int32 of lists of integer ids, each row's repeated ids
    dropped (first occurrence kept, order kept), without a Python loop per
    id: the rows are flattened, (row, id) keys that repeat are removed by
    their first index."""
    n = len(branch_ids_per_row)
    lens = np.fromiter(map(len, branch_ids_per_row), dtype=np.int64, count=n)
    flat = np.fromiter(itertools.chain.from_iterable(branch_ids_per_row), dtype=np.int64, count=int(lens.sum()))
    if flat.size and (flat.min() < np.iinfo(np.int32).min or flat.max() > np.iinfo(np.int32).max):
        raise OverflowError("branch id out of the int32 range")
    rid = np.repeat(np.arange(n, dtype=np.int64), lens)
    if flat.size:
        span = int(flat.max()) - int(flat.min()) + 1
        _, first = np.unique(rid * span + (flat - flat.min()), return_index=True)
        keep = np.sort(first)
        flat, rid = flat[keep], rid[keep]
    ptr = np.zeros(n + 1, dtype=np.int32)
    ptr[1:] = np.cumsum(np.bincount(rid, minlength=n))
    return ptr, flat.astype(np.int32)


def _ids_csr(rows):
    ptr = np.zeros(len(rows) + 1, dtype=np.int32)
    flat = []
    for r, ids in enumerate(rows):
        ids = [int(v) for v in (ids if ids is not None else [])]
        flat.extend(ids)
        ptr[r + 1] = len(flat)
    return ptr, np.asarray(flat, dtype=np.int32)


class _BatchSweep:
    def __init__(self, grid, *, init_from_n_powerflow=True, precision="fp64", nb_iter=4, max_iter_base=10,
                 tol_base=1e-8, device=None, scheduling=None, nb_iter_per_round=1, tol=None, start="base",
                 strategy="refactor_every", handle_disconnected_grid=False, scaling_max_voltage_change=None,
                 max_dVa=None, max_dVm=None, **_ignored):
        d = grid_arrays(grid)
        self._d = d
        self.scaling_max_voltage_change = scaling_max_voltage_change
        self.max_dVa = max_dVa
        self.max_dVm = max_dVm
        self._prec = resolve_precision(precision)
        self.nb_iter = int(nb_iter)
        self.scheduling = resolve_scheduling("chunked" if scheduling is None else scheduling)
        self.nb_iter_per_round = nb_iter_per_round
        self.tol = default_tol() if tol is None else float(tol)
        self._s = make_session(d, device)
        if init_from_n_powerflow:
            res = self._s.set_base_v(d["Vinit"])
            if not (res < tol_base):
                raise RuntimeError(f"init_from_n_powerflow: the base-case residual {res:.3e} is not below "
                                   f"tol_base = {tol_base:.1e}")
            self._base_iters = 0
        else:
            V, st, it, res = self._s.solve_base(int(max_iter_base), float(tol_base), self._prec, 0.0)
            if st != RowStatus.CONVERGED:
                raise RuntimeError(f"the base case did not converge (status {RowStatus(st).name}, "
                                   f"residual {res:.3e})")
            self._base_iters = it
        self.start = start
        self.strategy = strategy
        self.handle_disconnected_grid = handle_disconnected_grid
        self._refactor_ratio = None  # None: the strategy's default
        self._max_reuse = None
        # mixed precision, continuous schedule: rows that end MAX_ITER or
        # DIVERGED are re-solved in plain FP64 from Vinit, whose verdict stands
        self.fallback = "fp64"
        self._fallback_rows = 0
        self._learned = None
        self._warm = {}
        self._n_branches = None
        self._ran = False
        self._timings = BatchTimings()

    # -------------------------------------------------------------- options
    @property
    def nb_iter_per_round(self):
        """Continuous scheduling: Newton steps every row runs between two
        convergence tests (k >= 1).  A row runs a multiple of k steps, at
        least k, also when it starts converged; after each round it leaves
        DIVERGED (residual not finite), CONVERGED (below tol) or MAX_ITER
        (steps >= nb_iter), as the reference's rounds
        (``src/_cpp/contingency/batch_pf_driver.cu:2691-2724``).  Takes
        effect on the next compute()."""
        return self._nb_iter_per_round

    @nb_iter_per_round.setter
    def nb_iter_per_round(self, value):
        value = int(value)
        if value < 1:
            raise ValueError("nb_iter_per_round must be >= 1")
        self._nb_iter_per_round = value

    @property
    def handle_disconnected_grid(self):
        """A row whose trips split the grid: False (default) leaves it
        NOT_SIMULATED with NaN voltages; True solves its largest component
        (most buses; on a tie the one holding the lowest bus) with the other
        buses masked -- frozen during the iteration, NaN in the results -- as
        the reference's option of that name.  A split that strands a slack
        bus stays NOT_SIMULATED.  Takes effect on the next compute()."""
        return self._handle_disconnected

    @handle_disconnected_grid.setter
    def handle_disconnected_grid(self, value):
        self._handle_disconnected = bool(value)
        self._s.set_handle_disconnected(self._handle_disconnected)

    @property
    def results_to_host(self):
        """True: every later ``compute()`` also writes each row's final
        voltages into the page-locked buffer that ``results_view()`` returns,
        from the kernels as the row leaves, so the transfer of V to the host
        overlaps the sweep and ``results_view()`` copies only the residuals,
        statuses and iterations.  The device results are unchanged.  Default
        False (no counterpart in the reference, whose results stay on the
        device)."""
        return getattr(self, "_results_to_host", False)

    @results_to_host.setter
    def results_to_host(self, value):
        self._results_to_host = bool(value)
        self._s.set_results_mirror(self._results_to_host)

    @property
    def start(self):
        """'base' (the converged base case, default), 'flat' (``Vinit``),
        'rows' (``set_start_voltages``) or 'learned' (``set_learned_start``)."""
        return self._start

    @start.setter
    def start(self, value):
        if value not in _START:
            raise ValueError(f"Unknown start {value!r}. Choose from: {list(_START)}")
        if value == "learned" and getattr(self, "_learned", None) is None:
            raise ValueError("start='learned' needs set_learned_start() first")
        self._start = value

    def set_learned_start(self, learned, refactor_ratio=None, max_reuse=None):
        """Start every row from the voltages ``learned`` (a trained
        ``warmstart.LearnedStart`` of this grid) predicts for it, on the
        device, at every ``compute()``; switches ``start`` to 'learned'.
        A good start leaves only the fast-contracting end of Newton's
        iteration, so the adaptive strategy may keep one LU longer:
        ``refactor_ratio`` / ``max_reuse`` apply to learned runs."""
        if learned.grid.n_bus != self.n_bus:
            raise ValueError("the learned start belongs to a grid of another size")
        self._learned = learned
        self._learned_override = (refactor_ratio, max_reuse)
        self.start = "learned"

    @property
    def _learned_opts(self):
        """(refactor_ratio, max_reuse) of learned runs.  On the shared base
        factor (base_chord) a chord step is cheap -- several rows share each
        factor read -- so rows keep chording while a step contracts by 0.7 or
        better, for at most 8 steps (the kernel also leaves the chord when
        the remaining step budget could not reach tol at the observed rate).
        Under the adaptive strategy a row factors its own Jacobian as soon as
        a step contracts by less than 0.5, for at most 6 steps on one
        factor."""
        r, m = getattr(self, "_learned_override", (None, None))
        long_chord = self._strategy == "base_chord"
        return (float(r if r is not None else (0.7 if long_chord else 0.5)),
                int(m if m is not None else (8 if long_chord else 6)))

    def _rows_have_trips(self):
        return False

    def _row_defs(self):
        """(sbus_rows or None, trips CSR or None, n_rows) of the current rows."""
        raise NotImplementedError

    def _device_row_defs(self):
        """The current rows as ``_row_defs`` gives them, but read from the
        session's own device copies (no host round trip): Sbus rows as a
        (rows, n_bus) complex128 tensor, trips as a device CSR (ptr, ids)."""
        import torch
        sb, tp, ti = (self._s.device_rows(w) for w in ("sbus", "trip_ptr", "trip_ids"))
        sbus = torch.from_dlpack(sb) if sb is not None else None
        trips = (torch.from_dlpack(tp), torch.from_dlpack(ti)) if tp is not None else None
        if sbus is not None:
            n = sbus.shape[0]
        elif trips is not None:
            n = trips[0].numel() - 1
        else:
            n = self._row_defs()[2]
        return sbus, trips, n

    def autotune(self, dense_rates=(40.0, 80.0, 160.0, 320.0, 640.0), repeats=2, batch_size=512):
        """Pick the symbolic plan that solves the current rows fastest.  Each
        candidate re-plans the head/tail split with another dense/scatter
        cost ratio (``Session.replan``) and times ``repeats`` sweeps of the
        current rows with the current start, precision and strategy (device
        time of the sweep kernel); the fastest plan is kept.  Returns
        {dense_rate: (tail_dim, best ms)} and the chosen rate."""
        out = {}
        best = (float("inf"), None)
        for rate in dense_rates:
            self._s.replan(1, float(rate), -1)
            ms = []
            for _ in range(max(1, int(repeats))):
                self._run(batch_size)
                ms.append(self._timings.t_kernel_ms)
            out[float(rate)] = (int(self._s.info()["tail_dim"]), float(min(ms)))
            if min(ms) < best[0]:
                best = (min(ms), float(rate))
        self._s.replan(1, best[1], -1)
        self._ran = False
        return out, best[1]

    @property
    def warm_report(self):
        """Timings of the last learned start: predict_ms (host time to
        enqueue the network and V0; the device runs them ahead of the sweep
        on the same stream order), n_rescued (rows restarted), n_base_start
        (rows that began from the base case: its mismatch was the smaller)."""
        return dict(self._warm)

    @property
    def scaling_max_voltage_change(self):
        """The reference's MaxVoltageChange step scaling
        (``src/gpusim2grid/contingency_analysis/gpu_facade.py:203-226``): True
        multiplies every Newton step by alpha <= 1 so that max|dtheta| <=
        ``max_dVa`` and max|dVm| <= ``max_dVm`` (defaults 0.5 rad / 0.1 pu),
        damping steps taken far from the solution so that they do not land on
        another power-flow root.  In array-tuple mode there is no grid
        configuration to inherit, so None (default) means off.  Under
        ``base_chord`` a row whose chord step would be scaled moves to its own
        factor, where its steps are scaled."""
        return self._scaling

    @scaling_max_voltage_change.setter
    def scaling_max_voltage_change(self, value):
        self._scaling = bool(value) if value is not None else False

    def _scaling_kw(self):
        return dict(step_scaling=self._scaling, max_dva=float(self.max_dVa) if self.max_dVa is not None else 0.0,
                    max_dvm=float(self.max_dVm) if self.max_dVm is not None else 0.0)

    @property
    def refactor_ratio(self):
        """Contraction per step below which a row keeps its factor ('adaptive':
        its own LU, default 0.3; 'base_chord': the shared base factor, default
        0.7 -- a step on it is cheap, several rows share each factor read).
        Learned runs use ``set_learned_start``'s values."""
        if self._refactor_ratio is not None:
            return self._refactor_ratio
        return 0.7 if self._strategy == "base_chord" else 0.3

    @refactor_ratio.setter
    def refactor_ratio(self, value):
        self._refactor_ratio = None if value is None else float(value)

    @property
    def max_reuse(self):
        """Steps on one factor at most (defaults: 3 'adaptive', 8
        'base_chord'); see ``refactor_ratio``."""
        if self._max_reuse is not None:
            return self._max_reuse
        return 8 if self._strategy == "base_chord" else 3

    @max_reuse.setter
    def max_reuse(self, value):
        self._max_reuse = None if value is None else int(value)

    @property
    def strategy(self):
        """Linear-solve strategy.  'refactor_every' (default): a new LU every
        Newton step, the reference's 'direct_refactor_every'.  'adaptive':
        keep the last LU while ||F||inf shrinks by ``refactor_ratio`` per step
        (at most ``max_reuse`` steps), refactor otherwise; the FP64 mismatch
        still converges every row to ``tol``."""
        return self._strategy

    @strategy.setter
    def strategy(self, value):
        if value not in _STRATEGY:
            raise ValueError(f"Unknown strategy {value!r}. Choose from: {list(_STRATEGY)}")
        self._strategy = value

    # ----------------------------------------------------------------- data
    def set_branch_data(self, branch_from, branch_to, yff_eff, yft_eff, ytf_eff, ytt_eff, bus_vn_kv=None,
                        sn_mva=None):
        """π-model branch admittances (explicit-array mode); needed to trip
        branches.  ``bus_vn_kv`` / ``sn_mva`` are accepted for signature
        parity (they only serve branch-flow post-processing)."""
        c = lambda a: np.ascontiguousarray(a, dtype=np.complex128)
        self._s.set_branch_data(np.ascontiguousarray(branch_from, dtype=np.int32),
                                np.ascontiguousarray(branch_to, dtype=np.int32),
                                c(yff_eff), c(yft_eff), c(ytf_eff), c(ytt_eff))
        self._n_branches = len(branch_from)
        self._limits = False

    def set_branch_limits(self, rate_mva, sn_mva=100.0):
        """Branch limits in MVA (one per branch of ``set_branch_data``; <= 0:
        unlimited).  From then on every ``compute()`` also evaluates each
        converged row's branch flows and loadings on the GPU as the row
        finishes (the reference's ``compute_branch_flows`` +
        ``check_limit_violations``); read them with ``branch_loading()``.
        ``None`` turns it off."""
        if self._n_branches is None:
            raise RuntimeError("set_branch_data() must be called before set_branch_limits()")
        if rate_mva is None:
            self._s.set_branch_limits(np.zeros(0), float(sn_mva))
            self._limits = False
            return
        rate = np.ascontiguousarray(rate_mva, dtype=np.float64)
        if rate.shape != (self._n_branches,):
            raise ValueError(f"rate_mva must have one entry per branch ({self._n_branches})")
        self._s.set_branch_limits(rate, float(sn_mva))
        self._limits = True

    def branch_loading(self):
        """(loading, n_violations, max_loading) of the last ``compute()``:
        loading (n_rows, n_branches) float32 = max(|S_from|, |S_to|) / limit
        (0 for tripped or unlimited branches, NaN for rows that did not
        converge); n_violations (n_rows,) branches above their limit (-1: row
        not converged); max_loading (n_rows,)."""
        if not self._ran:
            raise RuntimeError("Call compute() first.")
        if not getattr(self, "_limits", False):
            raise RuntimeError("set_branch_limits() was not called")
        return self._s.branch_loading(int(self._n_branches))

    def set_start_voltages(self, V0):
        """Per-row start voltages (n_rows, n_bus) complex; switches ``start`` to 'rows'."""
        V0 = np.ascontiguousarray(V0, dtype=np.complex128)
        self._s.set_start_rows(V0)
        self.start = "rows"

    # ------------------------------------------------------------------ run
    def _run(self, batch_size):
        fixed = self.scheduling == "chunked"
        n_ctas = max(int(batch_size), 0)
        t0 = time.perf_counter()
        ratio, reuse = float(self.refactor_ratio), int(self.max_reuse)
        rescue = self._start in ("rows", "learned")
        if self._start == "learned":
            import torch
            sbus, trips, n = self._device_row_defs()
            # V0 is written in place into the session's start-row buffer on
            # torch's stream; the session stream waits for it on the device
            # (no host synchronisation between the network and the sweep)
            self._learned.start_voltages(sbus, trips, n, out_ptr=self._s.start_rows_buffer(n))
            self._s.wait_stream(torch.cuda.current_stream().cuda_stream)
            self._warm = dict(predict_ms=(time.perf_counter() - t0) * 1e3)
            ratio, reuse = self._learned_opts
        self._s.run(self.nb_iter, self.tol, fixed, self._prec, _START[self._start], 0.0, n_ctas, False,
                    _STRATEGY[self._strategy], ratio, reuse, rescue, self.nb_iter_per_round, **self._scaling_kw())
        tm = self._s.timings()
        if self._start == "learned":
            self._learned.net.check()  # the network's GEMMs finished before the sweep (stream order)
            self._warm["n_rescued"] = int(tm["n_rescued"])
            self._warm["n_base_start"] = int(tm["n_base_start"])
        kernel_ms = tm["kernel_ms"]
        kernel_ms += self.fp64_fallback(n_ctas, tm["n_failed"])
        tm = dict(tm, kernel_ms=kernel_ms)
        self._timings = BatchTimings(n_rows=self._s.n_rows(), total_iters=int(tm["total_iters"]),
                                     t_plan_ms=tm["plan_ms"], t_upload_ms=tm["upload_ms"],
                                     t_kernel_ms=tm["kernel_ms"], t_total_ms=(time.perf_counter() - t0) * 1e3)
        self._ran = True
        self._host = None

    def fp64_fallback(self, n_ctas=0, n_failed=None):
        """Re-solve, in plain FP64 from Vinit, the rows a mixed-precision
        continuous run left MAX_ITER or DIVERGED (the flat-start FP64 NR
        remains the fallback).  ``n_failed``: those rows' count when the
        caller has read the timings already.  Returns its kernel ms."""
        self._fallback_rows = 0
        if self.fallback != "fp64" or self._prec != lib.PREC_MIXED or self.scheduling != "continuous":
            return 0.0
        if (self._s.timings()["n_failed"] if n_failed is None else n_failed) == 0:
            return 0.0
        import torch
        st = torch.from_dlpack(self._s.dlpack("status"))
        bad = ((st == int(RowStatus.MAX_ITER)) | (st == int(RowStatus.DIVERGED))).nonzero().flatten()
        if bad.numel() == 0:
            return 0.0
        rows = bad.to(torch.int32).cpu().numpy()
        self._s.run_subset(rows, self.nb_iter, self.tol, False, lib.PREC_FP64, lib.START_VINIT, 0.0, n_ctas,
                           lib.REFACTOR_EVERY, 0.0, 0, False, self.nb_iter_per_round, **self._scaling_kw())
        self._fallback_rows = int(rows.size)
        self._host = None
        return float(self._s.timings()["kernel_ms"])

    @property
    def fallback_rows(self):
        """Rows the last ``compute()`` re-solved in FP64 (see ``fallback``)."""
        return self._fallback_rows

    def compute(self, batch_size=512):
        """Solve every row.  Returns a DLPack capsule (n_rows, n_bus) complex128
        aliasing device memory, valid until the next ``compute()``.
        ``batch_size`` caps the rows in flight (one per CTA of the persistent
        kernel)."""
        self._run(batch_size)
        return self._s.dlpack("v")

    def _results(self):
        if not self._ran:
            raise RuntimeError("Call compute() first.")
        if self._host is None:
            self._host = self._s.results()
        return self._host

    def last_residuals(self):
        """||F||inf per row of the last ``compute()``."""
        return self._results()[1].copy()

    def get_row_status(self):
        return self._results()[2].copy()

    def get_row_iterations(self):
        return self._results()[3].copy()

    def get_row_factorizations(self):
        """LU factorizations each row of the last ``compute()`` performed."""
        if not self._ran:
            raise RuntimeError("Call compute() first.")
        return self._s.factor_counts()

    @property
    def V_results(self):
        """(n_rows, n_bus) complex voltages of the last ``compute()`` (host copy)."""
        return self._results()[0]

    @property
    def dim_J(self):
        """Unknowns of a row: len(pv + pq) angles, then len(pq) magnitudes."""
        return int(self._s.info()["dim_j"])

    def solve_JT(self, rhs):
        """Batched adjoint of the last ``compute()``: for every row r,
        ``lam[r] = J_r^-T rhs[r]``, J_r the row's Jacobian (FP64) at its
        converged voltage, in the reference's J layout (theta rows on sorted
        pv + pq, then Vm rows on pq).  ``rhs`` is (n_rows, dim_J), numpy or a
        torch tensor (returned in the same kind); non-finite entries count as
        0; rows that did not converge give 0 (the reference's
        ``solve_JT_batch_dlpack``)."""
        if not self._ran:
            raise RuntimeError("Call compute() first.")
        import torch
        n = self._s.n_rows()
        is_torch = isinstance(rhs, torch.Tensor)
        dev = torch.device("cuda", self._device_index())
        r = rhs if is_torch else torch.as_tensor(np.asarray(rhs))
        r = r.to(device=dev, dtype=torch.float64).contiguous()
        if r.shape != (n, self.dim_J):
            raise ValueError(f"rhs must be ({n}, {self.dim_J}), got {tuple(r.shape)}")
        lam = torch.empty_like(r)
        torch.cuda.current_stream(dev).synchronize()
        self._s.solve_jt(n, r.data_ptr(), lam.data_ptr())
        return lam if is_torch else lam.cpu().numpy()

    def _device_index(self):
        import torch
        return int(torch.from_dlpack(self._s.dlpack("status")).device.index)

    def results_view(self):
        """(V, residuals, status, iterations) of the last ``compute()`` as
        numpy views of page-locked host memory the session owns, filled by
        one DMA per array (V already written by the kernels under
        ``results_to_host``): no further host copy.  Valid until the next
        ``compute()`` or ``results_view()`` -- the lifetime of the reference's
        ``V_results`` device buffer; copy what must outlive it."""
        if not self._ran:
            raise RuntimeError("Call compute() first.")
        return self._s.results_view()

    def converged(self, tol=None):
        res = self.last_residuals()
        return res < (self.tol if tol is None else tol)

    def converged_n(self, tol=None):
        return True

    def results_dlpack(self, what="v"):
        """DLPack capsule of 'v', 'residuals', 'status' or 'iters'."""
        return self._s.dlpack(what)

    @property
    def timings(self):
        return self._timings

    @property
    def n_bus(self):
        return self._d["n_bus"]

    @property
    def n_branches(self):
        return self._n_branches

    @property
    def session(self):
        return self._s


class ContingencyAnalysisGPU(_BatchSweep):
    """Batch N-k contingency analysis: every row trips a set of branches from
    the base case.  Rows whose trips island the grid are NOT_SIMULATED with NaN
    voltages (``contingency_analysis_helper.cpp:634-651``)."""

    def __init__(self, grid, **kw):
        super().__init__(grid, **kw)
        self._ctg = []
        self._ctg_csr = (np.zeros(1, dtype=np.int32), np.zeros(0, dtype=np.int32))

    def add_contingencies_by_branch_id(self, branch_ids_per_ctg):
        """One inner list per contingency (branch indices; a branch named twice
        is tripped once).  Replaces previously given contingencies."""
        if self._n_branches is None:
            raise RuntimeError("set_branch_data() must be called before add_contingencies_by_branch_id()")
        rows, ptr, ids = _rows_csr(branch_ids_per_ctg)
        self._s.set_contingencies(ptr, ids)
        self._ctg = rows  # None for single-branch rows: built from the CSR when asked for
        self._ctg_csr = (ptr, ids)

    def get_contingencies(self):
        if self._ctg is None:
            ptr, ids = self._ctg_csr
            return [ids[ptr[r]:ptr[r + 1]].tolist() for r in range(len(ptr) - 1)]
        return [list(r) for r in self._ctg]

    def _row_defs(self):
        return None, self._ctg_csr, len(self._ctg_csr[0]) - 1

    def _rows_have_trips(self):
        return True

    @property
    def n_contingencies(self):
        return len(self._ctg_csr[0]) - 1


class InjectionSweepGPU(_BatchSweep):
    """One row per injection scenario on a fixed topology."""

    def __init__(self, grid, **kw):
        super().__init__(grid, **kw)
        self._n_scen = 0
        self._inj = None

    def set_injections(self, p_mw, q_mvar, sn_mva):
        """Bus injections in MW / MVAr, (n_scenarios, n_bus); Sbus = (p + jq) / sn_mva
        (``injection_sweep_session.cu:239-245``)."""
        p = np.ascontiguousarray(p_mw, dtype=np.float64)
        q = np.ascontiguousarray(q_mvar, dtype=np.float64)
        if p.ndim != 2 or p.shape != q.shape or p.shape[1] != self.n_bus:
            raise ValueError("p_mw and q_mvar must both be (n_scenarios, n_bus)")
        self._s.set_injections(p, q, float(sn_mva))
        self._n_scen = p.shape[0]
        self._inj = (p, q, float(sn_mva))

    def _row_defs(self):
        if self._inj is None:
            raise RuntimeError("set_injections() must be called before compute()")
        p, q, sn = self._inj
        return (p + 1j * q) / sn, None, self._n_scen

    def set_injections_from_elements(self, load_p, load_q, gen_p):
        """Per-element injections (lightsim2grid's batch API,
        ``injection_sweep/gpu_facade.py:394``).  Mapping loads and generators
        to buses needs a lightsim2grid grid; a facade built from an array
        tuple has none, so this raises RuntimeError, as the reference does in
        that mode."""
        raise RuntimeError("set_injections_from_elements() needs a lightsim2grid grid; explicit-array (tuple) "
                           "mode has no loads/generators to read. Use set_injections(p_mw, q_mvar, sn_mva) instead.")

    @property
    def n_scenarios(self):
        return self._n_scen


class ScenarioSweepGPU(InjectionSweepGPU):
    """Injections and topology per row: row r uses injection scenario r and
    trips the branches of ``set_topology()[r]``."""

    def __init__(self, grid, **kw):
        super().__init__(grid, **kw)
        self._topo_csr = None

    def set_topology(self, branch_ids_per_scenario):
        if self._n_branches is None:
            raise RuntimeError("set_branch_data() must be called before set_topology()")
        _, ptr, ids = _rows_csr(branch_ids_per_scenario)
        self._s.set_contingencies(ptr, ids)
        self._topo_csr = (ptr, ids)

    def _row_defs(self):
        if self._inj is None:
            raise RuntimeError("set_injections() must be called before compute()")
        p, q, sn = self._inj
        return (p + 1j * q) / sn, self._topo_csr, self._n_scen

    def get_topology(self):
        """The tripped branch ids of every scenario row (``set_topology``,
        duplicates dropped), or None without a topology."""
        if self._topo_csr is None:
            return None
        ptr, ids = self._topo_csr
        return [ids[ptr[r]:ptr[r + 1]].tolist() for r in range(len(ptr) - 1)]

    def _rows_have_trips(self):
        return self._topo_csr is not None

    def get_disconnected(self):
        """(n_rows,) int: 1 for a row whose topology islands the grid and was
        not solved (NaN), 0 otherwise -- a split solved on its largest
        component under ``handle_disconnected_grid`` counts as solved."""
        return (self.get_row_status() == RowStatus.NOT_SIMULATED).astype(np.int64)


def compute_many(sweeps, batch_size=0):
    """Solve the current rows of several sweeps -- any mix of grids, each
    facade with its own grid, rows and start -- in ONE persistent kernel
    launch (``gs2g_run_multi``): the launch's CTAs take rows from one queue
    across the grids, each row on its own grid's symbolic plan, so a batch
    of small and large grids keeps every SM busy until the whole batch
    drains.  Precision, ``nb_iter``, ``tol``, scheduling and strategy must
    agree across the sweeps.  Afterwards every facade reads its own results
    as after its own ``compute()``; returns the launch's kernel time (ms)."""
    sweeps = list(sweeps)
    if not sweeps:
        raise ValueError("compute_many needs at least one sweep")
    f0 = sweeps[0]
    for f in sweeps[1:]:
        if (f._prec, f.nb_iter, f.tol, f.scheduling, f._strategy, f.nb_iter_per_round, f._scaling_kw()) != (
                f0._prec, f0.nb_iter, f0.tol, f0.scheduling, f0._strategy, f0.nb_iter_per_round, f0._scaling_kw()):
            raise ValueError("compute_many: precision, nb_iter, tol, scheduling, strategy, nb_iter_per_round and "
                             "the step scaling must agree")
    starts = {f._start for f in sweeps}
    if len(starts) != 1:
        raise ValueError("compute_many: every sweep must use the same start")
    start = starts.pop()
    t0 = time.perf_counter()
    ratio, reuse = float(f0.refactor_ratio), int(f0.max_reuse)
    if start == "learned":
        import torch
        for f in sweeps:
            sbus, trips, n = f._device_row_defs()
            f._learned.start_voltages(sbus, trips, n, out_ptr=f._s.start_rows_buffer(n))
        # every session stream waits for the networks on the device
        for f in sweeps:
            f._s.wait_stream(torch.cuda.current_stream().cuda_stream)
        ratio, reuse = f0._learned_opts
    lib.run_multi([f._s for f in sweeps], f0.nb_iter, f0.tol, f0.scheduling == "chunked", f0._prec, _START[start],
                  0.0, max(int(batch_size), 0), False, _STRATEGY[f0._strategy], ratio, reuse,
                  start in ("rows", "learned"), f0.nb_iter_per_round, **f0._scaling_kw())
    kernel_ms = sweeps[0]._s.timings()["kernel_ms"]
    if start == "learned":
        for f in sweeps:
            f._learned.net.check()
    for f in sweeps:
        f._ran = True
        kernel_ms += f.fp64_fallback()
    total_ms = (time.perf_counter() - t0) * 1e3
    for f in sweeps:
        tm = f._s.timings()
        f._timings = BatchTimings(n_rows=f._s.n_rows(), total_iters=int(tm["total_iters"]), t_plan_ms=tm["plan_ms"],
                                  t_upload_ms=tm["upload_ms"], t_kernel_ms=kernel_ms, t_total_ms=total_ms)
        f._ran = True
        f._host = None
    return kernel_ms

