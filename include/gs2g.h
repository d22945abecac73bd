/*
 * gs2g.h — C-ABI of the B200-native batched Newton–Raphson AC power flow.
 *
 * Plain C: opaque handles, plain pointers and sizes, int status codes
 * (0 = success) and a thread-local last-error string.  No CUDA, torch or C++
 * types cross this boundary.  Complex arrays are interleaved (re, im) doubles.
 *
 * The entry points replace the reference's pybind11 surface for its bare
 * [pvpq | pq] Newton–Raphson path (file:line of the reference project):
 *   gs2g_session_create      AcPfNrSession / ContingencyAnalysisSession /
 *                            InjectionSweepSession / ScenarioSweepSession
 *                            constructors in array-tuple mode
 *                            (src/_cpp/python_bindings.cpp:1369, :1745, :2167, :2424)
 *   gs2g_set_branch_data     ContingencyAnalysisSession.set_branch_data
 *                            (src/gpusim2grid/contingency_analysis/gpu_facade.py:569)
 *   gs2g_set_contingencies   build_contingencies / set_topology
 *                            (src/_cpp/contingency_analysis_session.cu:188,
 *                             src/_cpp/scenario_sweep_session.cu:1009)
 *   gs2g_set_injections      InjectionSweepSession::set_injections
 *                            (src/_cpp/injection_sweep_session.cu:144-169, :239-245)
 *   gs2g_run                 ContingencyAnalysisSession::run / InjectionSweepSession::run /
 *                            ScenarioSweepSession::run
 *                            (src/_cpp/contingency_analysis_session.cu:394,
 *                             src/_cpp/injection_sweep_session.cu:194,
 *                             src/_cpp/scenario_sweep_session.cu:1267)
 *   gs2g_get_*               V_results / last_residuals / get_row_status /
 *                            get_row_iterations accessors
 *                            (src/gpusim2grid/contingency_analysis/gpu_facade.py:1025, :1203)
 *   gs2g_acpf_nr             acpf_nr_gpu (src/_cpp/python_bindings.cpp:1266-1285,
 *                            src/_cpp/acpf_nr.hpp:27-40)
 */
#ifndef GS2G_H
#define GS2G_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GS2G_OK 0
#define GS2G_ERR_INVALID 1   /* bad argument (reference: ValueError / std::invalid_argument) */
#define GS2G_ERR_RUNTIME 2   /* runtime failure (reference: RuntimeError) */
#define GS2G_ERR_CUDA 3      /* a CUDA call failed */

/* row status codes (src/_cpp/contingency/row_status.hpp:33-42) */
#define GS2G_ROW_CONVERGED 0
#define GS2G_ROW_MAX_ITER 1
#define GS2G_ROW_DIVERGED 2
#define GS2G_ROW_NOT_SIMULATED 3

/* linear-algebra precision of the Newton step */
#define GS2G_PREC_FP64 0  /* J, LU and solves in FP64 */
#define GS2G_PREC_MIXED 1 /* J, LU and solves in FP32; mismatch, norm and V in FP64 */

/* start voltage of the rows */
#define GS2G_START_VINIT 0 /* the session's Vinit (flat start) for every row */
#define GS2G_START_BASE 1  /* the converged base case, as the reference's batch sources */
#define GS2G_START_ROWS 2  /* one start per row, given by gs2g_set_start_rows */

typedef struct gs2g_session gs2g_session;

typedef struct gs2g_grid_info {
  int n_bus, nnz_y, n_pvpq, n_pq, dim_j;
  int64_t nnz_j, nnz_lu;
  int head_dim, tail_dim, tail_dim_exact, n_levels, n_supernodes;
  int64_t head_madds, schur_madds, dense_madds;
  double plan_ms;
} gs2g_grid_info;

typedef struct gs2g_run_opts {
  int max_iter;       /* Newton steps allowed per row */
  double tol;         /* ||F||inf threshold, per unit */
  int fixed_iters;    /* 1: exactly max_iter steps, then the residual (the reference's
                         chunked schedule); 0: stop each row at tol (continuous) */
  int precision;      /* GS2G_PREC_* */
  int start;          /* GS2G_START_* */
  double pivot_floor; /* static-pivot floor, 0 disables */
  int n_ctas;         /* persistent CTAs, <= 0 for one full wave */
  int profile_phases; /* 1: record per-phase SM cycles (gs2g_timings.phase_*) */
  /* GS2G_REFACTOR_EVERY: a new LU every Newton step (the reference's default
   * 'direct_refactor_every' strategy).  GS2G_REFACTOR_ADAPTIVE: keep the last
   * LU while ||F||inf shrinks by at least refactor_ratio per step, for at most
   * max_reuse steps (the reference's 'direct_iter0_only' idea, made adaptive);
   * the FP64 mismatch still converges every row to tol. */
  int refactor_policy;
  double refactor_ratio; /* <= 0 selects 0.3 (adaptive) or 0.7 (base_chord) */
  int max_reuse;         /* <= 0 selects 3 (adaptive) or 8 (base_chord) */
  /* 1: with GS2G_START_ROWS and the continuous schedule, guard each row's
   * given start (a learned or otherwise predicted one) against a bad
   * prediction.  With a base case, a row whose mismatch at its given start
   * is not below its mismatch at the base V starts from the base V instead.
   * A row that ends unconverged (MAX_ITER or DIVERGED) restarts once, inside
   * the same launch, from the base V (from Vinit without a base case), with
   * a fresh max_iter budget and a new LU every step; its iteration and
   * factorization counts include both attempts.  A given start whose
   * mismatch is not finite goes to that restart at once, without a step. */
  int rescue;
  /* Continuous schedule: Newton steps between two convergence tests of a
   * row (the reference's nb_iter_per_round,
   * src/gpusim2grid/contingency_analysis/_scheduling.py:145-156, rounds of
   * src/_cpp/contingency/batch_pf_driver.cu:2691-2724).  After each round
   * of k steps a row leaves DIVERGED (residual not finite), CONVERGED
   * (residual < tol) or MAX_ITER (steps >= max_iter); a row therefore runs a
   * multiple of k steps and at least k, also when it starts converged.
   * <= 0 selects 1; above 1000 is rejected (GS2G_ERR_INVALID). */
  int iters_per_round;
  /* 1: the reference's single-solve order (src/_cpp/acpf_nr.cu:505-561):
   * every iteration takes a full Newton step and then tests the mismatch
   * evaluated before that step, so a converged solve reports one step more
   * than the steps needed and returns the voltage after it; a solve that
   * never passes the test within max_iter steps ends MAX_ITER (DIVERGED
   * when its last mismatch is not finite).  Continuous schedule only. */
  int step_then_check;
  /* 1: the reference's MaxVoltageChange step scaling
   * (reduce_step_norms_kernel / apply_step_scale_kernel,
   * src/_cpp/acpf_nr_kernels.cu:677-726; facade option
   * scaling_max_voltage_change, src/gpusim2grid/acpf_nr/gpu_facade.py:100-121):
   * every Newton step is multiplied by alpha = min(1, max_dva / max|dtheta|,
   * max_dvm / max|dVm|) before it is applied, which keeps a step from far
   * away (a flat start, a heavily loaded row) from jumping to another
   * power-flow solution.  Under GS2G_REFACTOR_BASE_CHORD a row whose chord
   * step would be scaled leaves the chord for its own factor, where its
   * steps are scaled.  0 (default): full steps. */
  int step_scaling;
  double max_dva; /* radians; <= 0 selects 0.5 */
  double max_dvm; /* per unit; <= 0 selects 0.1 */
} gs2g_run_opts;

#define GS2G_REFACTOR_EVERY 0
#define GS2G_REFACTOR_ADAPTIVE 1
/* As ADAPTIVE, but every row starts its chord steps on the base case's
 * factor (its Jacobian at the base V; computed once per session and
 * precision, shared read-only by all rows) and factors its own Jacobian only
 * when a step stops contracting.  Needs a base case (solve_base or
 * set_base_v). */
#define GS2G_REFACTOR_BASE_CHORD 2

/* mismatch, fill, head LU, Schur, dense LU, solve: head forward, tail forward,
 * dense tail, head backward; update */
#define GS2G_N_PHASES 10

typedef struct gs2g_timings {
  double plan_ms;      /* symbolic analysis, once per session */
  double upload_ms;    /* last host-to-device copy of row data (wall) */
  double kernel_ms;    /* last sweep, CUDA events on the session stream */
  double total_ms;     /* last gs2g_run, wall */
  int64_t total_iters; /* sum of Newton steps over the rows of the last run */
  /* with profile_phases: SM cycles per phase summed over all CTAs, and each
   * phase's share of their total */
  double phase_cycles[GS2G_N_PHASES];
  double phase_share[GS2G_N_PHASES];
  int n_rescued;    /* rows of the last run restarted (gs2g_run_opts.rescue) */
  int n_base_start; /* rows of the last run that began from the base V instead of their given start */
  int64_t chord_steps; /* Newton steps of the last run taken in the chord sweep on the shared base factor */
  /* GS2G_REFACTOR_BASE_CHORD: the last set-up of the shared base factor (its
   * factorization, explicit inverse and packed solve values; done once per
   * session, base case and precision, outside every gs2g_run that reuses it):
   * wall ms and the device bytes it holds */
  double base_setup_ms;
  int64_t base_setup_bytes;
  /* rows of the last run (gs2g_run_subset re-solves included) whose status
   * is MAX_ITER or DIVERGED, counted when the timings are read */
  int64_t n_failed;
} gs2g_timings;

const char* gs2g_last_error(void);
int gs2g_version(void);
int gs2g_max_edits_per_row(void);

/* Session over one grid given as the reference's array tuple
 * (Ybus CSR, Vinit, Sbus, pv, pq).  `device` < 0 means the current device. */
int gs2g_session_create(int device, int n_bus, const int* ybus_indptr, const int* ybus_indices,
                        const double* ybus_values, const double* vinit, const double* sbus,
                        const int* pv, int n_pv, const int* pq, int n_pq, int tail_policy,
                        gs2g_session** out);
int gs2g_session_destroy(gs2g_session* s);
/* Rebuild the session's symbolic plan with other head/tail options: the
 * dense tail is extended with head columns while the planner's cost model,
 * (tail^3 / 3) / dense_rate + Schur volume, says so (dense_rate <= 0 keeps
 * the default 40; force_tau >= 0 forces the tail-row threshold; policy 0 =
 * exact trailing clique only).  Row definitions stay valid.  Used by the
 * facades' autotuner, which times candidate plans on the caller's rows
 * (the reference's lu_plan builds one plan; no counterpart). */
int gs2g_session_replan(gs2g_session* s, int tail_policy, double dense_rate, int force_tau);
/* GS2G_REFACTOR_BASE_CHORD with the continuous schedule runs in two launches:
 * a chord sweep that steps several rows per CTA in lockstep on the shared
 * base factor (every factor read serves all of them), then the single-row
 * sweep for the rows that need their own LU or the rescue, continued from
 * where the chord sweep left them.  mode 2 (default): the chord steps are
 * Broyden steps on the base factor (superlinear instead of linear
 * convergence); mode 1: plain chord steps, the same decisions as the
 * single-row sweep; mode 0: every row in the single-row sweep. */
int gs2g_session_set_chord(gs2g_session* s, int mode);
/* Rows that factor their own Jacobian after a chord sweep (its hand-offs),
 * and the rows of a gs2g_run_subset when there are few of them (at most one
 * per 8 CTAs of a full launch: the FP64 re-solve of the rows a mixed sweep
 * did not converge): cluster = 1 (default) runs each such row on a cluster
 * of 16 CTAs (8 when 16 per row do not fit in one launch), the leading CTA
 * running the row and all of them sharing each of its head LUs, Schur
 * updates and dense tail LUs (bit-identical to the one-CTA factorization,
 * FP32 and FP64); 0 runs each on one CTA.  Grids whose dense tail is under
 * 64 always use one CTA.  No counterpart in the reference (its batch LU has
 * no per-row kernel). */
int gs2g_session_set_handoff(gs2g_session* s, int cluster);
/* Order in which the persistent sweeps take the rows: on = 1 (default) by a
 * difficulty estimate, largest first -- the row's distance from the base
 * injections (sum over buses of |dP| + |dQ|, from gs2g_set_injections) plus
 * the base-case flow of each branch it trips -- so that rows needing many
 * steps start early and a sweep does not end on a tail of a few long rows;
 * 0: in row order.  Results are written per row and do not depend on the
 * order.  No counterpart in the reference (its rounds take rows in order). */
int gs2g_session_set_row_order(gs2g_session* s, int on);
/* handle_disconnected_grid (the reference's facade option,
 * src/gpusim2grid/contingency_analysis/gpu_facade.py:349, :544): on = 1
 * solves a row whose trips split the grid on its largest component -- the
 * most buses, on a tie the component holding the lowest bus
 * (compute_component_masks, src/_cpp/contingency_analysis_helper.cpp:657)
 * -- with every other bus masked: identity Jacobian rows and zero mismatch
 * for its P/Q equations (apply_bus_mask_kernel, src/_cpp/acpf_nr_kernels.cu:219),
 * so its voltage stays frozen, and NaN voltages for it in the results.  A
 * row that would mask an angle-reference (slack) bus is NOT_SIMULATED, as
 * are all splitting rows with on = 0 (default). */
int gs2g_session_set_handle_disconnected(gs2g_session* s, int on);
int gs2g_grid_get_info(const gs2g_session* s, gs2g_grid_info* out);
int gs2g_get_device(const gs2g_session* s, int* device);

/* Symbolic analysis only (host, no GPU needed): the statistics a session on
 * this grid would have.  Counterpart of the reference's once-only ANALYSIS
 * (src/_cpp/acpf_nr.cu:1466-1509, src/_cpp/own_lu/lu_plan.cpp:88-287). */
int gs2g_plan_info(int n_bus, const int* ybus_indptr, const int* ybus_indices, const int* pv, int n_pv,
                   const int* pq, int n_pq, int tail_policy, gs2g_grid_info* out);

/* π-model branch admittances, needed to trip branches. */
int gs2g_set_branch_data(gs2g_session* s, int n_branch, const int* from, const int* to,
                         const double* yff, const double* yft, const double* ytf, const double* ytt);
/* Batch rows as tripped-branch lists (CSR: row r trips ids[ptr[r]..ptr[r+1])).
 * n_rows = 0 clears them.  With injections also set, rows combine both. */
int gs2g_set_contingencies(gs2g_session* s, int n_rows, const int* ptr, const int* ids);
/* Per-row injections in MW / MVAr, row-major [n_rows x n_bus]; Sbus = (p + jq)/sn_mva.
 * n_rows = 0 clears them. */
int gs2g_set_injections(gs2g_session* s, int n_rows, const double* p_mw, const double* q_mvar, double sn_mva);
/* Per-row start voltages, complex [n_rows x n_bus] (used with GS2G_START_ROWS). */
int gs2g_set_start_rows(gs2g_session* s, int n_rows, const double* v0);
/* Same, from device memory already on the session's device. */
int gs2g_set_start_rows_device(gs2g_session* s, int n_rows, const double* v0_dev);
/* The session's own start-row buffer, complex [n_rows x n_bus] on its
 * device, for callers that compute start voltages on the GPU and write them
 * in place (no copy).  Sizes the buffer and records n_rows start rows; its
 * contents are used by the next GS2G_START_ROWS run, so the caller's writes
 * must be complete (its stream synchronised, or ordered before the session
 * stream by gs2g_session_wait_stream) before gs2g_run.  Valid until
 * the next call that sets start rows or destroy. */
int gs2g_start_rows_buffer(gs2g_session* s, int n_rows, double** v0_dev);
/* Replace the base injections (single-solve resolve). */
int gs2g_set_sbus(gs2g_session* s, const double* sbus);
/* Replace Vinit. */
int gs2g_set_vinit(gs2g_session* s, const double* vinit);

/* Solve the base case (no trips, base Sbus) from Vinit; keeps it as the
 * GS2G_START_BASE start.  Fills status/iters/residual if not NULL. */
int gs2g_solve_base(gs2g_session* s, const gs2g_run_opts* o, double* v_out, int* status, int* iters, double* residual);
/* Validate a converged base V (the reference's init_from_n_powerflow path):
 * returns the residual of V and stores it as the base start. */
int gs2g_set_base_v(gs2g_session* s, const double* v, double* residual);

/* Run every row.  Results stay on the device until read. */
int gs2g_run(gs2g_session* s, const gs2g_run_opts* o);
/* Re-run some rows of the last full run in place (other options allowed,
 * e.g. FP64 from Vinit for the rows a mixed-precision run did not converge):
 * rows[0..n_sub) index the assembled rows; their outputs are overwritten,
 * every other row's stay.  Needs a full gs2g_run of the same rows first.
 * The facades use it for the FP64 fallback of mixed-precision sweeps. */
int gs2g_run_subset(gs2g_session* s, const gs2g_run_opts* o, int n_sub, const int* rows);
/* Several grids in ONE persistent launch: the current rows of every session
 * (as gs2g_run would run them, same options for all) are solved by one
 * kernel launch whose CTAs take rows from one queue across the grids, each
 * with its own symbolic plan.  Results land in each session's own buffers
 * (gs2g_get_results etc. per session).  All sessions on one device, each
 * listed once, at most 16.  The launch runs on the first session's stream;
 * gs2g_timings of every session get its kernel time (rescue count and phase
 * counters on the first).  The reference runs one grid per session; this
 * serves the heterogeneous batch (rows of 118- to 10000-bus grids). */
int gs2g_run_multi(gs2g_session* const* sessions, int n_sessions, const gs2g_run_opts* o);
int gs2g_n_rows(const gs2g_session* s);
int gs2g_get_results(const gs2g_session* s, double* v_out, double* residuals, int* status, int* iters);
/* LU factorizations each row of the last run performed. */
int gs2g_get_factor_counts(const gs2g_session* s, int* factors);
/* Branch flows and limit check as each row leaves the GPU (the reference's
 * compute_branch_flows_kernel, src/_cpp/acpf_nr_kernels.cu:87-183, and
 * check_limit_violations, src/_cpp/contingency/violation_kernels.cu:297,
 * done by the row's own CTA on its final V).  rate_mva: one limit per branch
 * of gs2g_set_branch_data (<= 0: unlimited); n_branch = 0 turns it off.
 * Per row and branch: loading = max(|S_from|, |S_to|) / rate (0 for tripped
 * or unlimited branches, NaN for rows that did not converge or were not
 * simulated); per row: branches with loading > 1 (-1: not converged) and the
 * largest loading.  Setting branch data again turns the limits off. */
int gs2g_set_branch_limits(gs2g_session* s, int n_branch, const double* rate_mva, double sn_mva);
/* loading [n_rows x n_branch], n_violations [n_rows], max_loading [n_rows]; any may be NULL. */
int gs2g_get_branch_loading(const gs2g_session* s, float* loading, int* n_violations, float* max_loading);
/* Host copies of the last run's results in page-locked memory the session
 * owns (one DMA per array at full link speed, no copy through pageable
 * memory): V [n_rows x n_bus] complex, residuals, status, iters.  The
 * pointers stay valid, and their contents unchanged, until the next call of
 * this function, the next run or destroy: the lifetime of the reference's
 * V_results device buffer (src/gpusim2grid/contingency_analysis/gpu_facade.py:1203)
 * and of its DLPack exports.  No counterpart for the pinned copy itself. */
int gs2g_get_results_host(gs2g_session* s, double** v, double** residuals, int** status, int** iters);
/* Results mirror: on = 1 makes every later run (gs2g_run, gs2g_run_subset,
 * gs2g_run_multi) also write each row's final voltages straight into the
 * page-locked buffer gs2g_get_results_host returns, from the kernels, as
 * the row leaves -- the device-to-host transfer of V overlaps the sweep,
 * and gs2g_get_results_host then copies only the residuals, statuses and
 * iterations.  A run overwrites that buffer while it runs.  The device
 * results (gs2g_get_results, the DLPack exports) are unchanged.  Default 0.
 * No counterpart in the reference (its results stay on the device). */
int gs2g_session_set_results_mirror(gs2g_session* s, int on);
/* Batched adjoint of the last run: for every row r of it, lam[r] = J_r^-T
 * rhs[r], J_r the row's Jacobian (FP64) at its converged voltage, with its
 * branch trips and masked buses; the sensitivity of the converged state to
 * the row's injections (dx/ds = J^-1, so dL/ds = J^-T dL/dx).  rhs and lam
 * are device arrays [n_rows x dim_J] in the reference's J layout (P/theta
 * rows on sorted pv+pq, then Q/Vm rows on pq); non-finite rhs entries count
 * as 0; rows that did not converge, and a masked bus's entries, get 0.
 * n_rows must equal the last run's rows.  Replaces the reference's
 * solve_JT_batch (src/_cpp/contingency/batch_pf_driver.cuh:180-224,
 * src/gpusim2grid/differentiable/_batch_pf.py backward); each row's J is
 * refactored here instead of keeping the forward factors. */
int gs2g_solve_jt(gs2g_session* s, int n_rows, const double* rhs, double* lam);
/* Device pointers of the last run's results (valid until the next run or destroy). */
int gs2g_get_device_results(const gs2g_session* s, double** v, double** residuals, int** status, int** iters);
/* Device copies of the current row definitions (uploaded first if they
 * changed): sbus_rows [n_rows x n_bus] complex per unit (NULL: the rows use
 * the base injections), trip_ptr [n_rows + 1] / trip_ids [n_trip_ids] CSR of
 * tripped branches (NULL: no trips).  Valid until the rows change.  A
 * device-resident caller (e.g. a learned start) reads them instead of
 * shipping the rows again.  The rows' Ybus edits, islanding verdicts and
 * order are built by the next run, so a caller's network on these rows and
 * that host work overlap. */
int gs2g_get_device_rows(gs2g_session* s, int* n_rows, const double** sbus_rows, const int** trip_ptr,
                         const int** trip_ids, int64_t* n_trip_ids);
int gs2g_get_timings(const gs2g_session* s, gs2g_timings* out);
/* Synchronise the session stream. */
int gs2g_sync(gs2g_session* s);
/* Order the session stream after the work enqueued so far on `stream` (NULL:
 * the legacy default stream) on the device, without a host
 * synchronisation: e.g. start voltages written into gs2g_start_rows_buffer
 * by a network on the caller's stream, then gs2g_run.  (The reference
 * synchronises instead; no counterpart.) */
int gs2g_session_wait_stream(gs2g_session* s, void* stream);

/* Allocation-free batch solve.  No counterpart in the reference: this entry
 * point exists for callers that must not allocate device memory while they
 * solve -- e.g. code running under a framework's memory pool or arena that
 * forbids cudaMalloc/cudaFree in its hot path, or real-time code that cannot
 * afford an allocation's implicit synchronisation.  It runs the same sweep
 * kernel as gs2g_run on rows that differ by start voltage and injections (no
 * branch trips), with every input and output in caller-provided device
 * memory, and keeps the kernel's scratch (the row queue and per-row
 * workspaces, max 64 MiB in total) in a static device array the library
 * holds on each GPU that loads it.  It calls no cudaMalloc, cudaFree or
 * allocating library routine.
 *   v0 / sbus: complex rows (interleaved doubles) with strides in complex
 *   elements (0: one row shared by all).  Outputs as gs2g_get_device_results.
 *   Grids whose per-row workspace exceeds the static scratch are rejected
 *   (GS2G_ERR_INVALID); fewer rows run at once when fewer workspaces fit.
 *   The first call on a device looks up the array's device address (make it
 *   before any stream capture).  Every call shares the array: calls that
 *   overlap on the GPU race.  Returns once the work is enqueued on `stream`
 *   (NULL = default stream); synchronise it before reading the outputs.
 *   The rescue option restarts from the session's Vinit; its count is not
 *   recorded (gs2g_timings is not touched).
 *   Of gs2g_run_opts it reads max_iter, tol, fixed_iters, precision,
 *   pivot_floor, refactor_policy (GS2G_REFACTOR_EVERY or _ADAPTIVE only;
 *   GS2G_REFACTOR_BASE_CHORD needs session buffers and is rejected),
 *   refactor_ratio, max_reuse, rescue, iters_per_round and step_then_check;
 *   start, n_ctas, profile_phases and the step scaling (step_scaling,
 *   max_dva, max_dvm) are ignored (the rows start from v0, the CTA count is
 *   what fits the scratch, no phase counters, full steps).
 *   The device address of the scratch array is looked up once per device
 *   and kept for the life of the process: after cudaDeviceReset (or any
 *   re-creation of the device's primary context) this entry point must not
 *   be called again in that process. */
int gs2g_run_rows_noalloc(const gs2g_session* s, int n_rows, const double* v0, int64_t v0_stride,
                          const double* sbus, int64_t sbus_stride, const gs2g_run_opts* o, double* v_out,
                          double* residuals, int* status, int* iters, void* stream);

/* ---- Warm-start MLP building blocks ------------------------------------
 * The learned start voltage (the reference's ScenarioSweepGPU warm_start
 * slot, src/gpusim2grid/scenario_sweep/gpu_facade.py, which takes any
 * per-row V0) is produced by an MLP trained and evaluated with these device
 * routines.  All pointers are device memory on the current device; `stream`
 * NULL = default stream; each call only enqueues work.  bf16 arrays are
 * passed as void*.  Row-major matrices, `ld*` in elements.
 *
 * D[M x N] (fp32) = A[M x K] . B[N x K]^T (+ D when accumulate), A, B bf16,
 * on tcgen05 tensor cores.  M, N multiples of 128, K of 64; lda, ldb
 * multiples of 8, ldd of 4; 16-byte aligned bases.  *err is set to 1 if a
 * bounded wait inside the kernel ran out (the tile is then not written). */
int gs2g_mlp_gemm_tn_bf16(const void* A, int lda, const void* B, int ldb, float* D, int ldd, int M, int N, int K,
                          int accumulate, int* err, void* stream);
/* pre += bias (per column); act = bf16(gelu(pre)) (exact erf GELU) or
 * bf16(pre) when gelu = 0; act may be NULL. */
int gs2g_mlp_bias_act(float* pre, int ldp, const float* bias, void* act_bf16, int lda, int rows, int cols, int gelu,
                      void* stream);
/* dpre = bf16(dact * gelu'(pre)) */
int gs2g_mlp_gelu_bwd(const float* dact, int ldg, const float* pre, int ldp, void* dpre_bf16, int ldo, int rows,
                      int cols, void* stream);
/* dy = bf16(scale * (y - t)) on the first cols_valid columns, 0 on the rest;
 * *loss += sum of (y - t)^2 over the valid entries (loss may be NULL). */
int gs2g_mlp_mse_grad(const float* y, const float* t, int ld, void* dy_bf16, int rows, int cols, int cols_valid,
                      float scale, float* loss, void* stream);
/* out[c] = sum over rows of x[r][c] (bf16 in, fp32 out) */
int gs2g_mlp_colsum_bf16(const void* x, int ld, int rows, int cols, float* out, void* stream);
/* out[c][r] = in[r][c] (bf16) */
int gs2g_mlp_transpose_bf16(const void* in, int ldi, void* out, int ldo, int rows, int cols, void* stream);
/* out = bf16(in), n elements */
int gs2g_mlp_to_bf16(const float* in, void* out, int64_t n, void* stream);
/* One Adam step (bias-corrected, step >= 1, L2 weight decay added to the
 * gradient) on fp32 master weights; also writes their bf16
 * copy when w_bf16 is not NULL. */
int gs2g_mlp_adam(float* w, const float* g, float* m, float* v, void* w_bf16, int64_t n, float lr, float beta1,
                  float beta2, float eps, int step, float weight_decay, void* stream);
/* The network's standardised bf16 input block X [rows_pad x ldx] of `rows`
 * rows in one pass: columns [0, n_pvpq) the rows' active injections minus
 * the base case at buses pvpq, [n_pvpq, n_pvpq + n_pq) the reactive ones at
 * buses pq (0 when sbus_rows is NULL; complex rows of n_bus per unit),
 * plus, for every tripped branch b of a row (CSR trip_ptr / trip_ids, NULL:
 * none), the four values br_val[4b + k] at columns br_col[4b + k] (a column
 * < 0 or >= n_in is dropped); then (x - x_mean) / x_std for the n_in input
 * columns and 0 in the padding columns and rows. */
int gs2g_mlp_features(const double* sbus_rows, const double* sbus_base, const int* pvpq, int n_pvpq, const int* pq,
                      int n_pq, const int* trip_ptr, const int* trip_ids, const int* br_col, const float* br_val,
                      const float* x_mean, const float* x_std, int n_in, void* x_bf16, int ldx, int rows,
                      int rows_pad, int n_bus, void* stream);
/* The first layer's pre-activations for rows without injection part
 * (gs2g_mlp_features with sbus_rows NULL), from the few input columns their
 * tripped branches reach: pre[r] = base + sum over those columns c of
 * (bf16(xs_c) - bf16(-x_mean_c / x_std_c)) * W0T[c], the column values
 * summed as gs2g_mlp_features sums them; pre [rows_pad x ldp] fp32, 0 in
 * the padding rows.  W0T = W0^T (bf16, [n_in x h] row-major; W0 is the
 * first layer's [h x k0] weight) and base = gs2g_mlp_first_layer_base of the
 * same weights.  Equals X W0^T of the standardised inputs up to fp32
 * summation order.  (The reference has no network; no counterpart.) */
int gs2g_mlp_sparse_first_layer(const float* base, const void* w0t_bf16, int h, const int* trip_ptr,
                                const int* trip_ids, const int* br_col, const float* br_val, const float* x_mean,
                                const float* x_std, int n_in, float* pre, int ldp, int rows, int rows_pad,
                                void* stream);
/* base[h] = sum over the n_in input columns of bf16(-x_mean_c / x_std_c) *
 * W0T[c] (the first layer's product with an all-zero raw input row). */
int gs2g_mlp_first_layer_base(const void* w0t_bf16, int h, const float* x_mean, const float* x_std, int n_in,
                              float* base, void* stream);
/* Start voltages from the network's standardised outputs y[rows x ldy]:
 * bus b takes Va = y[va_index[b]] * y_std + y_mean when va_index[b] >= 0
 * (pv and pq buses), else the angle of vinit[b]; Vm likewise through
 * vm_index (pq buses), else |vinit[b]|.  v0 = complex [rows x n_bus]. */
int gs2g_mlp_start_voltages(const float* y, int ldy, const float* y_mean, const float* y_std, const int* va_index,
                            const int* vm_index, const double* vinit, int n_bus, double* v0, int rows, void* stream);

/* acpf_nr_gpu: one solve from Vinit, V written back into `v_inout`.
 * Returns the status through *converged (1/0), *iters and *residual. */
int gs2g_acpf_nr(int device, int n_bus, const int* ybus_indptr, const int* ybus_indices,
                 const double* ybus_values, double* v_inout, const double* sbus,
                 const int* pv, int n_pv, const int* pq, int n_pq, int max_iter, double tol,
                 int precision, int* converged, int* iters, double* residual, double* kernel_ms);

#ifdef __cplusplus
}
#endif

#endif /* GS2G_H */
