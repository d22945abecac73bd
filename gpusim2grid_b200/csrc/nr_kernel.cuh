// Device-side interface of the persistent batched Newton–Raphson kernel.
// Plain structs of device pointers; no CUDA or torch types leak into the
// C-ABI headers.
#pragma once

#include <cstdint>

namespace gs2g {

// Status codes of one batch row, the reference's RowStatus
// (src/_cpp/contingency/row_status.hpp:33-42).
enum RowStatusCode : int { ROW_CONVERGED = 0, ROW_MAX_ITER = 1, ROW_DIVERGED = 2, ROW_NOT_SIMULATED = 3 };

// Device copy of a Plan (see plan.hpp); every pointer is device memory.
struct DevPlan {
  int n_bus, nnz_y, dim, p, nt, ld, n_hv, n_levels;
  const int* y_indptr;
  const int* y_indices;
  const int* y_row;
  const int* jmap;     // [4 * nnz_y]
  const int* fP;       // [n_bus]
  const int* fQ;       // [n_bus]
  const int* lev_ptr;  // [n_levels + 1] into tasks
  const int* lev_big;  // [n_levels]: tasks [lev_ptr[l], lev_big[l]) are long (warp per task)
  const int* task_out;
  const int* task_diag;
  const int* task_pbeg;
  const int* task_pend;
  const uint8_t* task_has_a;
  const int* pair_l;
  const int* pair_u;
  const int* lev_piv_ptr;  // [n_levels + 1] into lev_piv
  const int* lev_piv;      // head pivots by level
  const int* sn_w;
  const int* sn_t;
  const int* sn_L;
  const int* sn_U;
  const int* sn_tidx;
  const int* tidx;
  const int* sg_ptr;  // [nt + 1] Schur column groups per tail row
  const int* sg_col;  // tail column of each group
  const int* se_ptr;  // [groups + 1] entries per group
  const int4* se_rec;  // per entry: HV offset of its L values, of its first U value, w | t << 4 (U stride t)
  const int* fw_ptr;  // [dim + 1]
  const int* fw_col;
  const int* fw_pos;
  const int* bw_ptr;  // [p + 1]
  const int* bw_row;
  const int* bw_pos;
  // transposed solves (see plan.hpp) and the J-index -> factor position map
  const int* ut_ptr;
  const int* ut_row;
  const int* ut_pos;
  const int* lt_ptr;
  const int* lt_row;
  const int* lt_pos;
  const int* iperm;
};

// One launch = one sweep over a list of rows.
struct SweepArgs {
  int n_rows;             // rows of this launch (queue length)
  const int* row_map;     // [n_rows] row of the session solved for queue entry q (nullptr: q itself)
  const double* ybus;     // [2 * nnz_y] interleaved complex base Ybus values
  const double* v0;       // start voltage, complex, row r at v0 + 2 * r * v0_stride
  int64_t v0_stride;      // in complex elements (0: shared)
  const double* sbus;     // complex injections, row r at sbus + 2 * r * sbus_stride
  int64_t sbus_stride;
  const int* edit_ptr;    // [n_rows + 1] per-row Ybus edits (nullptr: none)
  const int* edit_k;      // Ybus entry index
  const double* edit_val; // complex delta to SUBTRACT
  const int* row_skip;    // [n_rows] nonzero: NOT_SIMULATED (nullptr: none)
  // handle_disconnected_grid: buses of row r outside its largest component,
  // mask_bus[mask_ptr[r] .. mask_ptr[r + 1]) (nullptr: none).  Their P/Q
  // equations become identity rows with zero mismatch (the voltage stays
  // frozen), they leave the norm, and their voltages are reported NaN.
  const int* mask_ptr;
  const int* mask_bus;
  int max_iter;
  double tol;
  int fixed_iters;        // 1: exactly max_iter steps then the residual; 0: stop at tol
  // continuous schedule: a row's mismatch is tested only after every
  // round_k-th step (so a row runs a multiple of round_k steps, at least
  // round_k), the reference's nb_iter_per_round
  int round_k;
  // 1: the reference's single-solve order: each step is taken, then the
  // mismatch evaluated before it decides convergence (no round rule)
  int step_first;
  int refactor_policy;    // 0: refactor every step; 1: reuse the LU while ||F|| contracts;
                          // 2: as 1, starting on the base case's factor (base_ws)
  double refactor_ratio;  // policy 1: refactor when ||F_k|| > ratio * ||F_{k-1}||
  int max_reuse;          // policy 1: refactor after this many steps on one LU
  int* factors_out;       // [n_rows] LU factorizations per row (nullptr: not recorded)
  // rescue: a row that ends unconverged (continuous schedule) restarts once
  // from this complex [n_bus] voltage (nullptr: no rescue); n_rescued counts
  // the restarts (nullptr: not counted)
  const double* rescue_v0;
  int* n_rescued;
  // start selection: a row whose first mismatch at its own start is not
  // below the mismatch at this complex [n_bus] voltage (the base case) starts
  // from it instead (nullptr: off); n_alt_start counts those rows
  const double* alt_v0;
  // per-row Newton steps already taken by another launch (nullptr: none);
  // may alias iters_out (read at the row's start, written at its end)
  const int* iters_in;
  // chord sweep (see launch_chord): rows it hands to the single-row kernel
  // are appended to handoff ([n_rows]) and counted in *n_handoff
  int* handoff;
  int* n_handoff;
  int handoff_base;  // added to the row id in handoff (multi-grid: the grid's first global row)
  // when set, the launch's row count is read here on the device (a launch
  // that follows the chord sweep on the same stream takes its hand-offs)
  const int* n_rows_dev;
  const double* alt_s;  // complex [n_bus] V conj(Y V) at alt_v0 on the unedited Ybus (nullptr: evaluate in full)
  // complex [n_bus] Y V at alt_v0 on the unedited Ybus, summed over each
  // Ybus row in the order of the sweep's mismatch (nullptr: evaluate in full)
  const double* alt_i;
  // chord sweep: per-row outage compensation records set up ahead of it by
  // launch_comp_setup ([n_rows] of comp_rec_bytes(); nullptr: set up in the
  // sweep)
  const char* comp_rec;
  int* n_alt_start;
  // chord sweep: Newton steps taken on the shared base factor, summed over rows
  unsigned long long* n_chord_steps;
  // chord sweep: Broyden updates of the base factor's steps (see chord_sweep.cuh)
  int broyden;
  // policy 2: workspace (ws_layout of this plan and precision) holding the
  // base case's factor, shared read-only by every CTA; factor_only: factor
  // the Jacobian at the start voltage into the CTA's workspace and stop
  const char* base_ws;
  const double* base_v;  // complex [n_bus]: the voltage the base factor was taken at
  const char* base_inv;  // [dim x dim] of the sweep's type: column c = M0^-1 e_c (outage compensation)
  // the base factor's head values in solve order (of the sweep's type):
  // base_fwv[q] = HV[fw_pos[q]], base_bwv[q] = HV[bw_pos[q]] (nullptr: gather)
  const char* base_fwv;
  const char* base_bwv;
  char* inverse_out;     // inverse mode: row r of the launch writes column r of M0^-1 here
  int factor_only;
  // branch flows and limit check when the row leaves (loading_out nullptr: off)
  int n_branch;
  const int* br_from;
  const int* br_to;
  const double* br_y;     // [n_branch * 4] complex: yff, yft, ytf, ytt
  const double* br_rate;  // [n_branch] limits, per unit (<= 0: no limit)
  const int* trip_ptr;    // [n_rows + 1] tripped branch ids per row (nullptr: none)
  const int* trip_ids;
  float* loading_out;     // [n_rows * n_branch] max(|S_from|, |S_to|) / rate (0: tripped or no limit)
  int* nviol_out;         // [n_rows] branches above their limit (-1: row not converged)
  float* maxload_out;     // [n_rows]
  // outputs
  double* v_out;          // [n_rows * n_bus] complex
  double* v_mirror;       // nullptr, or a host-mapped copy of v_out that gets each row's final V as it leaves
  int step_scaling;       // MaxVoltageChange: steps scaled so max|dtheta| <= max_dva, max|dVm| <= max_dvm
  double max_dva, max_dvm;
  double* res_out;        // [n_rows]
  int* status_out;        // [n_rows]
  int* iters_out;         // [n_rows]
  // scheduling
  int* queue;             // one int, zeroed before the launch
  char* workspace;        // per-CTA scratch
  int64_t ws_stride;      // bytes per CTA
  double pivot_floor;     // static-pivot floor (|u_kk| below it is raised to it)
  // optional: per-phase SM cycles summed over CTAs (nullptr: not recorded)
  unsigned long long* phase_cycles;  // [N_PHASES]
};

// Phases of one Newton iteration, as the reference's per-phase timings
// (AcPfTimings, src/_cpp/timing_utils.hpp:131-215) split them.
enum Phase : int {
  PH_MISMATCH = 0,  // SpMV + mismatch + norm
  PH_FILL = 1,      // zero the tail + Jacobian fill
  PH_HEAD = 2,      // sparse head LU
  PH_SCHUR = 3,     // Schur update of the tail
  PH_DENSE = 4,     // dense tail LU
  PH_SOLVE = 5,     // triangular solves: head forward
  PH_SOLVE_TAIL = 6,   // forward rows of the tail against the head
  PH_SOLVE_DENSE = 7,  // dense tail forward + backward
  PH_SOLVE_BACK = 8,   // head backward
  PH_UPDATE = 9,       // voltage update
  N_PHASES = 10
};

// Per-CTA workspace bytes for precision `prec` (0: fp64 LU, 1: fp32 LU).
int64_t workspace_bytes(const DevPlan& P, int prec);
// byte offset of the head factor values (n_hv of the precision's type) in a workspace
int64_t workspace_hv_offset(const DevPlan& P, int prec);

// Launch the sweep on `stream` with `n_ctas` CTAs (<= 0: one wave at full
// occupancy).  Returns the cudaError_t as int.
int launch_sweep(const DevPlan& P, const SweepArgs& a, int prec, int n_ctas, void* stream);

// Chord sweep (policy 2, continuous schedule): chord_rows_per_cta() rows per
// CTA step in lockstep on the base factor (a.base_ws) with its inverse
// (a.base_inv); converged rows are finished, the others are handed off to a
// following single-row launch (a.handoff / a.n_handoff, their V in v_out and
// steps in iters_out).  Workspace per CTA: chord_workspace_bytes.
int64_t chord_workspace_bytes(const DevPlan& P, int prec);
int chord_rows_per_cta();
int chord_ctas(const DevPlan& P, int prec, int device);
int launch_chord(const DevPlan& P, const SweepArgs& a, int prec, int n_ctas, void* stream);
// The outage compensation of every row (a.edit_ptr rows 0..n_rows-1) on the
// base factor (a.base_v, a.base_inv), one small CTA per row, into rec
// ([n_rows] x comp_rec_bytes()), for the chord sweep that follows on the
// stream (a.comp_rec).
int64_t comp_rec_bytes();
int launch_comp_setup(const DevPlan& P, const SweepArgs& a, int prec, int n_rows, void* rec, void* stream);

// CTAs that fit at once for `prec` (for sizing the workspace).
int sweep_ctas(int prec, int device);

// The single-row sweep (prec 1: FP32 factors, 0: FP64) with a cluster of
// `cluster` CTAs per row (8, or 16 up to handoff_cluster_size()): the
// cluster's leading CTA runs the row (its workspace: the leader's block
// index times ws_stride), and all of them share each of its head LUs, Schur
// updates and dense tail LUs.  n_ctas a multiple of the cluster size.
int handoff_cluster_size();

// Batched adjoint (FP64): lam[r] = J_r^-T rhs[r] for the a.n_rows rows of a
// sweep (a.v_out the converged voltages, a.status_out their statuses, the
// rows' edits and masks as in the sweep), J_r at the row's converged V; rows
// that did not converge get 0.  rhs / lam [n_rows x dim] in the reference's
// J layout.  Workspace a.workspace / a.ws_stride (double layout), queue
// zeroed by the caller.
int launch_adjoint(const DevPlan& P, const SweepArgs& a, const double* rhs, double* lam, int n_ctas, void* stream);
int launch_sweep_cluster(const DevPlan& P, const SweepArgs& a, int prec, int cluster, int n_ctas, void* stream);

// Several grids in one persistent launch (see sweep_kernel_multi): the plan
// and the per-grid launch arguments of each grid (SweepArgs fields n_rows,
// ybus, v0, sbus, edits, skip, options and outputs; its queue, workspace and
// phase_cycles are not used).
constexpr int MAX_GRIDS = 16;
struct GridEntry {
  DevPlan P;
  SweepArgs a;
};
// d_grids [n_grids] and d_row_begin [n_grids + 1] in device memory; queue
// zeroed by the caller; workspace n_ctas * ws_stride bytes, ws_stride >=
// workspace_bytes of every grid.
// With row_list, queue entry q solves global row row_list[q] and the entry
// count is read from *n_rows_dev (the hand-offs of a multi-grid chord sweep).
int launch_sweep_multi(const GridEntry* d_grids, int n_grids, const int* d_row_begin, int n_rows, int* queue,
                       char* workspace, int64_t ws_stride, unsigned long long* phase_cycles, int prec, int n_ctas,
                       void* stream, const int* row_list = nullptr, const int* n_rows_dev = nullptr);
// Multi-grid chord sweep over d_grids (policy 2, every grid with its base
// factor and inverse; each grid's a.queue its own zeroed counter; a.handoff
// one list for all grids, a.handoff_base the grid's first global row).
// smem: the largest chord_smem of the grids.
int launch_chord_multi(const GridEntry* d_grids, int n_grids, int smem, unsigned long long* phase_cycles, int prec,
                       int n_ctas, void* stream);
int chord_smem(const DevPlan& P, int prec);

// Size of the file-scope device array the allocation-free sweep uses as its
// scratch (row queue + per-CTA workspaces).
constexpr int64_t kStaticScratchBytes = int64_t(64) << 20;

// Launch the sweep with its scratch in that static array instead of caller
// memory: a.queue / a.workspace / a.ws_stride are filled in here.  `device`
// must be the current device.  Returns a cudaError_t as int;
// cudaErrorInvalidValue when one CTA's workspace does not fit the array.
// *n_ctas_used receives the CTA count (bounded by what fits).
int launch_sweep_static(const DevPlan& P, SweepArgs a, int prec, int device, void* stream, int* n_ctas_used);

}  // namespace gs2g
