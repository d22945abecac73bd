// Symbolic plan of the batched Newton–Raphson power flow on one grid.
//
// Everything here is integer work done once per grid on the host and shared,
// bit-identical, by every batch row: the Jacobian layout, the fill-reducing
// order, the elimination structure, the split of the factor into a sparse
// "head" and a dense "tail", and every index list the device code walks.
//
// Reference counterparts:
//   * J layout (P/θ on sorted(pv ∪ pq) at [0, n_pvpq), Q/Vm on pq in input
//     order at [n_pvpq, dim_J)): src/_cpp/acpf_nr.cu:130-236, :645-685.
//   * One symbolic analysis shared by the whole batch (cuDSS ANALYSIS once,
//     own-LU plan): src/_cpp/contingency/strategies/cudss_batch_solver.cuh:273-690,
//     src/_cpp/own_lu/lu_plan.cpp:88-287.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace gs2g {

// Encoded destination of one Jacobian coefficient in the per-row factor
// storage: >= 0 is an index into the head value array HV; <= -2 is an index
// into the dense tail S as -(off + 2); -1 means the coefficient does not exist.
inline int encode_tail(int off) { return -(off + 2); }

struct TailOptions {
  // 0: the tail is the exact dense trailing clique.  1: extend it with the
  // head columns a cost model says are cheaper as dense work (default).
  int policy = 1;
  // cost-model weights: dense madds per unit of cost and scatter volume per unit
  double dense_rate = 40.0;
  double scatter_rate = 1.0;
  // forced tail-row threshold (< 0: chosen by the cost model)
  int force_tau = -1;
};

struct Plan {
  // ---- grid -------------------------------------------------------------
  int n_bus = 0;
  int nnz_y = 0;
  std::vector<int> y_indptr, y_indices;  // CSR, sorted columns
  std::vector<int> y_row;                // row of every Ybus entry
  std::vector<int> y_diag;               // position of (i,i) per bus, -1 if absent

  // ---- Jacobian layout (reference order) --------------------------------
  int n_pvpq = 0, n_pq = 0, dim = 0;
  std::vector<int> pvpq, pq;  // sorted(pv ∪ pq); pq in input order

  // ---- factor order -----------------------------------------------------
  // perm[f] = J index of factor position f; iperm[j] = factor position.
  std::vector<int> perm, iperm;
  // per bus: factor position of its P row / θ column (or -1), Q row / Vm column (or -1)
  std::vector<int> fP, fQ;

  // ---- head / tail split ------------------------------------------------
  int p = 0;     // head size (variables)
  int nt = 0;    // tail size
  int ld = 0;    // leading dimension of the dense tail (row-major)
  int n_hv = 0;  // head value array length

  // head pivot levels: tasks of level l are [lev_ptr[l], lev_ptr[l+1])
  int n_levels = 0;
  std::vector<int> lev_ptr;
  // within level l, tasks [lev_ptr[l], lev_big[l]) have at least kBigTask
  // products (one warp each on the device), the rest one thread each
  std::vector<int> lev_big;
  static constexpr int kBigTask = 24;
  // head pivots by level (for the level-scheduled triangular solves)
  std::vector<int> lev_piv_ptr, lev_piv;
  // head tasks: out position in HV; has_a flag; diag position for L entries
  // (divide after accumulation) or -1; pair range.
  std::vector<int> task_out, task_diag, task_pbeg, task_pend;
  std::vector<uint8_t> task_has_a;
  std::vector<int> pair_l, pair_u;  // HV positions of l and u in each product
  int64_t head_madds = 0;

  // head supernodes (for the tail blocks and the Schur update)
  int n_sn = 0;
  std::vector<int> sn_first, sn_w, sn_t, sn_L, sn_U, sn_tidx;  // sn_tidx: offset into tidx
  std::vector<int> tidx;  // tail-local row index of every tail row of every supernode
  // Schur items per tail row: [schur_ptr[ti], schur_ptr[ti+1]) of (sn, a)
  std::vector<int> schur_ptr, schur_sn, schur_a;
  // The same update as column groups, the form the device runs: tail row ti
  // owns groups [sg_ptr[ti], sg_ptr[ti+1]); group g updates S[ti][sg_col[g]]
  // with the sum over entries [se_ptr[g], se_ptr[g+1]) of
  //   sum_{c < w} HV[se_L[e] + c] * HV[se_U[e] + c * t],  w | t << 4 = se_wt[e]
  // (entries of a group in supernode order).
  std::vector<int> sg_ptr, sg_col, se_ptr, se_L, se_U, se_wt;
  std::vector<int> se_rec;  // [4 * entries]: (se_L, se_U, se_wt, 0) packed for one 16-byte load
  int64_t schur_madds = 0, schur_volume = 0;
  int64_t dense_madds = 0;

  // solves (factor order)
  // forward: per row i, (m, HV pos of l_im) over head columns m
  std::vector<int> fw_ptr, fw_col, fw_pos;
  // backward: per head pivot k, (i, HV pos of u_ki) over i in struct(k)
  std::vector<int> bw_ptr, bw_row, bw_pos;
  std::vector<int> diag_pos;  // HV position of u_kk, k < p (== k)
  // transposed solves (the adjoint J^T x = b; the factor pattern is
  // structurally symmetric, so they follow the same level schedule):
  // per column j, (k, HV pos of u_kj) over head rows k < j;
  std::vector<int> ut_ptr, ut_row, ut_pos;  // [dim + 1]
  // per head column i, (r, HV pos of l_ri) over rows r > i (head or tail)
  std::vector<int> lt_ptr, lt_row, lt_pos;  // [p + 1]

  // ---- Jacobian fill map --------------------------------------------------
  // per Ybus entry k: destinations of its J11 (P-θ), J12 (P-Vm), J21 (Q-θ),
  // J22 (Q-Vm) coefficients, encoded as described above.
  std::vector<int> jmap;  // [4 * nnz_y]

  // ---- statistics --------------------------------------------------------
  int64_t nnz_j = 0, nnz_lu = 0;
  int n_tail_exact = 0;
  double build_ms = 0;
};

// Build the plan.  ybus_indptr/indices describe the CSR pattern (values are
// not needed).  Throws std::invalid_argument on malformed input.
Plan build_plan(int n_bus, const int* ybus_indptr, const int* ybus_indices,
                const int* pv, int n_pv, const int* pq, int n_pq,
                const TailOptions& opt = TailOptions());

// Bus-level minimum-degree order on an undirected graph with vertex weights
// (1 or 2 unknowns per bus).  Exposed for tests.
std::vector<int> min_degree_order(int n, const std::vector<std::vector<int>>& adj,
                                  const std::vector<int>& weight);

}  // namespace gs2g
