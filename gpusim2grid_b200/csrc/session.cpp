// Host side of the C-ABI (include/gs2g.h): sessions over one grid, batch-row
// assembly (branch trips -> Ybus edit lists, islanding pre-check, injection
// rows), device buffers and the launch of the persistent sweep kernel.
//
// Reference counterparts: the sessions of src/_cpp/contingency_analysis_session.cu,
// injection_sweep_session.cu and scenario_sweep_session.cu, the branch-trip
// deltas of contingency_analysis_helper.cpp:23-84 and the connectivity
// pre-check of contingency_analysis_helper.cpp:634-651.
#include "../../include/gs2g.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <complex>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include <pthread.h>

#include "nr_kernel.cuh"
#include "plan.hpp"

namespace {

thread_local std::string g_err;

constexpr int kMaxEdits = 64;  // must match MAX_EDITS in nr_kernel.cu
// a row runs at most max(max_iter, k) + k steps; k is bounded so that no
// option value can keep a row stepping for long
constexpr int kMaxItersPerRound = 1000;

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

struct DevBuf {
  void* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void ensure(size_t bytes) {
    if (bytes <= n && p) return;
    release();
    ck(cudaMalloc(&p, bytes ? bytes : 16), "cudaMalloc");
    n = bytes ? bytes : 16;
  }
  template <typename T>
  T* as() const { return static_cast<T*>(p); }
};

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

struct gs2g_session {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t ev_ext = nullptr;  // work of another stream the session stream waits for
  gs2g::Plan plan;
  gs2g::DevPlan dplan{};
  std::vector<int> y_ip, y_ix, pv, pq;  // canonical pattern and bus sets, for re-planning
  std::vector<std::unique_ptr<DevBuf>> plan_bufs;
  int n_bus = 0;
  std::vector<double> ybus;  // canonical values, interleaved complex
  std::vector<double> vinit, sbus, base_v;
  bool has_base = false;
  DevBuf d_ybus, d_vinit, d_sbus, d_basev;
  DevBuf d_bases;  // complex [n_bus] Vb conj(Y Vb): the power the base V draws on the unedited Ybus
  DevBuf d_basei;  // complex [n_bus] Y Vb, summed as the sweep's mismatch sums (fused multiply-adds, row order)
  DevBuf d_comp;   // per-row outage compensation records of the chord sweep

  // branch data
  int n_branch = 0;
  std::vector<int> br_from, br_to;
  std::vector<double> yff, yft, ytf, ytt;
  std::vector<int> k_ff, k_tt, k_ft, k_tf;  // Ybus entry of each branch term
  std::vector<uint8_t> is_bridge;           // branch whose loss alone islands the grid
  std::vector<uint64_t> cut_label;          // cycle-space label per branch (islanding pre-check)
  int base_components = 1;                  // connected components of the branch graph
  DevBuf d_br_from, d_br_to, d_br_y;        // branch data on the device (flows)
  DevBuf d_br_rate;                         // limits in per unit
  bool limits_on = false;
  DevBuf d_trip_ptr, d_trip_ids;            // tripped branches per assembled row
  DevBuf d_loading, d_nviol, d_maxload;     // flow outputs of the last run

  // row definitions
  int n_ctg = 0;
  std::vector<int> ctg_ptr, ctg_ids;
  int n_inj = 0;  // injection rows, already in d_sbus_rows (set_injections uploads them)
  std::vector<double> inj_key;  // per injection row: sum |dP| + |dQ| against the base Sbus
  // longest rows first: the queue takes rows by a difficulty estimate
  // (gs2g_session_set_row_order); d_row_order is that permutation
  int row_order = 1;
  DevBuf d_row_order;
  bool rows_have_order = false;
  int n_start = 0;
  DevBuf d_v0rows;
  bool rows_dirty = true;
  bool edits_dirty = true;  // the rows' Ybus edits, masks, skips and order still to build

  // assembled rows on the device
  int n_rows = 0;
  bool rows_have_sbus = false, rows_have_edits = false, rows_have_skip = false, rows_have_mask = false;
  DevBuf d_sbus_rows, d_edit_ptr, d_edit_k, d_edit_val, d_row_skip;
  // handle_disconnected_grid: a row whose trips split the grid solves the
  // largest component, the other buses masked (their voltages NaN)
  int handle_disconnected = 0;
  std::vector<uint8_t> is_slack;      // buses in neither pv nor pq (the angle reference)
  DevBuf d_mask_ptr, d_mask_bus;      // masked buses per assembled row (CSR)
  DevBuf d_v_out, d_res, d_status, d_iters, d_factors;
  DevBuf d_ws, d_queue, d_phase;
  DevBuf d_multi;  // grid table of gs2g_run_multi (when this session leads)
  DevBuf d_row_map;  // rows of gs2g_run_subset
  DevBuf d_base_ws;        // base case's factor for GS2G_REFACTOR_BASE_CHORD
  DevBuf d_base_inv;       // its inverse, column c = M0^-1 e_c (outage compensation)
  DevBuf d_base_fwv, d_base_bwv;  // its head values in forward / backward solve order
  DevBuf d_handoff;        // rows the chord sweep hands to the single-row sweep
  DevBuf d_chord_steps;    // Newton steps the last chord sweep took on the base factor
  int chord = 2;           // policy 2: 0 single-row sweep, 1 chord sweep, 2 chord sweep with Broyden steps
  int handoff_cluster = 1;  // the chord sweep's hand-offs and small subsets run with a cluster of CTAs per row
  int base_factor_prec = -1;  // precision it was computed in (-1: none or stale)
  // base-solve outputs (kept apart from the batch results)
  DevBuf b_v, b_res, b_status, b_iters;

  gs2g_timings tm{};
  int last_rows_run = 0;
  // pinned double buffer for large result copies (see d2h_staged)
  mutable void* h_stage = nullptr;
  // pinned host copy of the last run's results (gs2g_get_results_host)
  void* h_res = nullptr;
  size_t h_res_bytes = 0;
  // results mirror (gs2g_session_set_results_mirror): runs write each row's
  // final V into h_res as the row leaves; mirror_valid once a full run did
  bool mirror_on = false;
  bool mirror_valid = false;
  mutable cudaEvent_t ev_stage[2] = {nullptr, nullptr};
};

namespace {

template <typename T>
const T* upload_vec(gs2g_session* s, const std::vector<T>& v) {
  auto b = std::make_unique<DevBuf>();
  b->ensure(std::max<size_t>(v.size() * sizeof(T), 16));
  if (!v.empty()) ck(cudaMemcpy(b->p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "upload plan");
  const T* p = b->as<T>();
  s->plan_bufs.push_back(std::move(b));
  return p;
}

void upload_plan(gs2g_session* s) {
  const gs2g::Plan& P = s->plan;
  gs2g::DevPlan& D = s->dplan;
  D.n_bus = P.n_bus;
  D.nnz_y = P.nnz_y;
  D.dim = P.dim;
  D.p = P.p;
  D.nt = P.nt;
  D.ld = P.ld;
  D.n_hv = P.n_hv;
  D.n_levels = P.n_levels;
  D.y_indptr = upload_vec(s, P.y_indptr);
  D.y_indices = upload_vec(s, P.y_indices);
  D.y_row = upload_vec(s, P.y_row);
  D.jmap = upload_vec(s, P.jmap);
  D.fP = upload_vec(s, P.fP);
  D.fQ = upload_vec(s, P.fQ);
  D.lev_ptr = upload_vec(s, P.lev_ptr);
  D.lev_big = upload_vec(s, P.lev_big);
  D.task_out = upload_vec(s, P.task_out);
  D.task_diag = upload_vec(s, P.task_diag);
  D.task_pbeg = upload_vec(s, P.task_pbeg);
  D.task_pend = upload_vec(s, P.task_pend);
  D.task_has_a = upload_vec(s, P.task_has_a);
  D.pair_l = upload_vec(s, P.pair_l);
  D.pair_u = upload_vec(s, P.pair_u);
  D.lev_piv_ptr = upload_vec(s, P.lev_piv_ptr);
  D.lev_piv = upload_vec(s, P.lev_piv);
  D.sn_w = upload_vec(s, P.sn_w);
  D.sn_t = upload_vec(s, P.sn_t);
  D.sn_L = upload_vec(s, P.sn_L);
  D.sn_U = upload_vec(s, P.sn_U);
  D.sn_tidx = upload_vec(s, P.sn_tidx);
  D.tidx = upload_vec(s, P.tidx);
  D.sg_ptr = upload_vec(s, P.sg_ptr);
  D.sg_col = upload_vec(s, P.sg_col);
  D.se_ptr = upload_vec(s, P.se_ptr);
  D.se_rec = reinterpret_cast<const int4*>(upload_vec(s, P.se_rec));
  D.fw_ptr = upload_vec(s, P.fw_ptr);
  D.fw_col = upload_vec(s, P.fw_col);
  D.fw_pos = upload_vec(s, P.fw_pos);
  D.bw_ptr = upload_vec(s, P.bw_ptr);
  D.bw_row = upload_vec(s, P.bw_row);
  D.bw_pos = upload_vec(s, P.bw_pos);
  D.ut_ptr = upload_vec(s, P.ut_ptr);
  D.ut_row = upload_vec(s, P.ut_row);
  D.ut_pos = upload_vec(s, P.ut_pos);
  D.lt_ptr = upload_vec(s, P.lt_ptr);
  D.lt_row = upload_vec(s, P.lt_row);
  D.lt_pos = upload_vec(s, P.lt_pos);
  D.iperm = upload_vec(s, P.iperm);
}

// Ybus entry index of (i, j), -1 if not in the pattern.
int ybus_find(const gs2g::Plan& P, int i, int j) {
  const int* b = P.y_indices.data() + P.y_indptr[i];
  const int* e = P.y_indices.data() + P.y_indptr[i + 1];
  const int* it = std::lower_bound(b, e, j);
  return (it != e && *it == j) ? int(it - P.y_indices.data()) : -1;
}

struct DSU {
  std::vector<int> p;
  explicit DSU(int n) : p(n) { std::iota(p.begin(), p.end(), 0); }
  int f(int x) {
    while (p[x] != x) x = p[x] = p[p[x]];
    return x;
  }
  bool u(int a, int b) {
    a = f(a);
    b = f(b);
    if (a == b) return false;
    p[a] = b;
    return true;
  }
};

// Bridges of the branch graph (Tarjan's low-link, iterative, over branch ids
// so parallel branches are never bridges) and its component count.  A row
// that trips a bridge islands the grid; a row that trips one non-bridge
// branch does not, so the per-row connectivity check runs only for rows
// that trip two or more non-bridge branches.
void compute_bridges(gs2g_session* s) {
  const int n = s->n_bus, m = s->n_branch;
  // a branch open at one end (negative endpoint) joins no two buses
  auto edge = [&](int l) { return s->br_from[l] >= 0 && s->br_to[l] >= 0; };
  std::vector<int> deg(n + 1, 0);
  for (int l = 0; l < m; ++l) {
    if (!edge(l)) continue;
    ++deg[s->br_from[l] + 1];
    ++deg[s->br_to[l] + 1];
  }
  for (int v = 0; v < n; ++v) deg[v + 1] += deg[v];
  std::vector<int> adj_v(2 * m), adj_e(2 * m), fill(deg.begin(), deg.end() - 1);
  for (int l = 0; l < m; ++l) {
    if (!edge(l)) continue;
    const int f = s->br_from[l], t = s->br_to[l];
    adj_v[fill[f]] = t;
    adj_e[fill[f]++] = l;
    adj_v[fill[t]] = f;
    adj_e[fill[t]++] = l;
  }
  s->is_bridge.assign(m, 0);
  std::vector<int> tin(n, -1), low(n, 0), it(n, 0), pe(n, -1);
  std::vector<int> stack, post;
  post.reserve(n);
  int timer = 0, comps = 0;
  for (int root = 0; root < n; ++root) {
    if (tin[root] >= 0) continue;
    ++comps;
    stack.push_back(root);
    tin[root] = low[root] = timer++;
    it[root] = deg[root];
    while (!stack.empty()) {
      const int v = stack.back();
      if (it[v] < deg[v + 1]) {
        const int k = it[v]++;
        const int w = adj_v[k], e = adj_e[k];
        if (e == pe[v]) continue;
        if (tin[w] < 0) {
          pe[w] = e;
          tin[w] = low[w] = timer++;
          it[w] = deg[w];
          stack.push_back(w);
        } else {
          low[v] = std::min(low[v], tin[w]);
        }
      } else {
        stack.pop_back();
        post.push_back(v);
        if (!stack.empty()) {
          const int u = stack.back();
          low[u] = std::min(low[u], low[v]);
          if (low[v] > tin[u]) s->is_bridge[pe[v]] = 1;
        }
      }
    }
  }
  s->base_components = comps;

  // Cycle-space labels: a pseudo-random 64-bit value per non-tree branch of
  // the DFS forest, and for a tree branch the XOR of the values of the
  // non-tree branches whose fundamental cycle runs through it (the XOR of
  // the values incident to the subtree below it).  Every cycle crosses an
  // edge cut an even number of times, so the labels of any cut XOR to zero:
  // trips whose labels are linearly independent over GF(2) cannot contain a
  // cut and leave the grid connected, with certainty; dependent labels only
  // call for the exact check.  (Bridges are the branches labelled zero.)
  s->cut_label.assign(m, 0);
  std::vector<uint64_t> sub(n, 0);
  auto mix = [](uint64_t x) {  // splitmix64 finaliser
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
  };
  for (int l = 0; l < m; ++l) {
    if (!edge(l)) continue;
    const int f = s->br_from[l], t = s->br_to[l];
    if (pe[f] == l || pe[t] == l) continue;  // tree branch
    const uint64_t r = mix((uint64_t)l + 0x51ed27ull) | 1ull;
    s->cut_label[l] = r;
    sub[f] ^= r;
    sub[t] ^= r;
  }
  for (const int v : post) {  // children before parents
    const int l = pe[v];
    if (l < 0) continue;
    s->cut_label[l] = sub[v];
    const int u = s->br_from[l] == v ? s->br_to[l] : s->br_from[l];
    sub[u] ^= sub[v];
  }
}

// True when the labels of the given branches are linearly independent over
// GF(2) (no nonempty subset XORs to zero): removing them leaves the grid as
// connected as it was.  Branches open at one end join nothing and are left
// out.
bool trips_keep_connected(const gs2g_session* s, const std::vector<int>& ids) {
  uint64_t basis[64];
  int nb = 0;
  for (const int l : ids) {
    if (s->br_from[l] < 0 || s->br_to[l] < 0) continue;
    uint64_t x = s->cut_label[l];
    for (int i = 0; i < nb && x; ++i) x = std::min(x, x ^ basis[i]);
    if (x == 0) return false;
    basis[nb++] = x;
    // keep the basis sorted by leading bit, highest first, so the reduction
    // above clears each basis vector's leading bit in turn
    for (int i = nb - 1; i > 0 && basis[i] > basis[i - 1]; --i) std::swap(basis[i], basis[i - 1]);
    if (nb == 64) return false;  // more trips than label bits: check exactly
  }
  return true;
}

// The order in which the row queue takes the rows: by a difficulty estimate,
// largest first, so that rows needing many steps start early and the
// persistent sweep does not end on a tail of a few long rows (a row's
// results do not depend on when it runs).  Estimate: the row's distance
// from the base injections (sum |dP| + |dQ|) plus, per tripped branch, its
// flow at the base voltage (max |S_from|, |S_to|): both are the mismatch a
// row starts with at the base case.  Off, or without any estimate, the
// queue takes the rows in order.
void order_rows(gs2g_session* s, int nr) {
  s->rows_have_order = false;
  if (!s->row_order || nr < 2) return;
  std::vector<double> key(nr, 0.0);
  bool any = false;
  if (s->n_inj == nr && (int)s->inj_key.size() == nr) {
    key = s->inj_key;
    any = true;
  }
  if (s->n_ctg == nr && s->has_base && !s->yff.empty()) {
    const int m = s->n_branch;
    std::vector<double> fk(m, 0.0);
    const double* V = s->base_v.data();
    for (int l = 0; l < m; ++l) {
      const int f = s->br_from[l], t = s->br_to[l];
      const std::complex<double> vf = f >= 0 ? std::complex<double>(V[2 * f], V[2 * f + 1]) : 0.0;
      const std::complex<double> vt = t >= 0 ? std::complex<double>(V[2 * t], V[2 * t + 1]) : 0.0;
      auto c = [&](const std::vector<double>& y) { return std::complex<double>(y[2 * l], y[2 * l + 1]); };
      const std::complex<double> i_f = c(s->yff) * vf + c(s->yft) * vt, i_t = c(s->ytf) * vf + c(s->ytt) * vt;
      fk[l] = std::max(std::abs(vf * std::conj(i_f)), std::abs(vt * std::conj(i_t)));
    }
    for (int r = 0; r < nr; ++r)
      for (int q = s->ctg_ptr[r]; q < s->ctg_ptr[r + 1]; ++q) key[r] += fk[s->ctg_ids[q]];
    any = true;
  }
  if (!any) return;
  std::vector<int> order(nr);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return key[x] > key[y]; });
  s->d_row_order.ensure((size_t)nr * sizeof(int));
  ck(cudaMemcpy(s->d_row_order.p, order.data(), (size_t)nr * sizeof(int), cudaMemcpyHostToDevice), "upload row order");
  s->rows_have_order = true;
}

// Rows in two stages.  The first (row count, trip CSR on the device) is all
// gs2g_get_device_rows needs, so a caller's network can run on the rows
// while the host builds the second (every row's Ybus edits, islanding
// verdict, masks and the row order), which a run needs.
void assemble_rows(gs2g_session* s, bool full = true) {
  if (s->rows_dirty) {
    if (s->n_ctg > 0 && s->n_inj > 0 && s->n_ctg != s->n_inj)
      throw std::invalid_argument("topology rows (" + std::to_string(s->n_ctg) + ") and injection rows (" +
                                  std::to_string(s->n_inj) + ") differ in number");
    const int nr = std::max(s->n_ctg, s->n_inj);
    s->n_rows = nr;
    s->rows_have_sbus = s->n_inj > 0;
    s->rows_have_edits = s->n_ctg > 0;
    s->rows_have_skip = false;
    s->rows_have_mask = false;
    s->rows_have_order = false;
    if (nr > 0 && s->rows_have_edits) {
      s->d_trip_ptr.ensure((nr + 1) * sizeof(int));
      s->d_trip_ids.ensure(std::max<size_t>(s->ctg_ids.size(), 1) * sizeof(int));
      ck(cudaMemcpy(s->d_trip_ptr.p, s->ctg_ptr.data(), (nr + 1) * sizeof(int), cudaMemcpyHostToDevice),
         "upload trips");
      if (!s->ctg_ids.empty())
        ck(cudaMemcpy(s->d_trip_ids.p, s->ctg_ids.data(), s->ctg_ids.size() * sizeof(int), cudaMemcpyHostToDevice),
           "upload trips");
    }
    s->rows_dirty = false;
    s->edits_dirty = true;
  }
  if (!full || !s->edits_dirty) return;
  const int n = s->n_bus;
  const int nr = s->n_rows;
  if (nr == 0) {
    s->edits_dirty = false;
    return;
  }
  if (s->rows_have_edits) {
    std::vector<int> eptr(nr + 1, 0), ek;
    std::vector<double> ev;
    std::vector<uint8_t> skip(nr, 0);
    std::vector<int> uniq;
    bool any_skip = false;
    std::vector<int> mptr(nr + 1, 0), mbus;  // masked buses per row (handle_disconnected)
    std::vector<int> comp_size, comp_min;
    std::vector<std::pair<int, std::complex<double>>> acc;
    for (int r = 0; r < nr; ++r) {
      uniq.assign(s->ctg_ids.begin() + s->ctg_ptr[r], s->ctg_ids.begin() + s->ctg_ptr[r + 1]);
      std::sort(uniq.begin(), uniq.end());
      uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
      if (!uniq.empty()) {
        bool island = s->base_components > 1;
        for (size_t q = 0; q < uniq.size() && !island; ++q) island = s->is_bridge[uniq[q]] != 0;
        if (!island && uniq.size() >= 2 && !trips_keep_connected(s, uniq)) {
          DSU d(n);
          size_t ui = 0;
          int comps = n;
          for (int l = 0; l < s->n_branch; ++l) {
            while (ui < uniq.size() && uniq[ui] < l) ++ui;
            if (ui < uniq.size() && uniq[ui] == l) continue;
            if (s->br_from[l] < 0 || s->br_to[l] < 0) continue;  // open at one end: no edge
            if (d.u(s->br_from[l], s->br_to[l])) --comps;
          }
          island = comps > 1;
        }
        bool masked_ok = false;
        if (island && s->handle_disconnected && s->base_components == 1) {
          // the largest component is solved, the other buses are masked
          // (compute_component_masks, contingency_analysis_helper.cpp:657):
          // largest by bus count, on a tie the one holding the lowest bus;
          // a row that would mask an angle reference bus is not simulated
          DSU d(n);
          size_t ui = 0;
          for (int l = 0; l < s->n_branch; ++l) {
            while (ui < uniq.size() && uniq[ui] < l) ++ui;
            if (ui < uniq.size() && uniq[ui] == l) continue;
            if (s->br_from[l] < 0 || s->br_to[l] < 0) continue;
            d.u(s->br_from[l], s->br_to[l]);
          }
          comp_size.assign(n, 0);
          comp_min.assign(n, n);
          for (int b = 0; b < n; ++b) {
            const int c = d.f(b);
            ++comp_size[c];
            comp_min[c] = std::min(comp_min[c], b);
          }
          int main_c = -1;
          for (int b = 0; b < n; ++b) {
            const int c = d.f(b);
            if (c != b) continue;  // one visit per component (its root)
            if (main_c < 0 || comp_size[c] > comp_size[main_c] ||
                (comp_size[c] == comp_size[main_c] && comp_min[c] < comp_min[main_c]))
              main_c = c;
          }
          masked_ok = true;
          const size_t m0 = mbus.size();
          for (int b = 0; b < n && masked_ok; ++b) {
            if (d.f(b) == main_c) continue;
            if (s->is_slack[b]) masked_ok = false;
            mbus.push_back(b);
          }
          if (!masked_ok) mbus.resize(m0);
        }
        if (island && !masked_ok) {
          skip[r] = 1;
          any_skip = true;
          eptr[r + 1] = (int)ek.size();
          mptr[r + 1] = (int)mbus.size();
          continue;
        }
      }
      mptr[r + 1] = (int)mbus.size();
      // one edit per Ybus position the trips touch, in position order, the
      // trips' terms summed in trip and term order (from zero)
      acc.clear();
      for (int l : uniq) {
        const double* v[4] = {&s->yff[2 * l], &s->ytt[2 * l], &s->yft[2 * l], &s->ytf[2 * l]};
        const int kk[4] = {s->k_ff[l], s->k_tt[l], s->k_ft[l], s->k_tf[l]};
        // an open endpoint has no Ybus row or column: its terms are skipped
        // (contingency_analysis_helper.cpp:53-75)
        for (int q = 0; q < 4; ++q) {
          if (kk[q] < 0) continue;
          const std::complex<double> t(v[q][0], v[q][1]);
          size_t e = 0;
          while (e < acc.size() && acc[e].first != kk[q]) ++e;
          if (e == acc.size()) acc.emplace_back(kk[q], std::complex<double>(0.0, 0.0) + t);
          else acc[e].second += t;
        }
      }
      std::sort(acc.begin(), acc.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
      if ((int)acc.size() > kMaxEdits)
        throw std::invalid_argument("row " + std::to_string(r) + " trips too many branches (" +
                                    std::to_string(acc.size()) + " Ybus edits > " + std::to_string(kMaxEdits) + ")");
      for (auto& kv : acc) {
        ek.push_back(kv.first);
        ev.push_back(kv.second.real());
        ev.push_back(kv.second.imag());
      }
      eptr[r + 1] = (int)ek.size();
    }
    s->d_edit_ptr.ensure(eptr.size() * sizeof(int));
    ck(cudaMemcpy(s->d_edit_ptr.p, eptr.data(), eptr.size() * sizeof(int), cudaMemcpyHostToDevice), "upload edits");
    s->d_edit_k.ensure(std::max<size_t>(ek.size(), 1) * sizeof(int));
    s->d_edit_val.ensure(std::max<size_t>(ev.size(), 2) * sizeof(double));
    if (!ek.empty()) {
      ck(cudaMemcpy(s->d_edit_k.p, ek.data(), ek.size() * sizeof(int), cudaMemcpyHostToDevice), "upload edits");
      ck(cudaMemcpy(s->d_edit_val.p, ev.data(), ev.size() * sizeof(double), cudaMemcpyHostToDevice), "upload edits");
    }
    if (!mbus.empty()) {
      s->d_mask_ptr.ensure(mptr.size() * sizeof(int));
      s->d_mask_bus.ensure(mbus.size() * sizeof(int));
      ck(cudaMemcpy(s->d_mask_ptr.p, mptr.data(), mptr.size() * sizeof(int), cudaMemcpyHostToDevice), "upload masks");
      ck(cudaMemcpy(s->d_mask_bus.p, mbus.data(), mbus.size() * sizeof(int), cudaMemcpyHostToDevice), "upload masks");
      s->rows_have_mask = true;
    }
    if (any_skip) {
      std::vector<int> sk(skip.begin(), skip.end());
      s->d_row_skip.ensure(sk.size() * sizeof(int));
      ck(cudaMemcpy(s->d_row_skip.p, sk.data(), sk.size() * sizeof(int), cudaMemcpyHostToDevice), "upload skip");
      s->rows_have_skip = true;
    }
  }
  order_rows(s, nr);
  s->edits_dirty = false;
}

struct OutBufs {
  double* v;
  double* res;
  int* status;
  int* iters;
  int* factors = nullptr;
  double* v_mirror = nullptr;  // device address of a pinned host copy of v (nullptr: none)
};

// Launch arguments of one grid's rows (everything but the queue, the
// workspace and the phase counters).
gs2g::SweepArgs make_args(gs2g_session* s, const gs2g_run_opts& o, int n_rows, const double* v0, int64_t v0_stride,
                          const double* sbus, int64_t sbus_stride, bool use_rows, const OutBufs& out) {
  if (o.precision != GS2G_PREC_FP64 && o.precision != GS2G_PREC_MIXED)
    throw std::invalid_argument("precision must be GS2G_PREC_FP64 or GS2G_PREC_MIXED");
  if (o.max_iter < 0) throw std::invalid_argument("max_iter must be >= 0");
  gs2g::SweepArgs a{};
  a.n_rows = n_rows;
  a.ybus = s->d_ybus.as<double>();
  a.v0 = v0;
  a.v0_stride = v0_stride;
  a.sbus = sbus;
  a.sbus_stride = sbus_stride;
  a.edit_ptr = use_rows && s->rows_have_edits ? s->d_edit_ptr.as<int>() : nullptr;
  a.edit_k = use_rows && s->rows_have_edits ? s->d_edit_k.as<int>() : nullptr;
  a.edit_val = use_rows && s->rows_have_edits ? s->d_edit_val.as<double>() : nullptr;
  a.row_skip = use_rows && s->rows_have_skip ? s->d_row_skip.as<int>() : nullptr;
  a.mask_ptr = use_rows && s->rows_have_mask ? s->d_mask_ptr.as<int>() : nullptr;
  a.mask_bus = use_rows && s->rows_have_mask ? s->d_mask_bus.as<int>() : nullptr;
  a.row_map = use_rows && s->rows_have_order ? s->d_row_order.as<int>() : nullptr;
  a.max_iter = o.max_iter;
  a.tol = o.tol;
  a.fixed_iters = o.fixed_iters;
  if (o.iters_per_round > kMaxItersPerRound)
    throw std::invalid_argument("iters_per_round must be <= " + std::to_string(kMaxItersPerRound));
  a.round_k = o.iters_per_round > 0 ? o.iters_per_round : 1;
  a.step_first = o.step_then_check != 0 && !o.fixed_iters;
  a.step_scaling = o.step_scaling != 0;
  a.max_dva = o.max_dva > 0 ? o.max_dva : 0.5;
  a.max_dvm = o.max_dvm > 0 ? o.max_dvm : 0.1;
  a.v_out = out.v;
  a.v_mirror = out.v_mirror;
  a.res_out = out.res;
  a.status_out = out.status;
  a.iters_out = out.iters;
  a.pivot_floor = o.pivot_floor;
  if (o.refactor_policy != GS2G_REFACTOR_EVERY && o.refactor_policy != GS2G_REFACTOR_ADAPTIVE &&
      o.refactor_policy != GS2G_REFACTOR_BASE_CHORD)
    throw std::invalid_argument("refactor_policy must be GS2G_REFACTOR_EVERY, _ADAPTIVE or _BASE_CHORD");
  a.refactor_policy = o.refactor_policy;
  if (o.refactor_policy == GS2G_REFACTOR_BASE_CHORD && use_rows && s->base_factor_prec == o.precision) {
    a.base_ws = s->d_base_ws.as<char>();
    a.base_v = s->d_basev.as<double>();
    a.base_inv = s->d_base_inv.as<char>();
    a.base_fwv = s->d_base_fwv.as<char>();
    a.base_bwv = s->d_base_bwv.as<char>();
  }
  // defaults: a step on the shared base factor is cheap (several rows share
  // each factor read), so base_chord keeps it longer than adaptive keeps a
  // row's own LU
  const bool chord_policy = o.refactor_policy == GS2G_REFACTOR_BASE_CHORD;
  a.refactor_ratio = o.refactor_ratio > 0 ? o.refactor_ratio : (chord_policy ? 0.7 : 0.3);
  a.max_reuse = o.max_reuse > 0 ? o.max_reuse : (chord_policy ? 8 : 3);
  a.factors_out = out.factors;
  // rescue (per-row starts, continuous schedule): with a base case the row
  // starts from the base V when that has the smaller mismatch, and an
  // unconverged row restarts from the base V (from Vinit without one)
  const bool rescue = o.rescue != 0 && v0_stride != 0 && !o.fixed_iters;
  const bool base = rescue && s->has_base && use_rows;
  a.rescue_v0 = rescue ? (base ? s->d_basev.as<double>() : s->d_vinit.as<double>()) : nullptr;
  a.alt_v0 = base ? s->d_basev.as<double>() : nullptr;
  a.alt_s = base ? s->d_bases.as<double>() : nullptr;
  a.alt_i = base ? s->d_basei.as<double>() : nullptr;
  a.phase_cycles = nullptr;
  if (use_rows && s->limits_on) {
    const size_t nr = (size_t)std::max(n_rows, 1);
    s->d_loading.ensure(nr * s->n_branch * sizeof(float));
    s->d_nviol.ensure(nr * sizeof(int));
    s->d_maxload.ensure(nr * sizeof(float));
    a.n_branch = s->n_branch;
    a.br_from = s->d_br_from.as<int>();
    a.br_to = s->d_br_to.as<int>();
    a.br_y = s->d_br_y.as<double>();
    a.br_rate = s->d_br_rate.as<double>();
    a.trip_ptr = s->rows_have_edits ? s->d_trip_ptr.as<int>() : nullptr;
    a.trip_ids = s->rows_have_edits ? s->d_trip_ids.as<int>() : nullptr;
    a.loading_out = s->d_loading.as<float>();
    a.nviol_out = s->d_nviol.as<int>();
    a.maxload_out = s->d_maxload.as<float>();
  }
  return a;
}

// Cluster size for `rows` rows that each get a cluster within `n_ctas`
// CTAs: 16, else 8, else 0 (one CTA per row).
int cluster_for(int rows, int n_ctas) {
  if (rows <= 0) return 0;
  for (int c = gs2g::handoff_cluster_size(); c >= 8; c /= 2)
    if ((int64_t)rows * c <= n_ctas) return c;
  return 0;
}

float launch(gs2g_session* s, const gs2g_run_opts& o, int n_rows, const double* v0, int64_t v0_stride,
             const double* sbus, int64_t sbus_stride, bool use_rows, const OutBufs& out, int n_ctas_req) {
  gs2g::SweepArgs a = make_args(s, o, n_rows, v0, v0_stride, sbus, sbus_stride, use_rows, out);
  int n_ctas = n_ctas_req > 0 ? n_ctas_req : gs2g::sweep_ctas(o.precision, s->device);
  n_ctas = std::max(1, std::min(n_ctas, std::max(n_rows, 1)));
  const int64_t wsb = gs2g::workspace_bytes(s->dplan, o.precision);
  s->d_queue.ensure(4 * sizeof(int));  // [0] row queue, [1] rescue count, [2] alternative starts, [3] hand-offs
  // policy 2 (continuous): the chord sweep takes every row first, several
  // per CTA on the base factor, and hands the rows that need their own LU
  // (or the rescue) to the single-row sweep that follows on the stream
  const bool chord = s->chord > 0 && use_rows && n_rows > 0 && o.refactor_policy == GS2G_REFACTOR_BASE_CHORD &&
                     a.base_ws != nullptr && a.base_inv != nullptr && !o.fixed_iters;
  int n_chord = 0;
  int64_t cwsb = 0;
  if (chord) {
    n_chord = n_ctas_req > 0 ? n_ctas_req : gs2g::chord_ctas(s->dplan, o.precision, s->device);
    const int per = gs2g::chord_rows_per_cta();
    n_chord = std::max(1, std::min(n_chord, (n_rows + per - 1) / per));
    cwsb = gs2g::chord_workspace_bytes(s->dplan, o.precision);
    s->d_handoff.ensure((size_t)n_rows * sizeof(int));
    if (a.edit_ptr != nullptr && a.base_v != nullptr) s->d_comp.ensure((size_t)n_rows * gs2g::comp_rec_bytes());
  }
  s->d_ws.ensure(std::max((size_t)wsb * n_ctas, (size_t)cwsb * n_chord));
  a.queue = s->d_queue.as<int>();
  a.workspace = s->d_ws.as<char>();
  a.ws_stride = wsb;
  a.n_rescued = s->d_queue.as<int>() + 1;
  a.n_alt_start = s->d_queue.as<int>() + 2;
  if (o.profile_phases) {
    s->d_phase.ensure(gs2g::N_PHASES * sizeof(unsigned long long));
    ck(cudaMemsetAsync(s->d_phase.p, 0, gs2g::N_PHASES * sizeof(unsigned long long), s->stream), "phase reset");
    a.phase_cycles = s->d_phase.as<unsigned long long>();
  }
  ck(cudaMemsetAsync(s->d_queue.p, 0, 4 * sizeof(int), s->stream), "queue reset");
  s->d_chord_steps.ensure(sizeof(unsigned long long));
  ck(cudaMemsetAsync(s->d_chord_steps.p, 0, sizeof(unsigned long long), s->stream), "step count reset");
  ck(cudaEventRecord(s->ev0, s->stream), "event");
  int n_next = n_rows;  // rows of the single-row launch (the hand-offs after a chord sweep)
  if (chord) {
    gs2g::SweepArgs c = a;
    c.ws_stride = cwsb;
    c.handoff = s->d_handoff.as<int>();
    c.n_handoff = s->d_queue.as<int>() + 3;
    c.n_chord_steps = s->d_chord_steps.as<unsigned long long>();
    c.broyden = s->chord == 2;
    // every row's outage compensation, set up in parallel ahead of the sweep
    if (a.edit_ptr != nullptr && a.base_v != nullptr) {
      ck((cudaError_t)gs2g::launch_comp_setup(s->dplan, c, o.precision, n_rows, s->d_comp.p, s->stream),
         "compensation setup launch");
      c.comp_rec = s->d_comp.as<char>();
    }
    ck((cudaError_t)gs2g::launch_chord(s->dplan, c, o.precision, n_chord, s->stream), "chord sweep launch");
    ck(cudaMemsetAsync(s->d_queue.p, 0, sizeof(int), s->stream), "queue reset");
    // how many rows were handed off decides the next launch's shape
    ck(cudaMemcpyAsync(&n_next, s->d_queue.as<int>() + 3, sizeof(int), cudaMemcpyDeviceToHost, s->stream),
       "hand-off count");
    ck(cudaStreamSynchronize(s->stream), "chord sweep");
    // the hand-offs continue from where the chord sweep left them: their V
    // (v_out) and step count (iters_out), on their own factor (policy 1)
    a.row_map = s->d_handoff.as<int>();
    a.n_rows_dev = s->d_queue.as<int>() + 3;
    a.v0 = out.v;
    a.v0_stride = s->n_bus;
    a.iters_in = out.iters;
    a.refactor_policy = GS2G_REFACTOR_ADAPTIVE;
    a.base_ws = nullptr;
    a.base_v = nullptr;
    a.base_inv = nullptr;
    a.base_fwv = nullptr;
    a.base_bwv = nullptr;
    a.alt_v0 = nullptr;
    a.alt_s = nullptr;
    a.alt_i = nullptr;
  }
  // hand-offs with a dense tail worth sharing: a cluster of 16 (or 8) CTAs
  // per row when every row gets one (the rows are few and each of their
  // factorizations would otherwise run on one SM after every other row has
  // finished)
  const int csize = chord && s->handoff_cluster && s->dplan.nt >= 64 ? cluster_for(n_next, n_ctas) : 0;
  if (n_next > 0 && csize > 0) {
    ck((cudaError_t)gs2g::launch_sweep_cluster(s->dplan, a, o.precision, csize, n_next * csize, s->stream),
       "hand-off cluster launch");
  } else if (n_next > 0) {
    ck((cudaError_t)gs2g::launch_sweep(s->dplan, a, o.precision, std::min(n_ctas, n_next), s->stream),
       "sweep launch");
  }
  ck(cudaEventRecord(s->ev1, s->stream), "event");
  ck(cudaStreamSynchronize(s->stream), "sweep");
  float ms = 0;
  ck(cudaEventElapsedTime(&ms, s->ev0, s->ev1), "event time");
  for (int q = 0; q < GS2G_N_PHASES; ++q) s->tm.phase_cycles[q] = s->tm.phase_share[q] = 0;
  ck(cudaMemcpy(&s->tm.n_rescued, s->d_queue.as<int>() + 1, sizeof(int), cudaMemcpyDeviceToHost), "rescue count");
  ck(cudaMemcpy(&s->tm.n_base_start, s->d_queue.as<int>() + 2, sizeof(int), cudaMemcpyDeviceToHost), "start count");
  unsigned long long cs = 0;
  ck(cudaMemcpy(&cs, s->d_chord_steps.p, sizeof(cs), cudaMemcpyDeviceToHost), "step count");
  s->tm.chord_steps = (int64_t)cs;
  if (o.profile_phases) {
    unsigned long long c[gs2g::N_PHASES];
    ck(cudaMemcpy(c, s->d_phase.p, sizeof(c), cudaMemcpyDeviceToHost), "read phases");
    double tot = 0;
    for (int q = 0; q < gs2g::N_PHASES; ++q) tot += (double)c[q];
    for (int q = 0; q < gs2g::N_PHASES; ++q) {
      s->tm.phase_cycles[q] = (double)c[q];
      s->tm.phase_share[q] = tot > 0 ? c[q] / tot : 0;
    }
  }
  return ms;
}

}  // namespace

namespace gs2g {
// last-error text for the MLP entry points (mlp_kernels.cu)
void set_last_error(const char* msg) { g_err = msg ? msg : ""; }
}  // namespace gs2g

namespace {

int fail(const std::exception& e) {
  g_err = e.what();
  if (dynamic_cast<const std::invalid_argument*>(&e)) return GS2G_ERR_INVALID;
  if (dynamic_cast<const CudaError*>(&e)) return GS2G_ERR_CUDA;
  return GS2G_ERR_RUNTIME;
}

#define GS2G_TRY try {
#define GS2G_CATCH                                  \
  return GS2G_OK;                                   \
  }                                                 \
  catch (const std::exception& e) { return fail(e); } \
  catch (...) {                                     \
    g_err = "unknown error";                        \
    return GS2G_ERR_RUNTIME;                        \
  }

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (dev >= 0 && dev != prev) ck(cudaSetDevice(dev), "cudaSetDevice");
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

void canonical_csr(int n, const int* indptr, const int* indices, const double* values, std::vector<int>& ip,
                   std::vector<int>& ix, std::vector<double>& vals) {
  if (indptr[0] != 0) throw std::invalid_argument("Ybus indptr[0] must be 0");
  ip.assign(n + 1, 0);
  ix.clear();
  vals.clear();
  std::vector<std::pair<int, std::complex<double>>> rowv;
  for (int i = 0; i < n; ++i) {
    if (indptr[i + 1] < indptr[i]) throw std::invalid_argument("Ybus indptr must be non-decreasing");
    rowv.clear();
    for (int k = indptr[i]; k < indptr[i + 1]; ++k) {
      if (indices[k] < 0 || indices[k] >= n) throw std::invalid_argument("Ybus column index out of range");
      rowv.emplace_back(indices[k], std::complex<double>(values[2 * k], values[2 * k + 1]));
    }
    std::sort(rowv.begin(), rowv.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    for (size_t q = 0; q < rowv.size(); ++q) {
      if (!ix.empty() && (int)ix.size() > ip[i] && ix.back() == rowv[q].first) {
        vals[vals.size() - 2] += rowv[q].second.real();
        vals[vals.size() - 1] += rowv[q].second.imag();
      } else {
        ix.push_back(rowv[q].first);
        vals.push_back(rowv[q].second.real());
        vals.push_back(rowv[q].second.imag());
      }
    }
    ip[i + 1] = (int)ix.size();
  }
}

gs2g_run_opts checked(const gs2g_run_opts* o) {
  if (!o) throw std::invalid_argument("run options must not be NULL");
  return *o;
}

}  // namespace

extern "C" {

const char* gs2g_last_error(void) { return g_err.c_str(); }
int gs2g_version(void) { return 100; }
int gs2g_max_edits_per_row(void) { return kMaxEdits; }

int gs2g_session_create(int device, int n_bus, const int* ybus_indptr, const int* ybus_indices,
                        const double* ybus_values, const double* vinit, const double* sbus, const int* pv, int n_pv,
                        const int* pq, int n_pq, int tail_policy, gs2g_session** out) {
  GS2G_TRY
  if (!out) throw std::invalid_argument("out must not be NULL");
  *out = nullptr;
  if (n_bus <= 0 || !ybus_indptr || !ybus_indices || !ybus_values || !vinit || !sbus)
    throw std::invalid_argument("session_create: missing grid arrays");
  if ((n_pv > 0 && !pv) || (n_pq > 0 && !pq) || n_pv < 0 || n_pq < 0)
    throw std::invalid_argument("session_create: bad pv/pq");
  auto s = std::make_unique<gs2g_session>();
  if (device < 0) ck(cudaGetDevice(&device), "cudaGetDevice");
  s->device = device;
  DeviceGuard g(device);
  s->n_bus = n_bus;
  std::vector<int> ip, ix;
  canonical_csr(n_bus, ybus_indptr, ybus_indices, ybus_values, ip, ix, s->ybus);
  gs2g::TailOptions topt;
  topt.policy = tail_policy;
  s->plan = gs2g::build_plan(n_bus, ip.data(), ix.data(), pv, n_pv, pq, n_pq, topt);
  s->tm.plan_ms = s->plan.build_ms;
  s->y_ip = ip;
  s->y_ix = ix;
  s->pv.assign(pv, pv + n_pv);
  s->pq.assign(pq, pq + n_pq);
  s->is_slack.assign(n_bus, 1);
  for (int i = 0; i < n_pv; ++i) s->is_slack[pv[i]] = 0;
  for (int i = 0; i < n_pq; ++i) s->is_slack[pq[i]] = 0;
  s->vinit.assign(vinit, vinit + 2 * n_bus);
  s->sbus.assign(sbus, sbus + 2 * n_bus);
  ck(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "stream");
  ck(cudaEventCreate(&s->ev0), "event");
  ck(cudaEventCreate(&s->ev1), "event");
  upload_plan(s.get());
  s->d_ybus.ensure(s->ybus.size() * sizeof(double));
  ck(cudaMemcpy(s->d_ybus.p, s->ybus.data(), s->ybus.size() * sizeof(double), cudaMemcpyHostToDevice), "upload Ybus");
  s->d_vinit.ensure(2 * n_bus * sizeof(double));
  ck(cudaMemcpy(s->d_vinit.p, vinit, 2 * n_bus * sizeof(double), cudaMemcpyHostToDevice), "upload Vinit");
  s->d_sbus.ensure(2 * n_bus * sizeof(double));
  ck(cudaMemcpy(s->d_sbus.p, sbus, 2 * n_bus * sizeof(double), cudaMemcpyHostToDevice), "upload Sbus");
  *out = s.release();
  GS2G_CATCH
}

int gs2g_session_set_chord(gs2g_session* s, int mode) {
  GS2G_TRY
  if (!s) throw std::invalid_argument("session_set_chord: NULL session");
  if (mode < 0 || mode > 2) throw std::invalid_argument("session_set_chord: mode must be 0, 1 or 2");
  s->chord = mode;
  GS2G_CATCH
}

int gs2g_session_set_handle_disconnected(gs2g_session* s, int on) {
  GS2G_TRY
  if (!s) throw std::invalid_argument("session_set_handle_disconnected: NULL session");
  if (on != 0 && on != 1) throw std::invalid_argument("session_set_handle_disconnected: on must be 0 or 1");
  if (s->handle_disconnected != on) s->rows_dirty = true;
  s->handle_disconnected = on;
  GS2G_CATCH
}

int gs2g_session_set_results_mirror(gs2g_session* s, int on) {
  GS2G_TRY
  if (!s) throw std::invalid_argument("session_set_results_mirror: NULL session");
  if (on != 0 && on != 1) throw std::invalid_argument("session_set_results_mirror: on must be 0 or 1");
  s->mirror_on = on != 0;
  if (!s->mirror_on) s->mirror_valid = false;
  GS2G_CATCH
}

int gs2g_session_set_row_order(gs2g_session* s, int on) {
  GS2G_TRY
  if (!s) throw std::invalid_argument("session_set_row_order: NULL session");
  if (on != 0 && on != 1) throw std::invalid_argument("session_set_row_order: on must be 0 or 1");
  if (s->row_order != on) s->rows_dirty = true;
  s->row_order = on;
  GS2G_CATCH
}

int gs2g_session_set_handoff(gs2g_session* s, int cluster) {
  GS2G_TRY
  if (!s) throw std::invalid_argument("session_set_handoff: NULL session");
  if (cluster != 0 && cluster != 1) throw std::invalid_argument("session_set_handoff: cluster must be 0 or 1");
  s->handoff_cluster = cluster;
  GS2G_CATCH
}

int gs2g_session_replan(gs2g_session* s, int tail_policy, double dense_rate, int force_tau) {
  GS2G_TRY
  if (!s) throw std::invalid_argument("session_replan: NULL session");
  if (tail_policy != 0 && tail_policy != 1) throw std::invalid_argument("session_replan: tail_policy must be 0 or 1");
  if (!(dense_rate >= 0)) throw std::invalid_argument("session_replan: dense_rate must be >= 0");
  DeviceGuard g(s->device);
  gs2g::TailOptions topt;
  topt.policy = tail_policy;
  if (dense_rate > 0) topt.dense_rate = dense_rate;
  topt.force_tau = force_tau;
  gs2g::Plan P = gs2g::build_plan(s->n_bus, s->y_ip.data(), s->y_ix.data(), s->pv.data(), (int)s->pv.size(),
                                  s->pq.data(), (int)s->pq.size(), topt);
  ck(cudaStreamSynchronize(s->stream), "replan");
  s->plan = std::move(P);
  s->plan_bufs.clear();
  upload_plan(s);
  s->base_factor_prec = -1;
  s->tm.plan_ms = s->plan.build_ms;
  GS2G_CATCH
}

int gs2g_session_destroy(gs2g_session* s) {
  GS2G_TRY
  if (!s) return GS2G_OK;
  {
    DeviceGuard g(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->ev_ext) cudaEventDestroy(s->ev_ext);
    for (cudaEvent_t e : s->ev_stage)
      if (e) cudaEventDestroy(e);
    if (s->h_stage) cudaFreeHost(s->h_stage);
    if (s->h_res) cudaFreeHost(s->h_res);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
  }
  GS2G_CATCH
}

int gs2g_get_device(const gs2g_session* s, int* device) {
  GS2G_TRY
  if (!s || !device) throw std::invalid_argument("NULL argument");
  *device = s->device;
  GS2G_CATCH
}

int gs2g_plan_info(int n_bus, const int* ybus_indptr, const int* ybus_indices, const int* pv, int n_pv, const int* pq,
                   int n_pq, int tail_policy, gs2g_grid_info* out) {
  GS2G_TRY
  if (n_bus <= 0 || !ybus_indptr || !ybus_indices || !out) throw std::invalid_argument("plan_info: bad arguments");
  std::vector<int> ip, ix;
  std::vector<double> vals;
  std::vector<double> zeros(2 * (size_t)std::max(ybus_indptr[n_bus], 0), 0.0);
  canonical_csr(n_bus, ybus_indptr, ybus_indices, zeros.data(), ip, ix, vals);
  gs2g::TailOptions topt;
  topt.policy = tail_policy;
  const gs2g::Plan P = gs2g::build_plan(n_bus, ip.data(), ix.data(), pv, n_pv, pq, n_pq, topt);
  out->n_bus = P.n_bus;
  out->nnz_y = P.nnz_y;
  out->n_pvpq = P.n_pvpq;
  out->n_pq = P.n_pq;
  out->dim_j = P.dim;
  out->nnz_j = P.nnz_j;
  out->nnz_lu = P.nnz_lu;
  out->head_dim = P.p;
  out->tail_dim = P.nt;
  out->tail_dim_exact = P.n_tail_exact;
  out->n_levels = P.n_levels;
  out->n_supernodes = P.n_sn;
  out->head_madds = P.head_madds;
  out->schur_madds = P.schur_madds;
  out->dense_madds = P.dense_madds;
  out->plan_ms = P.build_ms;
  GS2G_CATCH
}

int gs2g_grid_get_info(const gs2g_session* s, gs2g_grid_info* out) {
  GS2G_TRY
  if (!s || !out) throw std::invalid_argument("NULL argument");
  const gs2g::Plan& P = s->plan;
  out->n_bus = P.n_bus;
  out->nnz_y = P.nnz_y;
  out->n_pvpq = P.n_pvpq;
  out->n_pq = P.n_pq;
  out->dim_j = P.dim;
  out->nnz_j = P.nnz_j;
  out->nnz_lu = P.nnz_lu;
  out->head_dim = P.p;
  out->tail_dim = P.nt;
  out->tail_dim_exact = P.n_tail_exact;
  out->n_levels = P.n_levels;
  out->n_supernodes = P.n_sn;
  out->head_madds = P.head_madds;
  out->schur_madds = P.schur_madds;
  out->dense_madds = P.dense_madds;
  out->plan_ms = P.build_ms;
  GS2G_CATCH
}

int gs2g_set_branch_data(gs2g_session* s, int n_branch, const int* from, const int* to, const double* yff,
                         const double* yft, const double* ytf, const double* ytt) {
  GS2G_TRY
  if (!s || n_branch < 0 || (n_branch > 0 && (!from || !to || !yff || !yft || !ytf || !ytt)))
    throw std::invalid_argument("set_branch_data: bad arguments");
  std::vector<int> kff(n_branch), ktt(n_branch), kft(n_branch), ktf(n_branch);
  for (int l = 0; l < n_branch; ++l) {
    // a negative endpoint is a side with no bus in the solved system (the
    // open end of a half-open line): the branch has only its other end's
    // self term (contingency_analysis_helper.cpp:53-75)
    const int f = from[l], t = to[l];
    if (f >= s->n_bus || t >= s->n_bus || (f >= 0 && f == t))
      throw std::invalid_argument("set_branch_data: branch " + std::to_string(l) + " has a bad endpoint");
    kff[l] = f >= 0 ? ybus_find(s->plan, f, f) : -1;
    ktt[l] = t >= 0 ? ybus_find(s->plan, t, t) : -1;
    kft[l] = f >= 0 && t >= 0 ? ybus_find(s->plan, f, t) : -1;
    ktf[l] = f >= 0 && t >= 0 ? ybus_find(s->plan, t, f) : -1;
    if ((f >= 0 && kff[l] < 0) || (t >= 0 && ktt[l] < 0) || (f >= 0 && t >= 0 && (kft[l] < 0 || ktf[l] < 0)))
      throw std::invalid_argument("set_branch_data: branch " + std::to_string(l) + " is not in the Ybus pattern");
  }
  s->n_branch = n_branch;
  s->br_from.assign(from, from + n_branch);
  s->br_to.assign(to, to + n_branch);
  s->yff.assign(yff, yff + 2 * n_branch);
  s->yft.assign(yft, yft + 2 * n_branch);
  s->ytf.assign(ytf, ytf + 2 * n_branch);
  s->ytt.assign(ytt, ytt + 2 * n_branch);
  s->k_ff.swap(kff);
  s->k_tt.swap(ktt);
  s->k_ft.swap(kft);
  s->k_tf.swap(ktf);
  compute_bridges(s);
  {
    DeviceGuard g(s->device);
    std::vector<double> y(8 * (size_t)n_branch);
    for (int l = 0; l < n_branch; ++l) {
      const double* src[4] = {yff, yft, ytf, ytt};
      for (int q = 0; q < 4; ++q) {
        y[8 * l + 2 * q] = src[q][2 * l];
        y[8 * l + 2 * q + 1] = src[q][2 * l + 1];
      }
    }
    s->d_br_from.ensure(std::max(n_branch, 1) * sizeof(int));
    s->d_br_to.ensure(std::max(n_branch, 1) * sizeof(int));
    s->d_br_y.ensure(std::max<size_t>(y.size(), 1) * sizeof(double));
    if (n_branch) {
      ck(cudaMemcpy(s->d_br_from.p, from, n_branch * sizeof(int), cudaMemcpyHostToDevice), "upload branches");
      ck(cudaMemcpy(s->d_br_to.p, to, n_branch * sizeof(int), cudaMemcpyHostToDevice), "upload branches");
      ck(cudaMemcpy(s->d_br_y.p, y.data(), y.size() * sizeof(double), cudaMemcpyHostToDevice), "upload branches");
    }
  }
  s->limits_on = false;  // limits belong to the branch set they were given for
  s->rows_dirty = true;
  GS2G_CATCH
}

int gs2g_set_contingencies(gs2g_session* s, int n_rows, const int* ptr, const int* ids) {
  GS2G_TRY
  if (!s || n_rows < 0) throw std::invalid_argument("set_contingencies: bad arguments");
  if (n_rows > 0) {
    if (!ptr || ptr[0] != 0) throw std::invalid_argument("set_contingencies: ptr[0] must be 0");
    for (int r = 0; r < n_rows; ++r)
      if (ptr[r + 1] < ptr[r]) throw std::invalid_argument("set_contingencies: ptr must be non-decreasing");
    const int nnz = ptr[n_rows];
    if (nnz > 0 && !ids) throw std::invalid_argument("set_contingencies: ids must not be NULL");
    for (int q = 0; q < nnz; ++q)
      if (ids[q] < 0 || ids[q] >= s->n_branch)
        // std::runtime_error, as build_contingency_from_branch_ids
        // (contingency_analysis_helper.cpp:46-48): RuntimeError in Python
        throw std::runtime_error("set_contingencies: branch index " + std::to_string(ids[q]) +
                                 " out of range (n_branches=" + std::to_string(s->n_branch) + ")");
    s->ctg_ptr.assign(ptr, ptr + n_rows + 1);
    s->ctg_ids.assign(ids, ids + nnz);
  } else {
    s->ctg_ptr.clear();
    s->ctg_ids.clear();
  }
  s->n_ctg = n_rows;
  s->rows_dirty = true;
  GS2G_CATCH
}

extern "C++" {
namespace {
// Host copies of large results: the destination is usually fresh pageable
// memory (a new numpy array), whose first touch costs a page fault per 4 KB,
// so one thread copies at a few GB/s while the DMA delivers tens.  The copy
// out of the pinned staging chunk is split over a small pool of persistent
// threads (created on first use, shared by all sessions).
class CopyPool {
 public:
  static CopyPool& get() {
    static CopyPool pool;
    return pool;
  }
  // f(begin, end) over [0, n) in up to size() + 1 parts of at least `grain`
  // items each; the caller runs the first part
  void parallel_for(size_t n, size_t grain, const std::function<void(size_t, size_t)>& f) {
    if (forked_) {  // a forked child has the pool object but not its threads
      f(0, n);
      return;
    }
    const int parts = (int)std::min<size_t>(workers_.size() + 1, std::max<size_t>(1, n / std::max<size_t>(grain, 1)));
    if (parts <= 1) {
      f(0, n);
      return;
    }
    const size_t step = (n + parts - 1) / parts;
    {
      std::unique_lock<std::mutex> lk(m_);
      for (int k = 1; k < parts; ++k) {
        const size_t b = (size_t)k * step, e = std::min(n, b + step);
        if (b < e) {
          tasks_.push_back([&f, b, e] { f(b, e); });
          ++pending_;
        }
      }
    }
    cv_.notify_all();
    f(0, std::min(n, step));
    std::unique_lock<std::mutex> lk(m_);
    done_.wait(lk, [&] { return pending_ == 0; });
  }
  // memcpy(dst, src, n), split by 1 MB parts
  void copy(void* dst, const void* src, size_t n) {
    parallel_for(n, size_t(1) << 20, [=](size_t b, size_t e) {
      std::memcpy(static_cast<char*>(dst) + b, static_cast<const char*>(src) + b, e - b);
    });
  }

 private:
  CopyPool() {
    pthread_atfork(nullptr, nullptr, [] { forked_ = true; });
    const unsigned hw = std::thread::hardware_concurrency();
    const int n = (int)std::min<unsigned>(7, hw > 1 ? hw - 1 : 0);
    for (int i = 0; i < n; ++i) workers_.emplace_back([this] { run(); });
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> lk(m_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
  }
  void run() {
    for (;;) {
      std::function<void()> f;
      {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return stop_ || !tasks_.empty(); });
        if (stop_ && tasks_.empty()) return;
        f = std::move(tasks_.back());
        tasks_.pop_back();
      }
      f();
      {
        std::lock_guard<std::mutex> lk(m_);
        if (--pending_ == 0) done_.notify_all();
      }
    }
  }
  std::vector<std::thread> workers_;
  std::vector<std::function<void()>> tasks_;
  std::mutex m_;
  std::condition_variable cv_, done_;
  int pending_ = 0;
  bool stop_ = false;
  static inline bool forked_ = false;
};

constexpr size_t kStageChunk = size_t(8) << 20;
// the session's pinned double buffer for large copies, made on first use
void ensure_stage(const gs2g_session* s) {
  if (!s->h_stage) {
    ck(cudaMallocHost(&s->h_stage, 2 * kStageChunk), "pinned staging buffer");
    for (cudaEvent_t& e : s->ev_stage) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
  }
}
// Large host-to-device uploads of generated data: `fill(dst, off, len)`
// writes bytes [off, off + len) of the payload into a pinned chunk, which is
// copied to the device while the next chunk is filled.  `len` is a multiple
// of 16 bytes except for the last chunk.
template <typename Fill>
void h2d_staged(const gs2g_session* s, void* dst, size_t bytes, Fill fill) {
  ensure_stage(s);
  char* buf[2] = {static_cast<char*>(s->h_stage), static_cast<char*>(s->h_stage) + kStageChunk};
  const size_t nch = (bytes + kStageChunk - 1) / kStageChunk;
  for (size_t i = 0; i < nch; ++i) {
    const size_t off = i * kStageChunk, len = std::min(kStageChunk, bytes - off);
    if (i >= 2) ck(cudaEventSynchronize(s->ev_stage[i & 1]), "upload rows");  // buffer free again
    fill(reinterpret_cast<double*>(buf[i & 1]), off, len);
    ck(cudaMemcpyAsync(static_cast<char*>(dst) + off, buf[i & 1], len, cudaMemcpyHostToDevice, s->stream),
       "upload rows");
    ck(cudaEventRecord(s->ev_stage[i & 1], s->stream), "event");
  }
  ck(cudaStreamSynchronize(s->stream), "upload rows");
}
}  // namespace
}  // extern "C++"

int gs2g_set_injections(gs2g_session* s, int n_rows, const double* p_mw, const double* q_mvar, double sn_mva) {
  GS2G_TRY
  if (!s || n_rows < 0) throw std::invalid_argument("set_injections: bad arguments");
  if (n_rows > 0) {
    if (!p_mw || !q_mvar) throw std::invalid_argument("set_injections: p_mw / q_mvar must not be NULL");
    if (!(sn_mva > 0)) throw std::invalid_argument("set_injections: sn_mva must be positive");
    DeviceGuard g(s->device);
    const size_t m = (size_t)n_rows * s->n_bus;
    s->d_sbus_rows.ensure(m * 2 * sizeof(double));
    // Sbus = (p + jq) / sn_mva, interleaved straight into pinned chunks that
    // are copied to the device while the next chunk is converted
    const double inv = 1.0 / sn_mva;
    // each row's distance from the base injections, sum over buses of
    // |dP| + |dQ| (the row-order key), accumulated in fixed point while the
    // rows are converted
    const size_t n = s->n_bus;
    std::unique_ptr<std::atomic<int64_t>[]> keyfx(new std::atomic<int64_t>[n_rows]);
    for (int r = 0; r < n_rows; ++r) keyfx[r].store(0, std::memory_order_relaxed);
    const double* sb = s->sbus.data();
    constexpr double kFix = 1e9;
    h2d_staged(s, s->d_sbus_rows.p, m * 2 * sizeof(double), [&](double* dst, size_t off, size_t len) {
      const size_t q0 = off / (2 * sizeof(double)), nq = len / (2 * sizeof(double));
      CopyPool::get().parallel_for(nq, size_t(1) << 16, [&](size_t b, size_t e) {
        size_t row = (q0 + b) / n, bus = (q0 + b) % n;
        double acc = 0.0;
        for (size_t q = b; q < e; ++q) {
          const double pr = p_mw[q0 + q] * inv, qr = q_mvar[q0 + q] * inv;
          dst[2 * q] = pr;
          dst[2 * q + 1] = qr;
          acc += std::fabs(pr - sb[2 * bus]) + std::fabs(qr - sb[2 * bus + 1]);
          if (++bus == n) {
            keyfx[row].fetch_add((int64_t)std::llround(std::min(acc, 1e9) * kFix), std::memory_order_relaxed);
            acc = 0.0;
            bus = 0;
            ++row;
          }
        }
        if (bus != 0) keyfx[row].fetch_add((int64_t)std::llround(std::min(acc, 1e9) * kFix), std::memory_order_relaxed);
      });
    });
    s->inj_key.resize(n_rows);
    for (int r = 0; r < n_rows; ++r) s->inj_key[r] = (double)keyfx[r].load(std::memory_order_relaxed) / kFix;
  } else {
    s->inj_key.clear();
  }
  s->n_inj = n_rows;
  s->rows_dirty = true;
  GS2G_CATCH
}

int gs2g_set_start_rows(gs2g_session* s, int n_rows, const double* v0) {
  GS2G_TRY
  if (!s || n_rows < 0 || (n_rows > 0 && !v0)) throw std::invalid_argument("set_start_rows: bad arguments");
  DeviceGuard g(s->device);
  const size_t bytes = (size_t)n_rows * s->n_bus * 2 * sizeof(double);
  s->d_v0rows.ensure(bytes);
  if (bytes) ck(cudaMemcpy(s->d_v0rows.p, v0, bytes, cudaMemcpyHostToDevice), "upload start rows");
  s->n_start = n_rows;
  GS2G_CATCH
}

int gs2g_set_start_rows_device(gs2g_session* s, int n_rows, const double* v0_dev) {
  GS2G_TRY
  if (!s || n_rows < 0 || (n_rows > 0 && !v0_dev)) throw std::invalid_argument("set_start_rows_device: bad arguments");
  DeviceGuard g(s->device);
  const size_t bytes = (size_t)n_rows * s->n_bus * 2 * sizeof(double);
  s->d_v0rows.ensure(bytes);
  if (bytes) ck(cudaMemcpyAsync(s->d_v0rows.p, v0_dev, bytes, cudaMemcpyDeviceToDevice, s->stream), "copy start rows");
  ck(cudaStreamSynchronize(s->stream), "copy start rows");
  s->n_start = n_rows;
  GS2G_CATCH
}

int gs2g_start_rows_buffer(gs2g_session* s, int n_rows, double** v0_dev) {
  GS2G_TRY
  if (!s || n_rows < 0 || !v0_dev) throw std::invalid_argument("start_rows_buffer: bad arguments");
  DeviceGuard g(s->device);
  s->d_v0rows.ensure((size_t)std::max(n_rows, 1) * s->n_bus * 2 * sizeof(double));
  s->n_start = n_rows;
  *v0_dev = s->d_v0rows.as<double>();
  GS2G_CATCH
}

int gs2g_set_sbus(gs2g_session* s, const double* sbus) {
  GS2G_TRY
  if (!s || !sbus) throw std::invalid_argument("set_sbus: bad arguments");
  DeviceGuard g(s->device);
  s->sbus.assign(sbus, sbus + 2 * s->n_bus);
  ck(cudaMemcpy(s->d_sbus.p, sbus, 2 * s->n_bus * sizeof(double), cudaMemcpyHostToDevice), "upload Sbus");
  GS2G_CATCH
}

int gs2g_set_vinit(gs2g_session* s, const double* vinit) {
  GS2G_TRY
  if (!s || !vinit) throw std::invalid_argument("set_vinit: bad arguments");
  DeviceGuard g(s->device);
  s->vinit.assign(vinit, vinit + 2 * s->n_bus);
  ck(cudaMemcpy(s->d_vinit.p, vinit, 2 * s->n_bus * sizeof(double), cudaMemcpyHostToDevice), "upload Vinit");
  GS2G_CATCH
}

namespace {
// Vb conj(Y Vb) per bus for the current base V (host, once per base case),
// so that a row's mismatch norm at the base V needs no sparse product; and
// Y Vb itself, summed with the fused multiply-adds of the sweep's mismatch
// in the same order (IEEE fma rounds the same on host and device), so that
// the chord sweep writes a row's F at the base V bit-identical to the sparse
// product it replaces.
void upload_base_power(gs2g_session* s) {
  const int n = s->n_bus;
  std::vector<double> S(2 * n), I(2 * n);
  for (int i = 0; i < n; ++i) {
    double ir = 0, ii = 0, fr = 0, fi = 0;
    for (int k = s->y_ip[i]; k < s->y_ip[i + 1]; ++k) {
      const double yr = s->ybus[2 * k], yi = s->ybus[2 * k + 1];
      const double vr = s->base_v[2 * s->y_ix[k]], vi = s->base_v[2 * s->y_ix[k] + 1];
      ir += yr * vr - yi * vi;
      ii += yr * vi + yi * vr;
      fr = std::fma(yr, vr, std::fma(-yi, vi, fr));
      fi = std::fma(yr, vi, std::fma(yi, vr, fi));
    }
    const double vr = s->base_v[2 * i], vi = s->base_v[2 * i + 1];
    S[2 * i] = vr * ir + vi * ii;  // V conj(I)
    S[2 * i + 1] = vi * ir - vr * ii;
    I[2 * i] = fr;
    I[2 * i + 1] = fi;
  }
  s->d_bases.ensure(2 * n * sizeof(double));
  ck(cudaMemcpy(s->d_bases.p, S.data(), 2 * n * sizeof(double), cudaMemcpyHostToDevice), "upload base power");
  s->d_basei.ensure(2 * n * sizeof(double));
  ck(cudaMemcpy(s->d_basei.p, I.data(), 2 * n * sizeof(double), cudaMemcpyHostToDevice), "upload base current");
}
}  // namespace

int gs2g_solve_base(gs2g_session* s, const gs2g_run_opts* o_, double* v_out, int* status, int* iters,
                    double* residual) {
  GS2G_TRY
  if (!s) throw std::invalid_argument("NULL session");
  gs2g_run_opts o = checked(o_);
  DeviceGuard g(s->device);
  const int n = s->n_bus;
  s->b_v.ensure(2 * n * sizeof(double));
  s->b_res.ensure(sizeof(double));
  s->b_status.ensure(sizeof(int));
  s->b_iters.ensure(sizeof(int));
  OutBufs ob{s->b_v.as<double>(), s->b_res.as<double>(), s->b_status.as<int>(), s->b_iters.as<int>()};
  const float ms = launch(s, o, 1, s->d_vinit.as<double>(), 0, s->d_sbus.as<double>(), 0, false, ob, 1);
  s->tm.kernel_ms = ms;
  int st = 0, it = 0;
  double res = 0;
  s->base_v.resize(2 * n);
  ck(cudaMemcpy(s->base_v.data(), s->b_v.p, 2 * n * sizeof(double), cudaMemcpyDeviceToHost), "read base V");
  ck(cudaMemcpy(&st, s->b_status.p, sizeof(int), cudaMemcpyDeviceToHost), "read base status");
  ck(cudaMemcpy(&it, s->b_iters.p, sizeof(int), cudaMemcpyDeviceToHost), "read base iters");
  ck(cudaMemcpy(&res, s->b_res.p, sizeof(double), cudaMemcpyDeviceToHost), "read base residual");
  s->d_basev.ensure(2 * n * sizeof(double));
  ck(cudaMemcpy(s->d_basev.p, s->b_v.p, 2 * n * sizeof(double), cudaMemcpyDeviceToDevice), "keep base V");
  s->has_base = true;
  s->base_factor_prec = -1;
  upload_base_power(s);
  if (v_out) std::memcpy(v_out, s->base_v.data(), 2 * n * sizeof(double));
  if (status) *status = st;
  if (iters) *iters = it;
  if (residual) *residual = res;
  GS2G_CATCH
}

int gs2g_set_base_v(gs2g_session* s, const double* v, double* residual) {
  GS2G_TRY
  if (!s || !v) throw std::invalid_argument("set_base_v: bad arguments");
  DeviceGuard g(s->device);
  const int n = s->n_bus;
  s->d_basev.ensure(2 * n * sizeof(double));
  ck(cudaMemcpy(s->d_basev.p, v, 2 * n * sizeof(double), cudaMemcpyHostToDevice), "upload base V");
  s->b_v.ensure(2 * n * sizeof(double));
  s->b_res.ensure(sizeof(double));
  s->b_status.ensure(sizeof(int));
  s->b_iters.ensure(sizeof(int));
  gs2g_run_opts o{};
  o.max_iter = 0;
  o.tol = 0;
  o.fixed_iters = 1;
  o.precision = GS2G_PREC_FP64;
  OutBufs ob{s->b_v.as<double>(), s->b_res.as<double>(), s->b_status.as<int>(), s->b_iters.as<int>()};
  launch(s, o, 1, s->d_basev.as<double>(), 0, s->d_sbus.as<double>(), 0, false, ob, 1);
  double res = 0;
  ck(cudaMemcpy(&res, s->b_res.p, sizeof(double), cudaMemcpyDeviceToHost), "read residual");
  s->base_v.assign(v, v + 2 * n);
  s->has_base = true;
  s->base_factor_prec = -1;
  upload_base_power(s);
  if (residual) *residual = res;
  GS2G_CATCH
}

namespace {
// Row sources and output buffers of a session's assembled rows.
struct RunPrep {
  int nr;
  const double* v0;
  int64_t v0s;
  const double* sb;
  int64_t sbs;
  OutBufs ob;
};

// Factor the base case's Jacobian (base V, base Ybus) once per precision
// into the session's base workspace: one CTA in factor-only mode whose
// workspace is that buffer.  GS2G_REFACTOR_BASE_CHORD rows start on it.
void ensure_base_factor(gs2g_session* s, int prec) {
  if (s->base_factor_prec == prec) return;
  if (!s->has_base)
    throw std::runtime_error("refactor policy BASE_CHORD needs a base case (solve_base or set_base_v first)");
  const auto t_setup = std::chrono::steady_clock::now();
  const int n = s->n_bus;
  const int64_t wsb = gs2g::workspace_bytes(s->dplan, prec);
  s->d_base_ws.ensure((size_t)wsb);
  s->b_v.ensure(2 * n * sizeof(double));
  s->b_res.ensure(sizeof(double));
  s->b_status.ensure(sizeof(int));
  s->b_iters.ensure(sizeof(int));
  gs2g_run_opts o{};
  o.max_iter = 1;
  o.precision = prec;
  o.refactor_policy = GS2G_REFACTOR_EVERY;
  OutBufs ob{s->b_v.as<double>(), s->b_res.as<double>(), s->b_status.as<int>(), s->b_iters.as<int>()};
  gs2g::SweepArgs a = make_args(s, o, 1, s->d_basev.as<double>(), 0, s->d_sbus.as<double>(), 0, false, ob);
  a.factor_only = 1;
  s->d_queue.ensure(3 * sizeof(int));
  a.queue = s->d_queue.as<int>();
  a.workspace = s->d_base_ws.as<char>();
  a.ws_stride = wsb;
  ck(cudaMemsetAsync(s->d_queue.p, 0, 3 * sizeof(int), s->stream), "queue reset");
  ck((cudaError_t)gs2g::launch_sweep(s->dplan, a, prec, 1, s->stream), "base factor launch");
  // its inverse, one column per row of an inverse-mode sweep over all CTAs
  const int dim = s->dplan.dim;
  const size_t elem = prec == GS2G_PREC_FP64 ? sizeof(double) : sizeof(float);
  s->d_base_inv.ensure((size_t)dim * dim * elem);
  int n_ctas = std::max(1, std::min(gs2g::sweep_ctas(prec, s->device), dim));
  s->d_ws.ensure((size_t)wsb * n_ctas);
  gs2g::SweepArgs ai = a;
  ai.factor_only = 0;
  ai.n_rows = dim;
  ai.base_ws = s->d_base_ws.as<char>();
  ai.inverse_out = s->d_base_inv.as<char>();
  ai.workspace = s->d_ws.as<char>();
  ck(cudaMemsetAsync(s->d_queue.p, 0, 3 * sizeof(int), s->stream), "queue reset");
  ck((cudaError_t)gs2g::launch_sweep(s->dplan, ai, prec, n_ctas, s->stream), "base inverse launch");
  ck(cudaStreamSynchronize(s->stream), "base factor");
  // its head values in solve order, so that the chord sweep streams them
  // beside the column indices instead of gathering them through fw_pos / bw_pos
  {
    const int64_t hv_off = gs2g::workspace_hv_offset(s->dplan, prec);
    const size_t n_hv = (size_t)s->dplan.n_hv;
    std::vector<char> hv(std::max<size_t>(n_hv, 1) * elem);
    if (n_hv)
      ck(cudaMemcpy(hv.data(), s->d_base_ws.as<char>() + hv_off, n_hv * elem, cudaMemcpyDeviceToHost),
         "read base factor");
    auto packed = [&](const std::vector<int>& pos, DevBuf& dst) {
      std::vector<char> v(std::max<size_t>(pos.size(), 1) * elem);
      for (size_t q = 0; q < pos.size(); ++q) std::memcpy(v.data() + q * elem, hv.data() + (size_t)pos[q] * elem, elem);
      dst.ensure(v.size());
      ck(cudaMemcpy(dst.p, v.data(), v.size(), cudaMemcpyHostToDevice), "upload base factor values");
    };
    packed(s->plan.fw_pos, s->d_base_fwv);
    packed(s->plan.bw_pos, s->d_base_bwv);
  }
  s->base_factor_prec = prec;
  s->tm.base_setup_ms = ms_since(t_setup);
  s->tm.base_setup_bytes = (int64_t)(s->d_base_ws.n + s->d_base_inv.n + s->d_base_fwv.n + s->d_base_bwv.n);
}

// The pinned result buffer for `nr` rows: V [nr x n] complex, then the
// residuals, statuses and iterations.  Grows only (a grown buffer loses its
// contents, and with them a valid mirror).
void ensure_host_results(gs2g_session* s, size_t nr) {
  const size_t n = s->n_bus;
  const size_t total = std::max<size_t>(nr * n * 2 * sizeof(double) + nr * (sizeof(double) + 2 * sizeof(int)), 16);
  if (s->h_res_bytes >= total) return;
  s->mirror_valid = false;
  if (s->h_res) ck(cudaFreeHost(s->h_res), "free pinned results");
  s->h_res = nullptr;
  s->h_res_bytes = 0;
  ck(cudaHostAlloc(&s->h_res, total, cudaHostAllocMapped), "pinned results");
  s->h_res_bytes = total;
}

RunPrep prepare_rows(gs2g_session* s, const gs2g_run_opts& o) {
  if (o.refactor_policy == GS2G_REFACTOR_BASE_CHORD) ensure_base_factor(s, o.precision);
  const int nr = s->n_rows;
  const int n = s->n_bus;
  const double* v0 = s->d_vinit.as<double>();
  int64_t v0s = 0;
  if (o.start == GS2G_START_BASE) {
    if (!s->has_base) throw std::runtime_error("start=BASE needs a base case (solve_base or set_base_v first)");
    v0 = s->d_basev.as<double>();
  } else if (o.start == GS2G_START_ROWS) {
    if (s->n_start != nr)
      throw std::invalid_argument("start=ROWS needs one start voltage per row (" + std::to_string(nr) + "), got " +
                                  std::to_string(s->n_start));
    v0 = s->d_v0rows.as<double>();
    v0s = n;
  } else if (o.start != GS2G_START_VINIT) {
    throw std::invalid_argument("unknown start mode");
  }
  const double* sb = s->rows_have_sbus ? s->d_sbus_rows.as<double>() : s->d_sbus.as<double>();
  const int64_t sbs = s->rows_have_sbus ? n : 0;
  s->d_v_out.ensure((size_t)std::max(nr, 1) * n * 2 * sizeof(double));
  s->d_res.ensure((size_t)std::max(nr, 1) * sizeof(double));
  s->d_status.ensure((size_t)std::max(nr, 1) * sizeof(int));
  s->d_iters.ensure((size_t)std::max(nr, 1) * sizeof(int));
  s->d_factors.ensure((size_t)std::max(nr, 1) * sizeof(int));
  OutBufs ob{s->d_v_out.as<double>(), s->d_res.as<double>(), s->d_status.as<int>(), s->d_iters.as<int>(),
             s->d_factors.as<int>()};
  if (s->mirror_on && nr > 0) {
    ensure_host_results(s, nr);
    void* d = nullptr;
    ck(cudaHostGetDevicePointer(&d, s->h_res, 0), "results mirror address");
    ob.v_mirror = static_cast<double*>(d);
  }
  return RunPrep{nr, v0, v0s, sb, sbs, ob};
}
}  // namespace

int gs2g_run(gs2g_session* s, const gs2g_run_opts* o_) {
  GS2G_TRY
  if (!s) throw std::invalid_argument("NULL session");
  gs2g_run_opts o = checked(o_);
  DeviceGuard g(s->device);
  auto t0 = std::chrono::steady_clock::now();
  assemble_rows(s);
  s->tm.upload_ms = ms_since(t0);
  s->mirror_valid = false;
  const RunPrep rp = prepare_rows(s, o);
  const int nr = rp.nr;
  s->tm.kernel_ms = launch(s, o, nr, rp.v0, rp.v0s, rp.sb, rp.sbs, true, rp.ob, o.n_ctas);
  s->last_rows_run = nr;
  s->mirror_valid = rp.ob.v_mirror != nullptr;
  s->tm.total_ms = ms_since(t0);
  s->tm.total_iters = -1;
  GS2G_CATCH
}

int gs2g_run_subset(gs2g_session* s, const gs2g_run_opts* o_, int n_sub, const int* rows) {
  GS2G_TRY
  if (!s) throw std::invalid_argument("NULL session");
  gs2g_run_opts o = checked(o_);
  if (n_sub < 0 || (n_sub > 0 && !rows)) throw std::invalid_argument("run_subset: bad row list");
  DeviceGuard g(s->device);
  auto t0 = std::chrono::steady_clock::now();
  assemble_rows(s);
  if (s->last_rows_run != s->n_rows)
    throw std::invalid_argument("run_subset: run the full batch (gs2g_run) before re-running a subset of it");
  for (int i = 0; i < n_sub; ++i)
    if (rows[i] < 0 || rows[i] >= s->n_rows) throw std::invalid_argument("run_subset: row index out of range");
  s->tm.upload_ms = ms_since(t0);
  const RunPrep rp = prepare_rows(s, o);
  // the subset's rows reach the mirror only when it is on (same rows, so
  // the buffer is not regrown)
  if (rp.ob.v_mirror == nullptr) s->mirror_valid = false;
  s->d_row_map.ensure(std::max(n_sub, 1) * sizeof(int));
  if (n_sub) ck(cudaMemcpy(s->d_row_map.p, rows, n_sub * sizeof(int), cudaMemcpyHostToDevice), "upload row map");
  gs2g::SweepArgs a = make_args(s, o, n_sub, rp.v0, rp.v0s, rp.sb, rp.sbs, true, rp.ob);
  a.row_map = s->d_row_map.as<int>();
  int n_ctas = o.n_ctas > 0 ? o.n_ctas : gs2g::sweep_ctas(o.precision, s->device);
  // few rows with a dense tail worth sharing (an FP64 re-solve of the rows
  // a mixed sweep did not converge): a cluster of CTAs per row
  const int csize = s->handoff_cluster && s->dplan.nt >= 64 ? cluster_for(n_sub, n_ctas) : 0;
  const bool cluster = n_sub > 0 && csize > 0;
  n_ctas = cluster ? n_sub * csize : std::max(1, std::min(n_ctas, std::max(n_sub, 1)));
  const int64_t wsb = gs2g::workspace_bytes(s->dplan, o.precision);
  s->d_ws.ensure((size_t)wsb * n_ctas);
  s->d_queue.ensure(3 * sizeof(int));
  a.queue = s->d_queue.as<int>();
  a.workspace = s->d_ws.as<char>();
  a.ws_stride = wsb;
  a.n_rescued = s->d_queue.as<int>() + 1;
  if (o.profile_phases) {
    s->d_phase.ensure(gs2g::N_PHASES * sizeof(unsigned long long));
    ck(cudaMemsetAsync(s->d_phase.p, 0, gs2g::N_PHASES * sizeof(unsigned long long), s->stream), "phase reset");
    a.phase_cycles = s->d_phase.as<unsigned long long>();
  }
  ck(cudaMemsetAsync(s->d_queue.p, 0, 3 * sizeof(int), s->stream), "queue reset");
  ck(cudaEventRecord(s->ev0, s->stream), "event");
  if (n_sub > 0 && cluster)
    ck((cudaError_t)gs2g::launch_sweep_cluster(s->dplan, a, o.precision, csize, n_ctas, s->stream),
       "subset cluster launch");
  else if (n_sub > 0)
    ck((cudaError_t)gs2g::launch_sweep(s->dplan, a, o.precision, n_ctas, s->stream), "subset launch");
  ck(cudaEventRecord(s->ev1, s->stream), "event");
  ck(cudaStreamSynchronize(s->stream), "subset sweep");
  float ms = 0;
  ck(cudaEventElapsedTime(&ms, s->ev0, s->ev1), "event time");
  s->tm.kernel_ms = ms;
  for (int q = 0; q < GS2G_N_PHASES; ++q) s->tm.phase_cycles[q] = s->tm.phase_share[q] = 0;
  if (o.profile_phases) {
    unsigned long long c[gs2g::N_PHASES];
    ck(cudaMemcpy(c, s->d_phase.p, sizeof(c), cudaMemcpyDeviceToHost), "read phases");
    double tot = 0;
    for (int q = 0; q < gs2g::N_PHASES; ++q) tot += (double)c[q];
    for (int q = 0; q < gs2g::N_PHASES; ++q) {
      s->tm.phase_cycles[q] = (double)c[q];
      s->tm.phase_share[q] = tot > 0 ? c[q] / tot : 0;
    }
  }
  s->tm.total_ms = ms_since(t0);
  s->tm.total_iters = -1;
  GS2G_CATCH
}

int gs2g_run_multi(gs2g_session* const* sessions, int n_sessions, const gs2g_run_opts* o_) {
  GS2G_TRY
  if (!sessions || n_sessions < 1 || n_sessions > gs2g::MAX_GRIDS)
    throw std::invalid_argument("run_multi: between 1 and " + std::to_string(gs2g::MAX_GRIDS) + " sessions");
  for (int i = 0; i < n_sessions; ++i) {
    if (!sessions[i]) throw std::invalid_argument("run_multi: NULL session");
    if (sessions[i]->device != sessions[0]->device) throw std::invalid_argument("run_multi: sessions on different devices");
    for (int j = 0; j < i; ++j)
      if (sessions[j] == sessions[i]) throw std::invalid_argument("run_multi: a session is listed twice");
  }
  gs2g_run_opts o = checked(o_);
  gs2g_session* s0 = sessions[0];
  DeviceGuard g(s0->device);
  auto t0 = std::chrono::steady_clock::now();
  std::vector<gs2g::GridEntry> ge(n_sessions);
  std::vector<int> begin(n_sessions + 1, 0);
  int64_t wsb = 0;
  // [0] row queue, [1] rescue count, [2] alternative starts, [3] hand-offs,
  // [4 + i] chord queue of grid i
  s0->d_queue.ensure((4 + n_sessions) * sizeof(int));
  for (int i = 0; i < n_sessions; ++i) {
    gs2g_session* s = sessions[i];
    assemble_rows(s);
    s->mirror_valid = false;
    const RunPrep rp = prepare_rows(s, o);
    ge[i].P = s->dplan;
    ge[i].a = make_args(s, o, rp.nr, rp.v0, rp.v0s, rp.sb, rp.sbs, true, rp.ob);
    ge[i].a.n_rescued = s0->d_queue.as<int>() + 1;
    ge[i].a.n_alt_start = s0->d_queue.as<int>() + 2;
    begin[i + 1] = begin[i] + rp.nr;
    wsb = std::max(wsb, gs2g::workspace_bytes(s->dplan, o.precision));
  }
  const double upload_ms = ms_since(t0);
  const int total = begin[n_sessions];
  int n_ctas = o.n_ctas > 0 ? o.n_ctas : gs2g::sweep_ctas(o.precision, s0->device);
  n_ctas = std::max(1, std::min(n_ctas, std::max(total, 1)));
  // policy 2 (continuous): a multi-grid chord sweep first (several rows per
  // CTA on each grid's base factor), then the single-row sweep continues the
  // rows it hands off, from v_out / iters_out on their own factors
  bool chord = s0->chord > 0 && total > 0 && o.refactor_policy == GS2G_REFACTOR_BASE_CHORD && !o.fixed_iters;
  for (int i = 0; i < n_sessions; ++i) chord = chord && ge[i].a.base_ws != nullptr && ge[i].a.base_inv != nullptr;
  std::vector<gs2g::GridEntry> gc;
  int64_t cwsb = 0;
  int csmem = 0, n_chord = 0;
  if (chord) {
    const int per = gs2g::chord_rows_per_cta();
    int big = 0;
    for (int i = 0; i < n_sessions; ++i) {
      cwsb = std::max(cwsb, gs2g::chord_workspace_bytes(sessions[i]->dplan, o.precision));
      const int sm = gs2g::chord_smem(sessions[i]->dplan, o.precision);
      if (sm > csmem) {
        csmem = sm;
        big = i;
      }
    }
    n_chord = o.n_ctas > 0 ? o.n_ctas : gs2g::chord_ctas(sessions[big]->dplan, o.precision, s0->device);
    n_chord = std::max(1, std::min(n_chord, (total + per - 1) / per));
    s0->d_handoff.ensure((size_t)total * sizeof(int));
    s0->d_chord_steps.ensure(sizeof(unsigned long long));
    gc = ge;
    for (int i = 0; i < n_sessions; ++i) {
      gs2g::SweepArgs& a = gc[i].a;
      a.queue = s0->d_queue.as<int>() + 4 + i;
      a.ws_stride = cwsb;
      a.handoff = s0->d_handoff.as<int>();
      a.n_handoff = s0->d_queue.as<int>() + 3;
      a.handoff_base = begin[i];
      a.n_chord_steps = s0->d_chord_steps.as<unsigned long long>();
      a.broyden = s0->chord == 2;
      // the hand-offs continue from where the chord sweep left them
      gs2g::SweepArgs& b = ge[i].a;
      b.v0 = b.v_out;
      b.v0_stride = sessions[i]->n_bus;
      b.iters_in = b.iters_out;
      b.refactor_policy = GS2G_REFACTOR_ADAPTIVE;
      b.base_ws = nullptr;
      b.base_v = nullptr;
      b.base_inv = nullptr;
      b.alt_v0 = nullptr;
      b.alt_s = nullptr;
      b.alt_i = nullptr;
    }
  }
  s0->d_ws.ensure(std::max((size_t)wsb * n_ctas, (size_t)cwsb * n_chord));
  for (auto& e : gc) e.a.workspace = s0->d_ws.as<char>();
  const size_t ge_bytes = sizeof(gs2g::GridEntry) * n_sessions;
  s0->d_multi.ensure(2 * ge_bytes + sizeof(int) * (n_sessions + 1));
  ck(cudaMemcpy(s0->d_multi.p, ge.data(), ge_bytes, cudaMemcpyHostToDevice), "upload grids");
  if (chord) ck(cudaMemcpy(s0->d_multi.as<char>() + ge_bytes, gc.data(), ge_bytes, cudaMemcpyHostToDevice), "upload grids");
  int* d_begin = reinterpret_cast<int*>(s0->d_multi.as<char>() + 2 * ge_bytes);
  ck(cudaMemcpy(d_begin, begin.data(), sizeof(int) * (n_sessions + 1), cudaMemcpyHostToDevice), "upload grids");
  unsigned long long* phase = nullptr;
  if (o.profile_phases) {
    s0->d_phase.ensure(gs2g::N_PHASES * sizeof(unsigned long long));
    ck(cudaMemsetAsync(s0->d_phase.p, 0, gs2g::N_PHASES * sizeof(unsigned long long), s0->stream), "phase reset");
    phase = s0->d_phase.as<unsigned long long>();
  }
  ck(cudaMemsetAsync(s0->d_queue.p, 0, (4 + n_sessions) * sizeof(int), s0->stream), "queue reset");
  if (chord) ck(cudaMemsetAsync(s0->d_chord_steps.p, 0, sizeof(unsigned long long), s0->stream), "step count reset");
  ck(cudaEventRecord(s0->ev0, s0->stream), "event");
  if (chord)
    ck((cudaError_t)gs2g::launch_chord_multi(
           reinterpret_cast<const gs2g::GridEntry*>(s0->d_multi.as<char>() + ge_bytes), n_sessions, csmem, phase,
           o.precision, n_chord, s0->stream),
       "multi-grid chord sweep launch");
  if (total > 0)
    ck((cudaError_t)gs2g::launch_sweep_multi(reinterpret_cast<const gs2g::GridEntry*>(s0->d_multi.p), n_sessions,
                                             d_begin, total, s0->d_queue.as<int>(), s0->d_ws.as<char>(), wsb, phase,
                                             o.precision, n_ctas, s0->stream,
                                             chord ? s0->d_handoff.as<int>() : nullptr,
                                             chord ? s0->d_queue.as<int>() + 3 : nullptr),
       "multi-grid sweep launch");
  ck(cudaEventRecord(s0->ev1, s0->stream), "event");
  ck(cudaStreamSynchronize(s0->stream), "multi-grid sweep");
  float ms = 0;
  ck(cudaEventElapsedTime(&ms, s0->ev0, s0->ev1), "event time");
  int counts[2] = {0, 0};
  ck(cudaMemcpy(counts, s0->d_queue.as<int>() + 1, sizeof(counts), cudaMemcpyDeviceToHost), "rescue count");
  for (int i = 0; i < n_sessions; ++i) {
    gs2g_session* s = sessions[i];
    s->last_rows_run = begin[i + 1] - begin[i];
    s->mirror_valid = s->mirror_on && s->last_rows_run > 0;
    s->tm.kernel_ms = ms;
    s->tm.upload_ms = upload_ms;
    s->tm.total_ms = ms_since(t0);
    s->tm.total_iters = -1;
    s->tm.n_rescued = i == 0 ? counts[0] : 0;
    s->tm.n_base_start = i == 0 ? counts[1] : 0;
    s->tm.chord_steps = 0;
    if (i == 0 && chord) {
      unsigned long long cs = 0;
      ck(cudaMemcpy(&cs, s0->d_chord_steps.p, sizeof(cs), cudaMemcpyDeviceToHost), "step count");
      s->tm.chord_steps = (int64_t)cs;
    }
    for (int q = 0; q < GS2G_N_PHASES; ++q) s->tm.phase_cycles[q] = s->tm.phase_share[q] = 0;
  }
  if (o.profile_phases) {
    unsigned long long cyc[gs2g::N_PHASES];
    ck(cudaMemcpy(cyc, s0->d_phase.p, sizeof(cyc), cudaMemcpyDeviceToHost), "read phases");
    double tot = 0;
    for (int q = 0; q < gs2g::N_PHASES; ++q) tot += (double)cyc[q];
    for (int q = 0; q < gs2g::N_PHASES; ++q) {
      s0->tm.phase_cycles[q] = (double)cyc[q];
      s0->tm.phase_share[q] = tot > 0 ? cyc[q] / tot : 0;
    }
  }
  GS2G_CATCH
}

int gs2g_n_rows(const gs2g_session* s) { return s ? s->last_rows_run : 0; }

namespace {
// Large device-to-host copies into the caller's (pageable) memory go through
// a pinned double buffer of the session: chunk i+1 is in flight while chunk
// i is copied out on the host (by the copy pool).
void d2h_staged(const gs2g_session* s, void* dst, const void* src, size_t bytes) {
  constexpr size_t kChunk = kStageChunk;
  if (bytes < 2 * kChunk) {
    ck(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost), "read results");
    return;
  }
  ensure_stage(s);
  char* buf[2] = {static_cast<char*>(s->h_stage), static_cast<char*>(s->h_stage) + kChunk};
  const size_t nch = (bytes + kChunk - 1) / kChunk;
  auto issue = [&](size_t i) {
    const size_t off = i * kChunk, len = std::min(kChunk, bytes - off);
    ck(cudaMemcpyAsync(buf[i & 1], static_cast<const char*>(src) + off, len, cudaMemcpyDeviceToHost, s->stream),
       "read results");
    ck(cudaEventRecord(s->ev_stage[i & 1], s->stream), "event");
  };
  issue(0);
  for (size_t i = 0; i < nch; ++i) {
    if (i + 1 < nch) issue(i + 1);  // into the buffer chunk i-1 left, already copied out
    ck(cudaEventSynchronize(s->ev_stage[i & 1]), "read results");
    const size_t off = i * kChunk, len = std::min(kChunk, bytes - off);
    CopyPool::get().copy(static_cast<char*>(dst) + off, buf[i & 1], len);
  }
}
}  // namespace

int gs2g_solve_jt(gs2g_session* s, int n_rows, const double* rhs, double* lam) {
  GS2G_TRY
  if (!s || n_rows < 0 || (n_rows > 0 && (!rhs || !lam))) throw std::invalid_argument("solve_jt: bad arguments");
  if (n_rows != s->last_rows_run)
    throw std::invalid_argument("solve_jt: n_rows (" + std::to_string(n_rows) + ") must be the rows of the last run (" +
                                std::to_string(s->last_rows_run) + ")");
  if (n_rows == 0) return GS2G_OK;
  DeviceGuard g(s->device);
  assemble_rows(s);
  gs2g_run_opts o{};
  o.precision = GS2G_PREC_FP64;
  OutBufs ob{s->d_v_out.as<double>(), s->d_res.as<double>(), s->d_status.as<int>(), s->d_iters.as<int>()};
  gs2g::SweepArgs a = make_args(s, o, n_rows, s->d_vinit.as<double>(), 0, s->d_sbus.as<double>(), 0, true, ob);
  const int64_t wsb = gs2g::workspace_bytes(s->dplan, GS2G_PREC_FP64);
  const int n_ctas = std::max(1, std::min(gs2g::sweep_ctas(GS2G_PREC_FP64, s->device), n_rows));
  s->d_ws.ensure((size_t)wsb * n_ctas);
  s->d_queue.ensure(4 * sizeof(int));
  a.queue = s->d_queue.as<int>();
  a.workspace = s->d_ws.as<char>();
  a.ws_stride = wsb;
  ck(cudaMemsetAsync(s->d_queue.p, 0, sizeof(int), s->stream), "queue reset");
  ck((cudaError_t)gs2g::launch_adjoint(s->dplan, a, rhs, lam, n_ctas, s->stream), "adjoint launch");
  ck(cudaStreamSynchronize(s->stream), "adjoint");
  GS2G_CATCH
}

int gs2g_get_results_host(gs2g_session* s, double** v, double** residuals, int** status, int** iters) {
  GS2G_TRY
  if (!s || !v || !residuals || !status || !iters) throw std::invalid_argument("get_results_host: NULL argument");
  DeviceGuard g(s->device);
  const size_t nr = s->last_rows_run, n = s->n_bus;
  const size_t bv = nr * n * 2 * sizeof(double), br = nr * sizeof(double), bi = nr * sizeof(int);
  const size_t o_r = bv, o_s = o_r + br, o_i = o_s + bi;
  ensure_host_results(s, nr);
  char* h = static_cast<char*>(s->h_res);
  if (nr) {
    // with a valid mirror the kernels already wrote V here
    if (!s->mirror_valid) ck(cudaMemcpyAsync(h, s->d_v_out.p, bv, cudaMemcpyDeviceToHost, s->stream), "read results");
    ck(cudaMemcpyAsync(h + o_r, s->d_res.p, br, cudaMemcpyDeviceToHost, s->stream), "read residuals");
    ck(cudaMemcpyAsync(h + o_s, s->d_status.p, bi, cudaMemcpyDeviceToHost, s->stream), "read status");
    ck(cudaMemcpyAsync(h + o_i, s->d_iters.p, bi, cudaMemcpyDeviceToHost, s->stream), "read iters");
    ck(cudaStreamSynchronize(s->stream), "read results");
  }
  *v = reinterpret_cast<double*>(h);
  *residuals = reinterpret_cast<double*>(h + o_r);
  *status = reinterpret_cast<int*>(h + o_s);
  *iters = reinterpret_cast<int*>(h + o_i);
  GS2G_CATCH
}

int gs2g_get_results(const gs2g_session* s, double* v_out, double* residuals, int* status, int* iters) {
  GS2G_TRY
  if (!s) throw std::invalid_argument("NULL session");
  DeviceGuard g(s->device);
  const size_t nr = s->last_rows_run, n = s->n_bus;
  if (v_out && nr) d2h_staged(s, v_out, s->d_v_out.p, nr * n * 2 * sizeof(double));
  if (residuals && nr) ck(cudaMemcpy(residuals, s->d_res.p, nr * sizeof(double), cudaMemcpyDeviceToHost), "read res");
  if (status && nr) ck(cudaMemcpy(status, s->d_status.p, nr * sizeof(int), cudaMemcpyDeviceToHost), "read status");
  if (iters && nr) ck(cudaMemcpy(iters, s->d_iters.p, nr * sizeof(int), cudaMemcpyDeviceToHost), "read iters");
  GS2G_CATCH
}

int gs2g_get_factor_counts(const gs2g_session* s, int* factors) {
  GS2G_TRY
  if (!s || !factors) throw std::invalid_argument("NULL argument");
  DeviceGuard g(s->device);
  if (s->last_rows_run)
    ck(cudaMemcpy(factors, s->d_factors.p, (size_t)s->last_rows_run * sizeof(int), cudaMemcpyDeviceToHost),
       "read factor counts");
  GS2G_CATCH
}

int gs2g_set_branch_limits(gs2g_session* s, int n_branch, const double* rate_mva, double sn_mva) {
  GS2G_TRY
  if (!s) throw std::invalid_argument("NULL session");
  if (n_branch == 0) {
    s->limits_on = false;
    return GS2G_OK;
  }
  if (n_branch != s->n_branch || !rate_mva || !(sn_mva > 0))
    throw std::invalid_argument("set_branch_limits: needs one limit per branch of set_branch_data and sn_mva > 0");
  DeviceGuard g(s->device);
  std::vector<double> pu(n_branch);
  for (int l = 0; l < n_branch; ++l) pu[l] = rate_mva[l] / sn_mva;
  s->d_br_rate.ensure(n_branch * sizeof(double));
  ck(cudaMemcpy(s->d_br_rate.p, pu.data(), n_branch * sizeof(double), cudaMemcpyHostToDevice), "upload limits");
  s->limits_on = true;
  GS2G_CATCH
}

int gs2g_get_branch_loading(const gs2g_session* s, float* loading, int* n_violations, float* max_loading) {
  GS2G_TRY
  if (!s) throw std::invalid_argument("NULL session");
  if (!s->limits_on || !s->d_loading.p) throw std::runtime_error("get_branch_loading: no limits were set for the last run");
  DeviceGuard g(s->device);
  const size_t nr = s->last_rows_run;
  if (loading && nr) d2h_staged(s, loading, s->d_loading.p, nr * s->n_branch * sizeof(float));
  if (n_violations && nr)
    ck(cudaMemcpy(n_violations, s->d_nviol.p, nr * sizeof(int), cudaMemcpyDeviceToHost), "read violations");
  if (max_loading && nr)
    ck(cudaMemcpy(max_loading, s->d_maxload.p, nr * sizeof(float), cudaMemcpyDeviceToHost), "read violations");
  GS2G_CATCH
}

int gs2g_get_device_results(const gs2g_session* s, double** v, double** residuals, int** status, int** iters) {
  GS2G_TRY
  if (!s) throw std::invalid_argument("NULL session");
  if (v) *v = s->d_v_out.as<double>();
  if (residuals) *residuals = s->d_res.as<double>();
  if (status) *status = s->d_status.as<int>();
  if (iters) *iters = s->d_iters.as<int>();
  GS2G_CATCH
}

int gs2g_get_device_rows(gs2g_session* s, int* n_rows, const double** sbus_rows, const int** trip_ptr,
                         const int** trip_ids, int64_t* n_trip_ids) {
  GS2G_TRY
  if (!s) throw std::invalid_argument("NULL session");
  DeviceGuard g(s->device);
  assemble_rows(s, false);
  if (n_rows) *n_rows = s->n_rows;
  if (sbus_rows) *sbus_rows = s->rows_have_sbus ? s->d_sbus_rows.as<double>() : nullptr;
  if (trip_ptr) *trip_ptr = s->rows_have_edits ? s->d_trip_ptr.as<int>() : nullptr;
  if (trip_ids) *trip_ids = s->rows_have_edits ? s->d_trip_ids.as<int>() : nullptr;
  if (n_trip_ids) *n_trip_ids = s->rows_have_edits ? (int64_t)s->ctg_ids.size() : 0;
  GS2G_CATCH
}

int gs2g_get_timings(const gs2g_session* s, gs2g_timings* out) {
  GS2G_TRY
  if (!s || !out) throw std::invalid_argument("NULL argument");
  *out = s->tm;
  out->n_failed = 0;
  if (s->last_rows_run > 0) {
    DeviceGuard g(s->device);
    std::vector<int> it(s->last_rows_run), st(s->last_rows_run);
    ck(cudaMemcpy(it.data(), s->d_iters.p, it.size() * sizeof(int), cudaMemcpyDeviceToHost), "read iters");
    ck(cudaMemcpy(st.data(), s->d_status.p, st.size() * sizeof(int), cudaMemcpyDeviceToHost), "read statuses");
    int64_t tot = 0, failed = 0;
    for (int v : it) tot += v;
    for (int v : st) failed += v == GS2G_ROW_MAX_ITER || v == GS2G_ROW_DIVERGED;
    out->total_iters = tot;
    out->n_failed = failed;
  }
  GS2G_CATCH
}

int gs2g_sync(gs2g_session* s) {
  GS2G_TRY
  if (!s) throw std::invalid_argument("NULL session");
  DeviceGuard g(s->device);
  ck(cudaStreamSynchronize(s->stream), "sync");
  GS2G_CATCH
}

int gs2g_session_wait_stream(gs2g_session* s, void* stream) {
  GS2G_TRY
  if (!s) throw std::invalid_argument("NULL session");
  DeviceGuard g(s->device);
  if (!s->ev_ext) ck(cudaEventCreateWithFlags(&s->ev_ext, cudaEventDisableTiming), "event");
  ck(cudaEventRecord(s->ev_ext, static_cast<cudaStream_t>(stream)), "record the other stream");
  ck(cudaStreamWaitEvent(s->stream, s->ev_ext, 0), "wait for the other stream");
  GS2G_CATCH
}

int gs2g_run_rows_noalloc(const gs2g_session* s, int n_rows, const double* v0, int64_t v0_stride,
                          const double* sbus, int64_t sbus_stride, const gs2g_run_opts* o, double* v_out,
                          double* residuals, int* status, int* iters, void* stream) {
  // Allocation-free path: uses only device buffers the session set up at
  // creation (plan, Ybus) and caller memory; the kernel's scratch is the
  // library's static device array (launch_sweep_static).
  GS2G_TRY
  if (!s || !o) throw std::invalid_argument("run_rows_noalloc: NULL session or options");
  if (n_rows < 0 || v0_stride < 0 || sbus_stride < 0) throw std::invalid_argument("run_rows_noalloc: negative size");
  if (n_rows > 0 && (!v0 || !sbus || !v_out || !residuals || !status || !iters))
    throw std::invalid_argument("run_rows_noalloc: NULL input or output");
  if (o->precision != GS2G_PREC_FP64 && o->precision != GS2G_PREC_MIXED)
    throw std::invalid_argument("precision must be GS2G_PREC_FP64 or GS2G_PREC_MIXED");
  if (o->refactor_policy == GS2G_REFACTOR_BASE_CHORD)
    throw std::invalid_argument("run_rows_noalloc: GS2G_REFACTOR_BASE_CHORD is not supported on the allocation-free "
                                "path (it needs the session's base-factor buffers); use GS2G_REFACTOR_EVERY or "
                                "GS2G_REFACTOR_ADAPTIVE");
  if (o->refactor_policy != GS2G_REFACTOR_EVERY && o->refactor_policy != GS2G_REFACTOR_ADAPTIVE)
    throw std::invalid_argument("refactor_policy must be GS2G_REFACTOR_EVERY or GS2G_REFACTOR_ADAPTIVE");
  if (o->max_iter < 0) throw std::invalid_argument("max_iter must be >= 0");
  const int64_t ws = gs2g::workspace_bytes(s->dplan, o->precision);
  if (ws + 256 > gs2g::kStaticScratchBytes)
    throw std::invalid_argument("run_rows_noalloc: one row's workspace (" + std::to_string(ws) +
                                " bytes) exceeds the static scratch (" +
                                std::to_string(gs2g::kStaticScratchBytes) + " bytes); use gs2g_run");
  DeviceGuard g(s->device);
  gs2g::SweepArgs a{};
  a.n_rows = n_rows;
  a.ybus = s->d_ybus.as<double>();
  a.v0 = v0;
  a.v0_stride = v0_stride;
  a.sbus = sbus;
  a.sbus_stride = sbus_stride;
  a.max_iter = o->max_iter;
  a.tol = o->tol;
  a.fixed_iters = o->fixed_iters;
  if (o->iters_per_round > kMaxItersPerRound)
    throw std::invalid_argument("iters_per_round must be <= " + std::to_string(kMaxItersPerRound));
  a.round_k = o->iters_per_round > 0 ? o->iters_per_round : 1;
  a.step_first = o->step_then_check != 0 && !o->fixed_iters;
  a.refactor_policy = o->refactor_policy;
  a.refactor_ratio = o->refactor_ratio > 0 ? o->refactor_ratio : 0.3;
  a.max_reuse = o->max_reuse > 0 ? o->max_reuse : 3;
  a.v_out = v_out;
  a.res_out = residuals;
  a.status_out = status;
  a.iters_out = iters;
  a.pivot_floor = o->pivot_floor;
  if (o->rescue != 0 && v0_stride != 0 && !o->fixed_iters) a.rescue_v0 = s->d_vinit.as<double>();
  int used = 0;
  ck((cudaError_t)gs2g::launch_sweep_static(s->dplan, a, o->precision, s->device, stream, &used),
     "allocation-free sweep launch");
  GS2G_CATCH
}

int gs2g_acpf_nr(int device, int n_bus, const int* ybus_indptr, const int* ybus_indices, const double* ybus_values,
                 double* v_inout, const double* sbus, const int* pv, int n_pv, const int* pq, int n_pq, int max_iter,
                 double tol, int precision, int* converged, int* iters, double* residual, double* kernel_ms) {
  gs2g_session* s = nullptr;
  int rc = gs2g_session_create(device, n_bus, ybus_indptr, ybus_indices, ybus_values, v_inout, sbus, pv, n_pv, pq,
                               n_pq, 1, &s);
  if (rc) return rc;
  gs2g_run_opts o{};
  o.max_iter = max_iter;
  o.tol = tol;
  o.fixed_iters = 0;
  o.precision = precision;
  o.start = GS2G_START_VINIT;
  o.step_then_check = 1;  // the reference's single-solve order (acpf_nr.cu:505-561)
  int st = 0, it = 0;
  double res = 0;
  rc = gs2g_solve_base(s, &o, v_inout, &st, &it, &res);
  if (rc == 0) {
    if (converged) *converged = st == GS2G_ROW_CONVERGED ? 1 : 0;
    if (iters) *iters = it;
    if (residual) *residual = res;
    if (kernel_ms) *kernel_ms = s->tm.kernel_ms;
  }
  std::string keep = g_err;
  gs2g_session_destroy(s);
  if (rc) g_err = keep;
  return rc;
}

}  // extern "C"
