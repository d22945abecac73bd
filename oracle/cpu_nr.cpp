// CPU FP64 Newton-Raphson AC power flow over a batch of rows, OpenMP over rows.
//
// TEST INFRASTRUCTURE ONLY: the compiled CPU baseline of bench.py (the
// cpu_baseline leg and the --impl reference arm) and a fast FP64 checker for
// the tests.  The product path never links or calls it.
//
// It restates, in C++, the same algorithm as oracle/nr_oracle.py -- the
// reference's bare [pvpq | pq] Newton-Raphson with its CPU oracle's linear
// algebra (lightsim2grid's KLU: a fill-reducing ordering, one symbolic
// analysis, a static-pivot numeric refactorization every step):
//   * J layout: P/theta on sorted(pv u pq) at [0, n_pvpq), Q/Vm on pq in input
//     order at [n_pvpq, dim)            (reference src/_cpp/acpf_nr.cu:145-236)
//   * mismatch F = -[Re, Im](V conj(Y V) - Sbus), NaN-sticky inf-norm
//                                        (src/_cpp/acpf_nr_kernels.cu:493-557)
//   * Jacobian dS/dVa, dS/dVm (MATPOWER) (src/_cpp/acpf_nr_kernels.cu:559-650)
//   * Va update on pvpq, then Vm on pq, polar (src/_cpp/acpf_nr_kernels.cu:728-790)
//   * continuous schedule with one step per round: after each step the
//     residual decides DIVERGED / CONVERGED / MAX_ITER
//                                        (src/_cpp/contingency/batch_pf_driver.cu:2691-2724)
//   * branch trips subtract yff@(f,f), ytt@(t,t), yft@(f,t), ytf@(t,f), an
//     open (negative) end skipping its terms; a branch named twice trips once
//                                        (src/_cpp/contingency_analysis_helper.cpp:23-84)
//   * a row whose trips disconnect the branch graph is NOT_SIMULATED with NaN
//     voltages                           (src/_cpp/contingency_analysis_helper.cpp:634-651)
//
// Linear algebra (its own design, not the engine's): a minimum-degree
// ordering of the bus graph (each bus's theta and Vm unknowns eliminated as a
// pair), stopped once the remaining graph is dense; the eliminated buses form
// a sparse head factored by precomputed scatter programs, the rest a dense
// tail factored by a blocked right-looking LU.  No pivoting, as the
// reference's own LU and KLU's refactorization on a fixed pivot sequence.
//
// C entry point: cpunr_sweep (see the end of this file).

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include <immintrin.h>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using cplx = std::complex<double>;
constexpr int CONVERGED = 0, MAX_ITER = 1, DIVERGED = 2, NOT_SIMULATED = 3;

// ------------------------------------------------------------------ grid
struct Plan {
  int n = 0, dim = 0, n_pvpq = 0;
  std::vector<int> yp, yi;      // Ybus CSR (sorted columns)
  std::vector<int> yrow;        // row of every entry
  std::vector<int> rowP, rowQ;  // bus -> F row of its P / Q equation, -1: none
  std::vector<int> pos;         // unknown (F row / J column index) -> pivot position
  int p = 0, T = 0;             // head positions [0, p), dense tail [p, dim)
  std::vector<int> adj_ptr, adj;       // head pivot k: later positions coupled to k (sorted)
  std::vector<int64_t> ustart, lstart; // value offsets of U row k / L column k
  int64_t nh = 0;                      // head values (diagonal, U rows, L columns)
  std::vector<int64_t> prog_ptr;       // per head pivot: scatter targets of its update
  std::vector<int64_t> prog;
  std::vector<int64_t> jdst;           // [4 * nnz_y]: J value of (entry, quadrant) -> value index, -1 unused
  double plan_ms = 0;

  int64_t val_index(int r, int c) const {
    if (r >= p && c >= p) return nh + (int64_t)(r - p) * T + (c - p);
    if (r == c) return r;
    const bool upper = r < c;
    const int k = upper ? r : c, o = upper ? c : r;
    const int* b = adj.data() + adj_ptr[k];
    const int* e = adj.data() + adj_ptr[k + 1];
    const int* it = std::lower_bound(b, e, o);
    if (it == e || *it != o) throw std::logic_error("position outside the filled pattern");
    return (upper ? ustart[k] : lstart[k]) + (it - b);
  }
};

// Minimum-degree elimination of the bus graph (explicit fill), stopped when
// the smallest degree reaches `dense_frac` of the buses left: those buses
// become the dense tail.  Returns the bus order and, for every eliminated
// bus, its neighbours at elimination (all later in the order).
void min_degree(int n, const std::vector<std::vector<int>>& g0, const std::vector<uint8_t>& has_unknowns,
                double dense_frac, std::vector<int>& order, std::vector<std::vector<int>>& elim_adj, int& n_head) {
  std::vector<std::vector<int>> g = g0;
  std::vector<uint8_t> gone(n, 0);
  std::set<std::pair<int, int>> pq;
  for (int v = 0; v < n; ++v) pq.insert({(int)g[v].size(), v});
  order.clear();
  elim_adj.assign(n, {});
  int left = n;
  while (!pq.empty()) {
    const auto [deg, v] = *pq.begin();
    if (deg >= dense_frac * left && left > 1) break;
    pq.erase(pq.begin());
    gone[v] = 1;
    order.push_back(v);
    elim_adj[v] = g[v];
    --left;
    const std::vector<int>& nb = g[v];
    for (int u : nb) {
      pq.erase({(int)g[u].size(), u});
      std::vector<int> merged;
      merged.reserve(g[u].size() + nb.size());
      std::set_union(g[u].begin(), g[u].end(), nb.begin(), nb.end(), std::back_inserter(merged));
      merged.erase(std::remove_if(merged.begin(), merged.end(), [&](int w) { return w == u || w == v; }),
                   merged.end());
      g[u].swap(merged);
      pq.insert({(int)g[u].size(), u});
    }
    g[v].clear();
  }
  n_head = (int)order.size();
  // the dense tail: the remaining buses, those with unknowns in their input order
  for (int v = 0; v < n; ++v)
    if (!gone[v]) order.push_back(v);
  (void)has_unknowns;
}

Plan build_plan(int n, const int* yp, const int* yi, const int* pv, int npv, const int* pq, int npq,
                double dense_frac) {
  const auto t0 = std::chrono::steady_clock::now();
  Plan P;
  P.n = n;
  P.yp.assign(yp, yp + n + 1);
  P.yi.assign(yi, yi + yp[n]);
  for (int i = 0; i < n; ++i)
    if (!std::is_sorted(P.yi.begin() + P.yp[i], P.yi.begin() + P.yp[i + 1]))
      std::sort(P.yi.begin() + P.yp[i], P.yi.begin() + P.yp[i + 1]);
  P.yrow.resize(P.yi.size());
  for (int i = 0; i < n; ++i)
    for (int k = P.yp[i]; k < P.yp[i + 1]; ++k) P.yrow[k] = i;
  // J layout
  std::vector<int> pvpq(pv, pv + npv);
  pvpq.insert(pvpq.end(), pq, pq + npq);
  std::sort(pvpq.begin(), pvpq.end());
  P.n_pvpq = (int)pvpq.size();
  P.dim = P.n_pvpq + npq;
  P.rowP.assign(n, -1);
  P.rowQ.assign(n, -1);
  for (int a = 0; a < P.n_pvpq; ++a) P.rowP[pvpq[a]] = a;
  for (int a = 0; a < npq; ++a) P.rowQ[pq[a]] = P.n_pvpq + a;
  // bus graph of the Ybus pattern, buses with unknowns only
  std::vector<uint8_t> hu(n, 0);
  for (int i = 0; i < n; ++i) hu[i] = P.rowP[i] >= 0 || P.rowQ[i] >= 0;
  std::vector<std::vector<int>> g(n);
  for (int i = 0; i < n; ++i) {
    if (!hu[i]) continue;
    for (int k = P.yp[i]; k < P.yp[i + 1]; ++k) {
      const int j = P.yi[k];
      if (j != i && hu[j]) g[i].push_back(j);
    }
    std::sort(g[i].begin(), g[i].end());
    g[i].erase(std::unique(g[i].begin(), g[i].end()), g[i].end());
  }
  std::vector<int> border;
  std::vector<std::vector<int>> eadj;
  int n_head_bus = 0;
  // buses without unknowns (the slack) take no part: give them an empty graph
  min_degree(n, g, hu, dense_frac, border, eadj, n_head_bus);
  // positions: theta then Vm of every bus in order
  P.pos.assign(P.dim, -1);
  std::vector<int> bus_first(n, -1);
  int q = 0;
  for (int idx = 0; idx < n; ++idx) {
    const int v = border[idx];
    if (idx == n_head_bus) P.p = q;
    if (!hu[v]) continue;
    bus_first[v] = q;
    if (P.rowP[v] >= 0) P.pos[P.rowP[v]] = q++;
    if (P.rowQ[v] >= 0) P.pos[P.rowQ[v]] = q++;
  }
  if (n_head_bus >= n) P.p = q;
  P.T = P.dim - P.p;
  auto unknowns = [&](int v, std::vector<int>& out) {
    if (P.rowP[v] >= 0) out.push_back(P.pos[P.rowP[v]]);
    if (P.rowQ[v] >= 0) out.push_back(P.pos[P.rowQ[v]]);
  };
  // filled adjacency of every head position (later positions only)
  P.adj_ptr.assign(P.p + 1, 0);
  std::vector<std::vector<int>> adjv(P.p);
  for (int idx = 0; idx < n_head_bus; ++idx) {
    const int v = border[idx];
    if (!hu[v]) continue;
    std::vector<int> later;
    for (int u : eadj[v]) unknowns(u, later);
    std::sort(later.begin(), later.end());
    const int f0 = bus_first[v];
    const bool two = P.rowP[v] >= 0 && P.rowQ[v] >= 0;
    adjv[f0] = later;
    if (two) {
      adjv[f0].insert(adjv[f0].begin(), f0 + 1);
      adjv[f0 + 1] = later;
    }
  }
  for (int k = 0; k < P.p; ++k) P.adj_ptr[k + 1] = P.adj_ptr[k] + (int)adjv[k].size();
  P.adj.resize(P.adj_ptr[P.p]);
  for (int k = 0; k < P.p; ++k) std::copy(adjv[k].begin(), adjv[k].end(), P.adj.begin() + P.adj_ptr[k]);
  P.ustart.resize(P.p);
  P.lstart.resize(P.p);
  int64_t o = P.p;
  for (int k = 0; k < P.p; ++k) {
    P.ustart[k] = o;
    o += adjv[k].size();
  }
  for (int k = 0; k < P.p; ++k) {
    P.lstart[k] = o;
    o += adjv[k].size();
  }
  P.nh = o;
  // update programs: pivot k subtracts L(i,k) U(k,j) from (i, j) for i, j in adj(k)
  P.prog_ptr.assign(P.p + 1, 0);
  for (int k = 0; k < P.p; ++k) {
    const int64_t m = adjv[k].size();
    P.prog_ptr[k + 1] = P.prog_ptr[k] + m * m;
  }
  P.prog.resize(P.prog_ptr[P.p]);
  for (int k = 0; k < P.p; ++k) {
    const auto& a = adjv[k];
    const int64_t m = a.size();
    int64_t* d = P.prog.data() + P.prog_ptr[k];
    for (int64_t x = 0; x < m; ++x)
      for (int64_t y = 0; y < m; ++y) d[x * m + y] = P.val_index(a[x], a[y]);
  }
  // J values of every (Ybus entry, quadrant): q = 0 dP/dtheta, 1 dP/dVm, 2 dQ/dtheta, 3 dQ/dVm
  P.jdst.assign(4 * P.yi.size(), -1);
  for (size_t k = 0; k < P.yi.size(); ++k) {
    const int i = P.yrow[k], j = P.yi[k];
    const int rows[2] = {P.rowP[i], P.rowQ[i]};
    const int cols[2] = {P.rowP[j], P.rowQ[j]};
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        if (rows[a] >= 0 && cols[b] >= 0) P.jdst[4 * k + 2 * a + b] = P.val_index(P.pos[rows[a]], P.pos[cols[b]]);
  }
  P.plan_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return P;
}

// ------------------------------------------------------------------ dense tail
// C[m x n] -= A[m x kb] B[kb x n], all row-major with leading dimension ld:
// 6 x 8 register blocks on AVX2 FMA (12 accumulators, two vectors of B and a
// broadcast of A per k), scalar edges.
void gemm_sub(const double* A, const double* B, double* C, int m, int n, int kb, int ld) {
  int i = 0;
  for (; i + 6 <= m; i += 6) {
    const double* a[6];
    for (int r = 0; r < 6; ++r) a[r] = A + (int64_t)(i + r) * ld;
    int j = 0;
    for (; j + 8 <= n; j += 8) {
      double* c[6];
      __m256d acc[6][2];
      for (int r = 0; r < 6; ++r) {
        c[r] = C + (int64_t)(i + r) * ld + j;
        acc[r][0] = _mm256_loadu_pd(c[r]);
        acc[r][1] = _mm256_loadu_pd(c[r] + 4);
      }
      const double* bk = B + j;
      for (int k = 0; k < kb; ++k, bk += ld) {
        const __m256d b0 = _mm256_loadu_pd(bk), b1 = _mm256_loadu_pd(bk + 4);
        for (int r = 0; r < 6; ++r) {
          const __m256d av = _mm256_broadcast_sd(a[r] + k);
          acc[r][0] = _mm256_fnmadd_pd(av, b0, acc[r][0]);
          acc[r][1] = _mm256_fnmadd_pd(av, b1, acc[r][1]);
        }
      }
      for (int r = 0; r < 6; ++r) {
        _mm256_storeu_pd(c[r], acc[r][0]);
        _mm256_storeu_pd(c[r] + 4, acc[r][1]);
      }
    }
    for (; j < n; ++j)
      for (int r = 0; r < 6; ++r) {
        double sacc = C[(int64_t)(i + r) * ld + j];
        for (int k = 0; k < kb; ++k) sacc -= a[r][k] * B[(int64_t)k * ld + j];
        C[(int64_t)(i + r) * ld + j] = sacc;
      }
  }
  for (; i < m; ++i)
    for (int k = 0; k < kb; ++k) {
      const double av = A[(int64_t)i * ld + k];
      const double* b = B + (int64_t)k * ld;
      double* c = C + (int64_t)i * ld;
      for (int j = 0; j < n; ++j) c[j] -= av * b[j];
    }
}

// In-place LU (unit L, no pivoting) of the n x n row-major matrix S.
void dense_lu(double* S, int n) {
  constexpr int NB = 32;  // measured: 32 beats 16-96 on n = 500-1200 (the panel is the slow part)
  const int ld = n;
  for (int k0 = 0; k0 < n; k0 += NB) {
    const int k1 = std::min(n, k0 + NB);
    // panel: columns [k0, k1), every row below the diagonal
    for (int k = k0; k < k1; ++k) {
      const double piv = S[(int64_t)k * ld + k];
      const double* uk = S + (int64_t)k * ld;
      for (int i = k + 1; i < n; ++i) {
        double* ri = S + (int64_t)i * ld;
        const double l = ri[k] / piv;
        ri[k] = l;
        for (int j = k + 1; j < k1; ++j) ri[j] -= l * uk[j];
      }
    }
    if (k1 >= n) break;
    // U12 = L11^-1 A12
    for (int k = k0; k < k1; ++k) {
      const double* uk = S + (int64_t)k * ld;
      for (int i = k + 1; i < k1; ++i) {
        double* ri = S + (int64_t)i * ld;
        const double l = ri[k];
        for (int j = k1; j < n; ++j) ri[j] -= l * uk[j];
      }
    }
    // A22 -= L21 U12
    gemm_sub(S + (int64_t)k1 * ld + k0, S + (int64_t)k0 * ld + k1, S + (int64_t)k1 * ld + k1, n - k1, n - k1,
             k1 - k0, ld);
  }
}

// ------------------------------------------------------------------ one row
struct Work {
  std::vector<cplx> Y, V, I;
  std::vector<double> vals, F, y;
};

double mismatch(const Plan& P, const cplx* Y, const cplx* V, cplx* I, const cplx* S, double* F) {
  double nrm = 0.0;
  bool nan = false;
  for (int i = 0; i < P.n; ++i) {
    cplx acc(0.0, 0.0);
    for (int k = P.yp[i]; k < P.yp[i + 1]; ++k) acc += Y[k] * V[P.yi[k]];
    I[i] = acc;
    const cplx s = V[i] * std::conj(acc) - S[i];
    if (P.rowP[i] >= 0) {
      F[P.rowP[i]] = -s.real();
      nan |= std::isnan(s.real());
      nrm = std::max(nrm, std::fabs(s.real()));
    }
    if (P.rowQ[i] >= 0) {
      F[P.rowQ[i]] = -s.imag();
      nan |= std::isnan(s.imag());
      nrm = std::max(nrm, std::fabs(s.imag()));
    }
  }
  return nan ? NAN : nrm;
}

// One Newton step: J(V) factored, dx = J^-1 F, polar update of V.
void newton_step(const Plan& P, Work& w) {
  const cplx* Y = w.Y.data();
  cplx* V = w.V.data();
  const cplx* I = w.I.data();
  double* vals = w.vals.data();
  std::fill(w.vals.begin(), w.vals.end(), 0.0);
  for (size_t k = 0; k < P.yi.size(); ++k) {
    const int i = P.yrow[k], j = P.yi[k];
    const int64_t* d = P.jdst.data() + 4 * k;
    if (d[0] < 0 && d[1] < 0 && d[2] < 0 && d[3] < 0) continue;
    const cplx vn = V[j] / std::abs(V[j]);
    cplx dva, dvm;
    if (i == j) {
      dva = cplx(0, 1) * V[i] * std::conj(I[i] - Y[k] * V[i]);
      dvm = V[i] * std::conj(Y[k] * vn) + std::conj(I[i]) * vn;
    } else {
      dva = -cplx(0, 1) * V[i] * std::conj(Y[k] * V[j]);
      dvm = V[i] * std::conj(Y[k] * vn);
    }
    const double v4[4] = {dva.real(), dvm.real(), dva.imag(), dvm.imag()};
    for (int q = 0; q < 4; ++q)
      if (d[q] >= 0) vals[d[q]] += v4[q];
  }
  // sparse head
  for (int k = 0; k < P.p; ++k) {
    const double piv = vals[k];
    const int64_t m = P.adj_ptr[k + 1] - P.adj_ptr[k];
    double* L = vals + P.lstart[k];
    const double* U = vals + P.ustart[k];
    for (int64_t a = 0; a < m; ++a) L[a] /= piv;
    const int64_t* d = P.prog.data() + P.prog_ptr[k];
    for (int64_t a = 0; a < m; ++a) {
      const double la = L[a];
      const int64_t* da = d + a * m;
      for (int64_t b = 0; b < m; ++b) vals[da[b]] -= la * U[b];
    }
  }
  double* S = vals + P.nh;
  if (P.T > 0) dense_lu(S, P.T);
  // solves
  double* y = w.y.data();
  for (int u = 0; u < P.dim; ++u) y[P.pos[u]] = w.F[u];
  for (int k = 0; k < P.p; ++k) {
    const double yk = y[k];
    const double* L = vals + P.lstart[k];
    for (int a = P.adj_ptr[k]; a < P.adj_ptr[k + 1]; ++a) y[P.adj[a]] -= L[a - P.adj_ptr[k]] * yk;
  }
  double* yt = y + P.p;
  for (int i = 0; i < P.T; ++i) {
    double s = yt[i];
    const double* r = S + (int64_t)i * P.T;
    for (int j = 0; j < i; ++j) s -= r[j] * yt[j];
    yt[i] = s;
  }
  for (int i = P.T - 1; i >= 0; --i) {
    double s = yt[i];
    const double* r = S + (int64_t)i * P.T;
    for (int j = i + 1; j < P.T; ++j) s -= r[j] * yt[j];
    yt[i] = s / r[i];
  }
  for (int k = P.p - 1; k >= 0; --k) {
    double s = y[k];
    const double* U = vals + P.ustart[k];
    for (int a = P.adj_ptr[k]; a < P.adj_ptr[k + 1]; ++a) s -= U[a - P.adj_ptr[k]] * y[P.adj[a]];
    y[k] = s / vals[k];
  }
  // Va on pvpq, then Vm on pq
  for (int i = 0; i < P.n; ++i) {
    const int fp = P.rowP[i], fq = P.rowQ[i];
    if (fp < 0 && fq < 0) continue;
    const double vm = std::abs(V[i]) + (fq >= 0 ? y[P.pos[fq]] : 0.0);
    const double va = std::arg(V[i]) + (fp >= 0 ? y[P.pos[fp]] : 0.0);
    V[i] = std::polar(vm, va);
  }
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

}  // namespace

extern "C" {

// Solve n_rows rows of one grid.  Complex arrays are interleaved (re, im)
// doubles.  Row r trips branches trip_ids[trip_ptr[r] .. trip_ptr[r+1])
// (trip_ptr NULL: no trips) and takes the injections sbus + 2 * r *
// sbus_stride (stride 0: the same for every row).  Every row starts from v0.
// Outputs per row: v_out [n_rows x n_bus], status, iters, residual.
// n_threads <= 0: all OpenMP threads.  Returns 0, or -1 on a bad argument
// (message in err, err_len bytes).
int cpunr_sweep(int n_bus, const int* yp, const int* yi, const double* yv, const double* v0, const double* sbus,
                int64_t sbus_stride, const int* pv, int npv, const int* pq, int npq, int n_branch, const int* bf,
                const int* bt, const double* yff, const double* yft, const double* ytf, const double* ytt,
                int n_rows, const int* trip_ptr, const int* trip_ids, int max_iter, double tol, int n_threads,
                double dense_frac, double* v_out, int* status, int* iters, double* residual, double* plan_ms,
                char* err, int err_len) {
  try {
    if (n_bus <= 0 || n_rows < 0 || !yp || !yi || !yv || !v0 || !sbus) throw std::invalid_argument("bad arguments");
    const Plan P = build_plan(n_bus, yp, yi, pv, npv, pq, npq, dense_frac > 0 ? dense_frac : 0.4);
    if (plan_ms) *plan_ms = P.plan_ms;
    // Ybus values in the plan's (sorted) entry order
    std::vector<cplx> Y0(P.yi.size());
    for (int i = 0; i < n_bus; ++i) {
      for (int k = yp[i]; k < yp[i + 1]; ++k) {
        const int* b = P.yi.data() + P.yp[i];
        const int* e = P.yi.data() + P.yp[i + 1];
        const int64_t kk = std::lower_bound(b, e, yi[k]) - P.yi.data();
        Y0[kk] += cplx(yv[2 * k], yv[2 * k + 1]);
      }
    }
    auto find = [&](int i, int j) -> int64_t {
      const int* b = P.yi.data() + P.yp[i];
      const int* e = P.yi.data() + P.yp[i + 1];
      const int* it = std::lower_bound(b, e, j);
      if (it == e || *it != j) throw std::invalid_argument("branch term outside the Ybus pattern");
      return it - P.yi.data();
    };
    if (trip_ptr)
      for (int q = 0; q < trip_ptr[n_rows]; ++q)
        if (trip_ids[q] < 0 || trip_ids[q] >= n_branch) throw std::invalid_argument("branch id out of range");
    // Ybus entries of every branch term (-1: an open end's term), found
    // before the parallel region so that nothing throws inside it
    std::vector<int64_t> kbr(4 * (size_t)std::max(n_branch, 0), -1);
    for (int l = 0; l < n_branch; ++l) {
      const int f = bf[l], t = bt[l];
      if (f >= n_bus || t >= n_bus) throw std::invalid_argument("branch endpoint out of range");
      if (f >= 0) kbr[4 * l] = find(f, f);
      if (t >= 0) kbr[4 * l + 1] = find(t, t);
      if (f >= 0 && t >= 0) {
        kbr[4 * l + 2] = find(f, t);
        kbr[4 * l + 3] = find(t, f);
      }
    }
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
#pragma omp parallel
    {
      Work w;
      w.Y.resize(Y0.size());
      w.V.resize(n_bus);
      w.I.resize(n_bus);
      w.vals.resize(P.nh + (int64_t)P.T * P.T);
      w.F.resize(P.dim);
      w.y.resize(P.dim);
#pragma omp for schedule(dynamic, 1)
      for (int r = 0; r < n_rows; ++r) {
        double* vo = v_out + 2 * (int64_t)r * n_bus;
        std::copy(Y0.begin(), Y0.end(), w.Y.begin());
        bool island = false;
        if (trip_ptr && trip_ptr[r + 1] > trip_ptr[r]) {
          std::vector<int> ids(trip_ids + trip_ptr[r], trip_ids + trip_ptr[r + 1]);
          std::sort(ids.begin(), ids.end());
          ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
          DSU d(n_bus);
          int comps = n_bus;
          size_t ui = 0;
          for (int l = 0; l < n_branch; ++l) {
            while (ui < ids.size() && ids[ui] < l) ++ui;
            if (ui < ids.size() && ids[ui] == l) continue;
            if (bf[l] < 0 || bt[l] < 0) continue;
            if (d.u(bf[l], bt[l])) --comps;
          }
          island = comps > 1;
          if (!island)
            for (int l : ids) {
              const double* yb[4] = {yff, ytt, yft, ytf};
              for (int q = 0; q < 4; ++q)
                if (kbr[4 * l + q] >= 0) w.Y[kbr[4 * l + q]] -= cplx(yb[q][2 * l], yb[q][2 * l + 1]);
            }
        }
        if (island) {
          for (int i = 0; i < 2 * n_bus; ++i) vo[i] = NAN;
          status[r] = NOT_SIMULATED;
          iters[r] = 0;
          residual[r] = NAN;
          continue;
        }
        const cplx* S = reinterpret_cast<const cplx*>(sbus) + (int64_t)r * sbus_stride;
        const cplx* V0 = reinterpret_cast<const cplx*>(v0);
        std::copy(V0, V0 + n_bus, w.V.begin());
        int it = 0, st = MAX_ITER;
        double nrm = NAN;
        for (;;) {
          nrm = mismatch(P, w.Y.data(), w.V.data(), w.I.data(), S, w.F.data());
          if (it > 0) {
            if (!std::isfinite(nrm)) { st = DIVERGED; break; }
            if (nrm < tol) { st = CONVERGED; break; }
            if (it >= max_iter) { st = MAX_ITER; break; }
          }
          newton_step(P, w);
          ++it;
        }
        std::memcpy(vo, w.V.data(), sizeof(cplx) * n_bus);
        status[r] = st;
        iters[r] = it;
        residual[r] = nrm;
      }
    }
    return 0;
  } catch (const std::exception& e) {
    if (err && err_len > 0) {
      std::strncpy(err, e.what(), err_len - 1);
      err[err_len - 1] = 0;
    }
    return -1;
  }
}

// Symbolic statistics of the plan cpunr_sweep would use: head pivots, dense
// tail size, head values and scatter-program length.
int cpunr_plan_info(int n_bus, const int* yp, const int* yi, const int* pv, int npv, const int* pq, int npq,
                    double dense_frac, int64_t* out4) {
  try {
    const Plan P = build_plan(n_bus, yp, yi, pv, npv, pq, npq, dense_frac > 0 ? dense_frac : 0.4);
    out4[0] = P.p;
    out4[1] = P.T;
    out4[2] = P.nh;
    out4[3] = (int64_t)P.prog.size();
    return 0;
  } catch (...) {
    return -1;
  }
}

}  // extern "C"
