// Symbolic plan of the batched Newton–Raphson power flow (see plan.hpp).
#include "plan.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <limits>
#include <numeric>
#include <stdexcept>

namespace gs2g {

namespace {

struct Bits {
  int n = 0, words = 0;
  std::vector<uint64_t> w;
  Bits() = default;
  Bits(int n_, int rows) : n(n_), words((n_ + 63) / 64), w(size_t(rows) * ((n_ + 63) / 64), 0) {}
  uint64_t* row(int r) { return w.data() + size_t(r) * words; }
  const uint64_t* row(int r) const { return w.data() + size_t(r) * words; }
};

inline void set_bit(uint64_t* r, int i) { r[i >> 6] |= (uint64_t(1) << (i & 63)); }
inline void clr_bit(uint64_t* r, int i) { r[i >> 6] &= ~(uint64_t(1) << (i & 63)); }
inline bool get_bit(const uint64_t* r, int i) { return (r[i >> 6] >> (i & 63)) & 1; }

// Elimination structure of a symmetric pattern in a given order, at bus level.
// order[k] = bus eliminated k-th; adj = bus adjacency (no self loops).
// Returns struct_[k] = sorted elimination indices j > k adjacent to k in the
// filled graph, and parent[k] (-1 for roots).
void bus_symbolic(int nb, const std::vector<int>& order, const std::vector<std::vector<int>>& adj,
                  std::vector<std::vector<int>>& st, std::vector<int>& parent) {
  std::vector<int> pos(nb);
  for (int k = 0; k < nb; ++k) pos[order[k]] = k;
  Bits B(nb, nb);
  for (int k = 0; k < nb; ++k) {
    uint64_t* r = B.row(k);
    for (int u : adj[order[k]]) {
      int j = pos[u];
      if (j > k) set_bit(r, j);
    }
  }
  st.assign(nb, {});
  parent.assign(nb, -1);
  for (int k = 0; k < nb; ++k) {
    uint64_t* r = B.row(k);
    // bits <= k are never set (only later indices are ever merged in)
    std::vector<int>& s = st[k];
    for (int wd = 0; wd < B.words; ++wd) {
      uint64_t x = r[wd];
      while (x) {
        int b = __builtin_ctzll(x);
        s.push_back(wd * 64 + b);
        x &= x - 1;
      }
    }
    if (!s.empty()) {
      int pa = s[0];
      parent[k] = pa;
      uint64_t* rp = B.row(pa);
      for (int wd = 0; wd < B.words; ++wd) rp[wd] |= r[wd];
      clr_bit(rp, pa);
    }
  }
}

}  // namespace

std::vector<int> min_degree_order(int n, const std::vector<std::vector<int>>& adj,
                                  const std::vector<int>& weight) {
  // Minimum (weighted external) degree on the explicit elimination graph held
  // as bitsets.  Ties go to the lowest index so the order is deterministic.
  // Once the remaining graph is a clique the rest is appended in index order.
  Bits B(n, n);
  std::vector<uint64_t> wmask(B.words, 0), alive(B.words, 0);
  for (int i = 0; i < n; ++i) {
    if (weight[i] == 2) set_bit(wmask.data(), i);
    set_bit(alive.data(), i);
    for (int u : adj[i])
      if (u != i) set_bit(B.row(i), u);
  }
  auto wdeg = [&](int i) {
    const uint64_t* r = B.row(i);
    int d = 0;
    for (int wd = 0; wd < B.words; ++wd) d += __builtin_popcountll(r[wd]) + __builtin_popcountll(r[wd] & wmask[wd]);
    return d;
  };
  std::vector<int> deg(n);
  for (int i = 0; i < n; ++i) deg[i] = wdeg(i);
  std::vector<char> done(n, 0);
  std::vector<int> order;
  order.reserve(n);
  int remaining = n;
  int remaining_w = 0;
  for (int i = 0; i < n; ++i) remaining_w += weight[i];
  while (remaining > 0) {
    int v = -1, bd = std::numeric_limits<int>::max();
    for (int i = 0; i < n; ++i)
      if (!done[i] && deg[i] < bd) { bd = deg[i]; v = i; }
    // clique check: the minimum-degree vertex is adjacent to every other
    // remaining vertex, and (since it has the minimum degree) so is everyone.
    if (bd == remaining_w - weight[v]) {
      bool clique = true;
      for (int i = 0; i < n && clique; ++i)
        if (!done[i] && deg[i] != remaining_w - weight[i]) clique = false;
      if (clique) {
        for (int i = 0; i < n; ++i)
          if (!done[i]) order.push_back(i);
        break;
      }
    }
    order.push_back(v);
    done[v] = 1;
    --remaining;
    remaining_w -= weight[v];
    clr_bit(alive.data(), v);
    uint64_t* rv = B.row(v);
    std::vector<int> nbrs;
    for (int wd = 0; wd < B.words; ++wd) {
      uint64_t x = rv[wd];
      while (x) {
        nbrs.push_back(wd * 64 + __builtin_ctzll(x));
        x &= x - 1;
      }
    }
    for (int u : nbrs) {
      uint64_t* ru = B.row(u);
      for (int wd = 0; wd < B.words; ++wd) ru[wd] |= rv[wd];
      clr_bit(ru, u);
      clr_bit(ru, v);
      deg[u] = wdeg(u);
    }
  }
  return order;
}

Plan build_plan(int n_bus, const int* ybus_indptr, const int* ybus_indices,
                const int* pv_in, int n_pv, const int* pq_in, int n_pq,
                const TailOptions& opt) {
  auto t0 = std::chrono::steady_clock::now();
  Plan P;
  if (n_bus <= 0) throw std::invalid_argument("build_plan: n_bus must be positive");
  P.n_bus = n_bus;
  P.nnz_y = ybus_indptr[n_bus];
  if (ybus_indptr[0] != 0 || P.nnz_y < 0) throw std::invalid_argument("build_plan: bad Ybus indptr");
  P.y_indptr.assign(ybus_indptr, ybus_indptr + n_bus + 1);
  P.y_indices.assign(ybus_indices, ybus_indices + P.nnz_y);
  P.y_row.resize(P.nnz_y);
  P.y_diag.assign(n_bus, -1);
  for (int i = 0; i < n_bus; ++i) {
    if (P.y_indptr[i + 1] < P.y_indptr[i]) throw std::invalid_argument("build_plan: Ybus indptr not monotone");
    for (int k = P.y_indptr[i]; k < P.y_indptr[i + 1]; ++k) {
      int j = P.y_indices[k];
      if (j < 0 || j >= n_bus) throw std::invalid_argument("build_plan: Ybus column index out of range");
      if (k > P.y_indptr[i] && P.y_indices[k - 1] >= j)
        throw std::invalid_argument("build_plan: Ybus columns must be sorted and unique per row");
      P.y_row[k] = i;
      if (j == i) P.y_diag[i] = k;
    }
  }

  // ---- J layout --------------------------------------------------------
  std::vector<int> kind(n_bus, 0);  // 0 slack/unused, 1 pv, 2 pq
  for (int i = 0; i < n_pv; ++i) {
    int b = pv_in[i];
    if (b < 0 || b >= n_bus) throw std::invalid_argument("build_plan: pv index out of range");
    if (kind[b]) throw std::invalid_argument("build_plan: bus listed twice in pv/pq");
    kind[b] = 1;
  }
  P.pq.resize(n_pq);
  for (int i = 0; i < n_pq; ++i) {
    int b = pq_in[i];
    if (b < 0 || b >= n_bus) throw std::invalid_argument("build_plan: pq index out of range");
    if (kind[b]) throw std::invalid_argument("build_plan: bus listed twice in pv/pq");
    kind[b] = 2;
    P.pq[i] = b;
  }
  for (int b = 0; b < n_bus; ++b)
    if (kind[b]) P.pvpq.push_back(b);
  P.n_pvpq = (int)P.pvpq.size();
  P.n_pq = n_pq;
  P.dim = P.n_pvpq + P.n_pq;
  if (P.dim == 0) throw std::invalid_argument("build_plan: no pv/pq bus");
  std::vector<int> jP(n_bus, -1), jQ(n_bus, -1);
  for (int i = 0; i < P.n_pvpq; ++i) jP[P.pvpq[i]] = i;
  for (int i = 0; i < n_pq; ++i) jQ[P.pq[i]] = P.n_pvpq + i;

  // ---- bus graph over the pv/pq buses ------------------------------------
  const int nb = P.n_pvpq;
  std::vector<int> node_of_bus(n_bus, -1);
  for (int i = 0; i < nb; ++i) node_of_bus[P.pvpq[i]] = i;
  std::vector<std::vector<int>> adj(nb);
  std::vector<int> wt(nb);
  for (int i = 0; i < nb; ++i) {
    int b = P.pvpq[i];
    wt[i] = kind[b] == 2 ? 2 : 1;
    for (int k = P.y_indptr[b]; k < P.y_indptr[b + 1]; ++k) {
      int c = P.y_indices[k];
      if (c != b && node_of_bus[c] >= 0) adj[i].push_back(node_of_bus[c]);
    }
  }
  // symmetrize (the pattern of a Ybus is symmetric; be safe)
  {
    std::vector<std::vector<int>> sym(nb);
    for (int i = 0; i < nb; ++i)
      for (int u : adj[i]) { sym[i].push_back(u); sym[u].push_back(i); }
    for (int i = 0; i < nb; ++i) {
      std::sort(sym[i].begin(), sym[i].end());
      sym[i].erase(std::unique(sym[i].begin(), sym[i].end()), sym[i].end());
    }
    adj.swap(sym);
  }

  std::vector<int> order = min_degree_order(nb, adj, wt);

  // ---- tail selection ------------------------------------------------------
  std::vector<std::vector<int>> st;
  std::vector<int> par;
  bus_symbolic(nb, order, adj, st, par);
  int tail_start = nb - 1;
  while (tail_start > 0 && (int)st[tail_start - 1].size() == nb - tail_start) --tail_start;
  {
    int w = 0;
    for (int k = tail_start; k < nb; ++k) w += wt[order[k]];
    P.n_tail_exact = w;
  }
  std::vector<char> intail(nb, 0);
  for (int k = tail_start; k < nb; ++k) intail[k] = 1;
  if (opt.policy == 1) {
    // tail-row weight of each head bus against the exact tail
    std::vector<int> trow(nb, 0);
    for (int k = 0; k < tail_start; ++k)
      for (int j : st[k])
        if (j >= tail_start) trow[k] += wt[order[j]];
    std::vector<int> cands;
    if (opt.force_tau >= 0) {
      cands.push_back(opt.force_tau);
    } else {
      cands = trow;
      std::sort(cands.begin(), cands.end());
      cands.erase(std::unique(cands.begin(), cands.end()), cands.end());
      // thin to at most ~64 candidates, plus "no extension"
      if (cands.size() > 64) {
        std::vector<int> thin;
        for (size_t q = 0; q < 64; ++q) thin.push_back(cands[q * cands.size() / 64]);
        cands.swap(thin);
      }
      cands.push_back(std::numeric_limits<int>::max());
    }
    double best = std::numeric_limits<double>::infinity();
    std::vector<char> best_set = intail;
    for (int tau : cands) {
      std::vector<char> in(intail);
      for (int k = 0; k < tail_start; ++k)
        if (trow[k] > tau) in[k] = 1;
      // ancestor closure (parents have larger indices)
      for (int k = 0; k < nb; ++k)
        if (in[k] && par[k] >= 0) in[par[k]] = 1;
      double N = 0, vol = 0;
      for (int k = 0; k < nb; ++k)
        if (in[k]) N += wt[order[k]];
      for (int k = 0; k < nb; ++k) {
        if (in[k]) continue;
        double tt = 0;
        for (int j : st[k])
          if (in[j]) tt += wt[order[j]];
        vol += wt[order[k]] * tt * tt;
      }
      double cost = (N * N * N / 3.0) / opt.dense_rate + vol / opt.scatter_rate;
      if (cost < best) { best = cost; best_set = in; }
    }
    intail = best_set;
  }
  // final bus order: head buses then tail buses, relative order kept.  This is
  // a topological order of the elimination tree (the tail is ancestor-closed),
  // so the fill is unchanged.
  std::vector<int> border;
  for (int k = 0; k < nb; ++k)
    if (!intail[k]) border.push_back(order[k]);
  int nb_head = (int)border.size();
  for (int k = 0; k < nb; ++k)
    if (intail[k]) border.push_back(order[k]);
  bus_symbolic(nb, border, adj, st, par);

  // ---- variable order --------------------------------------------------
  const int d = P.dim;
  P.perm.resize(d);
  P.iperm.assign(d, -1);
  std::vector<int> var0(nb + 1, 0);  // first factor position of elimination bus k
  std::vector<int> bus_of_var(d);    // elimination bus index of every factor position
  {
    int f = 0;
    for (int k = 0; k < nb; ++k) {
      var0[k] = f;
      int b = P.pvpq[border[k]];
      P.perm[f] = jP[b];
      bus_of_var[f++] = k;
      if (kind[b] == 2) {
        P.perm[f] = jQ[b];
        bus_of_var[f++] = k;
      }
    }
    var0[nb] = f;
  }
  for (int f = 0; f < d; ++f) P.iperm[P.perm[f]] = f;
  P.fP.assign(n_bus, -1);
  P.fQ.assign(n_bus, -1);
  for (int b = 0; b < n_bus; ++b) {
    if (jP[b] >= 0) P.fP[b] = P.iperm[jP[b]];
    if (jQ[b] >= 0) P.fQ[b] = P.iperm[jQ[b]];
  }
  const int p = var0[nb_head];
  P.p = p;
  P.nt = d - p;
  P.ld = ((P.nt + 7) / 8) * 8;
  if (P.nt == 0) P.ld = 0;

  // variable-level column structures (head columns only)
  std::vector<std::vector<int>> vst(p);
  for (int c = 0; c < p; ++c) {
    int k = bus_of_var[c];
    std::vector<int>& s = vst[c];
    for (int f = c + 1; f < var0[k + 1]; ++f) s.push_back(f);
    for (int j : st[k])
      for (int f = var0[j]; f < var0[j + 1]; ++f) s.push_back(f);
  }

  // ---- head supernodes ---------------------------------------------------
  std::vector<int> vpar(p, -1), nchild(d, 0);
  for (int c = 0; c < p; ++c)
    if (!vst[c].empty()) { vpar[c] = vst[c][0]; nchild[vpar[c]]++; }
  std::vector<int> sn_of(p, -1);
  {
    int s = -1;
    for (int c = 0; c < p; ++c) {
      bool join = c > 0 && vpar[c - 1] == c && nchild[c] == 1 && vst[c - 1].size() == vst[c].size() + 1;
      if (!join) {
        ++s;
        P.sn_first.push_back(c);
        P.sn_w.push_back(0);
      }
      sn_of[c] = s;
      P.sn_w[s]++;
    }
    P.n_sn = s + 1;
  }
  // head/tail split of every column's structure
  std::vector<int> nh(p, 0);
  for (int c = 0; c < p; ++c)
    for (int i : vst[c])
      if (i < p) nh[c]++;

  // ---- HV layout ---------------------------------------------------------
  std::vector<int> Lhh(p), Uhh(p);
  int pos = p;  // diag first
  for (int c = 0; c < p; ++c) { Lhh[c] = pos; pos += nh[c]; }
  for (int c = 0; c < p; ++c) { Uhh[c] = pos; pos += nh[c]; }
  P.sn_t.resize(P.n_sn);
  P.sn_L.resize(P.n_sn);
  P.sn_U.resize(P.n_sn);
  P.sn_tidx.resize(P.n_sn + 1);
  for (int s = 0; s < P.n_sn; ++s) {
    int c = P.sn_first[s];
    int t = (int)vst[c].size() - nh[c];
    P.sn_t[s] = t;
    P.sn_L[s] = pos; pos += t * P.sn_w[s];
    P.sn_U[s] = pos; pos += t * P.sn_w[s];
    P.sn_tidx[s] = (int)P.tidx.size();
    for (size_t q = nh[c]; q < vst[c].size(); ++q) P.tidx.push_back(vst[c][q] - p);
  }
  P.sn_tidx[P.n_sn] = (int)P.tidx.size();
  P.n_hv = pos;
  auto posL = [&](int i, int m, int rank) -> int {  // rank = index of i in vst[m]
    if (i < p) return Lhh[m] + rank;
    int s = sn_of[m];
    int a = rank - nh[m];
    return P.sn_L[s] + a * P.sn_w[s] + (m - P.sn_first[s]);
  };
  auto posU = [&](int m, int i, int rank) -> int {
    if (i < p) return Uhh[m] + rank;
    int s = sn_of[m];
    int a = rank - nh[m];
    return P.sn_U[s] + (m - P.sn_first[s]) * P.sn_t[s] + a;
  };

  // row lists over head columns: for row i, entries m (increasing) with positions
  std::vector<int> rptr(d + 1, 0);
  for (int c = 0; c < p; ++c)
    for (int i : vst[c]) rptr[i + 1]++;
  for (int i = 0; i < d; ++i) rptr[i + 1] += rptr[i];
  std::vector<int> rcol(rptr[d]), rL(rptr[d]), rU(rptr[d]);
  {
    std::vector<int> head(rptr.begin(), rptr.end() - 1);
    for (int c = 0; c < p; ++c)
      for (size_t q = 0; q < vst[c].size(); ++q) {
        int i = vst[c][q];
        int h = head[i]++;
        rcol[h] = c;
        rL[h] = posL(i, c, (int)q);
        rU[h] = posU(c, i, (int)q);
      }
  }

  // ---- J structure test: (r, c) factor positions -> is J nonzero? --------
  std::vector<std::vector<int>> ynb(n_bus);
  for (int b = 0; b < n_bus; ++b)
    for (int k = P.y_indptr[b]; k < P.y_indptr[b + 1]; ++k) ynb[b].push_back(P.y_indices[k]);
  auto bus_of_f = [&](int f) { return P.pvpq[border[bus_of_var[f]]]; };
  auto jnz = [&](int r, int c) {
    int br = bus_of_f(r), bc = bus_of_f(c);
    if (br == bc) return P.y_diag[br] >= 0;
    return std::binary_search(ynb[br].begin(), ynb[br].end(), bc);
  };

  // ---- levels and head tasks -------------------------------------------
  std::vector<int> level(p, 0);
  for (int k = 0; k < p; ++k) {
    int lv = 0;
    for (int h = rptr[k]; h < rptr[k + 1]; ++h) lv = std::max(lv, level[rcol[h]] + 1);
    level[k] = lv;
  }
  P.n_levels = p ? *std::max_element(level.begin(), level.end()) + 1 : 0;
  std::vector<std::vector<int>> by_level(P.n_levels);
  for (int k = 0; k < p; ++k) by_level[level[k]].push_back(k);
  P.lev_ptr.assign(1, 0);
  P.lev_piv_ptr.assign(1, 0);
  for (int lv = 0; lv < P.n_levels; ++lv) {
    for (int k : by_level[lv]) P.lev_piv.push_back(k);
    P.lev_piv_ptr.push_back((int)P.lev_piv.size());
  }
  auto add_task = [&](int out, bool has_a, int diag) {
    P.task_out.push_back(out);
    P.task_has_a.push_back(has_a ? 1 : 0);
    P.task_diag.push_back(diag);
    P.task_pbeg.push_back((int)P.pair_l.size());
  };
  auto end_task = [&]() { P.task_pend.push_back((int)P.pair_l.size()); };
  for (int lv = 0; lv < P.n_levels; ++lv) {
    for (int k : by_level[lv]) {
      // u_kk
      add_task(k, jnz(k, k), -1);
      for (int h = rptr[k]; h < rptr[k + 1]; ++h) { P.pair_l.push_back(rL[h]); P.pair_u.push_back(rU[h]); }
      end_task();
      for (size_t q = 0; q < vst[k].size(); ++q) {
        int i = vst[k][q];
        // merge S(i) and S(k) (both sorted, all < k for S(k); S(i) may hold k itself, skip m >= k)
        int a = rptr[i], ae = rptr[i + 1], b = rptr[k], be = rptr[k + 1];
        std::vector<int> mi, mk;
        while (a < ae && b < be) {
          int ma = rcol[a], mb = rcol[b];
          if (ma >= k) break;
          if (ma == mb) { mi.push_back(a); mk.push_back(b); ++a; ++b; }
          else if (ma < mb) ++a;
          else ++b;
        }
        // L entry l_ik
        add_task(posL(i, k, (int)q), jnz(i, k), k);
        for (size_t z = 0; z < mi.size(); ++z) { P.pair_l.push_back(rL[mi[z]]); P.pair_u.push_back(rU[mk[z]]); }
        end_task();
        // U entry u_ki
        add_task(posU(k, i, (int)q), jnz(k, i), -1);
        for (size_t z = 0; z < mi.size(); ++z) { P.pair_l.push_back(rL[mk[z]]); P.pair_u.push_back(rU[mi[z]]); }
        end_task();
      }
    }
    // long tasks first (a warp each on the device), longest first
    {
      const int t0 = P.lev_ptr.back(), t1 = (int)P.task_out.size();
      std::vector<int> idx(t1 - t0);
      std::iota(idx.begin(), idx.end(), t0);
      auto len = [&](int t) { return P.task_pend[t] - P.task_pbeg[t]; };
      std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
        const bool ba = len(a) >= Plan::kBigTask, bb = len(b) >= Plan::kBigTask;
        if (ba != bb) return ba;
        return ba ? len(a) > len(b) : false;
      });
      auto permute = [&](auto& v) {
        auto tmp = v;
        for (int q = 0; q < t1 - t0; ++q) v[t0 + q] = tmp[idx[q]];
      };
      permute(P.task_out);
      permute(P.task_diag);
      permute(P.task_pbeg);
      permute(P.task_pend);
      permute(P.task_has_a);
      int nbig = 0;
      for (int t = t0; t < t1; ++t)
        if (len(t) >= Plan::kBigTask) ++nbig;
      P.lev_big.push_back(t0 + nbig);
    }
    P.lev_ptr.push_back((int)P.task_out.size());
  }
  P.head_madds = (int64_t)P.pair_l.size();

  // ---- Schur items per tail row ----------------------------------------
  P.schur_ptr.assign(P.nt + 1, 0);
  for (int ti = 0; ti < P.nt; ++ti) {
    int i = p + ti;
    int last_s = -1;
    for (int h = rptr[i]; h < rptr[i + 1]; ++h) {
      int m = rcol[h];
      int s = sn_of[m];
      if (s == last_s) continue;
      last_s = s;
      // a = rank of ti in s's tail rows
      const int* tb = P.tidx.data() + P.sn_tidx[s];
      const int* te = P.tidx.data() + P.sn_tidx[s + 1];
      const int* it = std::lower_bound(tb, te, ti);
      if (it == te || *it != ti) throw std::logic_error("build_plan: inconsistent supernode tail rows");
      P.schur_sn.push_back(s);
      P.schur_a.push_back((int)(it - tb));
      P.schur_madds += (int64_t)P.sn_w[s] * P.sn_t[s];
      P.schur_volume += P.sn_t[s];
    }
    P.schur_ptr[ti + 1] = (int)P.schur_sn.size();
  }
  // column groups of the Schur update (see plan.hpp)
  {
    struct Ent {
      int col, L, U, wt, ord;
    };
    std::vector<Ent> ents;
    P.sg_ptr.assign(P.nt + 1, 0);
    P.se_ptr.assign(1, 0);
    for (int ti = 0; ti < P.nt; ++ti) {
      ents.clear();
      for (int q = P.schur_ptr[ti]; q < P.schur_ptr[ti + 1]; ++q) {
        const int s = P.schur_sn[q], a = P.schur_a[q], w = P.sn_w[s], t = P.sn_t[s];
        if (w >= 16 || t >= (1 << 27)) throw std::logic_error("build_plan: supernode too large for the Schur map");
        for (int b = 0; b < t; ++b)
          ents.push_back({P.tidx[P.sn_tidx[s] + b], P.sn_L[s] + a * w, P.sn_U[s] + b, w | (t << 4), (int)ents.size()});
      }
      std::sort(ents.begin(), ents.end(),
                [](const Ent& x, const Ent& y) { return x.col != y.col ? x.col < y.col : x.ord < y.ord; });
      for (size_t e = 0; e < ents.size(); ++e) {
        if (e == 0 || ents[e].col != ents[e - 1].col) {
          if (e > 0) P.se_ptr.push_back((int)P.se_L.size());
          P.sg_col.push_back(ents[e].col);
        }
        P.se_L.push_back(ents[e].L);
        P.se_U.push_back(ents[e].U);
        P.se_wt.push_back(ents[e].wt);
      }
      if (!ents.empty()) P.se_ptr.push_back((int)P.se_L.size());
      P.sg_ptr[ti + 1] = (int)P.sg_col.size();
    }
    P.se_rec.resize(4 * P.se_L.size());
    for (size_t e = 0; e < P.se_L.size(); ++e) {
      P.se_rec[4 * e] = P.se_L[e];
      P.se_rec[4 * e + 1] = P.se_U[e];
      P.se_rec[4 * e + 2] = P.se_wt[e];
      P.se_rec[4 * e + 3] = 0;
    }
  }
  for (int64_t k = 0; k < P.nt; ++k) P.dense_madds += (P.nt - 1 - k) * (P.nt - 1 - k);

  // ---- solves -------------------------------------------------------------
  P.fw_ptr = rptr;
  P.fw_col = rcol;
  P.fw_pos = rL;
  P.bw_ptr.assign(p + 1, 0);
  for (int k = 0; k < p; ++k) P.bw_ptr[k + 1] = P.bw_ptr[k] + (int)vst[k].size();
  P.bw_row.resize(P.bw_ptr[p]);
  P.bw_pos.resize(P.bw_ptr[p]);
  for (int k = 0; k < p; ++k)
    for (size_t q = 0; q < vst[k].size(); ++q) {
      P.bw_row[P.bw_ptr[k] + q] = vst[k][q];
      P.bw_pos[P.bw_ptr[k] + q] = posU(k, vst[k][q], (int)q);
    }
  P.diag_pos.resize(p);
  std::iota(P.diag_pos.begin(), P.diag_pos.end(), 0);
  // the same entries by column, for the transposed solves
  {
    P.ut_ptr.assign(d + 1, 0);
    for (int k = 0; k < p; ++k)
      for (int q = P.bw_ptr[k]; q < P.bw_ptr[k + 1]; ++q) ++P.ut_ptr[P.bw_row[q] + 1];
    for (int j = 0; j < d; ++j) P.ut_ptr[j + 1] += P.ut_ptr[j];
    P.ut_row.resize(P.ut_ptr[d]);
    P.ut_pos.resize(P.ut_ptr[d]);
    std::vector<int> fill(P.ut_ptr.begin(), P.ut_ptr.end() - 1);
    for (int k = 0; k < p; ++k)
      for (int q = P.bw_ptr[k]; q < P.bw_ptr[k + 1]; ++q) {
        const int j = P.bw_row[q];
        P.ut_row[fill[j]] = k;
        P.ut_pos[fill[j]++] = P.bw_pos[q];
      }
    P.lt_ptr.assign(p + 1, 0);
    for (int r = 0; r < d; ++r)
      for (int q = P.fw_ptr[r]; q < P.fw_ptr[r + 1]; ++q) ++P.lt_ptr[P.fw_col[q] + 1];
    for (int i = 0; i < p; ++i) P.lt_ptr[i + 1] += P.lt_ptr[i];
    P.lt_row.resize(P.lt_ptr[p]);
    P.lt_pos.resize(P.lt_ptr[p]);
    std::vector<int> fl(P.lt_ptr.begin(), P.lt_ptr.end() - 1);
    for (int r = 0; r < d; ++r)
      for (int q = P.fw_ptr[r]; q < P.fw_ptr[r + 1]; ++q) {
        const int i = P.fw_col[q];
        P.lt_row[fl[i]] = r;
        P.lt_pos[fl[i]++] = P.fw_pos[q];
      }
  }

  // ---- Jacobian fill map -------------------------------------------------
  auto dest = [&](int r, int c) -> int {
    if (r >= p && c >= p) return encode_tail((r - p) * P.ld + (c - p));
    if (r == c) return r;
    if (r > c) {  // l_rc, c head
      for (int h = rptr[r]; h < rptr[r + 1]; ++h)
        if (rcol[h] == c) return rL[h];
    } else {  // u_cr... u_rc with r head: row list of c holds (r, rU)
      for (int h = rptr[c]; h < rptr[c + 1]; ++h)
        if (rcol[h] == r) return rU[h];
    }
    throw std::logic_error("build_plan: Jacobian coefficient outside the factor pattern");
  };
  P.jmap.assign(size_t(4) * P.nnz_y, -1);
  for (int k = 0; k < P.nnz_y; ++k) {
    int i = P.y_row[k], j = P.y_indices[k];
    int rows[2] = {jP[i], jQ[i]};
    int cols[2] = {jP[j], jQ[j]};
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b) {
        if (rows[a] < 0 || cols[b] < 0) continue;
        P.jmap[size_t(4) * k + 2 * a + b] = dest(P.iperm[rows[a]], P.iperm[cols[b]]);
        P.nnz_j++;
      }
  }
  int64_t nl = 0;
  for (int c = 0; c < p; ++c) nl += (int64_t)vst[c].size();
  nl += (int64_t)P.nt * (P.nt - 1) / 2;
  P.nnz_lu = d + 2 * nl;
  P.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return P;
}

}  // namespace gs2g
