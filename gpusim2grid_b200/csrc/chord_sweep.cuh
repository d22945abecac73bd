// Chord sweep: several rows per CTA stepping in lockstep on the shared base
// factor (refactor policy 2, continuous schedule).
//
// Under policy 2 most Newton steps of most rows apply the same factor -- the
// base case's Jacobian, shared read-only by every CTA and resident in L2 --
// so a step is bound by the latency and the L2 bandwidth of streaming that
// factor, not by arithmetic.  Here each CTA holds CK rows ("slots") and every
// read of a factor entry or index serves all of them: the right-hand sides
// are stored interleaved (CK values per unknown, one vector load), the head
// levels and the tail rows are swept once for all slots, and the dense tail
// is one product of the tail block of the base inverse (the inverse of the
// dense Schur complement) with CK columns.  Every barrier is shared by the
// slots as well.
//
// A slot leaves the chord kernel when its row converges (outputs written
// here, branch flows included) or when the row needs more than the base
// factor can give: the step stopped contracting (ratio test or max_reuse),
// the mismatch is not finite, or the iteration budget is spent while a rescue
// voltage is set.  Those rows are handed off -- current V in v_out, steps so
// far in iters_out, row id in a device list -- to the single-row sweep
// kernel, which continues them with their own factor (policy 1) and, where
// needed, the rescue attempt.  The decisions are the single-row kernel's:
// the same ratio test, the same counters, the same statuses.
//
// With a.broyden set, the chord steps are Broyden's "good" method instead:
// the base factor (with the row's outage compensation) is the initial
// inverse Jacobian H0, and each step corrects H0 F by the rank-one updates
// of the steps taken so far, in the storage-efficient form of C. T. Kelley
// ("Iterative Methods for Linear and Nonlinear Equations", SIAM 1995, the
// brsol algorithm): with steps s_0..s_n stored,
//   z = H0 F;  z += s_{j+1} (s_j . z) / |s_j|^2  for j < n;
//   s_{n+1} = z / (1 - (s_n . z) / |s_n|^2),
// so a step costs one base solve plus a few dot products, and converges
// superlinearly where the plain chord converges linearly.  The same
// contraction, budget and hand-off tests apply to its steps.
//
// Included by nr_kernel.cu inside its anonymous namespace (it uses that
// file's helpers).

// CTAs per SM the chord kernels are compiled for (registers per thread
// follow: 3 -> 80).  The chord loop waits on dependent L2 loads, so more
// resident warps pay: 3 per SM was 15 % faster than 2 on the 2000- and
// 6500-bus sweeps.
#ifndef GS2G_CHORD_CTAS_PER_SM
#define GS2G_CHORD_CTAS_PER_SM 3
#endif

// Rows per CTA (build-time).  8 was measured against 4 on the 2000- and
// 6500-bus sweeps: 10-16 % slower at 2 CTAs per SM (128 registers) and
// 9-16 % slower at 3 (80 registers, more spills); 4 rows at 3 CTAs per SM
// is the default.
#ifndef GS2G_CHORD_ROWS
#define GS2G_CHORD_ROWS 4
#endif
constexpr int CK = GS2G_CHORD_ROWS;  // rows per CTA

// Unrolling of the chord loops whose loads form dependent chains (index ->
// right-hand side): the head and tail solves' entry loops and the dense
// product's column loop.  Build-time; the defaults were measured fastest.
#ifndef GS2G_CHORD_SOLVE_UNROLL
#define GS2G_CHORD_SOLVE_UNROLL 4
#endif
#ifndef GS2G_CHORD_DENSE_UNROLL
#define GS2G_CHORD_DENSE_UNROLL 8
#endif
#define GS2G_PRAGMA(x) _Pragma(#x)
#define GS2G_UNROLL(n) GS2G_PRAGMA(unroll n)
constexpr int CB_MAX = 10;  // Broyden steps kept per row (the memory restarts beyond)

// the CK right-hand sides of one unknown, loaded as one vector (or two)
template <typename T>
struct alignas(16) SlotVec {
  T v[CK];
};

template <typename T>
__device__ __forceinline__ void fms_slots(SlotVec<T>& acc, T a, const SlotVec<T>& b) {
#pragma unroll
  for (int s = 0; s < CK; ++s) acc.v[s] = fma(-a, b.v[s], acc.v[s]);
}

// Workspace of one chord CTA: the slots' voltages interleaved (V [n] x CK,
// slot s of bus i at i * CK + s), the interleaved right-hand sides
// y [dim] x CK (the mismatch writes F there), then the Broyden steps
// [CK][CB_MAX][dim].
struct ChordWs {
  int64_t V, y, S, total;
};

template <typename T>
__host__ __device__ ChordWs chord_ws(const DevPlan& P) {
  ChordWs w;
  int64_t o = 0;
  w.V = o; o = align256(o + (int64_t)CK * P.n_bus * 16);
  w.y = o; o = align256(o + (int64_t)P.dim * sizeof(SlotVec<T>));
  w.S = o; o = align256(o + (int64_t)CK * CB_MAX * P.dim * sizeof(T));
  w.total = o;
  return w;
}

// Per-slot state, in shared memory; written by thread 0 between barriers.
struct ChordSlot {
  int row;    // session row, -1: empty
  int it;     // Newton steps taken
  int since;  // steps on the factor since the last (here: base) factorization
  int fresh;  // first mismatch still to be compared with the alternative start
  int comp;   // outage compensation set up
  int act;    // this round: 1 solve, 2 converged, 3 diverged, 4 budget spent, 5 hand off
  int nb;     // Broyden steps stored
  int from_base;  // began from the rescue voltage (start selection): no rescue
  int masked;     // the row masks buses (handle_disconnected_grid): handed off at once
  double nrm, last;
};

// NaN-sticky block max of one value per slot at once (one pair of barriers).
__device__ __forceinline__ void block_nanmax_slots(double v[CK], double* s_red_slots) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int s = 0; s < CK; ++s) {
    for (int o = 16; o > 0; o >>= 1) {
      const double w = __shfl_xor_sync(0xffffffffu, v[s], o);
      v[s] = (isnan(w) || isnan(v[s])) ? NAN : fmax(v[s], w);
    }
  }
  if (lane == 0)
#pragma unroll
    for (int s = 0; s < CK; ++s) s_red_slots[warp * CK + s] = v[s];
  __syncthreads();
#pragma unroll
  for (int s = 0; s < CK; ++s) {
    double r = s_red_slots[s];
    for (int w = 1; w < NWARP; ++w) {
      const double x = s_red_slots[w * CK + s];
      r = (isnan(x) || isnan(r)) ? NAN : fmax(r, x);
    }
    v[s] = r;
  }
  __syncthreads();
}

// Block sum of one value per slot at once (one pair of barriers).
__device__ __forceinline__ void block_sum_slots(double v[CK], double* s_red_slots) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int s = 0; s < CK; ++s)
    for (int o = 16; o > 0; o >>= 1) v[s] += __shfl_xor_sync(0xffffffffu, v[s], o);
  if (lane == 0)
#pragma unroll
    for (int s = 0; s < CK; ++s) s_red_slots[warp * CK + s] = v[s];
  __syncthreads();
#pragma unroll
  for (int s = 0; s < CK; ++s) {
    double r = 0.0;
    for (int w = 0; w < NWARP; ++w) r += s_red_slots[w * CK + s];
    v[s] = r;
  }
  __syncthreads();
}

// Outage compensation of one unknown's right-hand sides (slots in `comp`):
// y_s[i] -= sum_c Minv[R_s[c], i] w_s[c], with w_s from chord_comp_solve.
template <typename T>
__device__ __forceinline__ void comp_apply(const int i, const int dim, const unsigned comp, SlotVec<T>& yi,
                                           const T* Minv, const int (*s_cr)[1 + MAX_COMP],
                                           const double (*s_cw)[MAX_COMP]) {
#pragma unroll
  for (int s = 0; s < CK; ++s) {
    if (!(comp >> s & 1)) continue;
    const int r = s_cr[s][0];
    T acc = T(0);
    for (int c = 0; c < r; ++c) acc += Minv[(int64_t)s_cr[s][1 + c] * dim + i] * (T)s_cw[s][c];
    yi.v[s] -= acc;
  }
}

// Broyden correction of the slots in `mask`: y holds x0 = M0^-1 F per slot on
// entry (before the outage compensation of the slots in `comp`, which the
// first pass applies) and the step s_{nb} on exit, which is also stored as
// the slot's next Broyden step (with its squared norm).  St: the CTA's steps
// [CK][CB_MAX][dim]; s_ss: their squared norms.
//
// Each pass over the unknowns reads one stored step per slot: the update
// z += c_j s_{j+1} and the next coefficient's dot product s_{j+1} . z share
// it (the dot is taken right after the update, on the same z), so n stored
// steps take n + 1 passes; the arithmetic and its order are the recursion's.
template <typename T>
__device__ __noinline__ void chord_broyden(const int dim, const unsigned mask, ChordSlot* sl, SlotVec<T>* y, T* St,
                                           double (*s_ss)[CB_MAX], double* s_red_slots, const unsigned comp,
                                           const T* Minv, const int (*s_cr)[1 + MAX_COMP],
                                           const double (*s_cw)[MAX_COMP]) {
  const int tid = threadIdx.x;
  int nb[CK];
  int maxnb = 0;
#pragma unroll
  for (int s = 0; s < CK; ++s) {
    nb[s] = (mask >> s & 1) ? sl[s].nb : 0;
    if (nb[s] >= CB_MAX) nb[s] = 0;  // memory full: restart from H0
    maxnb = max(maxnb, nb[s]);
  }
  auto step = [&](int s, int j) { return St + ((int64_t)s * CB_MAX + j) * dim; };
  // pass 0: the compensation (z = H0 F complete), and d = s_0 . z of every
  // slot holding steps (the first coefficient's, or the final one's when the
  // slot holds one step)
  double d[CK] = {};
  if (maxnb > 0 || comp) {
    for (int i = tid; i < dim; i += BS) {
      SlotVec<T> z = y[i];
      if (comp) {
        comp_apply(i, dim, comp, z, Minv, s_cr, s_cw);
        y[i] = z;
      }
#pragma unroll
      for (int s = 0; s < CK; ++s)
        if (nb[s] > 0) d[s] += (double)step(s, 0)[i] * (double)z.v[s];
    }
    if (maxnb > 0) block_sum_slots(d, s_red_slots);
    else __syncthreads();
  }
  // z += s_{j+1} (s_j . z) / |s_j|^2 for j < nb - 1; d ends as s_{nb-1} . z
  for (int j = 0; j + 1 < maxnb; ++j) {
    T cf[CK];
#pragma unroll
    for (int s = 0; s < CK; ++s) {
      const double ss = s_ss[s][j];
      cf[s] = (j + 1 < nb[s] && ss > 0.0) ? (T)(d[s] / ss) : T(0);
    }
    double dn[CK] = {};
    for (int i = tid; i < dim; i += BS) {
      SlotVec<T> z = y[i];
#pragma unroll
      for (int s = 0; s < CK; ++s)
        if (j + 1 < nb[s]) {
          const T st = step(s, j + 1)[i];
          z.v[s] = fma(cf[s], st, z.v[s]);
          dn[s] += (double)st * (double)z.v[s];
        }
      y[i] = z;
    }
    block_sum_slots(dn, s_red_slots);
#pragma unroll
    for (int s = 0; s < CK; ++s)
      if (j + 1 < nb[s]) d[s] = dn[s];
  }
  // s_{nb} = z / (1 - (s_{nb-1} . z) / |s_{nb-1}|^2); a vanishing denominator
  // (the update breaks down) restarts the memory with the plain step z
  T sc[CK];
#pragma unroll
  for (int s = 0; s < CK; ++s) {
    sc[s] = T(1);
    if (nb[s] > 0) {
      const double ss = s_ss[s][nb[s] - 1];
      const double den = ss > 0.0 ? 1.0 - d[s] / ss : 0.0;
      if (fabs(den) > 1e-6) sc[s] = (T)(1.0 / den);
      else nb[s] = 0;
    }
  }
  double q[CK] = {};
  for (int i = tid; i < dim; i += BS) {
    SlotVec<T> z = y[i];
#pragma unroll
    for (int s = 0; s < CK; ++s) {
      if (!(mask >> s & 1)) continue;
      z.v[s] *= sc[s];
      step(s, nb[s])[i] = z.v[s];
      q[s] += (double)z.v[s] * (double)z.v[s];
    }
    y[i] = z;
  }
  block_sum_slots(q, s_red_slots);
  if (tid == 0)
#pragma unroll
    for (int s = 0; s < CK; ++s)
      if (mask >> s & 1) {
        s_ss[s][nb[s]] = q[s];
        sl[s].nb = nb[s] + 1;
      }
  __syncthreads();
}

// F and ||F||inf of the slots in `mask` (bit s: slot s): one sweep over the
// Ybus rows, each entry read once for all slots.  Row edits are applied as
// corrections on the buses of the edited Ybus rows (edit e subtracts ev[e]
// from Y at the entry of row er[e], column ec[e]).  F goes straight into the
// slots' lanes of the interleaved right-hand sides y (the chord solve's
// input, in T); lanes of slots outside `mask` are kept only where `keep`
// has their bit (others are not read before they are written again).
template <typename T>
__device__ __noinline__ void chord_mismatch(const DevPlan P, const SweepArgs a, const unsigned mask,
                                            const unsigned keep, const ChordSlot* sl, const int* s_ne,
                                            const int (*s_er)[MAX_EDITS], const int (*s_ec)[MAX_EDITS],
                                            const double2 (*s_ev)[MAX_EDITS], const double2* Vs, SlotVec<T>* y,
                                            double* nrm_out, double* s_red_slots) {
  const int n = P.n_bus;
  const double2* Y = reinterpret_cast<const double2*>(a.ybus);
  const double2* sb[CK];
#pragma unroll
  for (int s = 0; s < CK; ++s)
    sb[s] = reinterpret_cast<const double2*>(a.sbus) + (int64_t)(sl[s].row < 0 ? 0 : sl[s].row) * a.sbus_stride;
  double lmax[CK] = {};
  for (int i = threadIdx.x; i < n; i += BS) {
    double2 acc[CK];
#pragma unroll
    for (int s = 0; s < CK; ++s) acc[s] = make_double2(0.0, 0.0);
    for (int k = P.y_indptr[i]; k < P.y_indptr[i + 1]; ++k) {
      const double2 yk = Y[k];
      const int j = P.y_indices[k];
#pragma unroll
      for (int s = 0; s < CK; ++s) {
        if (!(mask >> s & 1)) continue;
        const double2 vj = Vs[(int64_t)j * CK + s];
        acc[s].x = fma(yk.x, vj.x, fma(-yk.y, vj.y, acc[s].x));
        acc[s].y = fma(yk.x, vj.y, fma(yk.y, vj.x, acc[s].y));
      }
    }
    const int fp = P.fP[i], fq = P.fQ[i];
    SlotVec<T> rp{}, rq{};
    if (keep) {
      if (fp >= 0) rp = y[fp];
      if (fq >= 0) rq = y[fq];
    }
#pragma unroll
    for (int s = 0; s < CK; ++s) {
      if (!(mask >> s & 1)) continue;
      for (int e = 0; e < s_ne[s]; ++e) {
        if (s_er[s][e] != i) continue;
        const double2 vj = Vs[(int64_t)s_ec[s][e] * CK + s];
        acc[s] = csub(acc[s], cmul(s_ev[s][e], vj));
      }
      const double2 sv = csub(cmul(Vs[(int64_t)i * CK + s], conj2(acc[s])), sb[s][i]);
      if (fp >= 0) {
        rp.v[s] = (T)(-sv.x);
        lmax[s] = (isnan(sv.x) || isnan(lmax[s])) ? NAN : fmax(lmax[s], fabs(sv.x));
      }
      if (fq >= 0) {
        rq.v[s] = (T)(-sv.y);
        lmax[s] = (isnan(sv.y) || isnan(lmax[s])) ? NAN : fmax(lmax[s], fabs(sv.y));
      }
    }
    if (fp >= 0) y[fp] = rp;
    if (fq >= 0) y[fq] = rq;
  }
  block_nanmax_slots(lmax, s_red_slots);
  if (threadIdx.x == 0)
#pragma unroll
    for (int s = 0; s < CK; ++s)
      if (mask >> s & 1) nrm_out[s] = lmax[s];
  __syncthreads();
}

// F and ||F||inf of slot s at the alternative start (the base V, already in
// the slot's lane of Vs) without the sparse product: Ia = Y Va on the
// unedited Ybus, shared by all rows and summed with chord_mismatch's fused
// multiply-adds in its order, is corrected at the buses of the row's edited
// Ybus rows exactly as chord_mismatch corrects its sums, so F and the norm
// are bit-identical to chord_mismatch's for this slot.  Writes only the
// slot's lane of y.
template <typename T>
__device__ __noinline__ void chord_mismatch_alt(const DevPlan P, const SweepArgs a, const int s, const ChordSlot* sl,
                                                const int* s_ne, const int (*s_er)[MAX_EDITS],
                                                const int (*s_ec)[MAX_EDITS], const double2 (*s_ev)[MAX_EDITS],
                                                const double2* Vs, const double2* __restrict__ Ia, SlotVec<T>* y,
                                                double* nrm_out, double* s_red) {
  const double2* sb = reinterpret_cast<const double2*>(a.sbus) + (int64_t)(sl[s].row < 0 ? 0 : sl[s].row) * a.sbus_stride;
  double lmax = 0.0;
  for (int i = threadIdx.x; i < P.n_bus; i += BS) {
    double2 acc = Ia[i];
    for (int e = 0; e < s_ne[s]; ++e) {
      if (s_er[s][e] != i) continue;
      const double2 vj = Vs[(int64_t)s_ec[s][e] * CK + s];
      acc = csub(acc, cmul(s_ev[s][e], vj));
    }
    const double2 sv = csub(cmul(Vs[(int64_t)i * CK + s], conj2(acc)), sb[i]);
    const int fp = P.fP[i], fq = P.fQ[i];
    if (fp >= 0) {
      y[fp].v[s] = (T)(-sv.x);
      lmax = (isnan(sv.x) || isnan(lmax)) ? NAN : fmax(lmax, fabs(sv.x));
    }
    if (fq >= 0) {
      y[fq].v[s] = (T)(-sv.y);
      lmax = (isnan(sv.y) || isnan(lmax)) ? NAN : fmax(lmax, fabs(sv.y));
    }
  }
  lmax = block_nanmax(lmax, s_red);
  if (threadIdx.x == 0) nrm_out[s] = lmax;
  __syncthreads();
}

// Forward over the head levels, all slots at once.  fwv: the factor's
// values in solve order (one sequential stream beside fw_col).
template <typename T>
__device__ __noinline__ void chord_head_fw(const DevPlan P, const T* __restrict__ fwv, SlotVec<T>* y) {
  for (int lv = 0; lv < P.n_levels; ++lv) {
    for (int q0 = P.lev_piv_ptr[lv] + threadIdx.x; q0 < P.lev_piv_ptr[lv + 1]; q0 += BS) {
      const int i = P.lev_piv[q0];
      SlotVec<T> acc = y[i];
      GS2G_UNROLL(GS2G_CHORD_SOLVE_UNROLL)
      for (int q = P.fw_ptr[i]; q < P.fw_ptr[i + 1]; ++q) fms_slots(acc, fwv[q], y[P.fw_col[q]]);
      y[i] = acc;
    }
    __syncthreads();
  }
}

// The tail rows against the head.
template <typename T>
__device__ __noinline__ void chord_tail_fw(const DevPlan P, const T* __restrict__ fwv, SlotVec<T>* y) {
  for (int ti = threadIdx.x; ti < P.nt; ti += BS) {
    const int i = P.p + ti;
    SlotVec<T> acc = y[i];
    GS2G_UNROLL(GS2G_CHORD_SOLVE_UNROLL)
    for (int q = P.fw_ptr[i]; q < P.fw_ptr[i + 1]; ++q) fms_slots(acc, fwv[q], y[P.fw_col[q]]);
    y[i] = acc;
  }
  __syncthreads();
}

// y_t <- Sinv y_t for all slots: the tail block of the base inverse (column j
// at Minv + (p + j) * dim + p) times the CK columns held in shared memory.
// Each thread owns up to four tail rows per pass; for each column a warp
// reads 32 consecutive entries.
template <typename T>
__device__ __noinline__ void chord_dense(const DevPlan P, const T* __restrict__ Minv, SlotVec<T>* y, SlotVec<T>* ys) {
  const int tid = threadIdx.x, nt = P.nt;
  for (int i = tid; i < nt; i += BS) ys[i] = y[P.p + i];
  __syncthreads();
  const T* Sinv = Minv + (int64_t)P.p * P.dim + P.p;
  for (int r0 = 0; r0 < nt; r0 += 4 * BS) {
    SlotVec<T> acc[4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int s = 0; s < CK; ++s) acc[u].v[s] = T(0);
    const int nr = min(4, (nt - r0 - tid + BS - 1) / BS);  // rows of this thread in the pass (may be <= 0)
    const T* base = Sinv + r0 + tid;
    GS2G_UNROLL(GS2G_CHORD_DENSE_UNROLL)
    for (int j = 0; j < nt; ++j) {
      const SlotVec<T> yj = ys[j];
      const T* col = base + (int64_t)j * P.dim;
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (u < nr) fms_slots(acc[u], -col[u * BS], yj);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (u < nr) y[P.p + r0 + tid + u * BS] = acc[u];
  }
  __syncthreads();
}

// Backward over the head levels (bwv: values in solve order, fHV for the
// pivots).
template <typename T>
__device__ __noinline__ void chord_head_bw(const DevPlan P, const T* __restrict__ fHV, const T* __restrict__ bwv,
                                           SlotVec<T>* y) {
  for (int lv = P.n_levels - 1; lv >= 0; --lv) {
    for (int q0 = P.lev_piv_ptr[lv] + threadIdx.x; q0 < P.lev_piv_ptr[lv + 1]; q0 += BS) {
      const int k = P.lev_piv[q0];
      SlotVec<T> acc = y[k];
      GS2G_UNROLL(GS2G_CHORD_SOLVE_UNROLL)
      for (int q = P.bw_ptr[k]; q < P.bw_ptr[k + 1]; ++q) fms_slots(acc, bwv[q], y[P.bw_row[q]]);
      const T d = fHV[k];
#pragma unroll
      for (int s = 0; s < CK; ++s) acc.v[s] = acc.v[s] / d;
      y[k] = acc;
    }
    __syncthreads();
  }
}

// Outputs of a slot's row as it leaves: V (the slot's lane of the
// interleaved voltages, V[i * CK]), and either the final status (flows
// included, from the row's output copy) or the hand-off to the single-row
// kernel.
__device__ __noinline__ void chord_leave(const SweepArgs a, const ChordSlot sl, const double2* V, const int n,
                                         double* s_red) {
  const int tid = threadIdx.x;
  const int row = sl.row;
  double2* vout = reinterpret_cast<double2*>(a.v_out) + (int64_t)row * n;
  for (int i = tid; i < n; i += BS) vout[i] = V[(int64_t)i * CK];
  if (tid == 0 && a.n_chord_steps != nullptr) atomicAdd(a.n_chord_steps, (unsigned long long)sl.it);
  if (sl.act == 5) {
    if (tid == 0) {
      a.iters_out[row] = sl.it;
      a.handoff[atomicAdd(a.n_handoff, 1)] = (a.handoff_base + row) | (sl.from_base ? NO_RESCUE_BIT : 0);
    }
    __syncthreads();
    return;
  }
  if (a.v_mirror != nullptr) {
    double2* vm = reinterpret_cast<double2*>(a.v_mirror) + (int64_t)row * n;
    for (int i = tid; i < n; i += BS) vm[i] = V[(int64_t)i * CK];
  }
  const int status = sl.act == 2 ? ROW_CONVERGED : (sl.act == 3 ? ROW_DIVERGED : ROW_MAX_ITER);
  if (a.loading_out != nullptr) {
    __syncthreads();  // the row's output copy is complete
    row_flows(a, row, vout, status == ROW_CONVERGED, s_red);
  }
  if (tid == 0) {
    a.res_out[row] = sl.nrm;
    a.status_out[row] = status;
    a.iters_out[row] = sl.it;
    if (a.factors_out != nullptr) a.factors_out[row] = 0;
  }
  __syncthreads();
}

// Outage compensation of the slots in `comp`:
// y_s <- y_s - Z_s B_s (I + W_s B_s)^-1 y_s[R_s] (see setup_compensation and
// apply_compensation, the one-row form).  First the small solves, in
// parallel, one warp's leading thread per slot (w_s = B_s (I + W_s B_s)^-1
// y_s[R_s] into s_cw); then one sweep over the unknowns applies every slot's
// columns of the base inverse (comp_apply: chord_comp_apply, or the first
// pass of chord_broyden).
template <typename T>
__device__ __noinline__ void chord_comp_solve(const unsigned comp, const SlotVec<T>* y,
                                              const int (*s_cr)[1 + MAX_COMP],
                                              const double (*s_cB)[MAX_COMP * MAX_COMP],
                                              const double (*s_cLU)[MAX_COMP * MAX_COMP],
                                              const int (*s_cpiv)[MAX_COMP], double (*s_cw)[MAX_COMP]) {
  const int tid = threadIdx.x;
  const int s0 = tid >> 5;
  if (s0 < CK && (tid & 31) == 0 && (comp >> s0 & 1)) {
    const int s = s0;
    const int r = s_cr[s][0];
    const int* R = s_cr[s] + 1;
    double v[MAX_COMP];
    for (int q = 0; q < r; ++q) v[q] = (double)y[R[q]].v[s];
    const double* C = s_cLU[s];
    for (int k = 0; k < r; ++k) {  // P v, then L, then U
      const int pk = s_cpiv[s][k];
      if (pk != k) {
        const double t = v[k];
        v[k] = v[pk];
        v[pk] = t;
      }
    }
    for (int i2 = 1; i2 < r; ++i2)
      for (int k = 0; k < i2; ++k) v[i2] -= C[i2 * r + k] * v[k];
    for (int i2 = r - 1; i2 >= 0; --i2) {
      for (int k = i2 + 1; k < r; ++k) v[i2] -= C[i2 * r + k] * v[k];
      v[i2] /= C[i2 * r + i2];
    }
    for (int q = 0; q < r; ++q) {  // w = B v
      double acc = 0.0;
      for (int c = 0; c < r; ++c) acc += s_cB[s][q * r + c] * v[c];
      s_cw[s][q] = acc;
    }
  }
  __syncthreads();
}

template <typename T>
__device__ __noinline__ void chord_comp_apply(const int dim, const unsigned comp, SlotVec<T>* y, const T* Minv,
                                              const int (*s_cr)[1 + MAX_COMP], const double (*s_cw)[MAX_COMP]) {
  for (int i = threadIdx.x; i < dim; i += BS) {
    SlotVec<T> yi = y[i];
    comp_apply(i, dim, comp, yi, Minv, s_cr, s_cw);
    y[i] = yi;
  }
  __syncthreads();
}

// The chord loop over the rows of one grid (queue a.queue, a.n_rows), until
// that queue is exhausted and every slot has left.  Called by the
// single-grid kernel once and by the multi-grid kernel once per grid.
template <typename T, bool Y_SMEM = false>
__device__ __forceinline__ void chord_body(const DevPlan& P, const SweepArgs& a, PhaseProf& prof) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ ChordSlot sl[CK];
  __shared__ int s_pull, s_more;
  __shared__ int s_ne[CK];
  __shared__ int s_ek[CK][MAX_EDITS];
  __shared__ int s_er[CK][MAX_EDITS];  // Ybus row and column of each edit
  __shared__ int s_ec[CK][MAX_EDITS];
  __shared__ double2 s_ev[CK][MAX_EDITS];
  __shared__ double s_red[NWARP];
  __shared__ double s_red_slots[NWARP * CK];
  __shared__ double s_nrm[CK];
  __shared__ int s_cr[CK][1 + MAX_COMP];
  __shared__ double s_cB[CK][MAX_COMP * MAX_COMP];
  __shared__ double s_cLU[CK][MAX_COMP * MAX_COMP];
  __shared__ int s_cpiv[CK][MAX_COMP];
  __shared__ double s_cw[CK][MAX_COMP];
  __shared__ double s_ss[CK][CB_MAX];
  const int tid = threadIdx.x;
  const int n = P.n_bus;
  const ChordWs L = chord_ws<T>(P);
  char* ws = a.workspace + (int64_t)blockIdx.x * a.ws_stride;
  double2* Vs = reinterpret_cast<double2*>(ws + L.V);
  SlotVec<T>* ys = reinterpret_cast<SlotVec<T>*>(smem_raw);
  // the right-hand sides in the workspace, or (Y_SMEM) in shared memory
  // after the tail copy ys
  SlotVec<T>* y = Y_SMEM ? ys + (P.nt > 0 ? P.nt : 1) : reinterpret_cast<SlotVec<T>*>(ws + L.y);
  T* St = reinterpret_cast<T*>(ws + L.S);
  const WsLayout BL = ws_layout<T>(P);  // layout of the base factor's workspace
  const T* fHV = reinterpret_cast<const T*>(a.base_ws + BL.HV);
  const T* fwv = reinterpret_cast<const T*>(a.base_fwv);
  const T* bwv = reinterpret_cast<const T*>(a.base_bwv);
  const T* Minv = reinterpret_cast<const T*>(a.base_inv);
  const double2* Y = reinterpret_cast<const double2*>(a.ybus);
  const double2* Vbase = reinterpret_cast<const double2*>(a.base_v);
  auto shs = [&](int s) {
    return RowShared<T>{&s_ne[s], s_ek[s], s_ev[s], s_red, nullptr, nullptr, s_cr[s], s_cB[s], s_cLU[s], s_cpiv[s],
                        s_cw[s]};
  };
  if (tid == 0) {
    for (int s = 0; s < CK; ++s) sl[s].row = -1;
    s_more = 1;
  }
  __syncthreads();
  for (;;) {
    // ---- refill empty slots from the row queue ----------------------------
    for (int s = 0; s < CK; ++s) {
      if (sl[s].row >= 0) continue;
      for (;;) {
        // every thread reads the flag before thread 0 may pull (and clear it)
        const int more = s_more;
        __syncthreads();
        if (!more) break;
        if (tid == 0) {
          const int q = atomicAdd(a.queue, 1);
          s_pull = q < a.n_rows ? (a.row_map != nullptr ? a.row_map[q] : q) : -1;
          if (q >= a.n_rows) s_more = 0;
        }
        __syncthreads();
        const int row = s_pull;
        if (row < 0) break;
        if (a.row_skip != nullptr && a.row_skip[row]) {
          skip_row_outputs(a, row, n);
          continue;
        }
        if (tid == 0) {
          int ne = 0;
          if (a.edit_ptr != nullptr) {
            const int e0 = a.edit_ptr[row], e1 = a.edit_ptr[row + 1];
            ne = min(e1 - e0, MAX_EDITS);
            for (int e = 0; e < ne; ++e) {
              const int k = a.edit_k[e0 + e];
              s_ek[s][e] = k;
              s_er[s][e] = P.y_row[k];
              s_ec[s][e] = P.y_indices[k];
              s_ev[s][e] = reinterpret_cast<const double2*>(a.edit_val)[e0 + e];
            }
          }
          s_ne[s] = ne;
          sl[s].row = row;
          sl[s].it = 0;
          sl[s].since = 0;
          sl[s].masked = a.mask_ptr != nullptr && a.mask_ptr[row + 1] > a.mask_ptr[row];
          sl[s].fresh = a.alt_v0 != nullptr && !sl[s].masked;
          sl[s].comp = 0;
          sl[s].act = 0;
          sl[s].nb = 0;
          sl[s].from_base = 0;
          sl[s].last = INFINITY;
        }
        const double2* v0 = reinterpret_cast<const double2*>(a.v0) + (int64_t)row * a.v0_stride;
        for (int i = tid; i < n; i += BS) Vs[(int64_t)i * CK + s] = v0[i];
        __syncthreads();
        const RowEdits ed{s_ne[s], s_ek[s], s_ev[s]};
        bool c = false;
        if (ed.n > 0 && Minv != nullptr && Vbase != nullptr && !sl[s].masked) {
          // the record set up ahead of the sweep, else here
          const int lc = a.comp_rec != nullptr
                             ? load_compensation(reinterpret_cast<const CompRec*>(a.comp_rec) + row, s_cr[s],
                                                 s_cB[s], s_cLU[s], s_cpiv[s])
                             : -1;
          c = lc >= 0 ? lc > 0 : setup_compensation<T>(P, ed, Y, Vbase, Minv, shs(s));
        }
        if (tid == 0) sl[s].comp = c;
        __syncthreads();
        break;
      }
    }
    unsigned active = 0;
    for (int s = 0; s < CK; ++s) active |= (sl[s].row >= 0 ? 1u : 0u) << s;
    if (active == 0) break;

    // ---- mismatch of every slot, start selection for new rows --------------
    chord_mismatch<T>(P, a, active, 0u, sl, s_ne, s_er, s_ec, s_ev, Vs, y, s_nrm, s_red_slots);
    for (int s = 0; s < CK; ++s) {
      if (!(active >> s & 1) || !sl[s].fresh) continue;
      const RowEdits ed{s_ne[s], s_ek[s], s_ev[s]};
      const double2* va = reinterpret_cast<const double2*>(a.alt_v0);
      const double2* sb = reinterpret_cast<const double2*>(a.sbus) + (int64_t)sl[s].row * a.sbus_stride;
      const double na = a.alt_s != nullptr
                            ? alt_mismatch_norm(P, ed, va, reinterpret_cast<const double2*>(a.alt_s), sb, s_red)
                            : mismatch_norm(P, ed, Y, va, sb, s_red);
      const bool sw = !(s_nrm[s] < na) && isfinite(na);
      __syncthreads();
      if (tid == 0) {
        sl[s].fresh = 0;
        if (sw) sl[s].from_base = a.alt_v0 == a.rescue_v0;
      }
      if (sw) {
        for (int i = tid; i < n; i += BS) Vs[(int64_t)i * CK + s] = va[i];
        if (tid == 0 && a.n_alt_start != nullptr) atomicAdd(a.n_alt_start, 1);
        __syncthreads();
        if (a.alt_i != nullptr)
          chord_mismatch_alt<T>(P, a, s, sl, s_ne, s_er, s_ec, s_ev, Vs, reinterpret_cast<const double2*>(a.alt_i),
                                y, s_nrm, s_red);
        else
          chord_mismatch<T>(P, a, 1u << s, active & ~(1u << s), sl, s_ne, s_er, s_ec, s_ev, Vs, y, s_nrm,
                            s_red_slots);
      }
    }
    prof.mark(PH_MISMATCH);

    // ---- per-slot decisions (the single-row kernel's, in its order) ---------
    if (tid == 0) {
      for (int s = 0; s < CK; ++s) {
        if (!(active >> s & 1)) continue;
        ChordSlot& q = sl[s];
        const bool rescue = a.rescue_v0 != nullptr && !q.from_base;
        q.nrm = s_nrm[s];
        // the row is tested only at the end of a round of round_k steps (and
        // runs its first round whatever its mismatch); between tests a row
        // whose mismatch is not finite is handed off as well, and the
        // single-row sweep steps it to the end of its round
        const bool test = q.it > 0 && q.it % (a.round_k > 1 ? a.round_k : 1) == 0;
        if (q.masked) q.act = 5;  // masked rows are solved on their own factor
        else if (!isfinite(q.nrm)) q.act = (rescue || !test) ? 5 : 3;
        else if (test && q.nrm < a.tol) q.act = 2;
        else if (test && q.it >= a.max_iter) q.act = rescue ? 5 : 4;
        else if (!keep_factor(q.nrm, q.last, a.refactor_ratio, q.since, a.max_reuse, q.it, a.max_iter, a.tol))
          q.act = 5;  // needs its own LU
        else q.act = 1;
      }
    }
    __syncthreads();
    unsigned solve = 0;
    for (int s = 0; s < CK; ++s) {
      if (!(active >> s & 1)) continue;
      if (sl[s].act == 1) {
        solve |= 1u << s;
        continue;
      }
      chord_leave(a, sl[s], Vs + s, n, s_red);
      if (tid == 0) sl[s].row = -1;
      __syncthreads();
    }
    if (solve == 0) continue;

    // ---- one solve on the base factor for every remaining slot (F is in y;
    // the lanes of slots that left are not read) ------------------------------
    chord_head_fw<T>(P, fwv, y);
    prof.mark(PH_SOLVE);
    chord_tail_fw<T>(P, fwv, y);
    prof.mark(PH_SOLVE_TAIL);
    if (P.nt > 0) chord_dense<T>(P, Minv, y, ys);
    prof.mark(PH_SOLVE_DENSE);
    chord_head_bw<T>(P, fHV, bwv, y);
    {
      unsigned comp = 0;
      for (int s = 0; s < CK; ++s) comp |= ((solve >> s & 1) && sl[s].comp ? 1u : 0u) << s;
      if (comp) chord_comp_solve<T>(comp, y, s_cr, s_cB, s_cLU, s_cpiv, s_cw);
      if (a.broyden) chord_broyden<T>(P.dim, solve, sl, y, St, s_ss, s_red_slots, comp, Minv, s_cr, s_cw);
      else if (comp) chord_comp_apply<T>(P.dim, comp, y, Minv, s_cr, s_cw);
    }
    prof.mark(PH_SOLVE_BACK);

    // ---- step scaling (MaxVoltageChange): a slot whose chord step would be
    // scaled leaves the chord before the step, for its own factor, where
    // its steps are scaled (the Broyden recursion assumes full steps) ------
    if (a.step_scaling) {
      double mdt[CK] = {}, mdv[CK] = {};  // fmax skips NaN entries
      for (int i = tid; i < n; i += BS) {
        const int fp = P.fP[i], fq = P.fQ[i];
        const SlotVec<T> ya = fp >= 0 ? y[fp] : SlotVec<T>{};
        const SlotVec<T> ym = fq >= 0 ? y[fq] : SlotVec<T>{};
#pragma unroll
        for (int s = 0; s < CK; ++s) {
          if (fp >= 0) mdt[s] = fmax(mdt[s], fabs((double)ya.v[s]));
          if (fq >= 0) mdv[s] = fmax(mdv[s], fabs((double)ym.v[s]));
        }
      }
      block_nanmax_slots(mdt, s_red_slots);
      block_nanmax_slots(mdv, s_red_slots);
      unsigned scaled = 0;  // the same on every thread (the maxima are broadcast)
      for (int s = 0; s < CK; ++s)
        if ((solve >> s & 1) && step_alpha(mdt[s], mdv[s], a.max_dva, a.max_dvm) < 1.0) scaled |= 1u << s;
      solve &= ~scaled;
      for (int s = 0; s < CK; ++s) {
        if (!(scaled >> s & 1)) continue;
        if (tid == 0) sl[s].act = 5;
        __syncthreads();
        chord_leave(a, sl[s], Vs + s, n, s_red);
        if (tid == 0) sl[s].row = -1;
        __syncthreads();
      }
    }

    // ---- V update (FP64, polar) ---------------------------------------------
    for (int i = tid; i < n; i += BS) {
      const int fp = P.fP[i], fq = P.fQ[i];
      if (fp < 0 && fq < 0) continue;
      const SlotVec<T> ya = fp >= 0 ? y[fp] : SlotVec<T>{};
      const SlotVec<T> ym = fq >= 0 ? y[fq] : SlotVec<T>{};
#pragma unroll
      for (int s = 0; s < CK; ++s) {
        if (!(solve >> s & 1)) continue;
        double2* V = Vs + (int64_t)i * CK + s;
        const double2 v = *V;
        const double vm = hypot(v.x, v.y) + (fq >= 0 ? (double)ym.v[s] : 0.0);
        const double va = atan2(v.y, v.x) + (fp >= 0 ? (double)ya.v[s] : 0.0);
        double sn, cs;
        sincos(va, &sn, &cs);
        *V = make_double2(vm * cs, vm * sn);
      }
    }
    if (tid == 0)
      for (int s = 0; s < CK; ++s)
        if (solve >> s & 1) {
          sl[s].last = sl[s].nrm;
          ++sl[s].since;
          ++sl[s].it;
        }
    __syncthreads();
    prof.mark(PH_UPDATE);
  }
}

template <typename T>
__global__ void __launch_bounds__(BS, GS2G_CHORD_CTAS_PER_SM) chord_kernel(const DevPlan P, const SweepArgs a) {
  PhaseProf prof;
  prof.init(a.phase_cycles != nullptr && threadIdx.x == 0);
  chord_body<T>(P, a, prof);
  prof.flush(a.phase_cycles);
}

// The same chord sweep with the right-hand sides in shared memory (for grids
// whose dim x 4 values fit beside the tail copy): every solve's gathers are
// shared-memory loads, at 2 CTAs per SM instead of 3.
template <typename T>
__global__ void __launch_bounds__(BS, 2) chord_kernel_ysmem(const DevPlan P, const SweepArgs a) {
  PhaseProf prof;
  prof.init(a.phase_cycles != nullptr && threadIdx.x == 0);
  chord_body<T, true>(P, a, prof);
  prof.flush(a.phase_cycles);
}

// Multi-grid chord sweep: a CTA binds its slots to one grid at a time (the
// slots share that grid's base factor), draining the grids' own queues in
// cyclic order from grid blockIdx.x % n_grids, so the CTAs spread over the
// grids and move on as queues run dry.  The grid's plan and arguments are
// copied into shared memory while the CTA works on it.
template <typename T>
__global__ void __launch_bounds__(BS, GS2G_CHORD_CTAS_PER_SM)
    chord_kernel_multi(const GridEntry* __restrict__ grids, int n_grids, unsigned long long* phase_cycles) {
  __shared__ __align__(16) GridEntry s_grid;
  PhaseProf prof;
  prof.init(phase_cycles != nullptr && threadIdx.x == 0);
  for (int k = 0; k < n_grids; ++k) {
    const int g = (blockIdx.x + k) % n_grids;
    const int* src = reinterpret_cast<const int*>(grids + g);
    int* dst = reinterpret_cast<int*>(&s_grid);
    for (int i = threadIdx.x; i < (int)(sizeof(GridEntry) / sizeof(int)); i += BS) dst[i] = src[i];
    __syncthreads();
    chord_body<T>(s_grid.P, s_grid.a, prof);
    __syncthreads();  // every thread is done with this grid's entry before the next copy
  }
  prof.flush(phase_cycles);
}

template <typename T>
int chord_smem_bytes(const DevPlan& P) {
  return (int)(sizeof(SlotVec<T>) * (size_t)(P.nt > 0 ? P.nt : 1));
}
// dynamic shared memory of chord_kernel_ysmem: the tail copy, then y
template <typename T>
int chord_smem_bytes_ysmem(const DevPlan& P) {
  return chord_smem_bytes<T>(P) + (int)(sizeof(SlotVec<T>) * (size_t)P.dim);
}
// Right-hand sides in shared memory when they fit in this budget, which
// leaves room for 2 CTAs per SM (build-time; 0 keeps them in the workspace).
// Measured on the 2000-bus grid (67 KB): N-1 sweep -3 %, injection sweep
// -10 %, bit-identical.
#ifndef GS2G_CHORD_YSMEM_BYTES
#define GS2G_CHORD_YSMEM_BYTES (84 * 1024)
#endif
template <typename T>
bool chord_use_ysmem(const DevPlan& P) {
  return sizeof(T) == 4 && chord_smem_bytes_ysmem<T>(P) <= GS2G_CHORD_YSMEM_BYTES;
}
