// Persistent batched Newton–Raphson kernel for sm_100a.
//
// One CTA owns one batch row at a time and runs that row's whole Newton loop
// without leaving the kernel: mismatch SpMV (FP64) → ‖F‖∞ → Jacobian fill →
// sparse head LU (level-scheduled) → Schur update of the dense tail → dense
// tail LU → triangular solves → polar voltage update (FP64).  A row leaves the
// CTA as soon as it has converged, diverged or used its iteration budget, and
// the CTA takes the next row from a global queue: rows retire individually
// with no host round trip (the reference decides per round on the host,
// src/_cpp/contingency/batch_pf_driver.cu:2691-2720).
//
// The arithmetic of every step follows the reference:
//   mismatch  F = -[Re, Im](V∘conj(Y V) − Sbus)      acpf_nr_kernels.cu:493-557
//   Jacobian  dS/dVa, dS/dVm (MATPOWER)              acpf_nr_kernels.cu:559-650
//   update    Va += dθ on pvpq, then Vm += dVm on pq acpf_nr_kernels.cu:728-790
//   norm      NaN-sticky ‖F‖∞                         acpf_nr_kernels.cu:1076-1128
//   trips     Y −= {yff, ytt, yft, ytf} per branch    contingency_analysis_helper.cpp:23-84
// The linear algebra (LU of J, solves) runs in T = double or float; the
// mismatch, the norm and the voltages are always FP64.
#include "nr_kernel.cuh"

#include <cuda_runtime.h>

#include <type_traits>

#include "dense_lu.cuh"
#include "dense_lu_f32.cuh"
#include "dense_lu_f64.cuh"

#include <cmath>
#include <cstdint>
#include <mutex>

namespace gs2g {

namespace {

constexpr int BS = 256;        // threads per CTA
constexpr int NWARP = BS / 32;
constexpr int MAX_EDITS = 64;  // Ybus edits per row held in shared memory
static_assert(BS == dense::BS, "the dense LU assumes the sweep's CTA size");

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 conj2(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

struct RowEdits {
  int n;
  const int* k;
  const double2* v;
  __device__ __forceinline__ double2 apply(int kk, double2 y) const {
    for (int e = 0; e < n; ++e)
      if (k[e] == kk) y = csub(y, v[e]);
    return y;
  }
};

// NaN-sticky block max of |x| (a NaN anywhere makes the result NaN).
__device__ double block_nanmax(double v, double* s_red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    double w = __shfl_xor_sync(0xffffffffu, v, o);
    v = (isnan(w) || isnan(v)) ? NAN : fmax(v, w);
  }
  if (lane == 0) s_red[warp] = v;
  __syncthreads();
  double r = s_red[0];
  for (int i = 1; i < NWARP; ++i) {
    double w = s_red[i];
    r = (isnan(w) || isnan(r)) ? NAN : fmax(r, w);
  }
  __syncthreads();
  return r;
}

// Sum over the block (every thread gets it); s_red holds NWARP doubles.
__device__ double block_sum(double v, double* s_red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) s_red[warp] = v;
  __syncthreads();
  double r = 0.0;
  for (int w = 0; w < NWARP; ++w) r += s_red[w];
  __syncthreads();
  return r;
}

template <typename T>
__device__ __forceinline__ T clamp_pivot(T piv, double floor_) {
  const T f = (T)floor_;
  if (fabs(piv) < f) return piv < T(0) ? -f : f;
  return piv;
}

// Contribution of one Schur entry (see Plan::se_rec): sum_{c<w} L[c] U[c t].
// w <= 15 (1 or 2 here: supernodes are buses); the first two products are
// loaded together.
template <typename T>
__device__ __forceinline__ T schur_entry(const T* __restrict__ HV, int4 rec) {
  const T* Lr = HV + rec.x;
  const T* Ub = HV + rec.y;
  const int w = rec.z & 15, t = rec.z >> 4;
  const T l0 = Lr[0], u0 = Ub[0];
  const T l1 = w > 1 ? Lr[1] : T(0), u1 = w > 1 ? Ub[t] : T(0);
  T acc = l0 * u0 + l1 * u1;
  for (int c = 2; c < w; ++c) acc += Lr[c] * Ub[c * t];
  return acc;
}

// Schur update of the dense tail: warp per tail row, lane per column group
// (each lane sums every contribution to one entry S[ti][col] and writes it
// once), four groups per lane in flight: their entry records are loaded
// together, then their factor values.
// Sparse head LU, level by level, in place on the head factor values HV.
// With parts > 1 the `parts` CTAs of a cluster (this one: rank `part`) split
// each level's tasks and pass cluster barriers instead of block barriers;
// a task's arithmetic does not depend on who runs it.
template <typename T>
__device__ __noinline__ void head_lu(const DevPlan P, T* HV, const double pfloor, const int part, const int parts) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gwarp = part * NWARP + warp, nwarps = parts * NWARP;
  const int gtid = part * BS + tid, nthreads = parts * BS;
  auto barrier = [&]() {
    if (parts > 1)
      dense::cluster_barrier();
    else
      __syncthreads();
  };
  for (int lv = 0; lv < P.n_levels; ++lv) {
    const int t0 = P.lev_ptr[lv], tb = P.lev_big[lv], t1 = P.lev_ptr[lv + 1];
    // long tasks: one warp each, products split over the lanes
    for (int t = t0 + gwarp; t < tb; t += nwarps) {
      const int out = P.task_out[t];
      const int q1 = P.task_pend[t];
      T acc_p = T(0);
      for (int q = P.task_pbeg[t] + lane; q < q1; q += 32) acc_p += HV[P.pair_l[q]] * HV[P.pair_u[q]];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc_p += __shfl_xor_sync(0xffffffffu, acc_p, o);
      if (lane == 0) {
        T acc = (P.task_has_a[t] ? HV[out] : T(0)) - acc_p;
        if (out < P.p) acc = clamp_pivot(acc, pfloor);
        HV[out] = acc;
      }
    }
    for (int t = tb + gtid; t < t1; t += nthreads) {
      const int out = P.task_out[t];
      T acc = P.task_has_a[t] ? HV[out] : T(0);
      const int q1 = P.task_pend[t];
      for (int q = P.task_pbeg[t]; q < q1; ++q) acc -= HV[P.pair_l[q]] * HV[P.pair_u[q]];
      if (out < P.p) acc = clamp_pivot(acc, pfloor);
      HV[out] = acc;
    }
    barrier();
    for (int t = t0 + gtid; t < t1; t += nthreads) {
      const int dg = P.task_diag[t];
      if (dg >= 0) HV[P.task_out[t]] /= HV[dg];
    }
    barrier();
  }
}

template <typename T>
__device__ __noinline__ void schur_update(const DevPlan P, const T* __restrict__ HV, T* __restrict__ S, int part = 0,
                                          int parts = 1) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // with parts > 1 the CTAs of a cluster take every parts-th warp's rows
  for (int ti = part * NWARP + warp; ti < P.nt; ti += parts * NWARP) {
    T* Srow = S + (int64_t)ti * P.ld;
    const int g0 = P.sg_ptr[ti], g1 = P.sg_ptr[ti + 1];
    for (int gb = g0; gb < g1; gb += 128) {
      int ge[4], e0[4], e1[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        ge[u] = gb + lane + 32 * u;
        const bool in = ge[u] < g1;
        e0[u] = in ? P.se_ptr[ge[u]] : 0;
        e1[u] = in ? P.se_ptr[ge[u] + 1] : 0;
      }
      T acc[4] = {T(0), T(0), T(0), T(0)};
      // first entry of each group (nearly every group has one or two)
      int4 rec[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) rec[u] = e0[u] < e1[u] ? P.se_rec[e0[u]] : make_int4(0, 0, 0, 0);
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (e0[u] < e1[u]) acc[u] = schur_entry<T>(HV, rec[u]);
#pragma unroll
      for (int u = 0; u < 4; ++u)
        for (int e = e0[u] + 1; e < e1[u]; ++e) acc[u] += schur_entry<T>(HV, P.se_rec[e]);
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (ge[u] < g1) Srow[P.sg_col[ge[u]]] -= acc[u];
    }
  }
}

// The MaxVoltageChange scale of a Newton step with max|dtheta| = mdt and
// max|dVm| = mdv (apply_step_scale_kernel, acpf_nr_kernels.cu:708-726): 1
// unless a maximum exceeds its bound.
__device__ __forceinline__ double step_alpha(double mdt, double mdv, double max_dva, double max_dvm) {
  double alpha = 1.0;
  if (mdt > max_dva) alpha = fmin(alpha, max_dva / mdt);
  if (mdv > max_dvm) alpha = fmin(alpha, max_dvm / mdv);
  return alpha;
}

// Dense tail LU: FP32 on the SIMT kernel of dense_lu_f32.cuh, FP64 on its
// FP64 counterpart (dense_lu_f64.cuh; GS2G_FP64_LU=0 selects the older
// DMMA-tile LU of dense_lu.cuh); all use the dynamic shared memory as
// scratch.
#ifndef GS2G_FP64_LU
#define GS2G_FP64_LU 1
#endif
template <typename T>
__device__ __forceinline__ void dense_lu(T* S, int n, int ld, T* smem, double pfloor) {
  if constexpr (sizeof(T) == 4)
    gs2g::dense32::lu(S, n, ld, smem, pfloor);
  else if constexpr (GS2G_FP64_LU == 1)
    gs2g::dense64::lu(S, n, ld, smem, pfloor);
  else
    dense::lu<T>(S, n, ld, smem, pfloor);
}
// The same factorization by the `parts` CTAs of a cluster (this CTA: rank
// `part`), bit-identical to dense_lu.
template <typename T>
__device__ __forceinline__ void dense_lu_cluster(T* S, int n, int ld, T* smem, double pfloor, int part, int parts) {
  if constexpr (sizeof(T) == 4)
    gs2g::dense32::lu_cluster(S, n, ld, smem, pfloor, part, parts);
  else if constexpr (GS2G_FP64_LU == 1)
    gs2g::dense64::lu_cluster(S, n, ld, smem, pfloor, part, parts);
  else
    dense::lu_cluster(S, n, ld, smem, pfloor, part, parts);
}
static_assert(gs2g::dense64::Smem::elems <= dense::Smem<double>::elems, "FP64 LU scratch within the FP64 smem");
template <typename T>
__host__ __device__ constexpr int dense_smem_elems() {
  return sizeof(T) == 4 ? gs2g::dense32::Smem::elems : dense::Smem<T>::elems;
}

// Staging for the dense solves: warp 0 copies a 32 x 64 tile of the factor
// (rows r0.. (nr valid), columns c0.. (valid below n)) into shared memory
// with cp.async, one row per lane, zero-filling past column n.
template <typename T>
__host__ __device__ constexpr int stage_stride() {
  return 64 + 16 / (int)sizeof(T);
}
template <typename T>
__device__ __forceinline__ void stage_tile32x64(T* buf, const T* A, int ld, int n, int r0, int nr, int c0, int lane) {
  constexpr int EPC = 16 / sizeof(T);  // elements per 16-byte chunk
  if (lane < nr && c0 >= 0) {
    const T* rp = A + (int64_t)(r0 + lane) * ld + c0;
    T* dp = buf + lane * stage_stride<T>();
#pragma unroll
    for (int j = 0; j < 64 / EPC; ++j) {
      int bytes = (n - c0 - j * EPC) * (int)sizeof(T);
      bytes = bytes < 0 ? 0 : (bytes > 16 ? 16 : bytes);
      const unsigned sa = (unsigned)__cvta_generic_to_shared(dp + j * EPC);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(bytes ? rp + j * EPC : rp),
                   "r"(bytes));
    }
  }
  asm volatile("cp.async.commit_group;\n" ::);
}
__device__ __forceinline__ void wait_staged() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncwarp();
}

// Dense tail solves, y <- U^-1 L^-1 y on 32-wide block columns, pipelined.
// In step k of the forward pass warp 0 applies block k's solution x_k to
// the 32 rows of block k+1 and solves block k+1's diagonal block (from a
// 32 x 64 tile [L(k+1,k) | L(k+1,k+1)] staged one step ahead), while warps
// 1..7 apply x_k to every row below block k+1; one barrier per step.  The
// backward pass mirrors it (rows above, U, reciprocal pivots computed per
// lane).  x alternates between two 32-entry buffers in s_blk[0..63].
template <typename T>
__device__ __noinline__ void dense_solves(const T* __restrict__ A, int n, int ld, T* __restrict__ yg, T* s_blk, T* ys,
                                          T* sbuf) {
  constexpr int SS = stage_stride<T>();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (ys != yg) {
    for (int i = tid; i < n; i += BS) ys[i] = yg[i];
    __syncthreads();
  }
  const int nblk = (n + 31) / 32;
  // ---- forward, unit lower ----
  // prologue: solve block 0 (tile = [L(0,0) | ...], diagonal at column 0)
  if (warp == 0) {
    stage_tile32x64<T>(sbuf, A, ld, n, 0, min(32, n), 0, lane);
    wait_staged();
    const int cb = min(32, n);
    T v = lane < cb ? ys[lane] : T(0);
    const T* dr = sbuf + lane * SS;
#pragma unroll
    for (int c = 0; c < 32; ++c) {
      const T a = (lane < cb && c < lane) ? dr[c] : T(0);
      v = fma(-a, __shfl_sync(0xffffffffu, v, c), v);
    }
    if (lane < cb) ys[lane] = v;
    s_blk[lane] = lane < cb ? v : T(0);
    __syncwarp();
    // tile of block 1: [L(1,0) | L(1,1)]
    if (nblk > 1) stage_tile32x64<T>(sbuf, A, ld, n, 32, min(32, n - 32), 0, lane);
  }
  __syncthreads();
  for (int k = 0; k + 1 < nblk; ++k) {
    const int c0 = 32 * k;           // block k columns
    const int r1 = c0 + 32;          // block k+1 rows
    const int nb1 = min(32, n - r1);
    const T* xk = s_blk + 32 * (k & 1);
    T* xn = s_blk + 32 * ((k + 1) & 1);
    if (warp == 0) {
      wait_staged();
      const T* tr = sbuf + lane * SS;  // row r1 + lane: [L(k+1,k) | L(k+1,k+1)]
      T v = T(0);
      if (lane < nb1) {
        T acc0 = T(0), acc1 = T(0);
#pragma unroll
        for (int c = 0; c < 32; c += 2) {
          acc0 = fma(tr[c], xk[c], acc0);
          acc1 = fma(tr[c + 1], xk[c + 1], acc1);
        }
        v = ys[r1 + lane] - (acc0 + acc1);
      }
#pragma unroll
      for (int c = 0; c < 32; ++c) {
        const T a = (lane < nb1 && c < lane) ? tr[32 + c] : T(0);
        v = fma(-a, __shfl_sync(0xffffffffu, v, c), v);
      }
      if (lane < nb1) ys[r1 + lane] = v;
      xn[lane] = lane < nb1 ? v : T(0);
      __syncwarp();  // every lane has read the tile before it is refilled
      if (k + 2 < nblk) stage_tile32x64<T>(sbuf, A, ld, n, r1 + 32, min(32, n - r1 - 32), r1, lane);
    } else {
      // rows below block k+1 take x_k (warps 1..7)
      const int t = tid - 32;
      for (int i = r1 + 32 + t; i < n; i += BS - 32) {
        const T* row = A + (int64_t)i * ld + c0;
        T acc0 = T(0), acc1 = T(0), acc2 = T(0), acc3 = T(0);
        if constexpr (sizeof(T) == 4) {
          const float4* r4 = reinterpret_cast<const float4*>(row);
#pragma unroll
          for (int q = 0; q < 8; q += 2) {
            const float4 u = r4[q], w = r4[q + 1];
            acc0 = fma(u.x, xk[4 * q], acc0);
            acc1 = fma(u.y, xk[4 * q + 1], acc1);
            acc2 = fma(u.z, xk[4 * q + 2], acc2);
            acc3 = fma(u.w, xk[4 * q + 3], acc3);
            acc0 = fma(w.x, xk[4 * q + 4], acc0);
            acc1 = fma(w.y, xk[4 * q + 5], acc1);
            acc2 = fma(w.z, xk[4 * q + 6], acc2);
            acc3 = fma(w.w, xk[4 * q + 7], acc3);
          }
        } else {
          const double2* r2 = reinterpret_cast<const double2*>(row);
#pragma unroll
          for (int q = 0; q < 16; q += 2) {
            const double2 u = r2[q], w = r2[q + 1];
            acc0 = fma(u.x, xk[2 * q], acc0);
            acc1 = fma(u.y, xk[2 * q + 1], acc1);
            acc2 = fma(w.x, xk[2 * q + 2], acc2);
            acc3 = fma(w.y, xk[2 * q + 3], acc3);
          }
        }
        ys[i] -= (acc0 + acc1) + (acc2 + acc3);
      }
    }
    __syncthreads();
  }
  // ---- backward, upper ----
  // tile of block j: rows 32j.., columns 32j..32j+63 = [U(j,j) | U(j,j+1)]
  const int kl = nblk - 1;
  if (warp == 0) {
    const int c0 = 32 * kl, cb = n - c0;
    stage_tile32x64<T>(sbuf, A, ld, n, c0, cb, c0, lane);
    wait_staged();
    const T* dr = sbuf + lane * SS;
    const T rd = lane < cb ? T(1) / dr[lane] : T(1);
    T v = lane < cb ? ys[c0 + lane] : T(0);
#pragma unroll
    for (int c = 31; c >= 0; --c) {
      const T xc = __shfl_sync(0xffffffffu, v * rd, c);
      if (lane == c) v = xc;
      else if (lane < c) v = fma(-((lane < cb && c < cb) ? dr[c] : T(0)), xc, v);
    }
    if (lane < cb) ys[c0 + lane] = v;
    s_blk[32 * (kl & 1) + lane] = lane < cb ? v : T(0);  // no stale entries past cb
    __syncwarp();
    if (kl > 0) stage_tile32x64<T>(sbuf, A, ld, n, c0 - 32, 32, c0 - 32, lane);
  }
  __syncthreads();
  for (int k = kl; k > 0; --k) {
    const int c0 = 32 * k;        // block k columns (solved)
    const int cb = min(32, n - c0);
    const int r1 = c0 - 32;       // block k-1 rows
    const T* xk = s_blk + 32 * (k & 1);
    T* xn = s_blk + 32 * ((k - 1) & 1);
    if (warp == 0) {
      wait_staged();
      const T* tr = sbuf + lane * SS;  // row r1 + lane: [U(k-1,k-1) | U(k-1,k)]
      T acc0 = T(0), acc1 = T(0);
#pragma unroll
      for (int c = 0; c < 32; c += 2) {
        if (c < cb) acc0 = fma(tr[32 + c], xk[c], acc0);
        if (c + 1 < cb) acc1 = fma(tr[33 + c], xk[c + 1], acc1);
      }
      T v = ys[r1 + lane] - (acc0 + acc1);
      const T rd = T(1) / tr[lane];
#pragma unroll
      for (int c = 31; c >= 0; --c) {
        const T xc = __shfl_sync(0xffffffffu, v * rd, c);
        if (lane == c) v = xc;
        else if (lane < c) v = fma(-tr[c], xc, v);
      }
      ys[r1 + lane] = v;
      xn[lane] = v;
      __syncwarp();
      if (k - 1 > 0) stage_tile32x64<T>(sbuf, A, ld, n, r1 - 32, 32, r1 - 32, lane);
    } else {
      // rows above block k-1 take x_k (warps 1..7)
      const int t = tid - 32;
      for (int i = t; i < r1; i += BS - 32) {
        const T* row = A + (int64_t)i * ld + c0;
        T acc = T(0);
        if (cb == 32) {
          T acc1 = T(0), acc2 = T(0), acc3 = T(0);
          if constexpr (sizeof(T) == 4) {
            const float4* r4 = reinterpret_cast<const float4*>(row);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
              const float4 u = r4[q];
              acc = fma(u.x, xk[4 * q], acc);
              acc1 = fma(u.y, xk[4 * q + 1], acc1);
              acc2 = fma(u.z, xk[4 * q + 2], acc2);
              acc3 = fma(u.w, xk[4 * q + 3], acc3);
            }
          } else {
            const double2* r2 = reinterpret_cast<const double2*>(row);
#pragma unroll
            for (int q = 0; q < 16; q += 2) {
              const double2 u = r2[q], w = r2[q + 1];
              acc = fma(u.x, xk[2 * q], acc);
              acc1 = fma(u.y, xk[2 * q + 1], acc1);
              acc2 = fma(w.x, xk[2 * q + 2], acc2);
              acc3 = fma(w.y, xk[2 * q + 3], acc3);
            }
          }
          acc = (acc + acc1) + (acc2 + acc3);
        } else {
          for (int c = 0; c < cb; ++c) acc = fma(row[c], xk[c], acc);
        }
        ys[i] -= acc;
      }
    }
    __syncthreads();
  }
  if (ys != yg) {
    for (int i = tid; i < n; i += BS) yg[i] = ys[i];
    __syncthreads();
  }
}

// Whether a row keeps its current factor (an earlier iterate's, or the base
// case's) for one more step: the mismatch must contract by at least `ratio`
// per step and the factor must have served fewer than max_reuse steps.  Once
// BUDGET_STEPS or fewer steps are left (Newton from a near iterate needs
// about that many), the observed contraction rate -- settled by then -- held
// for the remaining steps must also reach tol: a chord that cannot converge
// in time is left for the row's own LU now, rather than after the budget is
// spent and the row has to be rescued.
constexpr int BUDGET_STEPS = 3;

__device__ __forceinline__ bool keep_factor(double nrm, double last, double ratio, int since, int max_reuse, int it,
                                            int max_iter, double tol) {
  if (!(nrm <= ratio * last) || since >= max_reuse) return false;
  if (max_iter - it <= BUDGET_STEPS && last < INFINITY && last > 0.0) {
    const double rho = nrm / last;
    if (rho > 0.0 && nrm * pow(rho, (double)(max_iter - it)) > tol) return false;
  }
  return true;
}

// Per-phase SM cycles, recorded by thread 0 of each CTA at the block-wide
// barriers that separate the phases, summed over CTAs at exit.
struct PhaseProf {
  unsigned long long acc[N_PHASES];
  long long t;
  bool on;
  __device__ void init(bool enabled) {
    on = enabled;
#pragma unroll
    for (int q = 0; q < N_PHASES; ++q) acc[q] = 0;
    t = clock64();
  }
  __device__ __forceinline__ void start() {
    if (on) t = clock64();
  }
  __device__ __forceinline__ void mark(int ph) {
    if (on) {
      const long long now = clock64();
      acc[ph] += (unsigned long long)(now - t);
      t = now;
    }
  }
  __device__ void flush(unsigned long long* out) {
    if (!on) return;
#pragma unroll
    for (int q = 0; q < N_PHASES; ++q) atomicAdd(out + q, acc[q]);
  }
};

__host__ __device__ __forceinline__ int64_t align256(int64_t x) { return (x + 255) & ~int64_t(255); }

constexpr int MAX_COMP = 16;  // compensated Jacobian positions per row (base_chord)

struct WsLayout {
  int64_t V, I, F, HV, S, y, M, total;
};

template <typename T>
__host__ __device__ WsLayout ws_layout(const DevPlan& P) {
  WsLayout w;
  int64_t o = 0;
  w.V = o; o = align256(o + (int64_t)P.n_bus * 16);
  w.I = o; o = align256(o + (int64_t)P.n_bus * 16);
  w.F = o; o = align256(o + (int64_t)P.dim * 8);
  w.HV = o; o = align256(o + (int64_t)P.n_hv * sizeof(T));
  w.S = o; o = align256(o + (int64_t)P.nt * P.ld * sizeof(T));
  w.y = o; o = align256(o + (int64_t)P.dim * sizeof(T));
  w.M = o; o = align256(o + (int64_t)((P.n_bus + 31) / 32) * 4);  // masked-bus bitmap
  w.total = o;
  return w;
}

// y_t <- Sinv y_t with an explicit inverse of the dense tail, column j at
// Sinv + j * ld (nt rows): one parallel product instead of the serial block
// chain of the triangular solves.  ys holds the input copy of y_t (shared
// memory); each thread owns up to four rows per pass, and for each column a
// warp reads 32 consecutive entries.
template <typename T>
__device__ __forceinline__ void tail_inverse_product(const T* Sinv, int64_t ld, int nt, const T* ys, T* yt) {
  const int tid = threadIdx.x;
  for (int r0 = 0; r0 < nt; r0 += 4 * BS) {
    T acc[4] = {T(0), T(0), T(0), T(0)};
    const T* base = Sinv + r0 + tid;
    const int nr = min(4, (nt - r0 - tid + BS - 1) / BS);  // rows of this thread in the pass (may be <= 0)
#pragma unroll 4
    for (int j = 0; j < nt; ++j) {
      const T yj = ys[j];
      const T* col = base + (int64_t)j * ld;
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (u < nr) acc[u] = fma(col[u * BS], yj, acc[u]);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (u < nr) yt[r0 + tid + u * BS] = acc[u];
  }
}

// y <- (LU)^-1 y with a factor (head values fHV, dense tail fS): forward
// over the head levels, the tail rows against the head, the dense tail
// forward + backward, backward over the head levels.  With Minv (the
// factor's explicit inverse, column c at Minv + c * dim, in the plan's
// ordering) the dense tail is applied as a product with its tail block,
// which is the inverse of the dense Schur complement.
template <typename T>
__device__ __forceinline__ void apply_factor(const DevPlan& P, const T* fHV, const T* fS, T* y, T* s_blk, T* s_dense,
                                             PhaseProf& prof, const T* Minv = nullptr) {
  const int tid = threadIdx.x;
  for (int lv = 0; lv < P.n_levels; ++lv) {
    for (int q0 = P.lev_piv_ptr[lv] + tid; q0 < P.lev_piv_ptr[lv + 1]; q0 += BS) {
      const int i = P.lev_piv[q0];
      T acc = y[i];
      for (int q = P.fw_ptr[i]; q < P.fw_ptr[i + 1]; ++q) acc -= fHV[P.fw_pos[q]] * y[P.fw_col[q]];
      y[i] = acc;
    }
    __syncthreads();
  }
  prof.mark(PH_SOLVE);
  for (int ti = tid; ti < P.nt; ti += BS) {
    const int i = P.p + ti;
    T acc = y[i];
    for (int q = P.fw_ptr[i]; q < P.fw_ptr[i + 1]; ++q) acc -= fHV[P.fw_pos[q]] * y[P.fw_col[q]];
    y[i] = acc;
  }
  __syncthreads();
  prof.mark(PH_SOLVE_TAIL);
  if (P.nt > 0 && Minv != nullptr && P.nt <= dense_smem_elems<T>()) {
    for (int i = tid; i < P.nt; i += BS) s_dense[i] = y[P.p + i];
    __syncthreads();
    tail_inverse_product<T>(Minv + (int64_t)P.p * P.dim + P.p, P.dim, P.nt, s_dense, y + P.p);
    __syncthreads();
  } else if (P.nt > 0)
  {
    // y tail in shared memory when it fits, the diagonal-block buffer after it
    const bool y_in_smem = P.nt + 32 * stage_stride<T>() + 32 <= dense_smem_elems<T>();
    T* ys = y_in_smem ? s_dense : y + P.p;
    T* sbuf = s_dense + (y_in_smem ? ((P.nt + 31) & ~31) : 0);
    dense_solves<T>(fS, P.nt, P.ld, y + P.p, s_blk, ys, sbuf);
  }
  prof.mark(PH_SOLVE_DENSE);
  for (int lv = P.n_levels - 1; lv >= 0; --lv) {
    for (int q0 = P.lev_piv_ptr[lv] + tid; q0 < P.lev_piv_ptr[lv + 1]; q0 += BS) {
      const int k = P.lev_piv[q0];
      T acc = y[k];
      for (int q = P.bw_ptr[k]; q < P.bw_ptr[k + 1]; ++q) acc -= fHV[P.bw_pos[q]] * y[P.bw_row[q]];
      y[k] = acc / fHV[k];
    }
    __syncthreads();
  }

  prof.mark(PH_SOLVE_BACK);
}

// Shared-memory scratch of one CTA, handed to solve_row.
template <typename T>
struct RowShared {
  int* s_ne;
  int* s_ek;
  double2* s_ev;
  double* s_red;
  T* s_blk;
  T* s_dense;
  // outage compensation on the base factor (see setup_compensation)
  int* s_cr;      // [1 + MAX_COMP]: r, then the compensated positions
  double* s_cB;   // [MAX_COMP^2] Delta J on those positions (row-major)
  double* s_cLU;  // [MAX_COMP^2] LU of I + W B (partial pivoting)
  int* s_cpiv;    // [MAX_COMP]
  double* s_cw;   // [MAX_COMP]
};

// One Jacobian entry pair of Ybus entry (i, j) with value yk at voltages
// Vi, Vj and current Ii (the J-fill formulas): out = {dP/dtheta_j,
// dP/dVm_j, dQ/dtheta_j, dQ/dVm_j}.
__device__ __forceinline__ void jac_entry(bool diag, double2 yk, double2 Vi, double2 Vj, double2 Ii, double out[4]) {
  double2 dVa, dVm;
  if (diag) {
    const double2 t = cmul(Vi, conj2(csub(Ii, cmul(yk, Vi))));
    dVa = make_double2(-t.y, t.x);
    const double inv = 1.0 / hypot(Vi.x, Vi.y);
    const double2 vn = make_double2(Vi.x * inv, Vi.y * inv);
    dVm = cadd(cmul(Vi, conj2(cmul(yk, vn))), cmul(conj2(Ii), vn));
  } else {
    const double2 t = cmul(Vi, conj2(cmul(yk, Vj)));
    dVa = make_double2(t.y, -t.x);
    const double inv = 1.0 / hypot(Vj.x, Vj.y);
    const double2 vn = make_double2(Vj.x * inv, Vj.y * inv);
    dVm = cmul(Vi, conj2(cmul(yk, vn)));
  }
  out[0] = dVa.x;
  out[1] = dVm.x;
  out[2] = dVa.y;
  out[3] = dVm.y;
}

// ||F||inf of the row (row-patched Ybus, its Sbus) at voltage Vx, NaN-sticky,
// without touching the row's workspace
__device__ __noinline__ double mismatch_norm(const DevPlan P, const RowEdits ed, const double2* Y, const double2* Vx,
                                             const double2* sb, double* s_red) {
  double lmax = 0.0;
  for (int i = threadIdx.x; i < P.n_bus; i += BS) {
    double2 acc = make_double2(0.0, 0.0);
    for (int k = P.y_indptr[i]; k < P.y_indptr[i + 1]; ++k) {
      const double2 yk = ed.apply(k, Y[k]);
      const double2 vj = Vx[P.y_indices[k]];
      acc.x = fma(yk.x, vj.x, fma(-yk.y, vj.y, acc.x));
      acc.y = fma(yk.x, vj.y, fma(yk.y, vj.x, acc.y));
    }
    const double2 s = csub(cmul(Vx[i], conj2(acc)), sb[i]);
    if (P.fP[i] >= 0) lmax = (isnan(s.x) || isnan(lmax)) ? NAN : fmax(lmax, fabs(s.x));
    if (P.fQ[i] >= 0) lmax = (isnan(s.y) || isnan(lmax)) ? NAN : fmax(lmax, fabs(s.y));
  }
  return block_nanmax(lmax, s_red);
}

// The same norm at the alternative start Va without a sparse product: Sa =
// Va conj(Y Va) on the unedited Ybus is shared by all rows, and a row's
// edits change S only at the buses of the edited Ybus rows, by
// Va_i conj(dY_k Va_j) per edited entry k = (i, j).
__device__ __noinline__ double alt_mismatch_norm(const DevPlan P, const RowEdits ed, const double2* Va,
                                                 const double2* Sa, const double2* sb, double* s_red) {
  double lmax = 0.0;
  for (int i = threadIdx.x; i < P.n_bus; i += BS) {
    double2 s = csub(Sa[i], sb[i]);
    for (int e = 0; e < ed.n; ++e) {
      const int k = ed.k[e];
      if (P.y_row[k] != i) continue;
      // edits subtract ed.v[e] from Y_k
      s = csub(s, cmul(Va[i], conj2(cmul(ed.v[e], Va[P.y_indices[k]]))));
    }
    if (P.fP[i] >= 0) lmax = (isnan(s.x) || isnan(lmax)) ? NAN : fmax(lmax, fabs(s.x));
    if (P.fQ[i] >= 0) lmax = (isnan(s.y) || isnan(lmax)) ? NAN : fmax(lmax, fabs(s.y));
  }
  return block_nanmax(lmax, s_red);
}

// Outage compensation (policy 2, rows with Ybus edits).  The chord matrix of
// a row is its Jacobian at the base voltage Vb, M = M0 + E B E^T, where M0 is
// the base factor and B = Delta J is confined to the P/Q rows and theta/Vm
// columns of the buses the edits touch (positions R, r <= MAX_COMP).  With
// Z = M0^-1 E -- columns R of the base inverse Minv, computed once per
// session (inverse mode of the sweep) -- and W = E^T Z, Woodbury gives
//   M^-1 F = x0 - Z B (I + W B)^-1 x0[R],   x0 = M0^-1 F.
// Returns false (no compensation) when the row touches too many positions.
// Run by a CTA of NT threads.
template <typename T, int NT = BS>
__device__ __noinline__ bool setup_compensation(const DevPlan P, const RowEdits ed, const double2* Y,
                                                const double2* Vb, const T* Minv, const RowShared<T> sh) {
  const int tid = threadIdx.x;
  int* R = sh.s_cr + 1;
  if (tid == 0) {
    int r = 0;
    bool ok = true;
    auto add = [&](int pos) {
      if (pos < 0) return;
      for (int q = 0; q < r; ++q)
        if (R[q] == pos) return;
      if (r < MAX_COMP) R[r++] = pos;
      else ok = false;
    };
    for (int e = 0; e < ed.n; ++e) {
      const int k = ed.k[e];
      const int i = P.y_row[k], j = P.y_indices[k];
      add(P.fP[i]);
      add(P.fQ[i]);
      add(P.fP[j]);
      add(P.fQ[j]);
    }
    sh.s_cr[0] = ok ? r : -1;
    // B = J(Vb, Y_row) - J(Vb, Y_base) on R x R: rows of the edited buses
    if (ok) {
      for (int q = 0; q < r * r; ++q) sh.s_cB[q] = 0.0;
      auto slot = [&](int pos) {
        for (int q = 0; q < r; ++q)
          if (R[q] == pos) return q;
        return -1;
      };
      for (int e = 0; e < ed.n; ++e) {
        const int i = P.y_row[ed.k[e]];
        bool seen = false;
        for (int e2 = 0; e2 < e; ++e2) seen |= P.y_row[ed.k[e2]] == i;
        if (seen) continue;  // each edited row once
        double2 Ib = make_double2(0.0, 0.0), Ir = make_double2(0.0, 0.0);
        for (int k = P.y_indptr[i]; k < P.y_indptr[i + 1]; ++k) {
          const double2 vj = Vb[P.y_indices[k]];
          Ib = cadd(Ib, cmul(Y[k], vj));
          Ir = cadd(Ir, cmul(ed.apply(k, Y[k]), vj));
        }
        const int rp = slot(P.fP[i]), rq = slot(P.fQ[i]);
        for (int k = P.y_indptr[i]; k < P.y_indptr[i + 1]; ++k) {
          const int j = P.y_indices[k];
          const int cp = slot(P.fP[j]), cq = slot(P.fQ[j]);
          if (cp < 0 && cq < 0) continue;
          double jb[4], jr[4];
          jac_entry(i == j, Y[k], Vb[i], Vb[j], Ib, jb);
          jac_entry(i == j, ed.apply(k, Y[k]), Vb[i], Vb[j], Ir, jr);
          const int rows[4] = {rp, rp, rq, rq}, cols[4] = {cp, cq, cp, cq};
          for (int q = 0; q < 4; ++q)
            if (rows[q] >= 0 && cols[q] >= 0) sh.s_cB[rows[q] * r + cols[q]] += jr[q] - jb[q];
        }
      }
    }
  }
  __syncthreads();
  const int r = sh.s_cr[0];
  if (r <= 0) return false;
  // C = I + W B, W[a][c] = Z_c[R[a]] = Minv[R[c]][R[a]], one entry per thread
  double* C = sh.s_cLU;
  for (int q = tid; q < r * r; q += NT) {
    const int i2 = q / r, j2 = q % r;
    double acc = i2 == j2 ? 1.0 : 0.0;
    for (int c = 0; c < r; ++c) acc += (double)Minv[(int64_t)R[c] * P.dim + R[i2]] * sh.s_cB[c * r + j2];
    C[q] = acc;
  }
  __syncthreads();
  // its LU with partial pivoting
  if (tid == 0) {
    for (int k = 0; k < r; ++k) {
      int pk = k;
      for (int i2 = k + 1; i2 < r; ++i2)
        if (fabs(C[i2 * r + k]) > fabs(C[pk * r + k])) pk = i2;
      sh.s_cpiv[k] = pk;
      if (pk != k)
        for (int j2 = 0; j2 < r; ++j2) {
          const double t = C[k * r + j2];
          C[k * r + j2] = C[pk * r + j2];
          C[pk * r + j2] = t;
        }
      const double d = C[k * r + k];
      for (int i2 = k + 1; i2 < r; ++i2) {
        const double l = C[i2 * r + k] / d;
        C[i2 * r + k] = l;
        for (int j2 = k + 1; j2 < r; ++j2) C[i2 * r + j2] -= l * C[k * r + j2];
      }
    }
  }
  __syncthreads();
  return true;
}

// A row's outage compensation as setup_compensation leaves it in shared
// memory, kept in global memory for the chord sweep: every row's record is
// set up by one launch ahead of the sweep (comp_setup_kernel, all rows in
// parallel), and the sweep's refill copies the record instead of building it
// on one thread of the CTA.  Rows touching more than COMP_REC positions
// (r = COMP_REC_NONE) build theirs in the sweep as before.
constexpr int COMP_REC = 8;
constexpr int COMP_REC_NONE = -2;
struct CompRec {
  int r;  // compensated positions; <= 0: none; COMP_REC_NONE: set up in the sweep
  int R[COMP_REC];
  int piv[COMP_REC];
  double B[COMP_REC * COMP_REC];   // row-major r x r
  double LU[COMP_REC * COMP_REC];  // row-major r x r
};

// One 32-thread CTA per session row: the row's edits as the chord refill
// takes them (the first MAX_EDITS), setup_compensation (the same arithmetic
// in the same order, so the record equals what the refill would compute),
// then the record.
template <typename T>
__global__ void __launch_bounds__(32) comp_setup_kernel(const DevPlan P, const SweepArgs a, CompRec* rec) {
  __shared__ int s_ek[MAX_EDITS];
  __shared__ double2 s_ev[MAX_EDITS];
  __shared__ int s_cr[1 + MAX_COMP];
  __shared__ double s_cB[MAX_COMP * MAX_COMP];
  __shared__ double s_cLU[MAX_COMP * MAX_COMP];
  __shared__ int s_cpiv[MAX_COMP];
  __shared__ int s_ne;
  const int row = blockIdx.x;
  const int tid = threadIdx.x;
  if (tid == 0) {
    const int e0 = a.edit_ptr[row], e1 = a.edit_ptr[row + 1];
    const int ne = min(e1 - e0, MAX_EDITS);
    for (int e = 0; e < ne; ++e) {
      s_ek[e] = a.edit_k[e0 + e];
      s_ev[e] = reinterpret_cast<const double2*>(a.edit_val)[e0 + e];
    }
    s_ne = ne;
  }
  __syncthreads();
  CompRec* out = rec + row;
  if (s_ne == 0) {
    if (tid == 0) out->r = 0;
    return;
  }
  const RowEdits ed{s_ne, s_ek, s_ev};
  const RowShared<T> sh{&s_ne, s_ek, s_ev, nullptr, nullptr, nullptr, s_cr, s_cB, s_cLU, s_cpiv, nullptr};
  const bool c = setup_compensation<T, 32>(P, ed, reinterpret_cast<const double2*>(a.ybus),
                                           reinterpret_cast<const double2*>(a.base_v),
                                           reinterpret_cast<const T*>(a.base_inv), sh);
  const int r = s_cr[0];
  if (!c) {
    if (tid == 0) out->r = 0;
    return;
  }
  if (r > COMP_REC) {
    if (tid == 0) out->r = COMP_REC_NONE;
    return;
  }
  if (tid == 0) out->r = r;
  for (int q = tid; q < r; q += 32) {
    out->R[q] = s_cr[1 + q];
    out->piv[q] = s_cpiv[q];
  }
  for (int q = tid; q < r * r; q += 32) {
    out->B[q] = s_cB[q];
    out->LU[q] = s_cLU[q];
  }
}

// The refill's copy of a record into the slot's shared arrays (every thread
// of the CTA); returns whether the row is compensated, or -1 when the record
// says to set it up in the sweep.
__device__ __forceinline__ int load_compensation(const CompRec* rec, int* s_cr, double* s_cB, double* s_cLU,
                                                 int* s_cpiv) {
  const int r = rec->r;
  if (r == COMP_REC_NONE) return -1;
  if (r <= 0) return 0;
  if (threadIdx.x == 0) s_cr[0] = r;
  for (int q = threadIdx.x; q < r; q += BS) {
    s_cr[1 + q] = rec->R[q];
    s_cpiv[q] = rec->piv[q];
  }
  for (int q = threadIdx.x; q < r * r; q += BS) {
    s_cB[q] = rec->B[q];
    s_cLU[q] = rec->LU[q];
  }
  __syncthreads();
  return 1;
}

// y <- y - Z B (I + W B)^-1 y[R]  (see setup_compensation)
template <typename T>
__device__ __noinline__ void apply_compensation(int dim, T* y, const T* Minv, const RowShared<T> sh,
                                                const int stride = 1) {
  const int tid = threadIdx.x;
  const int r = sh.s_cr[0];
  const int* R = sh.s_cr + 1;
  if (tid == 0) {
    double v[MAX_COMP];
    for (int q = 0; q < r; ++q) v[q] = (double)y[(int64_t)R[q] * stride];
    const double* C = sh.s_cLU;
    for (int k = 0; k < r; ++k) {  // P v, then L, then U
      const int pk = sh.s_cpiv[k];
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
      for (int c = 0; c < r; ++c) acc += sh.s_cB[q * r + c] * v[c];
      sh.s_cw[q] = acc;
    }
  }
  __syncthreads();
  for (int i = tid; i < dim; i += BS) {
    T acc = T(0);
    for (int c = 0; c < r; ++c) acc += Minv[(int64_t)R[c] * dim + i] * (T)sh.s_cw[c];
    y[(int64_t)i * stride] -= acc;
  }
  __syncthreads();
}

// Branch flows and the limit check of one row as it leaves, by the row's
// own CTA on the V it still holds (the reference's compute_branch_flows +
// check_limit_violations passes): per branch loading = max(|S_from|, |S_to|)
// / rate (0 for tripped or unlimited branches, NaN when not converged), the
// number of branches above 1 and the largest loading.
__device__ __noinline__ void row_flows(const SweepArgs a, const int row, const double2* V, const bool ok,
                                       double* s_red) {
  const int tid = threadIdx.x;
  const int q0 = a.trip_ptr != nullptr ? a.trip_ptr[row] : 0;
  const int q1 = a.trip_ptr != nullptr ? a.trip_ptr[row + 1] : 0;
  double lmax = 0.0;
  int nv = 0;
  for (int l = tid; l < a.n_branch; l += BS) {
    float ld = NAN;
    if (ok) {
      bool tripped = false;
      for (int q = q0; q < q1; ++q) tripped |= a.trip_ids[q] == l;
      ld = 0.f;
      if (!tripped && a.br_rate[l] > 0.0) {
        const double2* yb = reinterpret_cast<const double2*>(a.br_y) + 4 * (int64_t)l;
        // an open end (negative endpoint) has V = 0 and carries no power
        // (acpf_nr_kernels.cu:87-183)
        const int bf = a.br_from[l], bt = a.br_to[l];
        const double2 zero = make_double2(0.0, 0.0);
        const double2 Vf = bf >= 0 ? V[bf] : zero, Vt = bt >= 0 ? V[bt] : zero;
        const double2 Sf = bf >= 0 ? cmul(Vf, conj2(cadd(cmul(yb[0], Vf), cmul(yb[1], Vt)))) : zero;
        const double2 St = bt >= 0 ? cmul(Vt, conj2(cadd(cmul(yb[2], Vf), cmul(yb[3], Vt)))) : zero;
        const double r = fmax(hypot(Sf.x, Sf.y), hypot(St.x, St.y)) / a.br_rate[l];
        ld = (float)r;
        // a branch at a masked (NaN) bus has no flow to report: NaN, not counted
        if (!isnan(r)) {
          lmax = fmax(lmax, r);
          nv += r > 1.0;
        }
      }
    }
    a.loading_out[(int64_t)row * a.n_branch + l] = ld;
  }
  lmax = block_nanmax(lmax, s_red);
  const double nv_all = block_sum(double(nv), s_red);
  if (tid == 0) {
    a.nviol_out[row] = ok ? (int)nv_all : -1;
    a.maxload_out[row] = ok ? (float)lmax : NAN;
  }
}

// Outputs of a row that is not simulated (its outage islands the grid).
__device__ __noinline__ void skip_row_outputs(const SweepArgs a, const int row, const int n) {
  const int tid = threadIdx.x;
  double2* vout = reinterpret_cast<double2*>(a.v_out) + (int64_t)row * n;
  for (int i = tid; i < n; i += BS) vout[i] = make_double2(NAN, NAN);
  if (a.v_mirror != nullptr) {
    double2* vm = reinterpret_cast<double2*>(a.v_mirror) + (int64_t)row * n;
    for (int i = tid; i < n; i += BS) vm[i] = make_double2(NAN, NAN);
  }
  if (a.loading_out != nullptr) {
    for (int l = tid; l < a.n_branch; l += BS) a.loading_out[(int64_t)row * a.n_branch + l] = NAN;
    if (tid == 0) {
      a.nviol_out[row] = -1;
      a.maxload_out[row] = NAN;
    }
  }
  if (tid == 0) {
    a.res_out[row] = NAN;
    a.status_out[row] = ROW_NOT_SIMULATED;
    a.iters_out[row] = 0;
    if (a.factors_out != nullptr) a.factors_out[row] = 0;
  }
  __syncthreads();
}

// The whole Newton loop of one row of one grid, by the calling CTA: start
// voltage, edits, mismatch / Jacobian / factorization / solves / update
// until the row converges, diverges or uses its budget (with the optional
// rescue attempt), then the row's outputs.  ws: the CTA's workspace.
// A row id with this bit set (rows handed off by the chord sweep) is not
// rescued: it already began from the rescue voltage.
constexpr int NO_RESCUE_BIT = 1 << 30;

// A row solved by the leading CTA of a cluster whose other CTAs join its
// dense tail LU (sweep_kernel_cluster): the command word the leader posts in
// its shared memory, and the cluster size.
constexpr int CLUSTER_CMD_LU = 1, CLUSTER_CMD_DONE = 2;
struct ClusterLu {
  int* cmd;
  int parts;
};

template <typename T>
__device__ __forceinline__ void solve_row(const DevPlan& P, const SweepArgs& a, const int row_arg, char* ws,
                                          const RowShared<T>& sh, PhaseProf& prof, const ClusterLu* cl = nullptr) {
  const int tid = threadIdx.x;
  const int row = row_arg & ~NO_RESCUE_BIT;
  // a row that began from the rescue voltage (the base V, chosen by start
  // selection) is not restarted from it
  bool from_rescue_v = (row_arg & NO_RESCUE_BIT) != 0;
  const WsLayout L = ws_layout<T>(P);
  double2* V = reinterpret_cast<double2*>(ws + L.V);
  double2* I = reinterpret_cast<double2*>(ws + L.I);
  double* F = reinterpret_cast<double*>(ws + L.F);
  T* HV = reinterpret_cast<T*>(ws + L.HV);
  T* S = reinterpret_cast<T*>(ws + L.S);
  T* y = reinterpret_cast<T*>(ws + L.y);
  const double2* Y = reinterpret_cast<const double2*>(a.ybus);
  const int n = P.n_bus;
  int& s_ne = *sh.s_ne;
  int* s_ek = sh.s_ek;
  double2* s_ev = sh.s_ev;
  double* s_red = sh.s_red;
  T* s_blk = sh.s_blk;
  T* s_dense = sh.s_dense;
  if (a.inverse_out != nullptr) {
    // inverse mode: column `row` of the base factor's inverse (policy 2)
    for (int i = tid; i < P.dim; i += BS) y[i] = T(i == row ? 1 : 0);
    __syncthreads();
    apply_factor<T>(P, reinterpret_cast<const T*>(a.base_ws + L.HV), reinterpret_cast<const T*>(a.base_ws + L.S), y,
                    s_blk, s_dense, prof);
    T* col = reinterpret_cast<T*>(a.inverse_out) + (int64_t)row * P.dim;
    for (int i = tid; i < P.dim; i += BS) col[i] = y[i];
    __syncthreads();
    return;
  }
    double2* vout = reinterpret_cast<double2*>(a.v_out) + (int64_t)row * n;

    if (a.row_skip != nullptr && a.row_skip[row]) {
      skip_row_outputs(a, row, n);
      return;
    }
    if (tid == 0) {
      int ne = 0;
      if (a.edit_ptr != nullptr) {
        const int e0 = a.edit_ptr[row], e1 = a.edit_ptr[row + 1];
        ne = min(e1 - e0, MAX_EDITS);
        for (int e = 0; e < ne; ++e) {
          s_ek[e] = a.edit_k[e0 + e];
          s_ev[e] = reinterpret_cast<const double2*>(a.edit_val)[e0 + e];
        }
      }
      s_ne = ne;
    }
    const double2* v0 = reinterpret_cast<const double2*>(a.v0) + (int64_t)row * a.v0_stride;
    const double2* sb = reinterpret_cast<const double2*>(a.sbus) + (int64_t)row * a.sbus_stride;
    for (int i = tid; i < n; i += BS) V[i] = v0[i];
    // buses outside the row's largest component (handle_disconnected_grid)
    unsigned* mbits = reinterpret_cast<unsigned*>(ws + L.M);
    const bool has_mask = a.mask_ptr != nullptr && a.mask_ptr[row + 1] > a.mask_ptr[row];
    if (has_mask) {
      for (int w = tid; w < (n + 31) / 32; w += BS) mbits[w] = 0u;
      __syncthreads();
      for (int q = a.mask_ptr[row] + tid; q < a.mask_ptr[row + 1]; q += BS) {
        const int b = a.mask_bus[q];
        atomicOr(mbits + (b >> 5), 1u << (b & 31));
      }
    }
    auto masked = [&](int b) { return has_mask && ((mbits[b >> 5] >> (b & 31)) & 1u); };
    __syncthreads();
    const RowEdits ed{s_ne, s_ek, s_ev};
    prof.start();

    int it_total = 0, status = ROW_MAX_ITER, n_factor = 0;
    double nrm = NAN;
    // a masked row starts from its own start on its own factor (start
    // selection and the base factor know nothing of its masked rows)
    bool check_alt = a.alt_v0 != nullptr && !a.fixed_iters && !a.factor_only && !has_mask;
    // attempt 0 starts from the row's own start voltage; with a rescue
    // voltage, a row that ends unconverged there gets one more attempt from
    // it, with a fresh Newton budget (iterations and factorizations add up)
    for (int attempt = 0;; ++attempt) {
    // a row continued from another launch keeps counting its Newton steps
    int it = (attempt == 0 && a.iters_in != nullptr) ? a.iters_in[row] : 0;
    // policy 2 starts on the base case's factor (shared by every CTA, read
    // only) and moves to the row's own factor at its first refactor
    const bool on_base =
        a.refactor_policy == 2 && a.base_ws != nullptr && attempt == 0 && !a.factor_only && !has_mask;
    const T* fHV = on_base ? reinterpret_cast<const T*>(a.base_ws + L.HV) : HV;
    const T* fS = on_base ? reinterpret_cast<const T*>(a.base_ws + L.S) : S;
    bool have_factor = on_base;
    // rows with tripped branches correct the base factor for their outage
    bool comp_on = false;
    const T* Minv = reinterpret_cast<const T*>(a.base_inv);
    if (on_base && ed.n > 0 && a.base_v != nullptr && Minv != nullptr)
      comp_on = setup_compensation<T>(P, ed, Y, reinterpret_cast<const double2*>(a.base_v), Minv, sh);
    int since_factor = 0;
    double last_nrm = INFINITY;
    for (;;) {
      // ---- I = Y V (row-patched Ybus) ------------------------------------
      for (int i = tid; i < n; i += BS) {
        double2 acc = make_double2(0.0, 0.0);
        for (int k = P.y_indptr[i]; k < P.y_indptr[i + 1]; ++k) {
          const double2 yk = ed.apply(k, Y[k]);
          const double2 vj = V[P.y_indices[k]];
          acc.x = fma(yk.x, vj.x, fma(-yk.y, vj.y, acc.x));
          acc.y = fma(yk.x, vj.y, fma(yk.y, vj.x, acc.y));
        }
        I[i] = acc;
      }
      __syncthreads();
      // ---- F = -(V conj(I) - Sbus) at the P/Q rows, NaN-sticky inf-norm ---
      double lmax = 0.0;
      for (int i = tid; i < n; i += BS) {
        const double2 s = csub(cmul(V[i], conj2(I[i])), sb[i]);
        const int fp = P.fP[i], fq = P.fQ[i];
        if (masked(i)) {
          // a masked bus: identity row, zero mismatch, out of the norm
          if (fp >= 0) F[fp] = 0.0;
          if (fq >= 0) F[fq] = 0.0;
          continue;
        }
        if (fp >= 0) {
          F[fp] = -s.x;
          const double ax = fabs(s.x);
          lmax = (isnan(ax) || isnan(lmax)) ? NAN : fmax(lmax, ax);
        }
        if (fq >= 0) {
          F[fq] = -s.y;
          const double ay = fabs(s.y);
          lmax = (isnan(ay) || isnan(lmax)) ? NAN : fmax(lmax, ay);
        }
      }
      nrm = block_nanmax(lmax, s_red);
      if (check_alt) {
        // the row's own start stands only if its mismatch is below the
        // alternative start's (a NaN start never stands)
        check_alt = false;
        const double2* va = reinterpret_cast<const double2*>(a.alt_v0);
        const double na = a.alt_s != nullptr
                              ? alt_mismatch_norm(P, ed, va, reinterpret_cast<const double2*>(a.alt_s), sb, s_red)
                              : mismatch_norm(P, ed, Y, va, sb, s_red);
        if (!(nrm < na) && isfinite(na)) {
          for (int i = tid; i < n; i += BS) V[i] = va[i];
          if (tid == 0 && a.n_alt_start != nullptr) atomicAdd(a.n_alt_start, 1);
          from_rescue_v = a.alt_v0 == a.rescue_v0;
          __syncthreads();
          continue;  // mismatch again at the new start
        }
      }
      prof.mark(PH_MISMATCH);
      const bool finite = isfinite(nrm);
      // single-solve order: this step is taken whatever the mismatch, and the
      // mismatch before it decides convergence afterwards
      bool converged_after_step = false;
      if (a.factor_only) {
        // factor the Jacobian at the start voltage, nothing else
      } else if (a.fixed_iters) {
        // chunked schedule: exactly max_iter steps (a non-finite row keeps
        // stepping), then the residual of the final voltage decides
        if (it >= a.max_iter) {
          status = !finite ? ROW_DIVERGED : (nrm < a.tol ? ROW_CONVERGED : ROW_MAX_ITER);
          break;
        }
      } else if (a.step_first) {
        if (it >= a.max_iter) {
          status = !finite ? ROW_DIVERGED : ROW_MAX_ITER;
          break;
        }
        converged_after_step = nrm < a.tol;
      } else if (!finite && it == 0 && attempt == 0 && a.rescue_v0 != nullptr && !from_rescue_v) {
        // a given start whose mismatch is not finite is no start at all: the
        // row goes to its rescue attempt without a step
        status = ROW_DIVERGED;
        break;
      } else if (it > 0 && it % (a.round_k > 1 ? a.round_k : 1) == 0) {
        // continuous schedule: tested at the end of each round of round_k
        // steps only; a loaded row always runs its first round
        if (!finite) { status = ROW_DIVERGED; break; }
        if (nrm < a.tol) { status = ROW_CONVERGED; break; }
        if (it >= a.max_iter) { status = ROW_MAX_ITER; break; }
      }

      // ---- refactor, or reuse the factor of an earlier iterate ---------------
      // Policy 0 refactors every step (Newton).  Policy 1 keeps the last LU
      // while the mismatch contracts by at least refactor_ratio per step and
      // for at most max_reuse steps (an inexact Newton / chord step: the FP64
      // mismatch still drives the iterate to the same fixed point).  nrm is
      // block-uniform, so the branch is taken by the whole CTA.
      // (the rescue attempt restarts from Vinit, far from the solution: full
      // Newton there)
      const bool refactor = a.factor_only || !have_factor || a.refactor_policy == 0 || attempt > 0 ||
                            !keep_factor(nrm, last_nrm, a.refactor_ratio, since_factor, a.max_reuse, it, a.max_iter,
                                         a.tol);
      last_nrm = nrm;
      if (refactor) {
        have_factor = true;
        since_factor = 0;
        ++n_factor;
      // ---- zero the dense tail, then scatter J ------------------------------
      {
        const int64_t ns = (int64_t)P.nt * P.ld;
        for (int64_t q = tid; q < ns; q += BS) S[q] = T(0);
      }
      __syncthreads();
      for (int k = tid; k < P.nnz_y; k += BS) {
        const int i = P.y_row[k], j = P.y_indices[k];
        const double2 Vi = V[i], Ii = I[i];
        const double2 yk = ed.apply(k, Y[k]);
        double2 dVa, dVm;
        if (i == j) {
          const double2 t = cmul(Vi, conj2(csub(Ii, cmul(yk, Vi))));
          dVa = make_double2(-t.y, t.x);
          const double inv = 1.0 / hypot(Vi.x, Vi.y);
          const double2 vn = make_double2(Vi.x * inv, Vi.y * inv);
          dVm = cadd(cmul(Vi, conj2(cmul(yk, vn))), cmul(conj2(Ii), vn));
        } else {
          const double2 Vj = V[j];
          const double2 t = cmul(Vi, conj2(cmul(yk, Vj)));
          dVa = make_double2(t.y, -t.x);
          const double inv = 1.0 / hypot(Vj.x, Vj.y);
          const double2 vn = make_double2(Vj.x * inv, Vj.y * inv);
          dVm = cmul(Vi, conj2(cmul(yk, vn)));
        }
        double vals[4] = {dVa.x, dVm.x, dVa.y, dVm.y};
        if (masked(i) || masked(j)) {
          // a masked bus's rows are identity rows; live rows see no coupling to it
          const double one = (i == j) ? 1.0 : 0.0;
          vals[0] = one;
          vals[1] = 0.0;
          vals[2] = 0.0;
          vals[3] = one;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int dst = P.jmap[4 * k + q];
          if (dst >= 0) HV[dst] = (T)vals[q];
          else if (dst <= -2) S[-(dst + 2)] = (T)vals[q];
        }
      }
      __syncthreads();

      prof.mark(PH_FILL);
      // ---- sparse head LU, level by level (with a cluster: all its CTAs) ---
      const bool shared_factor = cl != nullptr && P.nt > 0;
      if (shared_factor) {
        // the cluster's other CTAs join: post the command, two barriers
        // (posted; read by all); the head factor's values and the scattered
        // tail are complete before the first of them
        if (tid == 0) *cl->cmd = CLUSTER_CMD_LU;
        dense::cluster_barrier();
        dense::cluster_barrier();
      }
      head_lu<T>(P, HV, a.pivot_floor, 0, shared_factor ? cl->parts : 1);

      prof.mark(PH_HEAD);
      if (shared_factor) {
        // the Schur update split by tail rows (a barrier), then the shared
        // dense factorization
        schur_update<T>(P, HV, S, 0, cl->parts);
        dense::cluster_barrier();
        prof.mark(PH_SCHUR);
        dense_lu_cluster<T>(S, P.nt, P.ld, s_dense, a.pivot_floor, 0, cl->parts);
      } else {
      // ---- Schur update of the dense tail ----------------------------------
      schur_update<T>(P, HV, S);
      __syncthreads();

      prof.mark(PH_SCHUR);
      // ---- dense tail LU --------------------------------------------------
      if (P.nt > 0) dense_lu<T>(S, P.nt, P.ld, s_dense, a.pivot_floor);
      }
      fHV = HV;
      fS = S;
      comp_on = false;
      }  // refactor
      ++since_factor;
      if (a.factor_only) break;

      prof.mark(PH_DENSE);
      // ---- solves -----------------------------------------------------------
      for (int i = tid; i < P.dim; i += BS) y[i] = (T)F[i];
      __syncthreads();
      // rows still on the base factor apply its dense tail through the base inverse
      apply_factor<T>(P, fHV, fS, y, s_blk, s_dense, prof, fHV != HV ? Minv : nullptr);
      if (comp_on) apply_compensation<T>(P.dim, y, Minv, sh);
      // ---- step scaling (MaxVoltageChange, acpf_nr_kernels.cu:677-726) -----
      double alpha = 1.0;
      if (a.step_scaling) {
        double mdt = 0.0, mdv = 0.0;  // fmax skips NaN entries
        for (int i = tid; i < n; i += BS) {
          const int fp = P.fP[i], fq = P.fQ[i];
          if (fp >= 0) mdt = fmax(mdt, fabs((double)y[fp]));
          if (fq >= 0) mdv = fmax(mdv, fabs((double)y[fq]));
        }
        mdt = block_nanmax(mdt, s_red);
        mdv = block_nanmax(mdv, s_red);
        alpha = step_alpha(mdt, mdv, a.max_dva, a.max_dvm);
      }
      // ---- V update (FP64, polar) -----------------------------------------
      for (int i = tid; i < n; i += BS) {
        const int fp = P.fP[i], fq = P.fQ[i];
        if (fp < 0 && fq < 0) continue;
        const double dva = fp >= 0 ? alpha * (double)y[fp] : 0.0;
        const double dvm = fq >= 0 ? alpha * (double)y[fq] : 0.0;
        const double2 v = V[i];
        const double vm = hypot(v.x, v.y) + dvm;
        const double va = atan2(v.y, v.x) + dva;
        double sn, cs;
        sincos(va, &sn, &cs);
        V[i] = make_double2(vm * cs, vm * sn);
      }
      __syncthreads();
      prof.mark(PH_UPDATE);
      ++it;
      if (converged_after_step) {
        status = ROW_CONVERGED;
        break;
      }
    }
    it_total += it;
    // status and attempt are block-uniform: the whole CTA restarts or leaves
    if (status == ROW_CONVERGED || a.fixed_iters || a.rescue_v0 == nullptr || attempt > 0 || from_rescue_v) break;
    const double2* rv = reinterpret_cast<const double2*>(a.rescue_v0);
    for (int i = tid; i < n; i += BS) V[i] = rv[i];
    if (tid == 0 && a.n_rescued != nullptr) atomicAdd(a.n_rescued, 1);
    __syncthreads();
    }  // attempts

    // masked buses are reported NaN (their voltage was frozen, not solved)
    if (has_mask) {
      for (int i = tid; i < n; i += BS)
        if (masked(i)) V[i] = make_double2(NAN, NAN);
      __syncthreads();
    }
    // ---- branch flows and limit check as the row leaves --------------------
    if (a.loading_out != nullptr) row_flows(a, row, V, status == ROW_CONVERGED, s_red);

    for (int i = tid; i < n; i += BS) vout[i] = V[i];
    if (a.v_mirror != nullptr) {
      double2* vm = reinterpret_cast<double2*>(a.v_mirror) + (int64_t)row * n;
      for (int i = tid; i < n; i += BS) vm[i] = V[i];
    }
    if (tid == 0) {
      a.res_out[row] = nrm;
      a.status_out[row] = status;
      a.iters_out[row] = it_total;
      if (a.factors_out != nullptr) a.factors_out[row] = n_factor;
    }
    __syncthreads();
}

template <typename T>
#ifndef GS2G_MIN_CTAS_PER_SM
#define GS2G_MIN_CTAS_PER_SM 2
#endif
__global__ void __launch_bounds__(BS, GS2G_MIN_CTAS_PER_SM) sweep_kernel(const DevPlan P, const SweepArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_row;
  __shared__ int s_ne;
  __shared__ int s_ek[MAX_EDITS];
  __shared__ double2 s_ev[MAX_EDITS];
  __shared__ double s_red[NWARP];
  __shared__ T s_blk[64];
  __shared__ int s_cr[1 + MAX_COMP];
  __shared__ double s_cB[MAX_COMP * MAX_COMP];
  __shared__ double s_cLU[MAX_COMP * MAX_COMP];
  __shared__ int s_cpiv[MAX_COMP];
  __shared__ double s_cw[MAX_COMP];
  const RowShared<T> sh{&s_ne, s_ek, s_ev, s_red, s_blk, reinterpret_cast<T*>(smem_raw), s_cr, s_cB, s_cLU, s_cpiv,
                        s_cw};
  char* ws = a.workspace + (int64_t)blockIdx.x * a.ws_stride;
  PhaseProf prof;
  prof.init(a.phase_cycles != nullptr && threadIdx.x == 0);
  const int n_rows = a.n_rows_dev != nullptr ? *a.n_rows_dev : a.n_rows;
  for (;;) {
    if (threadIdx.x == 0) s_row = atomicAdd(a.queue, 1);
    __syncthreads();
    const int q = s_row;
    if (q >= n_rows) {
      prof.flush(a.phase_cycles);
      return;
    }
    solve_row<T>(P, a, a.row_map != nullptr ? a.row_map[q] : q, ws, sh, prof);
  }
}

// The rank of this CTA in its cluster, and an int of the leading CTA's
// shared memory read through distributed shared memory.
__device__ __forceinline__ unsigned cluster_ctarank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  return r;
}
__device__ __forceinline__ int ld_shared_rank0(const int* p) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  unsigned ra;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(ra) : "r"(a), "r"(0));
  int v;
  asm volatile("ld.shared::cluster.u32 %0, [%1];\n" : "=r"(v) : "r"(ra) : "memory");
  return v;
}

// The single-row sweep with a cluster of HANDOFF_CLUSTER CTAs per row (FP32
// or FP64 factors): the leading CTA (rank 0) runs the row's whole Newton
// loop in its workspace as sweep_kernel does, and the other CTAs join each
// of its factorizations: the sparse head LU (each level's tasks split),
// the Schur update of the dense tail (split by tail rows) and the dense tail
// LU (dense_lu_cluster).  For the few rows the chord sweep
// hands off and the few rows of an FP64 re-solve, whose factorizations
// would otherwise each run on one SM after every other row has finished.
// When the rows outnumber the clusters, every CTA takes rows of its own.
// Protocol, all through cluster barriers (every CTA passes the same number):
// per row, the leader takes a queue entry and publishes it (barrier), every
// CTA reads it (barrier); then for each factorization the leader posts
// CLUSTER_CMD_LU (barrier, read, barrier) once the Jacobian is scattered,
// and all run the head LU (two barriers per level), their Schur rows
// (barrier) and the dense LU together; after the row it posts
// CLUSTER_CMD_DONE (barrier, read, barrier).
// Largest cluster a row gets (16 needs the non-portable cluster-size opt-in;
// the launch picks 16 or 8 by the number of rows, see launch_sweep_cluster).
constexpr int HANDOFF_CLUSTER = 16;

__device__ __forceinline__ unsigned cluster_nctarank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;\n" : "=r"(r));
  return r;
}

template <typename T>
__global__ void __launch_bounds__(BS, GS2G_MIN_CTAS_PER_SM)
    sweep_kernel_cluster(const DevPlan P, const SweepArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_row;
  __shared__ int s_cmd;
  __shared__ int s_ne;
  __shared__ int s_ek[MAX_EDITS];
  __shared__ double2 s_ev[MAX_EDITS];
  __shared__ double s_red[NWARP];
  __shared__ T s_blk[64];
  __shared__ int s_cr[1 + MAX_COMP];
  __shared__ double s_cB[MAX_COMP * MAX_COMP];
  __shared__ double s_cLU[MAX_COMP * MAX_COMP];
  __shared__ int s_cpiv[MAX_COMP];
  __shared__ double s_cw[MAX_COMP];
  const RowShared<T> sh{&s_ne, s_ek, s_ev, s_red, s_blk, reinterpret_cast<T*>(smem_raw), s_cr, s_cB, s_cLU, s_cpiv,
                        s_cw};
  const int rank = (int)cluster_ctarank();
  const int parts = (int)cluster_nctarank();  // the launch's cluster size
  const int n_rows = a.n_rows_dev != nullptr ? *a.n_rows_dev : a.n_rows;
  PhaseProf prof;
  if ((int64_t)n_rows * parts > gridDim.x) {
    // more rows than clusters: sharing the LUs would leave rows waiting for a
    // cluster, so every CTA runs rows of its own, as sweep_kernel does (the
    // choice is the same for the whole grid: no cluster barrier is used)
    prof.init(a.phase_cycles != nullptr && threadIdx.x == 0);
    char* own = a.workspace + (int64_t)blockIdx.x * a.ws_stride;
    for (;;) {
      if (threadIdx.x == 0) s_row = atomicAdd(a.queue, 1);
      __syncthreads();
      const int q = s_row;
      __syncthreads();  // every thread has read s_row before it is overwritten
      if (q >= n_rows) break;
      solve_row<T>(P, a, a.row_map != nullptr ? a.row_map[q] : q, own, sh, prof);
    }
    prof.flush(a.phase_cycles);
    return;
  }
  // the row lives in the leader's workspace
  char* ws = a.workspace + (int64_t)(blockIdx.x - rank) * a.ws_stride;
  T* S = reinterpret_cast<T*>(ws + ws_layout<T>(P).S);
  T* HV = reinterpret_cast<T*>(ws + ws_layout<T>(P).HV);
  prof.init(a.phase_cycles != nullptr && threadIdx.x == 0 && rank == 0);
  const ClusterLu cl{&s_cmd, parts};
  for (;;) {
    if (rank == 0 && threadIdx.x == 0) s_row = atomicAdd(a.queue, 1);
    dense::cluster_barrier();
    const int q = ld_shared_rank0(&s_row);
    dense::cluster_barrier();
    if (q >= n_rows) break;
    if (rank == 0) {
      solve_row<T>(P, a, a.row_map != nullptr ? a.row_map[q] : q, ws, sh, prof, &cl);
      if (threadIdx.x == 0) s_cmd = CLUSTER_CMD_DONE;
      dense::cluster_barrier();
      dense::cluster_barrier();
    } else {
      for (;;) {
        dense::cluster_barrier();
        const int cmd = ld_shared_rank0(&s_cmd);
        dense::cluster_barrier();
        if (cmd != CLUSTER_CMD_LU) break;
        // the leader's Jacobian values are in place (posted after them): the
        // head LU's share of each level, the Schur rows, a barrier, then the
        // shared dense LU
        head_lu<T>(P, HV, a.pivot_floor, rank, parts);
        schur_update<T>(P, HV, S, rank, parts);
        dense::cluster_barrier();
        dense_lu_cluster<T>(S, P.nt, P.ld, reinterpret_cast<T*>(smem_raw), a.pivot_floor, rank, parts);
      }
    }
  }
  prof.flush(a.phase_cycles);
}

// One persistent launch over the rows of several grids: row r of the
// launch is row r - row_begin[g] of grid g (row_begin ascending, n_grids
// <= MAX_GRIDS).  A CTA loads a grid's plan and arguments into shared
// memory when its next row belongs to another grid than its last one; the
// workspace stride covers the largest grid.
template <typename T>
__global__ void __launch_bounds__(BS, GS2G_MIN_CTAS_PER_SM)
    sweep_kernel_multi(const GridEntry* __restrict__ grids, int n_grids, const int* __restrict__ row_begin,
                       int n_rows, int* queue, char* workspace, int64_t ws_stride, unsigned long long* phase_cycles,
                       const int* __restrict__ row_list, const int* __restrict__ n_rows_dev) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_row;
  __shared__ int s_ne;
  __shared__ int s_ek[MAX_EDITS];
  __shared__ double2 s_ev[MAX_EDITS];
  __shared__ double s_red[NWARP];
  __shared__ T s_blk[64];
  __shared__ __align__(16) GridEntry s_grid;
  __shared__ int s_cr[1 + MAX_COMP];
  __shared__ double s_cB[MAX_COMP * MAX_COMP];
  __shared__ double s_cLU[MAX_COMP * MAX_COMP];
  __shared__ int s_cpiv[MAX_COMP];
  __shared__ double s_cw[MAX_COMP];
  const RowShared<T> sh{&s_ne, s_ek, s_ev, s_red, s_blk, reinterpret_cast<T*>(smem_raw), s_cr, s_cB, s_cLU, s_cpiv,
                        s_cw};
  char* ws = workspace + (int64_t)blockIdx.x * ws_stride;
  PhaseProf prof;
  prof.init(phase_cycles != nullptr && threadIdx.x == 0);
  int cur = -1;
  // with row_list, queue entry q solves global row row_list[q], and the
  // number of entries is read on the device (hand-offs of a chord sweep)
  const int n_entries = n_rows_dev != nullptr ? *n_rows_dev : n_rows;
  for (;;) {
    if (threadIdx.x == 0) s_row = atomicAdd(queue, 1);
    __syncthreads();
    const int q = s_row;
    if (q >= n_entries) {
      prof.flush(phase_cycles);
      return;
    }
    const int entry = row_list != nullptr ? row_list[q] : q;
    const int flag = entry & NO_RESCUE_BIT;
    const int row = entry & ~NO_RESCUE_BIT;
    int g = 0;
    while (g + 1 < n_grids && row >= row_begin[g + 1]) ++g;
    if (g != cur) {
      const int* src = reinterpret_cast<const int*>(grids + g);
      int* dst = reinterpret_cast<int*>(&s_grid);
      for (int i = threadIdx.x; i < (int)(sizeof(GridEntry) / sizeof(int)); i += BS) dst[i] = src[i];
      __syncthreads();
      cur = g;
    }
    const int lr = row - row_begin[g];
    // a queue position goes through the grid's row order; a hand-off entry
    // is already the grid's row
    const int srow = row_list == nullptr && s_grid.a.row_map != nullptr ? s_grid.a.row_map[lr] : lr;
    solve_row<T>(s_grid.P, s_grid.a, srow | flag, ws, sh, prof);
  }
}

#include "chord_sweep.cuh"
#include "adjoint.cuh"

template <typename T>
int smem_bytes() {
  return sizeof(T) == 4 ? gs2g::dense32::Smem::bytes : dense::Smem<T>::bytes;
}

}  // namespace

int64_t workspace_bytes(const DevPlan& P, int prec) {
  return prec == 1 ? ws_layout<float>(P).total : ws_layout<double>(P).total;
}

int64_t workspace_hv_offset(const DevPlan& P, int prec) {
  return prec == 1 ? ws_layout<float>(P).HV : ws_layout<double>(P).HV;
}

namespace {
// Dynamic shared memory above 48 KB needs an opt-in per kernel (per device
// context); cheap and idempotent, so it is set before every query / launch.
cudaError_t opt_in_smem() {
  cudaError_t e = cudaFuncSetAttribute(sweep_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       smem_bytes<float>());
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(sweep_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes<double>());
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(sweep_kernel_multi<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           smem_bytes<float>());
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(sweep_kernel_cluster<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           smem_bytes<float>());
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(sweep_kernel_cluster<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           smem_bytes<double>());
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(sweep_kernel_cluster<float>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(sweep_kernel_cluster<double>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(sweep_kernel_multi<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              smem_bytes<double>());
}
}  // namespace

int sweep_ctas(int prec, int device) {
  int n_sm = 0;
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device);
  opt_in_smem();
  int per_sm = 0;
  if (prec == 1)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_kernel<float>, BS, smem_bytes<float>());
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_kernel<double>, BS, smem_bytes<double>());
  if (per_sm < 1) per_sm = 1;
  return n_sm * per_sm;
}

int launch_sweep_multi(const GridEntry* d_grids, int n_grids, const int* d_row_begin, int n_rows, int* queue,
                       char* workspace, int64_t ws_stride, unsigned long long* phase_cycles, int prec, int n_ctas,
                       void* stream, const int* row_list, const int* n_rows_dev) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n_ctas <= 0 || n_grids <= 0 || n_grids > MAX_GRIDS) return (int)cudaErrorInvalidValue;
  const cudaError_t e = opt_in_smem();
  if (e != cudaSuccess) return (int)e;
  if (prec == 1)
    sweep_kernel_multi<float><<<n_ctas, BS, smem_bytes<float>(), st>>>(
        d_grids, n_grids, d_row_begin, n_rows, queue, workspace, ws_stride, phase_cycles, row_list, n_rows_dev);
  else
    sweep_kernel_multi<double><<<n_ctas, BS, smem_bytes<double>(), st>>>(
        d_grids, n_grids, d_row_begin, n_rows, queue, workspace, ws_stride, phase_cycles, row_list, n_rows_dev);
  return (int)cudaGetLastError();
}

int64_t chord_workspace_bytes(const DevPlan& P, int prec) {
  return prec == 1 ? chord_ws<float>(P).total : chord_ws<double>(P).total;
}

int chord_rows_per_cta() { return CK; }

namespace {
template <typename T>
cudaError_t chord_opt_in(const DevPlan& P) {
  return cudaFuncSetAttribute(chord_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, chord_smem_bytes<T>(P));
}
}  // namespace

int chord_ctas(const DevPlan& P, int prec, int device) {
  int n_sm = 0;
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device);
  int per_sm = 0;
  if (prec == 1 && chord_use_ysmem<float>(P)) {
    cudaFuncSetAttribute(chord_kernel_ysmem<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         chord_smem_bytes_ysmem<float>(P));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, chord_kernel_ysmem<float>, BS,
                                                  chord_smem_bytes_ysmem<float>(P));
  } else if (prec == 1) {
    chord_opt_in<float>(P);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, chord_kernel<float>, BS, chord_smem_bytes<float>(P));
  } else {
    chord_opt_in<double>(P);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, chord_kernel<double>, BS, chord_smem_bytes<double>(P));
  }
  if (per_sm < 1) per_sm = 1;
  return n_sm * per_sm;
}

int64_t comp_rec_bytes() { return (int64_t)sizeof(CompRec); }

int launch_comp_setup(const DevPlan& P, const SweepArgs& a, int prec, int n_rows, void* rec, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n_rows <= 0 || rec == nullptr || a.edit_ptr == nullptr || a.base_inv == nullptr || a.base_v == nullptr)
    return (int)cudaErrorInvalidValue;
  if (prec == 1)
    comp_setup_kernel<float><<<n_rows, 32, 0, st>>>(P, a, static_cast<CompRec*>(rec));
  else
    comp_setup_kernel<double><<<n_rows, 32, 0, st>>>(P, a, static_cast<CompRec*>(rec));
  return (int)cudaGetLastError();
}

int launch_chord(const DevPlan& P, const SweepArgs& a, int prec, int n_ctas, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n_ctas <= 0 || a.base_ws == nullptr || a.base_inv == nullptr || a.base_fwv == nullptr ||
      a.base_bwv == nullptr || a.handoff == nullptr || a.n_handoff == nullptr || a.fixed_iters)
    return (int)cudaErrorInvalidValue;
  if (prec == 1 && chord_use_ysmem<float>(P)) {
    const int sm = chord_smem_bytes_ysmem<float>(P);
    cudaError_t e = cudaFuncSetAttribute(chord_kernel_ysmem<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e != cudaSuccess) return (int)e;
    chord_kernel_ysmem<float><<<n_ctas, BS, sm, st>>>(P, a);
    return (int)cudaGetLastError();
  }
  cudaError_t e = prec == 1 ? chord_opt_in<float>(P) : chord_opt_in<double>(P);
  if (e != cudaSuccess) return (int)e;
  if (prec == 1)
    chord_kernel<float><<<n_ctas, BS, chord_smem_bytes<float>(P), st>>>(P, a);
  else
    chord_kernel<double><<<n_ctas, BS, chord_smem_bytes<double>(P), st>>>(P, a);
  return (int)cudaGetLastError();
}

int launch_chord_multi(const GridEntry* d_grids, int n_grids, int smem, unsigned long long* phase_cycles, int prec,
                       int n_ctas, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n_ctas <= 0 || n_grids <= 0 || n_grids > MAX_GRIDS || smem <= 0) return (int)cudaErrorInvalidValue;
  cudaError_t e = prec == 1 ? cudaFuncSetAttribute(chord_kernel_multi<float>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, smem)
                            : cudaFuncSetAttribute(chord_kernel_multi<double>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return (int)e;
  if (prec == 1)
    chord_kernel_multi<float><<<n_ctas, BS, smem, st>>>(d_grids, n_grids, phase_cycles);
  else
    chord_kernel_multi<double><<<n_ctas, BS, smem, st>>>(d_grids, n_grids, phase_cycles);
  return (int)cudaGetLastError();
}

int chord_smem(const DevPlan& P, int prec) { return prec == 1 ? chord_smem_bytes<float>(P) : chord_smem_bytes<double>(P); }

int launch_adjoint(const DevPlan& P, const SweepArgs& a, const double* rhs, double* lam, int n_ctas, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n_ctas <= 0 || a.v_out == nullptr || a.status_out == nullptr || a.queue == nullptr) return (int)cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(adjoint_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       smem_bytes<double>());
  if (e != cudaSuccess) return (int)e;
  adjoint_kernel<double><<<n_ctas, BS, smem_bytes<double>(), st>>>(P, a, rhs, lam);
  return (int)cudaGetLastError();
}

int handoff_cluster_size() { return HANDOFF_CLUSTER; }

int launch_sweep_cluster(const DevPlan& P, const SweepArgs& a, int prec, int cluster, int n_ctas, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if ((cluster != 8 && cluster != 16) || n_ctas <= 0 || n_ctas % cluster != 0 || a.inverse_out != nullptr ||
      a.factor_only)
    return (int)cudaErrorInvalidValue;
  cudaError_t e = opt_in_smem();
  if (e != cudaSuccess) return (int)e;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)n_ctas, 1, 1);
  cfg.blockDim = dim3(BS, 1, 1);
  cfg.dynamicSmemBytes = prec == 1 ? smem_bytes<float>() : smem_bytes<double>();
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (prec == 1)
    e = cudaLaunchKernelEx(&cfg, sweep_kernel_cluster<float>, P, a);
  else
    e = cudaLaunchKernelEx(&cfg, sweep_kernel_cluster<double>, P, a);
  if (e != cudaSuccess) return (int)e;
  return (int)cudaGetLastError();
}

int launch_sweep(const DevPlan& P, const SweepArgs& a, int prec, int n_ctas, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n_ctas <= 0) return (int)cudaErrorInvalidValue;
  const cudaError_t e = opt_in_smem();
  if (e != cudaSuccess) return (int)e;
  if (prec == 1)
    sweep_kernel<float><<<n_ctas, BS, smem_bytes<float>(), st>>>(P, a);
  else
    sweep_kernel<double><<<n_ctas, BS, smem_bytes<double>(), st>>>(P, a);
  return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Allocation-free sweep.  Its scratch -- the row-queue counter (first 256
// bytes) and the per-CTA workspaces -- lives in this file-scope device array,
// which every GPU that loads the library holds until the process exits.
// Host code must not use the array's name as an address: on the host it is
// a stand-in symbol.  The device address is looked up once per device with
// cudaGetSymbolAddress (the first call on a device does it, so that first
// call should come before any stream capture) and cached.  All calls share
// the array, so calls that overlap on the GPU race on it.
// ---------------------------------------------------------------------------
namespace {

static __device__ __align__(256) unsigned char g_sweep_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
char* g_scratch_ptr[kMaxDevices] = {};

cudaError_t scratch_address(int device, char** out) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_sweep_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[device] = static_cast<char*>(p);
  }
  *out = g_scratch_ptr[device];
  return cudaSuccess;
}

}  // namespace

int launch_sweep_static(const DevPlan& P, SweepArgs a, int prec, int device, void* stream, int* n_ctas_used) {
  const int64_t ws = workspace_bytes(P, prec);
  const int64_t room = kStaticScratchBytes - 256;
  if (ws <= 0 || ws > room) return (int)cudaErrorInvalidValue;
  char* base = nullptr;
  cudaError_t e = scratch_address(device, &base);
  if (e != cudaSuccess) return (int)e;
  int n_ctas = sweep_ctas(prec, device);
  const int64_t fit = room / ws;
  if (n_ctas > fit) n_ctas = (int)fit;
  if (n_ctas > a.n_rows) n_ctas = a.n_rows;
  if (n_ctas < 1) n_ctas = 1;
  a.queue = reinterpret_cast<int*>(base);
  a.workspace = base + 256;
  a.ws_stride = ws;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the queue must start at zero: the previous call left its final count there
  e = cudaMemsetAsync(base, 0, sizeof(int), st);
  if (e != cudaSuccess) return (int)e;
  if (n_ctas_used) *n_ctas_used = n_ctas;
  if (a.n_rows <= 0) return (int)cudaSuccess;
  return launch_sweep(P, a, prec, n_ctas, stream);
}

}  // namespace gs2g
