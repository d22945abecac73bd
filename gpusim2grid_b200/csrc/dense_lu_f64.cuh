// Dense FP64 LU (no pivoting) of one matrix by one CTA of 256 threads (or by
// the CTAs of a cluster), for the tail of the FP64 batched Newton–Raphson
// factorization: the FP64 arm, the FP64 re-solve of unconverged rows and
// the adjoint.  Device code only.  The design of dense_lu_f32.cuh with
// 32-wide panels, so that a row or column of a panel fits in 64 registers:
//   1. the kb x kb diagonal block is copied to shared memory (identity
//      padded to 32 x 32) and factored by one warp holding one row per lane
//      in registers (no block barrier inside);
//   2. L21 = A21 U11^-1: one thread per row of A21, the row in registers,
//      forward substitution against U11 rows read as broadcast double2;
//   3. U12 = L11^-1 A12: one thread per column of A12, the column in
//      registers, substitution against the rows of L11^T (unit diagonal);
//   4. A22 -= L21 U12 on 64 x 64 output tiles: the tile's A (64 x 32) and B
//      (32 x 64) operands are staged by cp.async in one piece, each thread
//      accumulates a 4 x 4 block (rows tr + 16 i, columns 2 tc + 32 h + e),
//      and the next tile's operands are in flight while a tile's results are
//      written back.
// A is row-major in global memory with leading dimension ld, a multiple of
// 2 (rows 16-byte aligned); panels start at multiples of 32.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace gs2g {
namespace dense64 {

constexpr int BS = 256;
constexpr int KP = 32;          // panel width
constexpr int SD = KP + 2;      // diagonal block stride (16-byte rows)
constexpr int TM = 64, TN = 64;
constexpr int SA = KP + 2;      // A tile [TM][SA]
constexpr int SB = TN + 2;      // B tile [KP][SB]

struct Smem {
  static constexpr int d_elems = KP * SD;
  static constexpr int r_elems = KP;  // reciprocal pivots
  static constexpr int a_elems = TM * SA;
  static constexpr int b_elems = KP * SB;
  static constexpr int elems = d_elems + r_elems + a_elems + b_elems;
  static constexpr int bytes = elems * 8;
};

__device__ __forceinline__ double clamp_piv(double piv, double floor_) {
  if (fabs(piv) < floor_) return piv < 0.0 ? -floor_ : floor_;
  return piv;
}

// Shared-memory loads issued in program order (asm volatile): the
// substitutions below hold 32 values per thread in registers, and letting
// the compiler hoist their broadcast loads ahead of the arithmetic would
// spill them.
__device__ __forceinline__ double2 lds2(const double* p) {
  double2 v;
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ld.shared.v2.f64 {%0,%1}, [%2];\n" : "=d"(v.x), "=d"(v.y) : "r"(a));
  return v;
}
__device__ __forceinline__ double lds1(const double* p) {
  double v;
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ld.shared.f64 %0, [%1];\n" : "=d"(v) : "r"(a));
  return v;
}

__device__ __forceinline__ void cp_async16(double* smem, const double* gmem, int src_bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}

// Stage the A (rows i0.., 32 columns) and B (32 rows, columns j0..) tiles of
// the trailing update, zero-filled outside [M) rows / [N) columns.
__device__ __forceinline__ void stage_tile(double* sA, double* sB, const double* A21, const double* A12, int ld, int M,
                                           int N, int i0, int j0) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int q = 0; q < (TM * KP / 2) / BS; ++q) {  // 4 chunks per thread
    const int c = tid + q * BS;
    const int r = c >> 4, k = (c & 15) * 2;
    const bool in = i0 + r < M;
    cp_async16(sA + r * SA + k, in ? A21 + (int64_t)(i0 + r) * ld + k : A21, in ? 16 : 0);
  }
#pragma unroll
  for (int q = 0; q < (KP * TN / 2) / BS; ++q) {  // 4 chunks per thread
    const int c = tid + q * BS;
    const int k = c >> 5, n = (c & 31) * 2;
    int bytes = (N - j0 - n) * 8;
    bytes = bytes < 0 ? 0 : (bytes > 16 ? 16 : bytes);
    cp_async16(sB + k * SB + n, bytes ? A12 + (int64_t)k * ld + j0 + n : A12, bytes);
  }
  asm volatile("cp.async.commit_group;\n" ::);
}

// A22[M x N] -= A21[M x 32] A12[32 x N].  With parts > 1 the CTA takes the
// output tiles part, part + parts, ... (the CTAs of a cluster split them).
__device__ __noinline__ void trailing_update(double* A22, const double* A21, const double* A12, int ld, int M, int N,
                                             double* sA, double* sB, int part = 0, int parts = 1) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tr = (warp >> 1) * 4 + (lane >> 3);  // 0..15
  const int tc = (warp & 1) * 8 + (lane & 7);    // 0..15
  const int n_ti = (M + TM - 1) / TM, n_tj = (N + TN - 1) / TN;
  const int n_tiles = n_ti * n_tj;
  if (part >= n_tiles) {
    __syncthreads();
    return;
  }
  stage_tile(sA, sB, A21, A12, ld, M, N, (part / n_tj) * TM, (part % n_tj) * TN);
  for (int t = part; t < n_tiles; t += parts) {
    const int i0 = (t / n_tj) * TM, j0 = (t % n_tj) * TN;
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
#pragma unroll 4
    for (int k = 0; k < KP; ++k) {
      double a[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = sA[(tr + 16 * i) * SA + k];
      const double2 b0 = *reinterpret_cast<const double2*>(sB + k * SB + 2 * tc);
      const double2 b1 = *reinterpret_cast<const double2*>(sB + k * SB + 32 + 2 * tc);
      const double b[4] = {b0.x, b0.y, b1.x, b1.y};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();  // every thread is done reading this tile's operands
    if (t + parts < n_tiles) {
      const int t1 = t + parts;
      stage_tile(sA, sB, A21, A12, ld, M, N, (t1 / n_tj) * TM, (t1 % n_tj) * TN);
    }
    // epilogue: all loads of the thread's block before its stores
    double2 cv[4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = i0 + tr + 16 * i;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int c = j0 + 32 * h + 2 * tc;
        cv[i][h] = (r < M && c + 1 < N) ? *reinterpret_cast<const double2*>(A22 + (int64_t)r * ld + c)
                                        : make_double2(0.0, 0.0);
      }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = i0 + tr + 16 * i;
      if (r >= M) continue;
      double* crow = A22 + (int64_t)r * ld;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int c = j0 + 32 * h + 2 * tc;
        const double* a = acc[i] + 2 * h;
        if (c + 1 < N)
          *reinterpret_cast<double2*>(crow + c) = make_double2(cv[i][h].x - a[0], cv[i][h].y - a[1]);
        else if (c < N)
          crow[c] -= a[0];
      }
    }
  }
  __syncthreads();
}

// Factor the identity-padded 32 x 32 block D (stride SD) in place; rp gets
// the reciprocal pivots.  Warp 0 holds one row per lane in registers.  Step
// j: lane j clamps its pivot and publishes its row (final: L part, pivot, U
// part) to D; the lanes below take l = x_j / u_jj and x_c -= l u_jc (c > j),
// reading row j as broadcast double2.  Warps 1..7 skip.
__device__ __noinline__ void factor_diag(double* D, double* rp, double pfloor) {
  const int r = threadIdx.x;
  if (r < KP) {
    double x[KP];
#pragma unroll
    for (int q = 0; q < KP / 2; ++q) {
      const double2 v = lds2(D + r * SD + 2 * q);
      x[2 * q] = v.x;
      x[2 * q + 1] = v.y;
    }
    __syncwarp();  // all rows read before any is rewritten
#pragma unroll
    for (int j = 0; j < KP; ++j) {
      if (r == j) {
        x[j] = clamp_piv(x[j], pfloor);
        rp[j] = 1.0 / x[j];
#pragma unroll
        for (int q = 0; q < KP / 2; ++q) *reinterpret_cast<double2*>(D + j * SD + 2 * q) = make_double2(x[2 * q], x[2 * q + 1]);
      }
      __syncwarp();
      if (r > j) {
        const double* uj = D + j * SD;
        const double l = x[j] * (1.0 / lds1(uj + j));
        x[j] = l;
        if (((j + 1) & 1) && j + 1 < KP) x[j + 1] = fma(-l, lds1(uj + j + 1), x[j + 1]);
#pragma unroll
        for (int c2 = ((j + 1) + 1) & ~1; c2 < KP; c2 += 2) {
          const double2 u = lds2(uj + c2);
          x[c2] = fma(-l, u.x, x[c2]);
          x[c2 + 1] = fma(-l, u.y, x[c2 + 1]);
        }
      }
    }
  }
  __syncthreads();
}

// x <- x M^-1 for the 32 values x of one thread, M upper triangular given by
// its rows (stride SD) in shared memory: after x_p is final, x_q -= x_p M_pq
// for q > p.  SCALE: x_p is multiplied by rp[p] (1 / M_pp) first; else M has
// a unit diagonal.
template <bool SCALE>
__device__ __forceinline__ void subst32(double (&x)[KP], const double* M, const double* rp) {
#pragma unroll
  for (int p = 0; p < KP; ++p) {
    if (SCALE) x[p] *= lds1(rp + p);
    const double xp = x[p];
    const double* mp = M + p * SD;
    if ((p + 1) & 1)
      if (p + 1 < KP) x[p + 1] = fma(-xp, lds1(mp + p + 1), x[p + 1]);
#pragma unroll
    for (int q2 = ((p + 1) + 1) & ~1; q2 < KP; q2 += 2) {
      const double2 u = lds2(mp + q2);
      x[q2] = fma(-xp, u.x, x[q2]);
      x[q2 + 1] = fma(-xp, u.y, x[q2 + 1]);
    }
  }
}

// L21 = A21 U11^-1 (x U11 = a per row), one thread per row (with parts > 1:
// rows part * BS + tid, then every parts * BS).
__device__ __noinline__ void trsm_rows(double* A21, int ld, int M, const double* D, const double* rp, int part = 0,
                                       int parts = 1) {
  for (int r = part * BS + threadIdx.x; r < M; r += BS * parts) {
    double2* row = reinterpret_cast<double2*>(A21 + (int64_t)r * ld);
    double x[KP];
#pragma unroll
    for (int q = 0; q < KP / 2; ++q) {
      const double2 v = row[q];
      x[2 * q] = v.x;
      x[2 * q + 1] = v.y;
    }
    subst32<true>(x, D, rp);
#pragma unroll
    for (int q = 0; q < KP / 2; ++q) row[q] = make_double2(x[2 * q], x[2 * q + 1]);
  }
}

// U12 = L11^-1 A12 (per column: y^T L11^T = a^T, L11^T upper with unit
// diagonal, given by its rows LT = rows of L11^T), one thread per column.
__device__ __noinline__ void trsm_cols(double* A12, int ld, int N, const double* LT, int part = 0, int parts = 1) {
  for (int c = part * BS + threadIdx.x; c < N; c += BS * parts) {
    double y[KP];
    const double* src = A12 + c;
#pragma unroll
    for (int r = 0; r < KP; ++r, src += ld) {
      y[r] = *src;
      if ((r & 15) == 15) asm volatile("" ::: "memory");  // at most 16 loads in flight
    }
    subst32<false>(y, LT, nullptr);
    // the stores walk the column again from an opaque copy of ld, so the 32
    // load addresses are not kept alive across the substitution
    int ld2;
    asm volatile("mov.b32 %0, %1;\n" : "=r"(ld2) : "r"(ld));
    double* dst = A12 + c;
#pragma unroll
    for (int r = 0; r < KP; ++r, dst += ld2) *dst = y[r];
  }
}

// Load the kb x kb diagonal block at Akk into D (identity padded).
__device__ __forceinline__ void load_diag(double* D, const double* Akk, int ld, int kb) {
  for (int idx = threadIdx.x; idx < KP * KP; idx += BS) {
    const int r = idx / KP, c = idx % KP;
    D[r * SD + c] = (r < kb && c < kb) ? Akk[(int64_t)r * ld + c] : (r == c ? 1.0 : 0.0);
  }
}

// L11^T into LT (the idle tile staging area) for the column solves.
__device__ __forceinline__ void transpose_l11(double* LT, const double* D) {
  for (int idx = threadIdx.x; idx < KP * KP; idx += BS) {
    const int r = idx / KP, c = idx % KP;
    LT[c * SD + r] = r > c ? D[r * SD + c] : 0.0;
  }
}

// LU of A (n x n, leading dimension ld) in place.
__device__ void lu(double* A, int n, int ld, double* smem, double pfloor) {
  double* D = smem;
  double* rp = D + Smem::d_elems;
  double* sA = rp + Smem::r_elems;
  double* sB = sA + Smem::a_elems;
  const int tid = threadIdx.x;
  for (int k0 = 0; k0 < n; k0 += KP) {
    const int kb = min(KP, n - k0);
    double* Akk = A + (int64_t)k0 * ld + k0;
    load_diag(D, Akk, ld, kb);
    __syncthreads();
    factor_diag(D, rp, pfloor);
    for (int idx = tid; idx < kb * kb; idx += BS) {
      const int r = idx / kb, c = idx % kb;
      Akk[(int64_t)r * ld + c] = D[r * SD + c];
    }
    const int m = n - k0 - kb;  // > 0 only with kb == 32
    if (m > 0) {
      double* A21 = A + (int64_t)(k0 + kb) * ld + k0;
      double* A12 = A + (int64_t)k0 * ld + k0 + kb;
      double* A22 = A + (int64_t)(k0 + kb) * ld + k0 + kb;
      double* LT = sA;
      transpose_l11(LT, D);
      __syncthreads();
      trsm_rows(A21, ld, m, D, rp);
      trsm_cols(A12, ld, m, LT);
      __syncthreads();  // L21 and U12 complete (global writes of other threads)
      trailing_update(A22, A21, A12, ld, m, m, sA, sB);
    }
    __syncthreads();
  }
}

// Barrier over every thread of every CTA of the cluster, ordering the
// memory accesses before it (global and distributed shared) before those
// after it.  Block-uniform calls only.
__device__ __forceinline__ void cluster_sync_all() {
  __threadfence();
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// The same LU as lu(), by the `parts` CTAs of a cluster together (this CTA
// has rank `part`); A in global memory, every CTA with its own scratch.
// Each CTA factors the diagonal block itself (every CTA needs it in its own
// shared memory), the row and column substitutions and the trailing-update
// tiles are split by rank, and three cluster barriers per panel order the
// stages.  Every element goes through the same operations in the same order
// as in lu(), so the factor is bit-identical.  Every CTA of the cluster must
// call it with the same n.
__device__ void lu_cluster(double* A, int n, int ld, double* smem, double pfloor, int part, int parts) {
  double* D = smem;
  double* rp = D + Smem::d_elems;
  double* sA = rp + Smem::r_elems;
  double* sB = sA + Smem::a_elems;
  const int tid = threadIdx.x;
  for (int k0 = 0; k0 < n; k0 += KP) {
    const int kb = min(KP, n - k0);
    double* Akk = A + (int64_t)k0 * ld + k0;
    load_diag(D, Akk, ld, kb);
    __syncthreads();
    factor_diag(D, rp, pfloor);
    cluster_sync_all();  // every CTA holds the block: rank 0 may write it back below
    const int m = n - k0 - kb;
    double* A21 = A + (int64_t)(k0 + kb) * ld + k0;
    double* A12 = A + (int64_t)k0 * ld + k0 + kb;
    double* A22 = A + (int64_t)(k0 + kb) * ld + k0 + kb;
    if (m > 0) {
      double* LT = sA;
      transpose_l11(LT, D);
      __syncthreads();
      trsm_rows(A21, ld, m, D, rp, part, parts);
      trsm_cols(A12, ld, m, LT, part, parts);
    }
    if (part == 0)
      for (int idx = tid; idx < kb * kb; idx += BS) {
        const int r = idx / kb, c = idx % kb;
        Akk[(int64_t)r * ld + c] = D[r * SD + c];
      }
    cluster_sync_all();  // L21, U12 and the diagonal block complete
    if (m > 0) trailing_update(A22, A21, A12, ld, m, m, sA, sB, part, parts);
    cluster_sync_all();  // A22 complete
  }
}

}  // namespace dense64
}  // namespace gs2g
