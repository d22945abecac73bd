// Dense FP32 LU (no pivoting) of one matrix by one CTA of 256 threads, for
// the tail of the mixed-precision batched Newton–Raphson factorization.
// Device code only.
//
// Right-looking, 64-wide panels.  Per panel k0 (width kb; kb < 64 only for
// the last panel, which has nothing below or to the right of it):
//   1. the kb x kb diagonal block is copied to shared memory (identity
//      padded to 64 x 64), factored by two warps holding one row per
//      thread in registers, and written back;
//   2. L21 = A21 U11^-1: one thread per row of A21, the row in registers,
//      forward substitution against U11 rows read as broadcast float4;
//   3. U12 = L11^-1 A12: one thread per column of A12, the column in
//      registers, substitution against the rows of L11^T (unit diagonal),
//      which is transposed into the idle tile staging area first;
//   4. A22 -= L21 U12 on 128 x 128 output tiles: the tile's A (128 x 64) and
//      B (64 x 128) operands are staged by cp.async in one piece, each
//      thread accumulates an 8 x 8 block (rows tr + 16 i, columns
//      4 tc + 64 h + e: within a warp 4 consecutive rows and 8 consecutive
//      float4 columns, so shared-memory reads are conflict-free), and the
//      next tile's operands are in flight while a tile's results are
//      written back.
// A is row-major in global memory with leading dimension ld, a multiple of
// 8 (rows 16-byte aligned); panels start at multiples of 64.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace gs2g {
namespace dense32 {

constexpr int BS = 256;
constexpr int KP = 64;          // panel width
constexpr int SD = KP + 4;      // diagonal block stride (16-byte rows)
constexpr int TM = 128, TN = 128;
constexpr int SA = KP + 4;      // A tile [TM][SA]
constexpr int SB = TN + 4;      // B tile [KP][SB]
#ifndef GS2G_DENSE32_EPI_ROWS
#define GS2G_DENSE32_EPI_ROWS 2  // rows per epilogue batch (1, 2, 4 or 8)
#endif

struct Smem {
  static constexpr int d_elems = KP * SD;
  static constexpr int r_elems = KP;  // reciprocal pivots
  static constexpr int a_elems = TM * SA;
  static constexpr int b_elems = KP * SB;
  static constexpr int elems = d_elems + r_elems + a_elems + b_elems;
  static constexpr int bytes = elems * 4;
};

__device__ __forceinline__ float clamp_piv(float piv, double floor_) {
  const float f = (float)floor_;
  if (fabsf(piv) < f) return piv < 0.f ? -f : f;
  return piv;
}

// Shared-memory loads issued in program order (asm volatile): the TRSM
// loops below hold 64 values per thread in registers, and letting the
// compiler hoist their ~500 broadcast loads ahead of the arithmetic would
// spill them.
__device__ __forceinline__ float4 lds4(const float* p) {
  float4 v;
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];\n" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
  return v;
}
__device__ __forceinline__ float lds1(const float* p) {
  float v;
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ld.shared.f32 %0, [%1];\n" : "=f"(v) : "r"(a));
  return v;
}

__device__ __forceinline__ void cp_async16(float* smem, const float* gmem, int src_bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}

// Stage the A (rows i0.., 64 columns) and B (64 rows, columns j0..) tiles of
// the trailing update, zero-filled outside [M) rows / [N) columns.
__device__ __forceinline__ void stage_tile(float* sA, float* sB, const float* A21, const float* A12, int ld, int M,
                                           int N, int i0, int j0) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int q = 0; q < (TM * KP / 4) / BS; ++q) {  // 8 chunks per thread
    const int c = tid + q * BS;
    const int r = c >> 4, k = (c & 15) * 4;
    const bool in = i0 + r < M;
    cp_async16(sA + r * SA + k, in ? A21 + (int64_t)(i0 + r) * ld + k : A21, in ? 16 : 0);
  }
#pragma unroll
  for (int q = 0; q < (KP * TN / 4) / BS; ++q) {  // 8 chunks per thread
    const int c = tid + q * BS;
    const int k = c >> 5, n = (c & 31) * 4;
    int bytes = (N - j0 - n) * 4;
    bytes = bytes < 0 ? 0 : (bytes > 16 ? 16 : bytes);
    cp_async16(sB + k * SB + n, bytes ? A12 + (int64_t)k * ld + j0 + n : A12, bytes);
  }
  asm volatile("cp.async.commit_group;\n" ::);
}

// A22[M x N] -= A21[M x 64] A12[64 x N].  With parts > 1 the CTA takes the
// output tiles part, part + parts, ... (the CTAs of a cluster split them).
__device__ __noinline__ void trailing_update(float* A22, const float* A21, const float* A12, int ld, int M, int N, float* sA,
                                float* sB, int part = 0, int parts = 1) {
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
    // bring this tile's output rows toward L2 while the tile computes
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int r = i0 + tr + 16 * i;
      if (r < M && j0 + 4 * tc < N)
        asm volatile("prefetch.global.L2 [%0];\n" ::"l"(A22 + (int64_t)r * ld + j0 + 4 * tc));
      if (r < M && j0 + 64 + 4 * tc < N)
        asm volatile("prefetch.global.L2 [%0];\n" ::"l"(A22 + (int64_t)r * ld + j0 + 64 + 4 * tc));
    }
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;
#pragma unroll 4
    for (int k = 0; k < KP; ++k) {
      float a[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = sA[(tr + 16 * i) * SA + k];
      const float4 b0 = *reinterpret_cast<const float4*>(sB + k * SB + 4 * tc);
      const float4 b1 = *reinterpret_cast<const float4*>(sB + k * SB + 64 + 4 * tc);
      const float b[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();  // every thread is done reading this tile's operands
    if (t + parts < n_tiles) {
      const int t1 = t + parts;
      stage_tile(sA, sB, A21, A12, ld, M, N, (t1 / n_tj) * TM, (t1 % n_tj) * TN);
    }
    // epilogue in batches of EB rows: all loads of a batch are issued before
    // its stores (the compiler cannot reorder them across the stores)
    constexpr int EB = GS2G_DENSE32_EPI_ROWS;
#pragma unroll
    for (int ib = 0; ib < 8; ib += EB) {
      float4 cv[EB][2];
#pragma unroll
      for (int i = 0; i < EB; ++i) {
        const int r = i0 + tr + 16 * (ib + i);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int c = j0 + 64 * h + 4 * tc;
          cv[i][h] = (r < M && c + 3 < N) ? *reinterpret_cast<const float4*>(A22 + (int64_t)r * ld + c)
                                          : make_float4(0.f, 0.f, 0.f, 0.f);
        }
      }
#pragma unroll
      for (int i = 0; i < EB; ++i) {
        const int r = i0 + tr + 16 * (ib + i);
        if (r >= M) continue;
        float* crow = A22 + (int64_t)r * ld;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int c = j0 + 64 * h + 4 * tc;
          const float* a = acc[ib + i] + 4 * h;
          if (c + 3 < N) {
            *reinterpret_cast<float4*>(crow + c) =
                make_float4(cv[i][h].x - a[0], cv[i][h].y - a[1], cv[i][h].z - a[2], cv[i][h].w - a[3]);
          } else {
#pragma unroll
            for (int e = 0; e < 4; ++e)
              if (c + e < N) crow[c + e] -= a[e];
          }
        }
      }
    }
  }
  __syncthreads();
}

// Factor the identity-padded 64 x 64 block D (stride SD) in place; rp gets
// the reciprocal pivots.  Warps 0 and 1 hold one row each in registers
// (thread r: row r).  Step j: thread j clamps its pivot and publishes its
// row (final: L part, pivot, U part) to D; a 64-thread named barrier; rows
// below j take l = x_j / u_jj and x_c -= l u_jc (c > j), reading row j as
// broadcast float4.  One lightweight barrier per step; warps 2..7 skip.
__device__ __noinline__ void factor_diag(float* D, float* rp, double pfloor) {
  const int r = threadIdx.x;
  if (r < KP) {
    float x[KP];
#pragma unroll
    for (int q = 0; q < KP / 4; ++q) {
      const float4 v = lds4(D + r * SD + 4 * q);
      x[4 * q] = v.x;
      x[4 * q + 1] = v.y;
      x[4 * q + 2] = v.z;
      x[4 * q + 3] = v.w;
    }
    asm volatile("bar.sync 1, 64;\n" ::: "memory");  // all rows read before any is rewritten
#pragma unroll
    for (int j = 0; j < KP; ++j) {
      if (r == j) {
        x[j] = clamp_piv(x[j], pfloor);
        rp[j] = 1.f / x[j];
#pragma unroll
        for (int q = 0; q < KP / 4; ++q)
          *reinterpret_cast<float4*>(D + j * SD + 4 * q) = make_float4(x[4 * q], x[4 * q + 1], x[4 * q + 2], x[4 * q + 3]);
      }
      asm volatile("bar.sync 1, 64;\n" ::: "memory");
      if (r > j) {
        const float* uj = D + j * SD;
        const float l = x[j] * (1.f / lds1(uj + j));
        x[j] = l;
#pragma unroll
        for (int c = j + 1; c < KP && (c & 3); ++c) x[c] = fmaf(-l, lds1(uj + c), x[c]);
#pragma unroll
        for (int c4 = ((j + 1) + 3) & ~3; c4 < KP; c4 += 4) {
          const float4 u = lds4(uj + c4);
          x[c4] = fmaf(-l, u.x, x[c4]);
          x[c4 + 1] = fmaf(-l, u.y, x[c4 + 1]);
          x[c4 + 2] = fmaf(-l, u.z, x[c4 + 2]);
          x[c4 + 3] = fmaf(-l, u.w, x[c4 + 3]);
        }
      }
    }
  }
  __syncthreads();
}

// x <- x M^-1 for the 64 values x of one thread, M upper triangular given by
// its rows (stride SD) in shared memory: after x_p is final, x_q -= x_p M_pq
// for q > p.  SCALE: x_p is multiplied by rp[p] (1 / M_pp) first; else M has
// a unit diagonal.
template <bool SCALE>
__device__ __forceinline__ void subst64(float (&x)[KP], const float* M, const float* rp) {
#pragma unroll
  for (int p = 0; p < KP; ++p) {
    if (SCALE) x[p] *= lds1(rp + p);
    const float xp = x[p];
    const float* mp = M + p * SD;
#pragma unroll
    for (int q = p + 1; q < KP && (q & 3); ++q) x[q] = fmaf(-xp, lds1(mp + q), x[q]);
#pragma unroll
    for (int q4 = ((p + 1) + 3) & ~3; q4 < KP; q4 += 4) {
      const float4 u = lds4(mp + q4);
      x[q4] = fmaf(-xp, u.x, x[q4]);
      x[q4 + 1] = fmaf(-xp, u.y, x[q4 + 1]);
      x[q4 + 2] = fmaf(-xp, u.z, x[q4 + 2]);
      x[q4 + 3] = fmaf(-xp, u.w, x[q4 + 3]);
    }
  }
}

// L21 = A21 U11^-1 (x U11 = a per row), one thread per row (with parts > 1:
// rows part * BS + tid, then every parts * BS).
__device__ __noinline__ void trsm_rows(float* A21, int ld, int M, const float* D, const float* rp, int part = 0,
                                       int parts = 1) {
  for (int r = part * BS + threadIdx.x; r < M; r += BS * parts) {
    float4* row = reinterpret_cast<float4*>(A21 + (int64_t)r * ld);
    float x[KP];
#pragma unroll
    for (int q = 0; q < KP / 4; ++q) {
      const float4 v = row[q];
      x[4 * q] = v.x;
      x[4 * q + 1] = v.y;
      x[4 * q + 2] = v.z;
      x[4 * q + 3] = v.w;
    }
    subst64<true>(x, D, rp);
#pragma unroll
    for (int q = 0; q < KP / 4; ++q) row[q] = make_float4(x[4 * q], x[4 * q + 1], x[4 * q + 2], x[4 * q + 3]);
  }
}

// U12 = L11^-1 A12 (per column: y^T L11^T = a^T, L11^T upper with unit
// diagonal, given by its rows LT = rows of L11^T), one thread per column.
__device__ __noinline__ void trsm_cols(float* A12, int ld, int N, const float* LT, int part = 0, int parts = 1) {
  for (int c = part * BS + threadIdx.x; c < N; c += BS * parts) {
    float y[KP];
    const float* src = A12 + c;
#pragma unroll
    for (int r = 0; r < KP; ++r, src += ld) {
      y[r] = *src;
      if ((r & 15) == 15) asm volatile("" ::: "memory");  // at most 16 loads in flight
    }
    subst64<false>(y, LT, nullptr);
    // the stores walk the column again from an opaque copy of ld, so the 64
    // load addresses are not kept alive across the substitution
    int ld2;
    asm volatile("mov.b32 %0, %1;\n" : "=r"(ld2) : "r"(ld));
    float* dst = A12 + c;
#pragma unroll
    for (int r = 0; r < KP; ++r, dst += ld2) *dst = y[r];
  }
}

// LU of A (n x n, leading dimension ld) in place.
__device__ void lu(float* A, int n, int ld, float* smem, double pfloor) {
  float* D = smem;
  float* rp = D + Smem::d_elems;
  float* sA = rp + Smem::r_elems;
  float* sB = sA + Smem::a_elems;
  const int tid = threadIdx.x;
  for (int k0 = 0; k0 < n; k0 += KP) {
    const int kb = min(KP, n - k0);
    float* Akk = A + (int64_t)k0 * ld + k0;
    for (int idx = tid; idx < KP * KP; idx += BS) {
      const int r = idx >> 6, c = idx & 63;
      D[r * SD + c] = (r < kb && c < kb) ? Akk[(int64_t)r * ld + c] : (r == c ? 1.f : 0.f);
    }
    __syncthreads();
    factor_diag(D, rp, pfloor);
    for (int idx = tid; idx < kb * kb; idx += BS) {
      const int r = idx / kb, c = idx % kb;
      Akk[(int64_t)r * ld + c] = D[r * SD + c];
    }
    const int m = n - k0 - kb;  // > 0 only with kb == 64
    if (m > 0) {
      float* A21 = A + (int64_t)(k0 + kb) * ld + k0;
      float* A12 = A + (int64_t)k0 * ld + k0 + kb;
      float* A22 = A + (int64_t)(k0 + kb) * ld + k0 + kb;
      // L11^T into the (idle) tile staging area for the column solves
      float* LT = sA;
      for (int idx = tid; idx < KP * KP; idx += BS) {
        const int r = idx >> 6, c = idx & 63;
        LT[c * SD + r] = r > c ? D[r * SD + c] : 0.f;
      }
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
// Each CTA factors the diagonal block itself (the 64 x 64 block is cheap and
// every CTA needs it in its own shared memory), the row and column
// substitutions and the trailing-update tiles are split by rank, and three
// cluster barriers per panel order the stages.  Every element goes through
// the same operations in the same order as in lu(), so the factor is
// bit-identical.  Every CTA of the cluster must call it with the same n.
__device__ void lu_cluster(float* A, int n, int ld, float* smem, double pfloor, int part, int parts) {
  float* D = smem;
  float* rp = D + Smem::d_elems;
  float* sA = rp + Smem::r_elems;
  float* sB = sA + Smem::a_elems;
  const int tid = threadIdx.x;
  for (int k0 = 0; k0 < n; k0 += KP) {
    const int kb = min(KP, n - k0);
    float* Akk = A + (int64_t)k0 * ld + k0;
    for (int idx = tid; idx < KP * KP; idx += BS) {
      const int r = idx >> 6, c = idx & 63;
      D[r * SD + c] = (r < kb && c < kb) ? Akk[(int64_t)r * ld + c] : (r == c ? 1.f : 0.f);
    }
    __syncthreads();
    factor_diag(D, rp, pfloor);
    cluster_sync_all();  // every CTA holds the block: rank 0 may write it back below
    const int m = n - k0 - kb;  // > 0 only with kb == 64
    float* A21 = A + (int64_t)(k0 + kb) * ld + k0;
    float* A12 = A + (int64_t)k0 * ld + k0 + kb;
    float* A22 = A + (int64_t)(k0 + kb) * ld + k0 + kb;
    if (m > 0) {
      float* LT = sA;
      for (int idx = tid; idx < KP * KP; idx += BS) {
        const int r = idx >> 6, c = idx & 63;
        LT[c * SD + r] = r > c ? D[r * SD + c] : 0.f;
      }
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

}  // namespace dense32
}  // namespace gs2g
