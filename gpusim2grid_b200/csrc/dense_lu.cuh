// Dense LU (no pivoting) of one matrix by one CTA, for the tail of the
// batched Newton–Raphson factorization.  Device code only.
//
// Right-looking with 64-wide panels.  Per panel:
//   1. the 64x64 diagonal block is factored in shared memory,
//   2. its triangular factors are inverted in shared memory (blocked 2x2 on
//      32x32 sub-blocks, the diagonal ones by one warp each in registers),
//   3. L21 = A21 U11^-1 and U12 = L11^-1 A12 run as CTA GEMM tiles,
//   4. the trailing matrix A22 -= L21 U12 runs as CTA GEMM tiles.
// GEMM tiles: FP64 DMMA (mma.sync m8n8k4) for double, a 4x8 register-tiled
// SIMT FFMA loop for float.  K streams through shared memory in KC-deep
// slabs with cp.async, double buffered across slabs and across tiles.  A tile
// accumulates all of K before writing its output, so an output tile may
// alias its own inputs (steps 3 and 4 work in place).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace gs2g {
namespace dense {

constexpr int BS = 256;  // threads per CTA (8 warps)
constexpr int KP = 64;   // panel width = largest K of a GEMM tile
#ifndef GS2G_DENSE_KC
#define GS2G_DENSE_KC 16
#endif
constexpr int KC = GS2G_DENSE_KC;  // K slab depth (build-time tunable)
constexpr int SD = KP + 1;  // diagonal block [KP][SD]
// The inverse buffer is read as a DMMA B operand (U11^-1, k rows x n cols:
// stride = 8 mod 16 avoids bank conflicts) or A operand (L11^-1, m rows x k
// cols: stride = 4 mod 16).
constexpr int SI_U = KP + 8;
constexpr int SI_L = KP + 4;
constexpr int SI_MAX = SI_U;

template <typename T>
struct Cfg;
template <>
struct Cfg<double> {
  static constexpr int TMt = 64, TNt = 64;  // CTA output tile
  static constexpr int SA = KC + 4;         // A slab [TMt][SA] (m, k): 4 mod 16
  static constexpr int SB = TNt + 8;        // B slab [KC][SB] (k, n): 8 mod 16
};
template <>
struct Cfg<float> {
  static constexpr int TMt = 64, TNt = 128;
  static constexpr int SA = KC + 4;
  static constexpr int SB = TNt + 4;
};

template <typename T>
struct Smem {
  static constexpr int d_elems = KP * SD;
  static constexpr int i_elems = KP * SI_MAX;
  static constexpr int a_elems = Cfg<T>::TMt * Cfg<T>::SA;
  static constexpr int b_elems = KC * Cfg<T>::SB;
  static constexpr int stage = a_elems + b_elems;
  // diagonal block, one triangular inverse, two slab stages
  static constexpr int elems = d_elems + i_elems + 2 * stage;
  static constexpr int bytes = elems * (int)sizeof(T);
};

template <typename T>
__device__ __forceinline__ T clamp_piv(T piv, double floor_) {
  const T f = (T)floor_;
  if (fabs(piv) < f) return piv < T(0) ? -f : f;
  return piv;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Stage one K slab of a tile into shared memory with 16-byte cp.async
// (zero-filled outside [M) x [K) and [K) x [N)).  Global operands must have
// 16-byte aligned rows and even (double) / multiple-of-4 (float) K offsets.
template <typename T, bool A_SMEM, bool B_SMEM>
__device__ __forceinline__ void stage_slab(T* sA, T* sB, const T* A, int lda, const T* B, int ldb, int M, int N,
                                           int K, int i0, int j0, int kc) {
  using CF = Cfg<T>;
  constexpr int EPC = 16 / sizeof(T);  // elements per 16-byte chunk
  const int tid = threadIdx.x;
  const int kn = min(KC, K - kc);
  if (!A_SMEM) {
    constexpr int CPR = KC / EPC;  // chunks per slab row
    for (int c = tid; c < CF::TMt * CPR; c += BS) {
      const int r = c / CPR, k = (c % CPR) * EPC;
      int bytes = (i0 + r < M) ? (kn - k) * (int)sizeof(T) : 0;
      bytes = bytes < 0 ? 0 : (bytes > 16 ? 16 : bytes);
      const T* src = bytes ? A + (int64_t)(i0 + r) * lda + kc + k : A;
      cp_async16(sA + r * CF::SA + k, src, bytes);
    }
  }
  if (!B_SMEM) {
    constexpr int CPR = CF::TNt / EPC;
    for (int c = tid; c < KC * CPR; c += BS) {
      const int k = c / CPR, n = (c % CPR) * EPC;
      int bytes = (k < kn) ? (N - j0 - n) * (int)sizeof(T) : 0;
      bytes = bytes < 0 ? 0 : (bytes > 16 ? 16 : bytes);
      const T* src = bytes ? B + (int64_t)(kc + k) * ldb + j0 + n : B;
      cp_async16(sB + k * CF::SB + n, src, bytes);
    }
  }
  cp_async_commit();
}

// ---------------------------------------------------------------------------
// CTA GEMM: C[M x N] (MODE 0: -=, MODE 1: =) A[M x K] B[K x N], K <= KP.
// A_SMEM / B_SMEM: that operand already sits in shared memory (stride
// lda / ldb) and is read in place; otherwise it streams from global memory.
// ---------------------------------------------------------------------------
// With parts > 1 the CTA computes the output tiles part, part + parts, ...
// (the CTAs of a cluster split them); a tile's arithmetic does not depend on
// which CTA computes it.
template <int MODE, bool A_SMEM, bool B_SMEM>
__device__ void gemm(double* C, int ldc, const double* A, int lda, const double* B, int ldb, int M, int N, int K,
                     double* stages, int part = 0, int parts = 1) {
  using CF = Cfg<double>;
  using SM = Smem<double>;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 2, wn = warp & 3;  // 2 x 4 warps, warp tile 32 x 16
  const int g = lane >> 2, q = lane & 3;
  const int n_tj = (N + CF::TNt - 1) / CF::TNt;
  const int n_sl = (K + KC - 1) / KC;
  const int n_tiles = ((M + CF::TMt - 1) / CF::TMt) * n_tj;
  const int my_tiles = part < n_tiles ? (n_tiles - part + parts - 1) / parts : 0;
  const int n_items = my_tiles * n_sl;
  if (n_items == 0) return;
  auto coords = [&](int item, int& i0, int& j0, int& kc) {
    const int tile = part + (item / n_sl) * parts;
    kc = (item % n_sl) * KC;
    i0 = (tile / n_tj) * CF::TMt;
    j0 = (tile % n_tj) * CF::TNt;
  };
  {
    int i0, j0, kc;
    coords(0, i0, j0, kc);
    stage_slab<double, A_SMEM, B_SMEM>(stages, stages + SM::a_elems, A, lda, B, ldb, M, N, K, i0, j0, kc);
  }
  const double sgn = MODE == 0 ? -1.0 : 1.0;
  double acc[4][2][2];
  for (int item = 0; item < n_items; ++item) {
    int i0, j0, kc;
    coords(item, i0, j0, kc);
    if (kc == 0) {
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) {
          const int r = i0 + wm * 32 + mt * 8 + g;
          const int c = j0 + wn * 16 + nt * 8 + 2 * q;
          double c0 = 0.0, c1 = 0.0;
          if (MODE == 0 && r < M) {
            if (c < N) c0 = C[(int64_t)r * ldc + c];
            if (c + 1 < N) c1 = C[(int64_t)r * ldc + c + 1];
          }
          acc[mt][nt][0] = c0;
          acc[mt][nt][1] = c1;
        }
    }
    cp_async_wait_all();
    __syncthreads();  // slab `item` visible; every warp is done with slab item-1
    const double* sA = stages + (item & 1) * SM::stage;
    const double* sB = sA + SM::a_elems;
    if (item + 1 < n_items) {
      int ni0, nj0, nkc;
      coords(item + 1, ni0, nj0, nkc);
      double* nA = stages + ((item + 1) & 1) * SM::stage;
      stage_slab<double, A_SMEM, B_SMEM>(nA, nA + SM::a_elems, A, lda, B, ldb, M, N, K, ni0, nj0, nkc);
    }
    const int kend = (min(KC, K - kc) + 3) & ~3;
    for (int k = 0; k < kend; k += 4) {
      double a[4], b[2];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        const int m = wm * 32 + mt * 8 + g;
        double v;
        if (A_SMEM)
          v = (i0 + m < M && kc + k + q < K) ? A[(int64_t)(i0 + m) * lda + kc + k + q] : 0.0;
        else
          v = sA[m * CF::SA + k + q];
        a[mt] = sgn * v;
      }
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) {
        const int n = wn * 16 + nt * 8 + g;
        if (B_SMEM)
          b[nt] = (kc + k + q < K && j0 + n < N) ? B[(int64_t)(kc + k + q) * ldb + j0 + n] : 0.0;
        else
          b[nt] = sB[(k + q) * CF::SB + n];
      }
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
          asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                       : "+d"(acc[mt][nt][0]), "+d"(acc[mt][nt][1])
                       : "d"(a[mt]), "d"(b[nt]));
    }
    if (kc + KC >= K) {
      // last slab of this tile: all of its inputs have been read into registers
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) {
          const int r = i0 + wm * 32 + mt * 8 + g;
          const int c = j0 + wn * 16 + nt * 8 + 2 * q;
          if (r < M) {
            if (c < N) C[(int64_t)r * ldc + c] = acc[mt][nt][0];
            if (c + 1 < N) C[(int64_t)r * ldc + c + 1] = acc[mt][nt][1];
          }
        }
    }
  }
  __syncthreads();
}

template <int MODE, bool A_SMEM, bool B_SMEM>
__device__ void gemm(float* C, int ldc, const float* A, int lda, const float* B, int ldb, int M, int N, int K,
                     float* stages) {
  using CF = Cfg<float>;
  using SM = Smem<float>;
  const int tid = threadIdx.x;
  const int tr = tid >> 4, tc = tid & 15;  // 16 x 16 threads, 4 x 8 each
  const int n_tj = (N + CF::TNt - 1) / CF::TNt;
  const int n_sl = (K + KC - 1) / KC;
  const int n_items = ((M + CF::TMt - 1) / CF::TMt) * n_tj * n_sl;
  if (n_items == 0) return;
  auto coords = [&](int item, int& i0, int& j0, int& kc) {
    const int tile = item / n_sl;
    kc = (item % n_sl) * KC;
    i0 = (tile / n_tj) * CF::TMt;
    j0 = (tile % n_tj) * CF::TNt;
  };
  {
    int i0, j0, kc;
    coords(0, i0, j0, kc);
    stage_slab<float, A_SMEM, B_SMEM>(stages, stages + SM::a_elems, A, lda, B, ldb, M, N, K, i0, j0, kc);
  }
  const float sgn = MODE == 0 ? -1.f : 1.f;
  float acc[4][8];
  for (int item = 0; item < n_items; ++item) {
    int i0, j0, kc;
    coords(item, i0, j0, kc);
    if (kc == 0) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int r = i0 + tr * 4 + i;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int c = j0 + tc * 8 + j;
          acc[i][j] = (MODE == 0 && r < M && c < N) ? C[(int64_t)r * ldc + c] : 0.f;
        }
      }
    }
    cp_async_wait_all();
    __syncthreads();
    const float* sA = stages + (item & 1) * SM::stage;
    const float* sB = sA + SM::a_elems;
    if (item + 1 < n_items) {
      int ni0, nj0, nkc;
      coords(item + 1, ni0, nj0, nkc);
      float* nA = stages + ((item + 1) & 1) * SM::stage;
      stage_slab<float, A_SMEM, B_SMEM>(nA, nA + SM::a_elems, A, lda, B, ldb, M, N, K, ni0, nj0, nkc);
    }
    const int kn = min(KC, K - kc);
    for (int k = 0; k < kn; ++k) {
      float a[4], b[8];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int m = tr * 4 + i;
        const float v = A_SMEM ? ((i0 + m < M) ? A[(int64_t)(i0 + m) * lda + kc + k] : 0.f) : sA[m * CF::SA + k];
        a[i] = sgn * v;
      }
      if (B_SMEM) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int n = j0 + tc * 8 + j;
          b[j] = n < N ? B[(int64_t)(kc + k) * ldb + n] : 0.f;
        }
      } else {
        const float4 b0 = *reinterpret_cast<const float4*>(sB + k * CF::SB + tc * 8);
        const float4 b1 = *reinterpret_cast<const float4*>(sB + k * CF::SB + tc * 8 + 4);
        b[0] = b0.x; b[1] = b0.y; b[2] = b0.z; b[3] = b0.w;
        b[4] = b1.x; b[5] = b1.y; b[6] = b1.z; b[7] = b1.w;
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    if (kc + KC >= K) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int r = i0 + tr * 4 + i;
        if (r >= M) continue;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int c = j0 + tc * 8 + j;
          if (c < N) C[(int64_t)r * ldc + c] = acc[i][j];
        }
      }
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// The diagonal tile D is always a full KP x KP block: rows/columns past the
// panel width kb are padded with the identity, so the warp routines below run
// fixed-size, predicate-free loops (the padding factors trivially and its
// couplings to the real block are zero).
// ---------------------------------------------------------------------------

// 32x32 LU of a diagonal sub-block by the calling warp, one row per lane in
// registers.  D points at the sub-block inside the [KP][SD] tile.
template <typename T>
__device__ __noinline__ void warp_lu32(T* D, double pfloor) {
  const int lane = threadIdx.x & 31;
  T x[32];
#pragma unroll
  for (int c = 0; c < 32; ++c) x[c] = D[lane * SD + c];
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    const T piv = clamp_piv(__shfl_sync(0xffffffffu, x[j], j), pfloor);
    if (lane == j) x[j] = piv;
    const T l = x[j] / piv;
    const bool below = lane > j;
    if (below) x[j] = l;
#pragma unroll
    for (int c = j + 1; c < 32; ++c) {
      const T u = __shfl_sync(0xffffffffu, x[c], j);
      if (below) x[c] = fma(-l, u, x[c]);
    }
  }
#pragma unroll
  for (int c = 0; c < 32; ++c) D[lane * SD + c] = x[c];
}

// Row lane of D21 <- D21 U11^{-1} (U11 = upper part of D11).
template <typename T>
__device__ __noinline__ void warp_row_trsm32(T* D) {
  const int r = 32 + (threadIdx.x & 31);
  T x[32];
#pragma unroll
  for (int c = 0; c < 32; ++c) x[c] = D[r * SD + c];
#pragma unroll
  for (int c = 0; c < 32; ++c) {
    T v = x[c];
#pragma unroll
    for (int p = 0; p < c; ++p) v = fma(-x[p], D[p * SD + c], v);
    x[c] = v / D[c * SD + c];
  }
#pragma unroll
  for (int c = 0; c < 32; ++c) D[r * SD + c] = x[c];
}

// Column lane of D12 <- L11^{-1} D12 (L11 = unit-lower part of D11).
template <typename T>
__device__ __noinline__ void warp_col_trsm32(T* D) {
  const int c = 32 + (threadIdx.x & 31);
  T x[32];
#pragma unroll
  for (int r = 0; r < 32; ++r) x[r] = D[r * SD + c];
#pragma unroll
  for (int r = 1; r < 32; ++r) {
    T v = x[r];
#pragma unroll
    for (int p = 0; p < r; ++p) v = fma(-D[r * SD + p], x[p], v);
    x[r] = v;
  }
#pragma unroll
  for (int r = 0; r < 32; ++r) D[r * SD + c] = x[r];
}

// LU of the (identity-padded) KP x KP diagonal tile in shared memory.
template <typename T>
__device__ void diag_lu(T* D, double pfloor) {
  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) warp_lu32(D, pfloor);
  __syncthreads();
  if (warp == 1) warp_row_trsm32(D);
  else if (warp == 2) warp_col_trsm32(D);
  __syncthreads();
  // D22 -= L21 U12 (32 x 32 x 32)
  T out[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int idx = tid + t * BS;
    const int r = 32 + (idx >> 5), c = 32 + (idx & 31);
    T v = D[r * SD + c];
#pragma unroll 8
    for (int p = 0; p < 32; ++p) v = fma(-D[r * SD + p], D[p * SD + c], v);
    out[t] = v;
  }
  __syncthreads();
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int idx = tid + t * BS;
    D[(32 + (idx >> 5)) * SD + 32 + (idx & 31)] = out[t];
  }
  __syncthreads();
  if (warp == 0) warp_lu32(D + 32 * SD + 32, pfloor);
  __syncthreads();
}

// Inverse of the 32x32 triangular block at D (stride SD) into Inv (stride
// si), by the calling warp: lane j computes column j in registers.
// UPPER: U^{-1}; else unit-lower L^{-1}.
template <bool UPPER, typename T>
__device__ __noinline__ void warp_tri_inv32(const T* D, T* Inv, int si) {
  const int j = threadIdx.x & 31;
  T x[32];
  if (UPPER) {
#pragma unroll
    for (int i = 31; i >= 0; --i) {
      T v = (i == j) ? T(1) : T(0);
#pragma unroll
      for (int k = i + 1; k < 32; ++k) v = fma(-D[i * SD + k], x[k], v);
      x[i] = v / D[i * SD + i];
    }
  } else {
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      T v = (i == j) ? T(1) : T(0);
#pragma unroll
      for (int k = 0; k < i; ++k) v = fma(-D[i * SD + k], x[k], v);
      x[i] = v;
    }
  }
#pragma unroll
  for (int i = 0; i < 32; ++i) Inv[i * si + j] = x[i];
}

// Inverse of a triangular factor of the kb x kb diagonal tile D into Inv
// (stride si, zero elsewhere up to KP), blocked on 32x32 sub-blocks:
//   U^{-1} = [U11^-1, -U11^-1 U12 U22^-1; 0, U22^-1]
//   L^{-1} = [L11^-1, 0; -L22^-1 L21 L11^-1, L22^-1]
template <bool UPPER, typename T>
__device__ void diag_inverse(const T* D, T* Inv, int si) {
  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) warp_tri_inv32<UPPER>(D, Inv, si);
  if (warp == 1) warp_tri_inv32<UPPER>(D + 32 * SD + 32, Inv + 32 * si + 32, si);
  __syncthreads();
  T out[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {  // X = U12 U22^-1, or X = L21 L11^-1
    const int idx = tid + t * BS;
    const int r = idx >> 5, c = idx & 31;
    T v = T(0);
#pragma unroll 8
    for (int p = 0; p < 32; ++p)
      v = UPPER ? fma(D[r * SD + 32 + p], Inv[(32 + p) * si + 32 + c], v)
                : fma(D[(32 + r) * SD + p], Inv[p * si + c], v);
    out[t] = v;
  }
  // the block that is zero in the result holds X meanwhile
  T* X = UPPER ? Inv + 32 * si : Inv + 32;
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int idx = tid + t * BS;
    X[(idx >> 5) * si + (idx & 31)] = out[t];
  }
  __syncthreads();
#pragma unroll
  for (int t = 0; t < 4; ++t) {  // Inv12 = -U11^-1 X, or Inv21 = -L22^-1 X
    const int idx = tid + t * BS;
    const int r = idx >> 5, c = idx & 31;
    T v = T(0);
#pragma unroll 8
    for (int p = 0; p < 32; ++p)
      v = UPPER ? fma(Inv[r * si + p], X[p * si + c], v) : fma(Inv[(32 + r) * si + 32 + p], X[p * si + c], v);
    out[t] = -v;
  }
  __syncthreads();
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int idx = tid + t * BS;
    const int r = idx >> 5, c = idx & 31;
    X[r * si + c] = T(0);
    if (UPPER)
      Inv[r * si + 32 + c] = out[t];
    else
      Inv[(32 + r) * si + c] = out[t];
  }
  __syncthreads();
}

// LU of A (n x n, row-major, leading dimension ld, global memory, rows
// 16-byte aligned), in place.
template <typename T>
__device__ void lu(T* A, int n, int ld, T* smem, double pfloor) {
  using SM = Smem<T>;
  T* D = smem;
  T* Inv = D + SM::d_elems;
  T* stages = Inv + SM::i_elems;
  const int tid = threadIdx.x;
  for (int k0 = 0; k0 < n; k0 += KP) {
    const int kb = min(KP, n - k0);
    T* Akk = A + (int64_t)k0 * ld + k0;
    for (int idx = tid; idx < KP * KP; idx += BS) {
      const int r = idx / KP, c = idx % KP;
      D[r * SD + c] = (r < kb && c < kb) ? Akk[(int64_t)r * ld + c] : T(r == c ? 1 : 0);
    }
    __syncthreads();
    diag_lu(D, pfloor);
    for (int idx = tid; idx < kb * kb; idx += BS) {
      const int r = idx / kb, c = idx % kb;
      Akk[(int64_t)r * ld + c] = D[r * SD + c];
    }
    const int m = n - k0 - kb;
    if (m > 0) {
      T* A21 = A + (int64_t)(k0 + kb) * ld + k0;
      T* A12 = A + (int64_t)k0 * ld + k0 + kb;
      T* A22 = A + (int64_t)(k0 + kb) * ld + k0 + kb;
      diag_inverse<true>(D, Inv, SI_U);
      gemm<1, false, true>(A21, ld, A21, ld, Inv, SI_U, m, kb, kb, stages);  // L21 = A21 U11^-1
      diag_inverse<false>(D, Inv, SI_L);
      gemm<1, true, false>(A12, ld, Inv, SI_L, A12, ld, kb, m, kb, stages);  // U12 = L11^-1 A12
      gemm<0, false, false>(A22, ld, A21, ld, A12, ld, m, m, kb, stages);    // A22 -= L21 U12
    }
    __syncthreads();
  }
}

// Barrier over every thread of every CTA of the cluster, ordering the
// memory accesses before it (global and distributed shared) before those
// after it.  Block-uniform calls only.
__device__ __forceinline__ void cluster_barrier() {
  __threadfence();
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// The same FP64 LU as lu(), by the `parts` CTAs of a cluster together (this
// CTA has rank `part`); A in global memory, every CTA with its own scratch.
// Every CTA factors and inverts the 64 x 64 diagonal block itself (cheap,
// and each needs it in its own shared memory); the tiles of L21, U12 and the
// trailing update are split by rank, and three cluster barriers per panel
// order the stages.  Each element goes through the same operations in the
// same order as in lu(), so the factor is bit-identical.  Every CTA of the
// cluster must call it with the same n.
__device__ void lu_cluster(double* A, int n, int ld, double* smem, double pfloor, int part, int parts) {
  using SM = Smem<double>;
  double* D = smem;
  double* Inv = D + SM::d_elems;
  double* stages = Inv + SM::i_elems;
  const int tid = threadIdx.x;
  for (int k0 = 0; k0 < n; k0 += KP) {
    const int kb = min(KP, n - k0);
    double* Akk = A + (int64_t)k0 * ld + k0;
    for (int idx = tid; idx < KP * KP; idx += BS) {
      const int r = idx / KP, c = idx % KP;
      D[r * SD + c] = (r < kb && c < kb) ? Akk[(int64_t)r * ld + c] : (r == c ? 1.0 : 0.0);
    }
    __syncthreads();
    diag_lu(D, pfloor);
    cluster_barrier();  // every CTA holds the block: rank 0 may write it back below
    const int m = n - k0 - kb;
    if (m > 0) {
      double* A21 = A + (int64_t)(k0 + kb) * ld + k0;
      double* A12 = A + (int64_t)k0 * ld + k0 + kb;
      diag_inverse<true>(D, Inv, SI_U);
      gemm<1, false, true>(A21, ld, A21, ld, Inv, SI_U, m, kb, kb, stages, part, parts);  // L21 = A21 U11^-1
      __syncthreads();
      diag_inverse<false>(D, Inv, SI_L);
      gemm<1, true, false>(A12, ld, Inv, SI_L, A12, ld, kb, m, kb, stages, part, parts);  // U12 = L11^-1 A12
    }
    if (part == 0)
      for (int idx = tid; idx < kb * kb; idx += BS) {
        const int r = idx / kb, c = idx % kb;
        Akk[(int64_t)r * ld + c] = D[r * SD + c];
      }
    cluster_barrier();  // L21, U12 and the diagonal block complete
    if (m > 0) {
      double* A21 = A + (int64_t)(k0 + kb) * ld + k0;
      double* A12 = A + (int64_t)k0 * ld + k0 + kb;
      double* A22 = A + (int64_t)(k0 + kb) * ld + k0 + kb;
      gemm<0, false, false>(A22, ld, A21, ld, A12, ld, m, m, kb, stages, part, parts);  // A22 -= L21 U12
    }
    cluster_barrier();  // A22 complete
  }
}

}  // namespace dense
}  // namespace gs2g
