// Kernels of the warm-start MLP: a BF16 GEMM on the 5th-generation tensor
// cores (tcgen05.mma, accumulator in tensor memory) and the elementwise
// pieces of the forward pass, the backward pass and the Adam step.
//
// GEMM form: D[M x N] (fp32) = A[M x K] . B[N x K]^T (+ D), A and B bf16,
// row-major with K contiguous ("TN"); every other product of the MLP is
// brought to this form by explicit transposes.  M, N multiples of 128, K a
// multiple of 64, leading dimensions multiples of 8 elements.
//
// One CTA (4 warps) computes one 128 x 128 tile.  K streams in 64-deep
// stages through a 3-stage shared-memory ring filled with cp.async; each
// stage is laid out in the canonical no-swizzle K-major UMMA layout (8-row x
// 16-byte core matrices; LBO = 128 B between the two K halves of one MMA,
// SBO = 1024 B between 8-row groups).  Thread 0 issues four
// tcgen05.mma.kind::f16 (M=128, N=128, K=16) per stage and commits them to
// the stage's mbarrier; producers wait on that mbarrier before refilling the
// stage.  The epilogue reads the 128 x 128 fp32 accumulator from TMEM
// (tcgen05.ld 32x32b: warp w owns lanes 32w..32w+31 = tile rows) and stores
// it.  Every mbarrier wait is bounded; on timeout the kernel sets *err and
// finishes without touching further data.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace gs2g {
namespace mlp {

constexpr int GT = 128;     // tile M = tile N
constexpr int GK = 64;      // K per stage
// operand ring depth: a stage is reloaded once the MMAs of the k-tile before
// it have completed (STAGES - 2 k-tiles of operands in flight).  6 stages
// (one CTA per SM) measured no faster than 3 (two CTAs per SM fit): with
// 128 x 128 tiles the operands are re-read from L2 at about 3.7 TB/s, which
// bounds the kernel before the ring depth does
#ifndef GS2G_GEMM_STAGES
#define GS2G_GEMM_STAGES 3
#endif
constexpr int STAGES = GS2G_GEMM_STAGES;
constexpr int GEMM_THREADS = 128;
constexpr int TILE_BYTES = GT * GK * 2;  // one operand tile per stage (16 KB)
constexpr int GEMM_SMEM = STAGES * 2 * TILE_BYTES + 1024;
constexpr uint64_t WAIT_NS = 2000000000ull;  // bound of one mbarrier wait (2 s)

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src));
}

// UMMA shared-memory descriptor, K-major, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, legacy LBO mode, layout SWIZZLE_NONE
}

// Instruction descriptor: kind::f16, A = B = bf16, D = f32, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for the phase with the given parity; false after WAIT_NS.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const uint64_t t0 = global_ns();
  for (uint32_t i = 0;; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if ((i & 255) == 255 && global_ns() - t0 > WAIT_NS) return false;
  }
}

__global__ void __launch_bounds__(GEMM_THREADS) gemm_tn_bf16_kernel(const __nv_bfloat16* __restrict__ A, int lda,
                                                                    const __nv_bfloat16* __restrict__ B, int ldb,
                                                                    float* __restrict__ D, int ldd, int K,
                                                                    int accumulate, int* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar[STAGES];
  __shared__ uint32_t tmem_base_s;
  __shared__ int s_fail;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * GT, n0 = blockIdx.x * GT;
  // 1024-byte aligned operand ring
  const uint32_t ring = (smem_u32(smem) + 1023) & ~1023u;
  auto a_tile = [&](int s) { return ring + (uint32_t)(s * 2 * TILE_BYTES); };
  auto b_tile = [&](int s) { return ring + (uint32_t)(s * 2 * TILE_BYTES + TILE_BYTES); };

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&mbar[s])));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
    s_fail = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_base_s)),
                 "r"(GT));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = tmem_base_s;

  const int KT = K / GK;
  // canonical layout offset of (row r, 16-byte k-chunk c) inside a tile
  auto load_stage = [&](int kt, int s) {
    const int k0 = kt * GK;
#pragma unroll
    for (int i = 0; i < (GT * GK / 8) / GEMM_THREADS; ++i) {
      const int idx = tid + i * GEMM_THREADS;  // 0 .. 1023
      const int r = idx >> 3, c = idx & 7;
      const uint32_t off = (uint32_t)((r >> 3) * 1024 + c * 128 + (r & 7) * 16);
      cp_async16(a_tile(s) + off, A + (int64_t)(m0 + r) * lda + k0 + c * 8);
      cp_async16(b_tile(s) + off, B + (int64_t)(n0 + r) * ldb + k0 + c * 8);
    }
  };
  // Group bookkeeping: the prologue commits k-tiles 0..STAGES-2 as groups
  // 0..STAGES-2; iteration kt commits one group (k-tile kt+STAGES-1, or
  // empty), so k-tile kt is always group kt, and at iteration kt the
  // STAGES-2 most recent groups may still be in flight.
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < KT) load_stage(s, s);
    asm volatile("cp.async.commit_group;\n" ::);
  }
  constexpr uint32_t idesc = umma_idesc_bf16(GT, GT);
  bool ok = true;
  int last = -1;  // last k-tile whose MMAs were committed
  for (int kt = 0; kt < KT; ++kt) {
    const int s = kt % STAGES;
    asm volatile("cp.async.wait_group %0;\n" ::"n"(STAGES - 2) : "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    if (__syncthreads_or(!ok)) {  // a timed-out wait anywhere stops every thread here
      ok = false;
      break;
    }
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
#pragma unroll
      for (int j = 0; j < GK / 16; ++j) {
        const uint64_t ad = umma_desc(a_tile(s) + j * 256, 128, 1024);
        const uint64_t bd = umma_desc(b_tile(s) + j * 256, 128, 1024);
        const uint32_t en = (kt > 0 || j > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(en), "r"(0), "r"(0), "r"(0), "r"(0));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
          smem_u32(&mbar[s])));
    }
    last = kt;
    // load k-tile kt+STAGES-1 into the stage k-tile kt-1 used (at kt = 0: the
    // still unused last stage), once k-tile kt-1's MMAs are done
    const int nk = kt + STAGES - 1;
    if (nk < KT) {
      const int ns = nk % STAGES;
      if (kt >= 1 && !mbar_wait(smem_u32(&mbar[ns]), (uint32_t)(((kt - 1) / STAGES) & 1))) ok = false;
      if (ok) load_stage(nk, ns);
    }
    asm volatile("cp.async.commit_group;\n" ::);
  }
  // wait for the last committed MMAs (after a failure too: TMEM is freed
  // only once they are done, or their wait has run out as well)
  if (last >= 0 && !mbar_wait(smem_u32(&mbar[last % STAGES]), (uint32_t)((last / STAGES) & 1))) ok = false;
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  if (__syncthreads_or(!ok) && tid == 0) s_fail = 1;
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  if (s_fail) {
    if (tid == 0) atomicExch(err, 1);
  } else {
    // epilogue: warp w reads TMEM lanes 32w..32w+31 (tile rows), 16 columns per load
    const int row = m0 + warp * 32 + lane;
    float* drow = D + (int64_t)row * ldd + n0;
#pragma unroll 1
    for (int c0 = 0; c0 < GT; c0 += 16) {
      uint32_t v[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
      for (int q = 0; q < 16; q += 4) {
        float4 o = make_float4(__uint_as_float(v[q]), __uint_as_float(v[q + 1]), __uint_as_float(v[q + 2]),
                               __uint_as_float(v[q + 3]));
        float4* dst = reinterpret_cast<float4*>(drow + c0 + q);
        if (accumulate) {
          const float4 old = *dst;
          o.x += old.x;
          o.y += old.y;
          o.z += old.z;
          o.w += old.w;
        }
        *dst = o;
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(GT));
  }
}

// ------------------------------------------------------------ elementwise
__device__ __forceinline__ float gelu_f(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad_f(float x) {
  const float cdf = 0.5f * (1.f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
  return cdf + x * pdf;
}

// pre[r][c] += bias[c]; act[r][c] = bf16(gelu(pre)) (or bf16(pre) when !gelu)
__global__ void bias_act_kernel(float* pre, int ldp, const float* bias, __nv_bfloat16* act, int lda, int rows,
                                int cols, int gelu) {
  const int64_t n = (int64_t)rows * cols;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / cols), c = (int)(i % cols);
    const float v = pre[(int64_t)r * ldp + c] + bias[c];
    pre[(int64_t)r * ldp + c] = v;
    if (act) act[(int64_t)r * lda + c] = __float2bfloat16(gelu ? gelu_f(v) : v);
  }
}

// dpre = dact * gelu'(pre) (fp32 in, bf16 out)
__global__ void gelu_bwd_kernel(const float* dact, int ldg, const float* pre, int ldp, __nv_bfloat16* dpre, int ldo,
                                int rows, int cols) {
  const int64_t n = (int64_t)rows * cols;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / cols), c = (int)(i % cols);
    dpre[(int64_t)r * ldo + c] =
        __float2bfloat16(dact[(int64_t)r * ldg + c] * gelu_grad_f(pre[(int64_t)r * ldp + c]));
  }
}

// dy = scale * (y - t) over the first `cols_valid` columns (0 elsewhere),
// bf16; loss += sum (y - t)^2 over valid entries.
__global__ void mse_grad_kernel(const float* y, const float* t, int ld, __nv_bfloat16* dy, int rows, int cols,
                                int cols_valid, float scale, float* loss) {
  const int64_t n = (int64_t)rows * cols;
  float acc = 0.f;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % cols);
    float g = 0.f;
    if (c < cols_valid) {
      const float d = y[i] - t[i];
      acc += d * d;
      g = scale * d;
    }
    dy[i] = __float2bfloat16(g);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, acc);
}

// column sums of a bf16 matrix: out[c] += sum_r x[r][c]; block (128 columns)
// x (a chunk of COLSUM_ROWS rows), one atomicAdd per column and chunk
constexpr int COLSUM_ROWS = 256;
__global__ void colsum_bf16_kernel(const __nv_bfloat16* x, int ld, int rows, int cols, float* out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  const int r0 = blockIdx.y * COLSUM_ROWS;
  const int r1 = min(rows, r0 + COLSUM_ROWS);
  float s = 0.f;
#pragma unroll 8
  for (int r = r0; r < r1; ++r) s += __bfloat162float(x[(int64_t)r * ld + c]);
  atomicAdd(out + c, s);
}

// out[c][r] = in[r][c] (bf16), 32x32 tiles through shared memory
__global__ void transpose_bf16_kernel(const __nv_bfloat16* in, int ldi, __nv_bfloat16* out, int ldo, int rows,
                                      int cols) {
  __shared__ __nv_bfloat16 t[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = r0 + k, c = c0 + threadIdx.x;
    t[k][threadIdx.x] = (r < rows && c < cols) ? in[(int64_t)r * ldi + c] : __float2bfloat16(0.f);
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int c = c0 + k, r = r0 + threadIdx.x;
    if (c < cols && r < rows) out[(int64_t)c * ldo + r] = t[threadIdx.x][k];
  }
}

__global__ void f32_to_bf16_kernel(const float* in, __nv_bfloat16* out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16(in[i]);
}

// Adam on fp32 master weights; writes the bf16 copy used by the GEMMs.
__global__ void adam_kernel(float* w, const float* g, float* m, float* v, __nv_bfloat16* wb, int64_t n, float lr,
                            float b1, float b2, float eps, float c1, float c2, float wd) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i] + wd * w[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16(wi);
  }
}

// Start voltages from predicted, standardised unknowns: for bus b of row r,
// Va = y[r][ia[b]] * std + mean when b is a pv/pq bus (ia[b] >= 0), else the
// angle of vinit[b]; Vm = y[r][im[b]] * std + mean when b is a pq bus
// (im[b] >= 0), else |vinit[b]|; V0 = Vm e^{j Va} (FP64).
__global__ void start_voltages_kernel(const float* y, int ldy, const float* ymean, const float* ystd, const int* ia,
                                      const int* im, const double2* vinit, int n_bus, double2* v0, int rows) {
  const int64_t n = (int64_t)rows * n_bus;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / n_bus), b = (int)(i % n_bus);
    const double2 v = vinit[b];
    double va = atan2(v.y, v.x), vm = hypot(v.x, v.y);
    const int a = ia[b], m = im[b];
    if (a >= 0) va = (double)y[(int64_t)r * ldy + a] * ystd[a] + ymean[a];
    if (m >= 0) vm = (double)y[(int64_t)r * ldy + m] * ystd[m] + ymean[m];
    double s, c;
    sincos(va, &s, &c);
    v0[i] = make_double2(vm * c, vm * s);
  }
}

// Standardised bf16 network inputs of the rows, in one pass (one CTA per
// row of the padded input block X [rows_pad x ldx]):
//   column c < n_pvpq:            Re(S_r - S_base) at bus pvpq[c]
//   column n_pvpq + c', c' < n_pq: Im(S_r - S_base) at bus pq[c']
//   (0 without injection rows)
//   plus, for every branch the row trips, the four contributions
//   br_val[4 b + k] at column br_col[4 b + k] (columns >= n_in dropped)
// then (x - mean) / std for c < n_in, 0 in the padding.  At most
// FEAT_MAX_TERMS trip contributions per row are held; more are read back
// from global memory per column.
constexpr int FEAT_MAX_TERMS = 256;
__global__ void features_kernel(const double2* __restrict__ sbus_rows, const double2* __restrict__ sbus_base,
                                const int* __restrict__ pvpq, int n_pvpq, const int* __restrict__ pq, int n_pq,
                                const int* __restrict__ trip_ptr, const int* __restrict__ trip_ids,
                                const int* __restrict__ br_col, const float* __restrict__ br_val,
                                const float* __restrict__ x_mean, const float* __restrict__ x_std, int n_in,
                                __nv_bfloat16* __restrict__ X, int ldx, int rows, int n_bus) {
  __shared__ int s_c[FEAT_MAX_TERMS];
  __shared__ float s_v[FEAT_MAX_TERMS];
  __shared__ int s_n;
  const int r = blockIdx.x;
  __nv_bfloat16* xr = X + (int64_t)r * ldx;
  if (r >= rows) {
    for (int c = threadIdx.x; c < ldx; c += blockDim.x) xr[c] = __float2bfloat16(0.f);
    return;
  }
  const int q0 = trip_ptr != nullptr ? trip_ptr[r] : 0, q1 = trip_ptr != nullptr ? trip_ptr[r + 1] : 0;
  if (threadIdx.x == 0) {
    int n = 0;
    for (int q = q0; q < q1 && n + 4 <= FEAT_MAX_TERMS; ++q) {
      const int b = trip_ids[q];
      for (int k = 0; k < 4; ++k) {
        const int c = br_col[4 * b + k];
        if (c >= 0 && c < n_in) {
          s_c[n] = c;
          s_v[n] = br_val[4 * b + k];
          ++n;
        }
      }
    }
    s_n = n;
  }
  __syncthreads();
  const int n_terms = s_n;
  const bool overflow = (q1 - q0) * 4 > FEAT_MAX_TERMS;
  const double2* sr = sbus_rows != nullptr ? sbus_rows + (int64_t)r * n_bus : nullptr;
  const int dim = n_pvpq + n_pq;
  for (int c = threadIdx.x; c < ldx; c += blockDim.x) {
    float v = 0.f;
    if (c < n_in) {
      if (sr != nullptr && c < dim) {
        const int b = c < n_pvpq ? pvpq[c] : pq[c - n_pvpq];
        v = c < n_pvpq ? (float)(sr[b].x - sbus_base[b].x) : (float)(sr[b].y - sbus_base[b].y);
      }
      if (!overflow) {
        for (int e = 0; e < n_terms; ++e)
          if (s_c[e] == c) v += s_v[e];
      } else {
        for (int q = q0; q < q1; ++q)
          for (int k = 0; k < 4; ++k)
            if (br_col[4 * trip_ids[q] + k] == c) v += br_val[4 * trip_ids[q] + k];
      }
      v = (v - x_mean[c]) / x_std[c];
    }
    xr[c] = __float2bfloat16(v);
  }
}

// First layer of the network for rows whose inputs have no injection part
// (sbus_rows NULL in features_kernel: outage rows at the base injections).
// Such a row's standardised input differs from the constant row
// xb_c = bf16((0 - mean_c) / std_c) only in the columns its tripped branches
// reach, so X W0^T = base + sum over those columns of
// (bf16(xs_c) - xb_c) W0[:, c], with base = xb W0^T (first_layer_base_kernel,
// once per set of weights) and W0T = W0^T [k0 x h] (coalesced over the
// outputs).  The column values are summed as features_kernel sums them.  A
// row with more than FEAT_MAX_TERMS contributions computes its full input
// row in shared memory and the whole dot product instead.  pre [rows_pad x
// ldp] fp32 (0 in the padding rows, as the GEMM of zero rows gives).
__global__ void sparse_first_layer_kernel(const float* __restrict__ base, const __nv_bfloat16* __restrict__ w0t,
                                          int h, const int* __restrict__ trip_ptr, const int* __restrict__ trip_ids,
                                          const int* __restrict__ br_col, const float* __restrict__ br_val,
                                          const float* __restrict__ x_mean, const float* __restrict__ x_std,
                                          int n_in, float* __restrict__ pre, int ldp, int rows) {
  extern __shared__ float s_x[];  // [n_in]: overflow rows only
  __shared__ int s_c[FEAT_MAX_TERMS];
  __shared__ float s_d[FEAT_MAX_TERMS];
  __shared__ int s_n;
  const int r = blockIdx.x;
  float* pr = pre + (int64_t)r * ldp;
  if (r >= rows) {
    for (int n = threadIdx.x; n < h; n += blockDim.x) pr[n] = 0.f;
    return;
  }
  const int q0 = trip_ptr[r], q1 = trip_ptr[r + 1];
  const bool overflow = (q1 - q0) * 4 > FEAT_MAX_TERMS;
  if (overflow) {
    // the row's full standardised input (features_kernel's overflow form)
    for (int c = threadIdx.x; c < n_in; c += blockDim.x) {
      float v = 0.f;
      for (int q = q0; q < q1; ++q)
        for (int k = 0; k < 4; ++k)
          if (br_col[4 * trip_ids[q] + k] == c) v += br_val[4 * trip_ids[q] + k];
      s_x[c] = __bfloat162float(__float2bfloat16((v - x_mean[c]) / x_std[c]));
    }
    __syncthreads();
    for (int n = threadIdx.x; n < h; n += blockDim.x) {
      float acc = 0.f;
      for (int c = 0; c < n_in; ++c) acc = fmaf(s_x[c], __bfloat162float(w0t[(int64_t)c * h + n]), acc);
      pr[n] = acc;
    }
    return;
  }
  if (threadIdx.x == 0) {
    int n = 0;
    for (int q = q0; q < q1; ++q) {
      const int b = trip_ids[q];
      for (int k = 0; k < 4; ++k) {
        const int c = br_col[4 * b + k];
        if (c < 0 || c >= n_in) continue;
        int e = 0;
        while (e < n && s_c[e] != c) ++e;
        if (e == n) {
          s_c[n] = c;
          s_d[n] = 0.f;
          ++n;
        }
        s_d[e] += br_val[4 * b + k];
      }
    }
    for (int e = 0; e < n; ++e) {
      const int c = s_c[e];
      const float xs = __bfloat162float(__float2bfloat16((s_d[e] - x_mean[c]) / x_std[c]));
      const float xb = __bfloat162float(__float2bfloat16((0.f - x_mean[c]) / x_std[c]));
      s_d[e] = xs - xb;
    }
    s_n = n;
  }
  __syncthreads();
  const int nt = s_n;
  for (int n = threadIdx.x; n < h; n += blockDim.x) {
    float acc = base[n];
    for (int e = 0; e < nt; ++e) acc = fmaf(s_d[e], __bfloat162float(w0t[(int64_t)s_c[e] * h + n]), acc);
    pr[n] = acc;
  }
}

// base[n] = sum_c bf16((0 - mean_c) / std_c) W0T[c][n] over the n_in input
// columns (one thread per output, fp32).
__global__ void first_layer_base_kernel(const __nv_bfloat16* __restrict__ w0t, int h,
                                        const float* __restrict__ x_mean, const float* __restrict__ x_std, int n_in,
                                        float* __restrict__ base) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= h) return;
  float acc = 0.f;
  for (int c = 0; c < n_in; ++c)
    acc = fmaf(__bfloat162float(__float2bfloat16((0.f - x_mean[c]) / x_std[c])),
               __bfloat162float(w0t[(int64_t)c * h + n]), acc);
  base[n] = acc;
}

inline int grid_for(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  if (b > 148 * 32) b = 148 * 32;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace mlp
}  // namespace gs2g

// ------------------------------------------------------------ C-ABI
// Status: 0 ok, 1 invalid argument, 3 CUDA error (see include/gs2g.h).
namespace gs2g {
void set_last_error(const char* msg);  // session.cpp
}
namespace {
using namespace gs2g::mlp;
int status_of(cudaError_t e) {
  if (e == cudaSuccess) return 0;
  gs2g::set_last_error(cudaGetErrorString(e));
  return e == cudaErrorInvalidValue ? 1 : 3;
}
int invalid(const char* what) {
  gs2g::set_last_error(what);
  return 1;
}
}  // namespace

extern "C" {

int gs2g_mlp_gemm_tn_bf16(const void* A, int lda, const void* B, int ldb, float* D, int ldd, int M, int N, int K,
                          int accumulate, int* err, void* stream) {
  if (M % GT || N % GT || K % GK || M <= 0 || N <= 0 || K <= 0)
    return invalid("gemm_tn_bf16: M, N must be positive multiples of 128 and K of 64");
  if (lda % 8 || ldb % 8 || ldd % 4 || lda < K || ldb < K || ldd < N || !err)
    return invalid("gemm_tn_bf16: leading dimensions must cover the rows and be 16-byte multiples");
  if (((uintptr_t)A | (uintptr_t)B | (uintptr_t)D) & 15) return invalid("gemm_tn_bf16: operands must be 16-byte aligned");
  cudaError_t e = cudaFuncSetAttribute(gemm_tn_bf16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM);
  if (e != cudaSuccess) return status_of(e);
  dim3 grid(N / GT, M / GT);
  gemm_tn_bf16_kernel<<<grid, GEMM_THREADS, GEMM_SMEM, (cudaStream_t)stream>>>(
      (const __nv_bfloat16*)A, lda, (const __nv_bfloat16*)B, ldb, D, ldd, K, accumulate, err);
  return status_of(cudaGetLastError());
}

int gs2g_mlp_bias_act(float* pre, int ldp, const float* bias, void* act_bf16, int lda, int rows, int cols, int gelu,
                      void* stream) {
  const int64_t n = (int64_t)rows * cols;
  if (n <= 0) return n < 0 ? invalid("bias_act: negative size") : 0;
  bias_act_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(pre, ldp, bias, (__nv_bfloat16*)act_bf16, lda,
                                                                      rows, cols, gelu);
  return status_of(cudaGetLastError());
}

int gs2g_mlp_gelu_bwd(const float* dact, int ldg, const float* pre, int ldp, void* dpre_bf16, int ldo, int rows,
                      int cols, void* stream) {
  const int64_t n = (int64_t)rows * cols;
  if (n <= 0) return n < 0 ? invalid("gelu_bwd: negative size") : 0;
  gelu_bwd_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(dact, ldg, pre, ldp, (__nv_bfloat16*)dpre_bf16,
                                                                      ldo, rows, cols);
  return status_of(cudaGetLastError());
}

int gs2g_mlp_mse_grad(const float* y, const float* t, int ld, void* dy_bf16, int rows, int cols, int cols_valid,
                      float scale, float* loss, void* stream) {
  const int64_t n = (int64_t)rows * cols;
  if (n == 0) return 0;
  if (n < 0 || ld != cols || cols_valid > cols) return invalid("mse_grad: ld must equal cols >= cols_valid");
  mse_grad_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(y, t, ld, (__nv_bfloat16*)dy_bf16, rows, cols,
                                                                      cols_valid, scale, loss);
  return status_of(cudaGetLastError());
}

int gs2g_mlp_colsum_bf16(const void* x, int ld, int rows, int cols, float* out, void* stream) {
  if (cols == 0) return 0;
  if (cols < 0 || rows < 0) return invalid("colsum: negative size");
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(float) * (size_t)cols, (cudaStream_t)stream);
  if (e != cudaSuccess || rows == 0) return status_of(e);
  dim3 grid((cols + 127) / 128, (rows + COLSUM_ROWS - 1) / COLSUM_ROWS);
  colsum_bf16_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)x, ld, rows, cols, out);
  return status_of(cudaGetLastError());
}

int gs2g_mlp_transpose_bf16(const void* in, int ldi, void* out, int ldo, int rows, int cols, void* stream) {
  if (rows < 0 || cols < 0) return invalid("transpose: negative size");
  if (rows == 0 || cols == 0) return 0;
  dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
  transpose_bf16_kernel<<<grid, block, 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)in, ldi, (__nv_bfloat16*)out,
                                                                  ldo, rows, cols);
  return status_of(cudaGetLastError());
}

int gs2g_mlp_to_bf16(const float* in, void* out, int64_t n, void* stream) {
  if (n <= 0) return n < 0 ? invalid("to_bf16: negative size") : 0;
  f32_to_bf16_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(in, (__nv_bfloat16*)out, n);
  return status_of(cudaGetLastError());
}

int gs2g_mlp_adam(float* w, const float* g, float* m, float* v, void* w_bf16, int64_t n, float lr, float beta1,
                  float beta2, float eps, int step, float weight_decay, void* stream) {
  if (n == 0) return 0;
  if (n < 0 || step < 1) return invalid("adam: negative size or step < 1");
  float c1 = 1.f, c2 = 1.f;
  for (int i = 0; i < step; ++i) {
    c1 *= beta1;
    c2 *= beta2;
  }
  adam_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, (__nv_bfloat16*)w_bf16, n, lr, beta1,
                                                                  beta2, eps, 1.f - c1, 1.f - c2, weight_decay);
  return status_of(cudaGetLastError());
}

int gs2g_mlp_features(const double* sbus_rows, const double* sbus_base, const int* pvpq, int n_pvpq, const int* pq,
                      int n_pq, const int* trip_ptr, const int* trip_ids, const int* br_col, const float* br_val,
                      const float* x_mean, const float* x_std, int n_in, void* x_bf16, int ldx, int rows,
                      int rows_pad, int n_bus, void* stream) {
  if (rows < 0 || rows_pad < rows || n_in < 0 || ldx < n_in || n_bus <= 0 || n_pvpq < 0 || n_pq < 0 || !x_bf16 ||
      !x_mean || !x_std || !sbus_base || (trip_ptr && (!trip_ids || !br_col || !br_val)))
    return invalid("features: bad arguments");
  if (rows_pad == 0) return 0;
  gs2g::mlp::features_kernel<<<rows_pad, 256, 0, (cudaStream_t)stream>>>(
      (const double2*)sbus_rows, (const double2*)sbus_base, pvpq, n_pvpq, pq, n_pq, trip_ptr, trip_ids, br_col,
      br_val, x_mean, x_std, n_in, (__nv_bfloat16*)x_bf16, ldx, rows, n_bus);
  return status_of(cudaGetLastError());
}

int gs2g_mlp_first_layer_base(const void* w0t_bf16, int h, const float* x_mean, const float* x_std, int n_in,
                              float* base, void* stream) {
  if (h <= 0 || n_in < 0 || !w0t_bf16 || !x_mean || !x_std || !base) return invalid("first_layer_base: bad arguments");
  gs2g::mlp::first_layer_base_kernel<<<(h + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
      (const __nv_bfloat16*)w0t_bf16, h, x_mean, x_std, n_in, base);
  return status_of(cudaGetLastError());
}

int gs2g_mlp_sparse_first_layer(const float* base, const void* w0t_bf16, int h, const int* trip_ptr,
                                const int* trip_ids, const int* br_col, const float* br_val, const float* x_mean,
                                const float* x_std, int n_in, float* pre, int ldp, int rows, int rows_pad,
                                void* stream) {
  if (h <= 0 || ldp < h || rows < 0 || rows_pad < rows || n_in < 0 || !base || !w0t_bf16 || !trip_ptr ||
      !trip_ids || !br_col || !br_val || !x_mean || !x_std || !pre)
    return invalid("sparse_first_layer: bad arguments");
  if (rows_pad == 0) return 0;
  const int smem = n_in * (int)sizeof(float);
  if (smem > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(gs2g::mlp::sparse_first_layer_kernel,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return status_of(e);
  }
  gs2g::mlp::sparse_first_layer_kernel<<<rows_pad, 256, smem, (cudaStream_t)stream>>>(
      base, (const __nv_bfloat16*)w0t_bf16, h, trip_ptr, trip_ids, br_col, br_val, x_mean, x_std, n_in, pre, ldp,
      rows);
  return status_of(cudaGetLastError());
}

int gs2g_mlp_start_voltages(const float* y, int ldy, const float* y_mean, const float* y_std, const int* va_index,
                            const int* vm_index, const double* vinit, int n_bus, double* v0, int rows, void* stream) {
  if (rows < 0 || n_bus <= 0) return invalid("start_voltages: bad sizes");
  const int64_t n = (int64_t)rows * n_bus;
  if (n == 0) return 0;
  start_voltages_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
      y, ldy, y_mean, y_std, va_index, vm_index, (const double2*)vinit, n_bus, (double2*)v0, rows);
  return status_of(cudaGetLastError());
}

}  // extern "C"
