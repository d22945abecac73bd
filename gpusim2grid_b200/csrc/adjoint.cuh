// Batched adjoint: J^T x = b for every converged row of the last sweep, J
// the row's Jacobian at its converged voltage (with its branch trips and, for
// a split row, its masked buses), in FP64.  The reference keeps the factors
// of its forward batch and solves the transposed systems with them
// (src/_cpp/contingency/batch_pf_driver.cuh:180-224, the backward pass of
// src/gpusim2grid/differentiable/_batch_pf.py); here a CTA refactors the
// row's Jacobian in its own workspace and runs the transposed solves:
//   J = L U  =>  J^T x = b  is  U^T w = b (forward), then L^T x = w (backward),
// on the same level schedule as the forward solves (the factor pattern is
// structurally symmetric), with the factor entries gathered by column (the
// plan's ut / lt lists) and the dense tail solved in 32-wide blocks.
//
// Included by nr_kernel.cu inside its anonymous namespace.

// I = Y V, the Jacobian at V scattered into HV / S, head LU, Schur update,
// dense tail LU (the factorization section of solve_row, without its
// mismatch and policies).
template <typename T>
__device__ __noinline__ void factor_at(const DevPlan& P, const SweepArgs& a, const RowEdits& ed, const double2* V,
                                       double2* I, T* HV, T* S, T* s_dense, const unsigned* mbits, bool has_mask) {
  const int tid = threadIdx.x;
  const double2* Y = reinterpret_cast<const double2*>(a.ybus);
  auto masked = [&](int b) { return has_mask && ((mbits[b >> 5] >> (b & 31)) & 1u); };
  for (int i = tid; i < P.n_bus; i += BS) {
    double2 acc = make_double2(0.0, 0.0);
    for (int k = P.y_indptr[i]; k < P.y_indptr[i + 1]; ++k) {
      const double2 yk = ed.apply(k, Y[k]);
      const double2 vj = V[P.y_indices[k]];
      acc.x = fma(yk.x, vj.x, fma(-yk.y, vj.y, acc.x));
      acc.y = fma(yk.x, vj.y, fma(yk.y, vj.x, acc.y));
    }
    I[i] = acc;
  }
  {
    const int64_t ns = (int64_t)P.nt * P.ld;
    for (int64_t q = tid; q < ns; q += BS) S[q] = T(0);
  }
  __syncthreads();
  for (int k = tid; k < P.nnz_y; k += BS) {
    const int i = P.y_row[k], j = P.y_indices[k];
    double out[4];
    jac_entry(i == j, ed.apply(k, Y[k]), V[i], V[j], I[i], out);
    if (masked(i) || masked(j)) {
      const double one = (i == j) ? 1.0 : 0.0;
      out[0] = one;
      out[1] = 0.0;
      out[2] = 0.0;
      out[3] = one;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int dst = P.jmap[4 * k + q];
      if (dst >= 0) HV[dst] = (T)out[q];
      else if (dst <= -2) S[-(dst + 2)] = (T)out[q];
    }
  }
  __syncthreads();
  for (int lv = 0; lv < P.n_levels; ++lv) {
    const int t0 = P.lev_ptr[lv], t1 = P.lev_ptr[lv + 1];
    for (int t = t0 + tid; t < t1; t += BS) {
      const int out = P.task_out[t];
      T acc = P.task_has_a[t] ? HV[out] : T(0);
      for (int q = P.task_pbeg[t]; q < P.task_pend[t]; ++q) acc -= HV[P.pair_l[q]] * HV[P.pair_u[q]];
      if (out < P.p) acc = clamp_pivot(acc, a.pivot_floor);
      HV[out] = acc;
    }
    __syncthreads();
    for (int t = t0 + tid; t < t1; t += BS) {
      const int dg = P.task_diag[t];
      if (dg >= 0) HV[P.task_out[t]] /= HV[dg];
    }
    __syncthreads();
  }
  schur_update<T>(P, HV, S);
  __syncthreads();
  if (P.nt > 0) dense_lu<T>(S, P.nt, P.ld, s_dense, a.pivot_floor);
  __syncthreads();
}

// y <- (LU)^-T y, the factor of factor_at; y in factor order.
template <typename T>
__device__ __noinline__ void solve_transposed(const DevPlan& P, const T* __restrict__ HV, const T* __restrict__ S,
                                              T* y) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // U^T forward over the head levels: y_j = (y_j - sum_k u_kj y_k) / u_jj
  for (int lv = 0; lv < P.n_levels; ++lv) {
    for (int q0 = P.lev_piv_ptr[lv] + tid; q0 < P.lev_piv_ptr[lv + 1]; q0 += BS) {
      const int j = P.lev_piv[q0];
      T acc = y[j];
      for (int q = P.ut_ptr[j]; q < P.ut_ptr[j + 1]; ++q) acc -= HV[P.ut_pos[q]] * y[P.ut_row[q]];
      y[j] = acc / HV[j];
    }
    __syncthreads();
  }
  // the tail entries against the head (u_kj, k head, j tail)
  const int nt = P.nt, ld = P.ld;
  T* yt = y + P.p;
  for (int ti = tid; ti < nt; ti += BS) {
    const int j = P.p + ti;
    T acc = y[j];
    for (int q = P.ut_ptr[j]; q < P.ut_ptr[j + 1]; ++q) acc -= HV[P.ut_pos[q]] * y[P.ut_row[q]];
    y[j] = acc;
  }
  __syncthreads();
  // dense U_tt^T forward in 32-wide blocks: warp 0 solves the diagonal block
  // (lane l holds entry k0 + l), then every thread applies the block to the
  // entries after it (row k of S is contiguous in the column index)
  for (int k0 = 0; k0 < nt; k0 += 32) {
    const int kb = min(32, nt - k0);
    if (warp == 0) {
      T v = lane < kb ? yt[k0 + lane] : T(0);
      for (int k = 0; k < kb; ++k) {
        const T wk = __shfl_sync(0xffffffffu, v, k) / S[(int64_t)(k0 + k) * ld + k0 + k];
        if (lane == k) v = wk;
        if (lane > k && lane < kb) v -= S[(int64_t)(k0 + k) * ld + k0 + lane] * wk;
      }
      if (lane < kb) yt[k0 + lane] = v;
    }
    __syncthreads();
    for (int j = k0 + kb + tid; j < nt; j += BS) {
      T acc = yt[j];
      for (int k = 0; k < kb; ++k) acc -= S[(int64_t)(k0 + k) * ld + j] * yt[k0 + k];
      yt[j] = acc;
    }
    __syncthreads();
  }
  // dense L_tt^T backward (unit diagonal), blocks from the bottom
  for (int r1 = nt; r1 > 0; r1 -= 32) {
    const int r0 = max(0, r1 - 32), rb = r1 - r0;
    if (warp == 0) {
      T v = lane < rb ? yt[r0 + lane] : T(0);
      for (int r = rb - 1; r >= 0; --r) {
        const T xr = __shfl_sync(0xffffffffu, v, r);
        if (lane < r) v -= S[(int64_t)(r0 + r) * ld + r0 + lane] * xr;
      }
      if (lane < rb) yt[r0 + lane] = v;
    }
    __syncthreads();
    for (int i = tid; i < r0; i += BS) {
      T acc = yt[i];
      for (int r = 0; r < rb; ++r) acc -= S[(int64_t)(r0 + r) * ld + i] * yt[r0 + r];
      yt[i] = acc;
    }
    __syncthreads();
  }
  // L^T backward over the head levels: y_i -= sum_r l_ri y_r (unit diagonal)
  for (int lv = P.n_levels - 1; lv >= 0; --lv) {
    for (int q0 = P.lev_piv_ptr[lv] + tid; q0 < P.lev_piv_ptr[lv + 1]; q0 += BS) {
      const int i = P.lev_piv[q0];
      T acc = y[i];
      for (int q = P.lt_ptr[i]; q < P.lt_ptr[i + 1]; ++q) acc -= HV[P.lt_pos[q]] * y[P.lt_row[q]];
      y[i] = acc;
    }
    __syncthreads();
  }
}

// One CTA per row (persistent, rows from a.queue): x = J^-T b for every row
// that converged, with b = rhs [n_rows x dim] and x = lam [n_rows x dim] in
// the reference's J layout (P/theta rows on sorted pv+pq, then Q/Vm rows on
// pq); non-finite b entries count as 0; rows that did not converge, and the
// entries of masked buses, get 0.
template <typename T>
__global__ void __launch_bounds__(BS, GS2G_MIN_CTAS_PER_SM)
    adjoint_kernel(const DevPlan P, const SweepArgs a, const double* __restrict__ rhs, double* __restrict__ lam) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_row;
  __shared__ int s_ne;
  __shared__ int s_ek[MAX_EDITS];
  __shared__ double2 s_ev[MAX_EDITS];
  const int tid = threadIdx.x;
  char* ws = a.workspace + (int64_t)blockIdx.x * a.ws_stride;
  const WsLayout L = ws_layout<T>(P);
  double2* V = reinterpret_cast<double2*>(ws + L.V);
  double2* I = reinterpret_cast<double2*>(ws + L.I);
  T* HV = reinterpret_cast<T*>(ws + L.HV);
  T* S = reinterpret_cast<T*>(ws + L.S);
  T* y = reinterpret_cast<T*>(ws + L.y);
  unsigned* mbits = reinterpret_cast<unsigned*>(ws + L.M);
  const int n = P.n_bus, dim = P.dim;
  for (;;) {
    if (tid == 0) s_row = atomicAdd(a.queue, 1);
    __syncthreads();
    const int row = s_row;
    __syncthreads();
    if (row >= a.n_rows) return;
    const double* b = rhs + (int64_t)row * dim;
    double* x = lam + (int64_t)row * dim;
    if (a.status_out[row] != ROW_CONVERGED) {
      for (int r = tid; r < dim; r += BS) x[r] = 0.0;
      continue;
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
    const bool has_mask = a.mask_ptr != nullptr && a.mask_ptr[row + 1] > a.mask_ptr[row];
    if (has_mask) {
      for (int w = tid; w < (n + 31) / 32; w += BS) mbits[w] = 0u;
      __syncthreads();
      for (int q = a.mask_ptr[row] + tid; q < a.mask_ptr[row + 1]; q += BS) {
        const int bus = a.mask_bus[q];
        atomicOr(mbits + (bus >> 5), 1u << (bus & 31));
      }
    }
    // the converged voltage (a masked bus's NaN stands for 0: it is decoupled)
    const double2* vr = reinterpret_cast<const double2*>(a.v_out) + (int64_t)row * n;
    for (int i = tid; i < n; i += BS) {
      const double2 v = vr[i];
      V[i] = (isnan(v.x) || isnan(v.y)) ? make_double2(0.0, 0.0) : v;
    }
    __syncthreads();
    const RowEdits ed{s_ne, s_ek, s_ev};
    factor_at<T>(P, a, ed, V, I, HV, S, reinterpret_cast<T*>(smem_raw), mbits, has_mask);
    for (int r = tid; r < dim; r += BS) {
      const double v = b[r];
      y[P.iperm[r]] = (T)(isfinite(v) ? v : 0.0);
    }
    __syncthreads();
    solve_transposed<T>(P, HV, S, y);
    if (has_mask) {
      // a masked bus's rows are identity rows: its entries carry no sensitivity
      for (int i = tid; i < n; i += BS) {
        if (!((mbits[i >> 5] >> (i & 31)) & 1u)) continue;
        if (P.fP[i] >= 0) y[P.fP[i]] = T(0);
        if (P.fQ[i] >= 0) y[P.fQ[i]] = T(0);
      }
      __syncthreads();
    }
    for (int r = tid; r < dim; r += BS) x[r] = (double)y[P.iperm[r]];
    __syncthreads();
  }
}
