// Device pieces of the adjoint of the on-shell solve: dU/dtheta for
// perturbations dV/dtheta of the two-body potential.
//
// With A = OP(C)^T (2 P123) OP(V C) (the block operators of the 2N structure,
// A built by k_abuild) and x_d = (1 - A G)^{-1} A e_d the on-shell columns,
//   dU[d'][d] = lambda_d'^T dA w_d,  lambda_d' = (1 - A G)^{-T} e_d',
//   w_d = e_d + G o x_d,  dA = OP(C)^T (2 P123) OP(dV C),
// so that per parameter only g_d'^T OP(dV C) w_d is needed, with
// g_d' = 2 P123^T OP(C) lambda_d' computed once.  lambda comes from one
// transposed solve with the stored LU factors (lu.cu), refined in FP64 through
// y = A^T lambda for the mixed-precision factor.

#include "tt_kernels.h"

namespace tt {
namespace {

// In-place transpose of a row-major n x n matrix: block (bx, by) with
// bx >= by swaps tiles (by, bx) and (bx, by) through shared memory (a diagonal
// tile is transposed onto itself); blocks below the diagonal exit at once.
template <typename T>
__global__ void k_transpose_inplace(T* __restrict__ a, int n) {
  if (blockIdx.x < blockIdx.y) return;
  __shared__ T t0[32][33], t1[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  const bool diag = blockIdx.x == blockIdx.y;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int c = threadIdx.x;
    if (by + i < n && bx + c < n) t0[i][c] = a[(size_t)(by + i) * n + bx + c];  // tile (by, bx)
    if (!diag && bx + i < n && by + c < n) t1[i][c] = a[(size_t)(bx + i) * n + by + c];  // tile (bx, by)
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int c = threadIdx.x;
    // (bx + i, by + c) <- old (by + c, bx + i)
    if (bx + i < n && by + c < n) a[(size_t)(bx + i) * n + by + c] = t0[c][i];
    // (by + i, bx + c) <- old (bx + c, by + i)
    if (!diag && by + i < n && bx + c < n) a[(size_t)(by + i) * n + bx + c] = t1[c][i];
  }
}

// y_k += A^T v_k for k < nrhs <= GT_MAXV: CTA = 256 columns x 256 rows of A,
// one column per thread (coalesced rows), partial sums added atomically
constexpr int GT_ROWS = 256;
constexpr int GT_MAXV = 8;
__global__ void __launch_bounds__(256) k_gemv_t(const double* __restrict__ A, int n, const double2* __restrict__ v,
                                                int nrhs, double2* __restrict__ y) {
  __shared__ double2 sv[GT_MAXV][GT_ROWS];
  const int c = blockIdx.x * 256 + threadIdx.x;
  const int r0 = blockIdx.y * GT_ROWS, rn = min(GT_ROWS, n - r0);
  for (int t = threadIdx.x; t < GT_MAXV * GT_ROWS; t += blockDim.x) {
    const int k = t / GT_ROWS, i = t % GT_ROWS;
    sv[k][i] = (k < nrhs && i < rn) ? v[(size_t)k * n + r0 + i] : make_double2(0, 0);
  }
  __syncthreads();
  if (c >= n) return;
  double ar[GT_MAXV], ai[GT_MAXV];
#pragma unroll
  for (int k = 0; k < GT_MAXV; k++) ar[k] = ai[k] = 0;
  const double* Ac = A + (size_t)r0 * n + c;
  for (int i = 0; i < rn; i++) {
    const double a = Ac[(size_t)i * n];
#pragma unroll
    for (int k = 0; k < GT_MAXV; k++) {
      if (k < nrhs) {
        ar[k] += a * sv[k][i].x;
        ai[k] += a * sv[k][i].y;
      }
    }
  }
#pragma unroll
  for (int k = 0; k < GT_MAXV; k++) {
    if (k < nrhs) {
      atomicAdd(&y[(size_t)k * n + c].x, ar[k]);
      atomicAdd(&y[(size_t)k * n + c].y, ai[k]);
    }
  }
}

// r_k = e_{rows[k]} - lam_k + G o y_k
__global__ void k_residual_t(const double2* __restrict__ lam, const double2* __restrict__ y,
                             const double2* __restrict__ G, const int32_t* __restrict__ rows, int n, int nrhs,
                             double2* __restrict__ r) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)n * nrhs) return;
  const int k = (int)(t / n), i = (int)(t % n);
  const double2 g = G[i], yy = y[t], l = lam[t];
  r[t] = make_double2((i == rows[k] ? 1.0 : 0.0) - l.x + g.x * yy.x - g.y * yy.y, -l.y + g.x * yy.y + g.y * yy.x);
}

// x_k = e_{rows[k]}
__global__ void k_unit_rhs(const int32_t* __restrict__ rows, int n, int nrhs, double2* __restrict__ x) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)n * nrhs) return;
  const int k = (int)(t / n), i = (int)(t % n);
  x[t] = make_double2(i == rows[k] ? 1.0 : 0.0, 0.0);
}

// w_k = e_{rows[k]} + G o x_k
__global__ void k_make_w(const double2* __restrict__ x, const double2* __restrict__ G,
                         const int32_t* __restrict__ rows, int n, int nrhs, double2* __restrict__ w) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)n * nrhs) return;
  const int k = (int)(t / n), i = (int)(t % n);
  const double2 g = G[i], v = x[t];
  w[t] = make_double2((i == rows[k] ? 1.0 : 0.0) + g.x * v.x - g.y * v.y, g.x * v.y + g.y * v.x);
}

// out_k = OP(X) in_k: out[(a, q, p)] = sum over partners a' of a and p' of
// X_b[(part_a Np + p) dim + part_a' Np + p'] in[(a', q, p')]
__global__ void k_block_apply(int Na, int Nq, int Np, const int32_t* __restrict__ blk, const int32_t* __restrict__ part,
                              const int32_t* __restrict__ cpl_off, const int32_t* __restrict__ cpl,
                              const int64_t* __restrict__ blk_off, const int32_t* __restrict__ blk_dim,
                              const double* __restrict__ X, const double2* __restrict__ in, int nrhs,
                              double2* __restrict__ out) {
  const int n = Na * Nq * Np;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)n * nrhs) return;
  const int k = (int)(t / n), i = (int)(t % n);
  const int a = i / (Nq * Np), q = (i / Np) % Nq, p = i % Np;
  const int b = blk[a], dim = blk_dim[b];
  const double* Xb = X + blk_off[b] + (size_t)(part[a] * Np + p) * dim;
  double re = 0, im = 0;
  for (int s = cpl_off[a]; s < cpl_off[a + 1]; s++) {
    const int ac = cpl[s];
    const double* xr = Xb + part[ac] * Np;
    const double2* v = in + (size_t)k * n + (size_t)ac * Nq * Np + (size_t)q * Np;
    for (int pc = 0; pc < Np; pc++) {
      re += xr[pc] * v[pc].x;
      im += xr[pc] * v[pc].y;
    }
  }
  out[t] = make_double2(re, im);
}

// g_k += 2 P^T u_k over the CSR rows, warp per row
// out_k = 2 P u_k (CSR rows, one warp per row)
__global__ void k_spmv(const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                       const double* __restrict__ val, int n, const double2* __restrict__ u, int nrhs,
                       double2* __restrict__ out) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int r = (int)warp;
  for (int k = 0; k < nrhs; k++) {
    double sr = 0, si = 0;
    for (int64_t e = rowptr[r] + lane; e < rowptr[r + 1]; e += 32) {
      const double2 uu = u[(size_t)k * n + col[e]];
      sr += val[e] * uu.x;
      si += val[e] * uu.y;
    }
    for (int o = 16; o > 0; o >>= 1) {
      sr += __shfl_xor_sync(0xffffffffu, sr, o);
      si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    if (lane == 0) out[(size_t)k * n + r] = make_double2(2.0 * sr, 2.0 * si);
  }
}

__global__ void k_spmv_t(const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                         const double* __restrict__ val, int n, const double2* __restrict__ u, int nrhs,
                         double2* __restrict__ g) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int r = (int)warp;
  for (int64_t e = rowptr[r] + lane; e < rowptr[r + 1]; e += 32) {
    const int c = col[e];
    const double v2 = 2.0 * val[e];
    for (int k = 0; k < nrhs; k++) {
      const double2 uu = u[(size_t)k * n + r];
      atomicAdd(&g[(size_t)k * n + c].x, v2 * uu.x);
      atomicAdd(&g[(size_t)k * n + c].y, v2 * uu.y);
    }
  }
}

// out[a * nb + b] += sum_i ga[i] hb[i] (complex, no conjugation), a < na, b < nb, na nb <= 16
__global__ void __launch_bounds__(256) k_bilinear(int n, const double2* __restrict__ g, int na,
                                                  const double2* __restrict__ h, int nb, double2* __restrict__ out) {
  double re[16], im[16];
#pragma unroll
  for (int j = 0; j < 16; j++) re[j] = im[j] = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n; i += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int j = 0; j < 16; j++) {
      const int a = j / 4, b = j % 4;
      if (a < na && b < nb) {
        const double2 x = g[(size_t)a * n + i], y = h[(size_t)b * n + i];
        re[j] += x.x * y.x - x.y * y.y;
        im[j] += x.x * y.y + x.y * y.x;
      }
    }
  }
  __shared__ double sr[8][16], si[8][16];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < 16; j++) {
    for (int o = 16; o > 0; o >>= 1) {
      re[j] += __shfl_xor_sync(0xffffffffu, re[j], o);
      im[j] += __shfl_xor_sync(0xffffffffu, im[j], o);
    }
    if (lane == 0) {
      sr[warp][j] = re[j];
      si[warp][j] = im[j];
    }
  }
  __syncthreads();
  if (threadIdx.x < 16) {
    const int j = threadIdx.x, a = j / 4, b = j % 4;
    if (a < na && b < nb) {
      double tr = 0, ti = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
        tr += sr[w][j];
        ti += si[w][j];
      }
      atomicAdd(&out[a * nb + b].x, tr);
      atomicAdd(&out[a * nb + b].y, ti);
    }
  }
}

// R[k][c] = A[rows[k] n + c] (complex, zero imaginary part)
__global__ void k_gather_rows(const double* __restrict__ A, int n, const int32_t* __restrict__ rows, int nrows,
                              double2* __restrict__ R) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)n * nrows) return;
  const int k = (int)(t / n), c = (int)(t % n);
  R[t] = make_double2(A[(size_t)rows[k] * n + c], 0.0);
}

// V[k][c] = R[k][c] G[e[k]][c]
__global__ void k_scale_rows(const double2* __restrict__ R, const double2* __restrict__ G,
                             const int32_t* __restrict__ e, int n, int nrows, double2* __restrict__ V) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)n * nrows) return;
  const int k = (int)(t / n), c = (int)(t % n);
  const double2 r = R[t], g = G[(size_t)e[k] * n + c];
  V[t] = make_double2(r.x * g.x - r.y * g.y, r.x * g.y + r.y * g.x);
}

// out[i] = R[src_row[i]][src_col[i]]
__global__ void k_pick(const double2* __restrict__ R, int n, const int32_t* __restrict__ src_row,
                       const int32_t* __restrict__ src_col, int m, double2* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) out[i] = R[(size_t)src_row[i] * n + src_col[i]];
}

}  // namespace

int gather_rows_device(const double* d_A, int n, const int32_t* d_rows, int nrows, double* d_R, cudaStream_t st) {
  k_gather_rows<<<ceil_div((size_t)n * nrows, 256), 256, 0, st>>>(d_A, n, d_rows, nrows, reinterpret_cast<double2*>(d_R));
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

int scale_rows_device(const double* d_R, const double* d_G, const int32_t* d_e, int n, int nrows, double* d_V,
                      cudaStream_t st) {
  k_scale_rows<<<ceil_div((size_t)n * nrows, 256), 256, 0, st>>>(reinterpret_cast<const double2*>(d_R),
                                                                 reinterpret_cast<const double2*>(d_G), d_e, n, nrows,
                                                                 reinterpret_cast<double2*>(d_V));
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

int pick_device(const double* d_R, int n, const int32_t* d_row, const int32_t* d_col, int m, double* d_out,
                cudaStream_t st) {
  if (m <= 0) return TT_OK;
  k_pick<<<ceil_div(m, 128), 128, 0, st>>>(reinterpret_cast<const double2*>(d_R), n, d_row, d_col, m,
                                           reinterpret_cast<double2*>(d_out));
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

template <typename T>
int transpose_inplace_device(T* a, int n, cudaStream_t st) {
  dim3 grid(ceil_div(n, 32), ceil_div(n, 32)), block(32, 8);
  k_transpose_inplace<T><<<grid, block, 0, st>>>(a, n);
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}
template int transpose_inplace_device<float2>(float2*, int, cudaStream_t);
template int transpose_inplace_device<double2>(double2*, int, cudaStream_t);

int gemv_t_device(const double* d_A, int n, const double* d_v, int nrhs, double* d_y, cudaStream_t st) {
  if (nrhs > GT_MAXV) {
    set_error("A^T products take at most 8 vectors per call");
    return TT_ERR_BADARG;
  }
  ProfScope prof(TT_PROF_RESIDUAL, st, 4.0 * n * (double)n * nrhs, 8.0 * n * (double)n);
  TT_CUDA_TRY(cudaMemsetAsync(d_y, 0, sizeof(double2) * (size_t)n * nrhs, st));
  dim3 grid(ceil_div(n, 256), ceil_div(n, GT_ROWS));
  k_gemv_t<<<grid, 256, 0, st>>>(d_A, n, reinterpret_cast<const double2*>(d_v), nrhs, reinterpret_cast<double2*>(d_y));
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

int residual_t_device(const double* d_lam, const double* d_y, const double* d_G, const int32_t* d_rows, int n,
                      int nrhs, double* d_r, cudaStream_t st) {
  k_residual_t<<<ceil_div((size_t)n * nrhs, 256), 256, 0, st>>>(
      reinterpret_cast<const double2*>(d_lam), reinterpret_cast<const double2*>(d_y),
      reinterpret_cast<const double2*>(d_G), d_rows, n, nrhs, reinterpret_cast<double2*>(d_r));
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

int unit_rhs_device(const int32_t* d_rows, int n, int nrhs, double* d_x, cudaStream_t st) {
  k_unit_rhs<<<ceil_div((size_t)n * nrhs, 256), 256, 0, st>>>(d_rows, n, nrhs, reinterpret_cast<double2*>(d_x));
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

int make_w_device(const double* d_x, const double* d_G, const int32_t* d_rows, int n, int nrhs, double* d_w,
                  cudaStream_t st) {
  k_make_w<<<ceil_div((size_t)n * nrhs, 256), 256, 0, st>>>(reinterpret_cast<const double2*>(d_x),
                                                           reinterpret_cast<const double2*>(d_G), d_rows, n, nrhs,
                                                           reinterpret_cast<double2*>(d_w));
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

int block_apply_device(const DeviceLayout& L, const double* d_X, const double* d_in, int nrhs, double* d_out,
                       cudaStream_t st) {
  const size_t total = (size_t)L.n * nrhs;
  if (total == 0) return TT_OK;
  k_block_apply<<<ceil_div(total, 256), 256, 0, st>>>(L.Nalpha, L.Nq, L.Np, L.blk.ptr, L.part.ptr, L.cpl_off.ptr,
                                                      L.cpl.ptr, L.blk_off.ptr, L.blk_dim.ptr, d_X,
                                                      reinterpret_cast<const double2*>(d_in), nrhs,
                                                      reinterpret_cast<double2*>(d_out));
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

int spmv_device(const DeviceCSR& P, const double* d_u, int nrhs, double* d_out, cudaStream_t st) {
  const int n = P.n;
  if (n == 0) return TT_OK;
  if (P.nnz == 0) {
    TT_CUDA_TRY(cudaMemsetAsync(d_out, 0, sizeof(double2) * (size_t)n * nrhs, st));
    return TT_OK;
  }
  k_spmv<<<ceil_div((size_t)n * 32, 256), 256, 0, st>>>(P.rowptr.ptr, P.col.ptr, P.val.ptr, n,
                                                      reinterpret_cast<const double2*>(d_u), nrhs,
                                                      reinterpret_cast<double2*>(d_out));
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

int spmv_t_device(const DeviceCSR& P, const double* d_u, int nrhs, double* d_g, cudaStream_t st) {
  const int n = P.n;
  TT_CUDA_TRY(cudaMemsetAsync(d_g, 0, sizeof(double2) * (size_t)n * nrhs, st));
  if (P.nnz == 0 || n == 0) return TT_OK;
  k_spmv_t<<<ceil_div((size_t)n * 32, 256), 256, 0, st>>>(P.rowptr.ptr, P.col.ptr, P.val.ptr, n,
                                                          reinterpret_cast<const double2*>(d_u), nrhs,
                                                          reinterpret_cast<double2*>(d_g));
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

int bilinear_device(int n, const double* d_g, int na, const double* d_h, int nb, double* d_out, cudaStream_t st) {
  if (na > 4 || nb > 4) {
    set_error("adjoint products take at most 4 deuteron states");
    return TT_ERR_UNSUPPORTED;
  }
  TT_CUDA_TRY(cudaMemsetAsync(d_out, 0, sizeof(double2) * na * nb, st));
  const int grid = (int)std::min<size_t>(ceil_div((size_t)n, 256), (size_t)4 * device_sm_count());
  k_bilinear<<<grid, 256, 0, st>>>(n, reinterpret_cast<const double2*>(d_g), na, reinterpret_cast<const double2*>(d_h),
                                   nb, reinterpret_cast<double2*>(d_out));
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

}  // namespace tt
