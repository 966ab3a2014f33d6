// Dense complex LU with partial pivoting (row-major, in place) and the
// triangular solves that use it.  This replaces the LAPACK zgetrf/zgetrs pair
// of the reference's dense Faddeev solver (General_functions/matrix_routines.cpp:73-80).
//
// Right-looking blocked algorithm, panel width NB:
//   panel  : cooperative kernel, one grid barrier pair per column (pivot search, swap)
//   laswp  : row interchanges applied to the columns left and right of the panel
//   trsm   : U12 <- L11^{-1} A12 (unit lower)
//   update : A22 <- A22 - L21 U12   (complex GEMM; SIMT here, tensor cores in gemm_tc.cu)
#include <cooperative_groups.h>

#include <cstring>
#include <vector>

#include "tt_kernels.h"
#include "tt_lu_internal.h"

namespace cg = cooperative_groups;

namespace tt {

template <typename T>
struct CT;
template <>
struct CT<double2> {
  using R = double;
};
template <>
struct CT<float2> {
  using R = float;
};

template <typename T>
__device__ __forceinline__ T cmul(T a, T b) {
  T r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename T>
__device__ __forceinline__ T cdiv(T a, T b) {
  using R = typename CT<T>::R;
  // Smith's algorithm
  T r;
  if (fabs((double)b.x) >= fabs((double)b.y)) {
    const R t = b.y / b.x, d = b.x + b.y * t;
    r.x = (a.x + a.y * t) / d;
    r.y = (a.y - a.x * t) / d;
  } else {
    const R t = b.x / b.y, d = b.y + b.x * t;
    r.x = (a.x * t + a.y) / d;
    r.y = (a.y * t - a.x) / d;
  }
  return r;
}

// ---------------------------------------------------------------------------
// Panel: rows [k, n), columns [k, k+nb).  Grid-wide cooperative kernel.
template <typename T>
__global__ void __launch_bounds__(256) k_panel(T* __restrict__ A, int n, int k, int nb, int32_t* __restrict__ ipiv,
                                               double* __restrict__ red_val, int* __restrict__ red_idx,
                                               int* __restrict__ info) {
  cg::grid_group grid = cg::this_grid();
  const int G = gridDim.x;
  const int m = n - k;
  const int chunk = (m + G - 1) / G;
  const int lo = k + blockIdx.x * chunk;
  const int hi = min(n, lo + chunk);
  __shared__ double s_val[256];
  __shared__ int s_idx[256];
  __shared__ int s_piv;
  __shared__ double s_pval;
  for (int jj = 0; jj < nb; jj++) {
    const int j = k + jj;
    // local argmax of |re|+|im| over rows >= j
    double best = -1.0;
    int bidx = -1;
    for (int i = max(lo, j) + threadIdx.x; i < hi; i += blockDim.x) {
      const T v = A[(size_t)i * n + j];
      const double a = fabs((double)v.x) + fabs((double)v.y);
      if (a > best) {
        best = a;
        bidx = i;
      }
    }
    s_val[threadIdx.x] = best;
    s_idx[threadIdx.x] = bidx;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) {
        const double o = s_val[threadIdx.x + s];
        const int oi = s_idx[threadIdx.x + s];
        if (o > s_val[threadIdx.x] || (o == s_val[threadIdx.x] && oi >= 0 && (s_idx[threadIdx.x] < 0 || oi < s_idx[threadIdx.x]))) {
          s_val[threadIdx.x] = o;
          s_idx[threadIdx.x] = oi;
        }
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      red_val[blockIdx.x] = s_val[0];
      red_idx[blockIdx.x] = s_idx[0];
    }
    grid.sync();
    if (threadIdx.x == 0) {
      double bv = -1.0;
      int bi = -1;
      for (int g = 0; g < G; g++) {
        const double v = red_val[g];
        const int vi = red_idx[g];
        if (vi < 0) continue;
        if (v > bv || (v == bv && vi < bi)) {
          bv = v;
          bi = vi;
        }
      }
      s_piv = bi;
      s_pval = bv;
    }
    __syncthreads();
    const int piv = s_piv;
    const bool zero_pivot = !(s_pval > 0.0);
    if (blockIdx.x == 0) {
      if (threadIdx.x == 0) {
        ipiv[j] = zero_pivot ? j : piv;
        if (zero_pivot && *info == 0) *info = j + 1;
      }
      if (!zero_pivot && piv != j) {
        for (int c = k + threadIdx.x; c < k + nb; c += blockDim.x) {
          const T t = A[(size_t)j * n + c];
          A[(size_t)j * n + c] = A[(size_t)piv * n + c];
          A[(size_t)piv * n + c] = t;
        }
      }
    }
    grid.sync();
    if (!zero_pivot) {
      const T d = A[(size_t)j * n + j];
      const int r0 = max(lo, j + 1);
      const int nrow = hi - r0;
      if (nrow > 0) {
        for (int i = r0 + threadIdx.x; i < hi; i += blockDim.x) A[(size_t)i * n + j] = cdiv(A[(size_t)i * n + j], d);
        __syncthreads();
        const int ncol = k + nb - (j + 1);
        if (ncol > 0) {
          for (int t = threadIdx.x; t < nrow * ncol; t += blockDim.x) {
            const int i = r0 + t / ncol, c = j + 1 + t % ncol;
            const T l = A[(size_t)i * n + j];
            const T u = A[(size_t)j * n + c];
            T a = A[(size_t)i * n + c];
            a.x -= l.x * u.x - l.y * u.y;
            a.y -= l.x * u.y + l.y * u.x;
            A[(size_t)i * n + c] = a;
          }
        }
      }
    }
    __syncthreads();
  }
}

// row interchanges of the panel applied to columns [c0, c1)
template <typename T>
__global__ void k_laswp(T* __restrict__ A, int n, int k, int nb, const int32_t* __restrict__ ipiv, int c0, int c1) {
  const int c = c0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= c1) return;
  for (int jj = 0; jj < nb; jj++) {
    const int j = k + jj, p = ipiv[j];
    if (p != j) {
      const T t = A[(size_t)j * n + c];
      A[(size_t)j * n + c] = A[(size_t)p * n + c];
      A[(size_t)p * n + c] = t;
    }
  }
}

// U12 <- L11^{-1} A12 : one block per 32 columns, L11 and the column tile in shared memory
template <typename T>
__global__ void __launch_bounds__(256) k_trsm(T* __restrict__ A, int n, int k, int nb) {
  extern __shared__ unsigned char smem_raw[];
  T* sL = reinterpret_cast<T*>(smem_raw);  // [nb][nb]
  T* sX = sL + nb * nb;                    // [nb][32]
  const int c0 = k + nb + blockIdx.x * 32;
  for (int t = threadIdx.x; t < nb * nb; t += blockDim.x) {
    const int i = t / nb, j = t % nb;
    sL[t] = A[(size_t)(k + i) * n + k + j];
  }
  for (int t = threadIdx.x; t < nb * 32; t += blockDim.x) {
    const int i = t / 32, cc = t % 32;
    const int c = c0 + cc;
    T v;
    v.x = 0;
    v.y = 0;
    if (c < n) v = A[(size_t)(k + i) * n + c];
    sX[t] = v;
  }
  __syncthreads();
  // 8 warps: warp w handles columns; lanes over rows below the pivot row
  const int cc = threadIdx.x % 32;
  const int grp = threadIdx.x / 32;  // 8 groups of 32 threads split the row updates
  for (int i = 0; i < nb; i++) {
    const T xi = sX[i * 32 + cc];
    for (int r = i + 1 + grp; r < nb; r += 8) {
      const T l = sL[r * nb + i];
      T v = sX[r * 32 + cc];
      v.x -= l.x * xi.x - l.y * xi.y;
      v.y -= l.x * xi.y + l.y * xi.x;
      sX[r * 32 + cc] = v;
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < nb * 32; t += blockDim.x) {
    const int i = t / 32, c = c0 + t % 32;
    if (c < n) A[(size_t)(k + i) * n + c] = sX[t];
  }
}

// C[m x p] -= L[m x nb] U[nb x p] on the trailing matrix; 64x64 complex tile,
// 256 threads with a 4x4 complex register tile each.
template <typename T>
__global__ void __launch_bounds__(256) k_gemm_update(T* __restrict__ A, int n, int k, int nb) {
  using R = typename CT<T>::R;
  constexpr int BM = 64, BN = 64, BK = 16;
  __shared__ T sA[BK][BM + 1];
  __shared__ T sB[BK][BN + 1];
  const int r0 = k + nb + blockIdx.y * BM;
  const int c0 = k + nb + blockIdx.x * BN;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  R accr[4][4], acci[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) accr[i][j] = acci[i][j] = 0;
  for (int kk0 = 0; kk0 < nb; kk0 += BK) {
    for (int t = threadIdx.x; t < BM * BK; t += 256) {
      const int i = t / BK, q = t % BK;
      const int r = r0 + i, kc = k + kk0 + q;
      T v;
      v.x = 0;
      v.y = 0;
      if (r < n && kk0 + q < nb) v = A[(size_t)r * n + kc];
      sA[q][i] = v;
    }
    for (int t = threadIdx.x; t < BK * BN; t += 256) {
      const int q = t / BN, j = t % BN;
      const int c = c0 + j, kr = k + kk0 + q;
      T v;
      v.x = 0;
      v.y = 0;
      if (c < n && kk0 + q < nb) v = A[(size_t)kr * n + c];
      sB[q][j] = v;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < BK; q++) {
      T a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = sA[q][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = sB[q][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
          accr[i][j] += a[i].x * b[j].x - a[i].y * b[j].y;
          acci[i][j] += a[i].x * b[j].y + a[i].y * b[j].x;
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int r = r0 + ty + 16 * i;
    if (r >= n) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int c = c0 + tx + 16 * j;
      if (c >= n) continue;
      T v = A[(size_t)r * n + c];
      v.x -= accr[i][j];
      v.y -= acci[i][j];
      A[(size_t)r * n + c] = v;
    }
  }
}

template <typename T>
int lu_factor_device(T* d_L, int n, int32_t* d_ipiv, cudaStream_t st, int use_tensor_cores, int* info) {
  const int nb = 64;
  const int sms = device_sm_count();
  DevBuf<double> red_val;
  DevBuf<int> red_idx, d_info;
  TT_TRY(red_val.alloc(sms));
  TT_TRY(red_idx.alloc(sms));
  TT_TRY(d_info.alloc(1));
  TT_CUDA_TRY(cudaMemsetAsync(d_info.ptr, 0, sizeof(int), st));
  const size_t trsm_smem = (size_t)(nb * nb + nb * 32) * sizeof(T);
  TT_CUDA_TRY(cudaFuncSetAttribute(k_trsm<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsm_smem));
  for (int k = 0; k < n; k += nb) {
    const int kb = min(nb, n - k);
    {
      int nn = n, kk = k, kbb = kb;
      T* Ap = d_L;
      int32_t* ip = d_ipiv;
      double* rv = red_val.ptr;
      int* ri = red_idx.ptr;
      int* inf = d_info.ptr;
      void* args[] = {&Ap, &nn, &kk, &kbb, &ip, &rv, &ri, &inf};
      TT_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_panel<T>, dim3(sms), dim3(256), args, 0, st));
      count_launch();
    }
    if (k > 0) {
      k_laswp<T><<<ceil_div(k, 256), 256, 0, st>>>(d_L, n, k, kb, d_ipiv, 0, k);
      count_launch();
      TT_CUDA_TRY(cudaGetLastError());
    }
    const int rest = n - k - kb;
    if (rest > 0) {
      k_laswp<T><<<ceil_div(rest, 256), 256, 0, st>>>(d_L, n, k, kb, d_ipiv, k + kb, n);
      count_launch();
      TT_CUDA_TRY(cudaGetLastError());
      k_trsm<T><<<ceil_div(rest, 32), 256, trsm_smem, st>>>(d_L, n, k, kb);
      count_launch();
      TT_CUDA_TRY(cudaGetLastError());
      if (use_tensor_cores) {
        TT_TRY(lu_update_tc(d_L, n, k, kb, st));
      } else {
        dim3 grid(ceil_div(rest, 64), ceil_div(rest, 64));
        k_gemm_update<T><<<grid, 256, 0, st>>>(d_L, n, k, kb);
        count_launch();
        TT_CUDA_TRY(cudaGetLastError());
      }
    }
  }
  if (use_tensor_cores) TT_TRY(tc_check_error(st));
  if (info) {
    TT_CUDA_TRY(cudaMemcpyAsync(info, d_info.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
    TT_CUDA_TRY(cudaStreamSynchronize(st));
  }
  return TT_OK;
}
template int lu_factor_device<double2>(double2*, int, int32_t*, cudaStream_t, int, int*);
template int lu_factor_device<float2>(float2*, int, int32_t*, cudaStream_t, int, int*);

// ---------------------------------------------------------------------------
// Triangular solves on nrhs complex128 columns x[k][n].
__global__ void k_permute(const double2* __restrict__ b, const int32_t* __restrict__ perm, int n, int nrhs,
                          double2* __restrict__ x) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)n * nrhs) return;
  const int k = (int)(t / n), i = (int)(t % n);
  x[t] = b[(size_t)k * n + perm[i]];
}

constexpr int SB = 64;  // substitution block

// diagonal block solve, one CTA; lower: unit diagonal, forward; upper: backward
template <typename T, bool LOWER>
__global__ void k_diag_solve(const T* __restrict__ A, int n, int i0, int bs, double2* __restrict__ x, int nrhs) {
  __shared__ double2 sx[SB][8];
  for (int k0 = 0; k0 < nrhs; k0 += 8) {
    const int kn = min(8, nrhs - k0);
    for (int t = threadIdx.x; t < bs * kn; t += blockDim.x) {
      const int i = t / kn, k = t % kn;
      sx[i][k] = x[(size_t)(k0 + k) * n + i0 + i];
    }
    __syncthreads();
    for (int s = 0; s < bs; s++) {
      const int i = LOWER ? s : bs - 1 - s;
      if (!LOWER) {
        if (threadIdx.x < kn) {
          const T d = A[(size_t)(i0 + i) * n + i0 + i];
          const double dr = d.x, di = d.y;
          const double2 v = sx[i][threadIdx.x];
          const double den = dr * dr + di * di;
          sx[i][threadIdx.x] = make_double2((v.x * dr + v.y * di) / den, (v.y * dr - v.x * di) / den);
        }
        __syncthreads();
      }
      const double2 xi_dummy = make_double2(0, 0);
      (void)xi_dummy;
      for (int t = threadIdx.x; t < bs * kn; t += blockDim.x) {
        const int r = t / kn, k = t % kn;
        const bool active = LOWER ? (r > i) : (r < i);
        if (!active) continue;
        const T l = A[(size_t)(i0 + r) * n + i0 + i];
        const double2 xi = sx[i][k];
        double2 v = sx[r][k];
        v.x -= (double)l.x * xi.x - (double)l.y * xi.y;
        v.y -= (double)l.x * xi.y + (double)l.y * xi.x;
        sx[r][k] = v;
      }
      __syncthreads();
    }
    for (int t = threadIdx.x; t < bs * kn; t += blockDim.x) {
      const int i = t / kn, k = t % kn;
      x[(size_t)(k0 + k) * n + i0 + i] = sx[i][k];
    }
    __syncthreads();
  }
}

// rows outside the solved block: x[r] -= A[r, i0:i0+bs] x[i0:i0+bs]; warp per row
template <typename T>
__global__ void k_block_update(const T* __restrict__ A, int n, int i0, int bs, int r_lo, int r_hi,
                               double2* __restrict__ x, int nrhs) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int r = r_lo + (int)warp;
  if (r >= r_hi) return;
  const T* Ar = A + (size_t)r * n + i0;
  for (int k = 0; k < nrhs; k++) {
    double sr = 0, si = 0;
    const double2* xb = x + (size_t)k * n + i0;
    for (int c = lane; c < bs; c += 32) {
      const T a = Ar[c];
      const double2 v = xb[c];
      sr += (double)a.x * v.x - (double)a.y * v.y;
      si += (double)a.x * v.y + (double)a.y * v.x;
    }
    for (int o = 16; o > 0; o >>= 1) {
      sr += __shfl_down_sync(0xffffffffu, sr, o);
      si += __shfl_down_sync(0xffffffffu, si, o);
    }
    if (lane == 0) {
      double2 v = x[(size_t)k * n + r];
      v.x -= sr;
      v.y -= si;
      x[(size_t)k * n + r] = v;
    }
  }
}

template <typename T>
int lu_solve_device(const T* d_LU, int n, const int32_t* d_ipiv, double* d_x, int nrhs, cudaStream_t st) {
  // compose the interchange sequence into one permutation (host, O(n))
  std::vector<int32_t> ipiv(n), perm(n);
  TT_CUDA_TRY(cudaMemcpyAsync(ipiv.data(), d_ipiv, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
  TT_CUDA_TRY(cudaStreamSynchronize(st));
  for (int i = 0; i < n; i++) perm[i] = i;
  for (int j = 0; j < n; j++) {
    const int p = ipiv[j];
    if (p < 0 || p >= n) {
      set_error("corrupt pivot sequence");
      return TT_ERR_CUDA;
    }
    std::swap(perm[j], perm[p]);
  }
  DevBuf<int32_t> d_perm;
  DevBuf<double2> d_tmp;
  TT_TRY(d_perm.upload(perm, st));
  TT_TRY(d_tmp.alloc((size_t)n * nrhs));
  TT_CUDA_TRY(cudaMemcpyAsync(d_tmp.ptr, d_x, sizeof(double2) * (size_t)n * nrhs, cudaMemcpyDeviceToDevice, st));
  double2* x = reinterpret_cast<double2*>(d_x);
  k_permute<<<ceil_div((size_t)n * nrhs, 256), 256, 0, st>>>(d_tmp.ptr, d_perm.ptr, n, nrhs, x);
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  // forward: unit lower
  for (int i0 = 0; i0 < n; i0 += SB) {
    const int bs = min(SB, n - i0);
    k_diag_solve<T, true><<<1, 256, 0, st>>>(d_LU, n, i0, bs, x, nrhs);
    count_launch();
    const int r_lo = i0 + bs;
    if (r_lo < n) k_block_update<T><<<ceil_div((size_t)(n - r_lo) * 32, 256), 256, 0, st>>>(d_LU, n, i0, bs, r_lo, n, x, nrhs);
    count_launch();
  }
  TT_CUDA_TRY(cudaGetLastError());
  // backward: upper with diagonal
  const int nblk = (n + SB - 1) / SB;
  for (int b = nblk - 1; b >= 0; b--) {
    const int i0 = b * SB, bs = min(SB, n - i0);
    k_diag_solve<T, false><<<1, 256, 0, st>>>(d_LU, n, i0, bs, x, nrhs);
    count_launch();
    if (i0 > 0) k_block_update<T><<<ceil_div((size_t)i0 * 32, 256), 256, 0, st>>>(d_LU, n, i0, bs, 0, i0, x, nrhs);
    count_launch();
  }
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}
template int lu_solve_device<double2>(const double2*, int, const int32_t*, double*, int, cudaStream_t);
template int lu_solve_device<float2>(const float2*, int, const int32_t*, double*, int, cudaStream_t);

}  // namespace tt
