// Triangular solves with the LU factor of lu_factor.cu (the zgetrs half of the
// reference's LAPACK solve, General_functions/matrix_routines.cpp:73-80), for a
// few right-hand sides at a time: forward substitution with the unit lower
// factor and back substitution with the upper factor, in FP64 arithmetic on a
// complex128 or complex64 factor.

#include <cstring>
#include <vector>

#include "tt_kernels.h"
#include "tt_lu_internal.h"

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
// Triangular solves on nrhs complex128 columns x[k][n].
__global__ void k_permute(const double2* __restrict__ b, const int32_t* __restrict__ perm, int n, int nrhs,
                          double2* __restrict__ x) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)n * nrhs) return;
  const int k = (int)(t / n), i = (int)(t % n);
  x[t] = b[(size_t)k * n + perm[i]];
}

constexpr int SB = 64;  // substitution block

// diagonal block solve, one CTA; the bs x bs block is staged in shared memory
// first; lower: unit diagonal, forward; upper: backward with the diagonal
template <typename T, bool LOWER>
__global__ void __launch_bounds__(256) k_diag_solve(const T* __restrict__ A, int n, int i0, int bs,
                                                     double2* __restrict__ x, int nrhs) {
  extern __shared__ unsigned char dsm[];
  T* sA = reinterpret_cast<T*>(dsm);  // [bs][bs]
  __shared__ double2 sx[SB][8];
  for (int t = threadIdx.x; t < bs * bs; t += blockDim.x) sA[t] = A[(size_t)(i0 + t / bs) * n + i0 + t % bs];
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
          const T d = sA[i * bs + i];
          const double dr = d.x, di = d.y;
          const double2 v = sx[i][threadIdx.x];
          const double den = dr * dr + di * di;
          sx[i][threadIdx.x] = make_double2((v.x * dr + v.y * di) / den, (v.y * dr - v.x * di) / den);
        }
        __syncthreads();
      }
      for (int t = threadIdx.x; t < bs * kn; t += blockDim.x) {
        const int r = t / kn, k = t % kn;
        const bool active = LOWER ? (r > i) : (r < i);
        if (!active) continue;
        const T l = sA[r * bs + i];
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

int lu_permutation(const int32_t* d_ipiv, int n, std::vector<int32_t>& perm, cudaStream_t st) {
  std::vector<int32_t> ipiv(n);
  TT_CUDA_TRY(cudaMemcpyAsync(ipiv.data(), d_ipiv, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
  TT_CUDA_TRY(cudaStreamSynchronize(st));
  perm.resize(n);
  for (int i = 0; i < n; i++) perm[i] = i;
  for (int j = 0; j < n; j++) {
    const int p = ipiv[j];
    if (p < 0 || p >= n) {
      set_error("corrupt pivot sequence");
      return TT_ERR_CUDA;
    }
    std::swap(perm[j], perm[p]);
  }
  return TT_OK;
}

template <typename T>
int lu_solve_device(const T* d_LU, int n, const int32_t* d_perm, double* d_x, double* d_tmp, int nrhs,
                    cudaStream_t st) {
  ProfScope prof(TT_PROF_TRSV, st, 8.0 * n * (double)n * nrhs, (double)n * n * sizeof(T));
  TT_CUDA_TRY(cudaMemcpyAsync(d_tmp, d_x, sizeof(double2) * (size_t)n * nrhs, cudaMemcpyDeviceToDevice, st));
  double2* x = reinterpret_cast<double2*>(d_x);
  k_permute<<<ceil_div((size_t)n * nrhs, 256), 256, 0, st>>>(reinterpret_cast<const double2*>(d_tmp), d_perm, n,
                                                            nrhs, x);
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  const size_t dsm = (size_t)SB * SB * sizeof(T);
  static bool attr_set = false;
  if (!attr_set) {
    TT_CUDA_TRY(cudaFuncSetAttribute(k_diag_solve<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm));
    TT_CUDA_TRY(cudaFuncSetAttribute(k_diag_solve<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm));
    attr_set = true;
  }
  // forward: unit lower
  for (int i0 = 0; i0 < n; i0 += SB) {
    const int bs = min(SB, n - i0);
    k_diag_solve<T, true><<<1, 256, (size_t)bs * bs * sizeof(T), st>>>(d_LU, n, i0, bs, x, nrhs);
    count_launch();
    const int r_lo = i0 + bs;
    if (r_lo < n) {
      k_block_update<T><<<ceil_div((size_t)(n - r_lo) * 32, 256), 256, 0, st>>>(d_LU, n, i0, bs, r_lo, n, x, nrhs);
      count_launch();
    }
  }
  TT_CUDA_TRY(cudaGetLastError());
  // backward: upper with diagonal
  const int nblk = (n + SB - 1) / SB;
  for (int b = nblk - 1; b >= 0; b--) {
    const int i0 = b * SB, bs = min(SB, n - i0);
    k_diag_solve<T, false><<<1, 256, (size_t)bs * bs * sizeof(T), st>>>(d_LU, n, i0, bs, x, nrhs);
    count_launch();
    if (i0 > 0) {
      k_block_update<T><<<ceil_div((size_t)i0 * 32, 256), 256, 0, st>>>(d_LU, n, i0, bs, 0, i0, x, nrhs);
      count_launch();
    }
  }
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}
template int lu_solve_device<double2>(const double2*, int, const int32_t*, double*, double*, int, cudaStream_t);
template int lu_solve_device<float2>(const float2*, int, const int32_t*, double*, double*, int, cudaStream_t);

}  // namespace tt
