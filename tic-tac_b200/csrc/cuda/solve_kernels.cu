// Kernels of the Faddeev-solve stage other than the LU factorisation and the
// A build (a_build.cu): resolvent diagonals, L = 1 - A diag(G), right-hand
// sides and the FP64 refinement residual.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <map>
#include <utility>

#include "tt_kernels.h"

namespace tt {

constexpr double kMp_d = 938.272;
constexpr double kMn_d = 939.565;

int DeviceLayout::upload(const ChannelLayout& L, const std::vector<double>& qwp, cudaStream_t st) {
  Nalpha = L.Nalpha;
  Np = L.Np;
  Nq = L.Nq;
  n = L.Nalpha * L.Np * L.Nq;
  TT_TRY(blk.upload(L.blk, st));
  TT_TRY(part.upload(L.part, st));
  TT_TRY(dim.upload(L.dim, st));
  TT_TRY(cpl_off.upload(L.cpl_off, st));
  TT_TRY(cpl.upload(L.cpl, st));
  TT_TRY(blk_off.upload(L.blk_off, st));
  TT_TRY(blk_dim.upload(L.blk_dim, st));
  TT_TRY(C.upload(L.C, st));
  TT_TRY(VC.upload(L.VC, st));
  TT_TRY(e_off.upload(L.e_off, st));
  TT_TRY(e_swp.upload(L.e_swp, st));
  TT_TRY(q_WP.upload(qwp, st));
  return TT_OK;
}

namespace {

__device__ __forceinline__ double heaviside(double v) { return v < 0 ? 0.0 : 1.0; }

// make_resolvent.cpp:14-80 (bound-continuum and continuum-continuum terms)
__global__ void k_resolvent(int Na, int Nq, int Np, const int32_t* __restrict__ e_off,
                            const double* __restrict__ e_swp, const double* __restrict__ qwp,
                            const double* __restrict__ E, int nE, double2* __restrict__ G) {
  const int n = Na * Nq * Np;
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (size_t)n * nE) return;
  const int j = (int)(tid / n), idx = (int)(tid % n);
  const int a = idx / (Nq * Np), q = (idx / Np) % Nq, p = idx % Np;
  const double e_lo = e_swp[e_off[a] + p], e_hi = e_swp[e_off[a] + p + 1];
  const double q_lo = qwp[q], q_hi = qwp[q + 1];
  const double En = E[j];
  double re, im;
  if (e_lo < 0) {
    const double Eb = e_lo;
    const double mu1 = kMn_d * (kMn_d + kMp_d + Eb) / (kMn_d + kMn_d + kMp_d + Eb);
    const double Eq_lo = q_lo * q_lo / (2 * mu1), Eq_hi = q_hi * q_hi / (2 * mu1);
    const double Dq = Eq_hi - Eq_lo;
    re = log(fabs((Eq_lo + Eb - En) / (Eq_hi + Eb - En))) / (Dq);
    im = (heaviside(Eq_hi + Eb - En) - heaviside(Eq_lo + Eb - En)) * (-M_PI) / (Dq);
  } else {
    const double Eb = 0;
    const double mu1 = kMn_d * (kMn_d + kMp_d + Eb) / (kMn_d + kMn_d + kMp_d + Eb);
    const double Eq_lo = q_lo * q_lo / (2 * mu1), Eq_hi = q_hi * q_hi / (2 * mu1);
    const double Ep = 0.5 * (e_lo + e_hi), Eq = 0.5 * (Eq_lo + Eq_hi);
    const double Dq = Eq_hi - Eq_lo, Dp = e_hi - e_lo;
    const double DM = 0.5 * (Dp - Dq), DP = 0.5 * (Dp + Dq), D = Ep + Eq - En;
    re = ((D + DM) * log(fabs(D + DM)) + (D - DM) * log(fabs(D - DM)) - (D + DP) * log(fabs(D + DP)) -
          (D - DP) * log(fabs(D - DP))) /
         (Dp * Dq);
    im = ((D + DM) * heaviside(D + DM) + (D - DM) * heaviside(D - DM) - (D + DP) * heaviside(D + DP) -
          (D - DP) * heaviside(D - DP)) *
         M_PI / (Dp * Dq);
  }
  G[tid] = make_double2(re, im);
}

// First-order change dG of the resolvents of k_resolvent for a change de of
// the SWP energy boundaries (layout of e_swp; a bound state's lower boundary
// is E_bound, which also sets the n-d reduced mass of its bins) and dEn of the
// energies E_j = E_com,j + E_bound (make_resolvent.cpp:14-80 differentiated;
// d(x ln|x|) = (ln|x| + 1) dx, d(x theta(x)) = theta(x) dx).
__global__ void k_dresolvent(int Na, int Nq, int Np, const int32_t* __restrict__ e_off,
                             const double* __restrict__ e_swp, const double* __restrict__ de_swp,
                             const double* __restrict__ qwp, const double* __restrict__ E, int nE, double dEn,
                             double2* __restrict__ dG) {
  const int n = Na * Nq * Np;
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (size_t)n * nE) return;
  const int j = (int)(tid / n), idx = (int)(tid % n);
  const int a = idx / (Nq * Np), q = (idx / Np) % Nq, p = idx % Np;
  const double e_lo = e_swp[e_off[a] + p], e_hi = e_swp[e_off[a] + p + 1];
  const double de_lo = de_swp[e_off[a] + p], de_hi = de_swp[e_off[a] + p + 1];
  const double q_lo = qwp[q], q_hi = qwp[q + 1];
  const double En = E[j], dE = dEn;
  double dre, dim;
  if (e_lo < 0) {
    const double Eb = e_lo, dEbl = de_lo;
    const double den = kMn_d + kMn_d + kMp_d + Eb;
    const double mu1 = kMn_d * (kMn_d + kMp_d + Eb) / den;
    const double dmu1 = kMn_d * kMn_d / (den * den) * dEbl;
    const double Eq_lo = q_lo * q_lo / (2 * mu1), Eq_hi = q_hi * q_hi / (2 * mu1);
    const double dEq_lo = -Eq_lo * dmu1 / mu1, dEq_hi = -Eq_hi * dmu1 / mu1;
    const double Dq = Eq_hi - Eq_lo, dDq = dEq_hi - dEq_lo;
    const double x = Eq_lo + Eb - En, y = Eq_hi + Eb - En;
    const double dx = dEq_lo + dEbl - dE, dy = dEq_hi + dEbl - dE;
    const double re = log(fabs(x / y)) / Dq;
    const double im = (heaviside(y) - heaviside(x)) * (-M_PI) / Dq;
    dre = (dx / x - dy / y) / Dq - re * dDq / Dq;
    dim = -im * dDq / Dq;
  } else {
    const double mu1 = kMn_d * (kMn_d + kMp_d) / (kMn_d + kMn_d + kMp_d);
    const double Eq_lo = q_lo * q_lo / (2 * mu1), Eq_hi = q_hi * q_hi / (2 * mu1);
    const double Ep = 0.5 * (e_lo + e_hi), Eq = 0.5 * (Eq_lo + Eq_hi);
    const double Dq = Eq_hi - Eq_lo, Dp = e_hi - e_lo;
    const double DM = 0.5 * (Dp - Dq), DP = 0.5 * (Dp + Dq), D = Ep + Eq - En;
    const double dDp = de_hi - de_lo, dD = 0.5 * (de_lo + de_hi) - dE;
    const double xs[4] = {D + DM, D - DM, D + DP, D - DP};
    const double dxs[4] = {dD + 0.5 * dDp, dD - 0.5 * dDp, dD + 0.5 * dDp, dD - 0.5 * dDp};
    const double sg[4] = {1.0, 1.0, -1.0, -1.0};
    double nre = 0, nim = 0, dnre = 0, dnim = 0;
    for (int t = 0; t < 4; t++) {
      nre += sg[t] * xs[t] * log(fabs(xs[t]));
      nim += sg[t] * xs[t] * heaviside(xs[t]);
      dnre += sg[t] * (log(fabs(xs[t])) + 1.0) * dxs[t];
      dnim += sg[t] * heaviside(xs[t]) * dxs[t];
    }
    const double re = nre / (Dp * Dq), im = nim * M_PI / (Dp * Dq);
    dre = dnre / (Dp * Dq) - re * dDp / Dp;
    dim = dnim * M_PI / (Dp * Dq) - im * dDp / Dp;
  }
  dG[tid] = make_double2(dre, dim);
}

template <typename T>
__device__ __forceinline__ T make_c(double re, double im);
template <>
__device__ __forceinline__ double2 make_c<double2>(double re, double im) { return make_double2(re, im); }
template <>
__device__ __forceinline__ float2 make_c<float2>(double re, double im) {
  return make_float2((float)re, (float)im);
}

template <typename T>
__global__ void k_form_L(const double* __restrict__ A, const double2* __restrict__ G, int n, T* __restrict__ L) {
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (size_t)n * n) return;
  const int i = (int)(tid / n), c = (int)(tid % n);
  const double a = A[tid];
  const double2 g = G[c];
  L[tid] = make_c<T>((i == c ? 1.0 : 0.0) - a * g.x, -a * g.y);
}

__global__ void k_gather_rhs(const double* __restrict__ A, int n, const int32_t* __restrict__ cols, int nrhs,
                             double2* __restrict__ b) {
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (size_t)n * nrhs) return;
  const int k = (int)(tid / n), i = (int)(tid % n);
  b[tid] = make_double2(A[(size_t)i * n + cols[k]], 0.0);
}

// r_k = b_k - x_k + A y_k, y_k = G o x_k; warp per row, up to 8 rhs per pass.
constexpr int RES_MAXR = 4;
// r_k = b_k - x_k + A y_k for up to RES_MAXR right-hand sides per pass; each
// warp takes RES_ROWS rows so that every y element fetched serves 4 rows of A,
// and each lane keeps 4 rows x 4 columns of A in flight.
constexpr int RES_ROWS = 4;
__global__ void __launch_bounds__(256) k_residual(const double* __restrict__ A, int n, const double2* __restrict__ y,
                                                  const double2* __restrict__ b, const double2* __restrict__ x,
                                                  int nrhs, double2* __restrict__ r) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t r0 = warp * RES_ROWS;
  if (r0 >= n) return;
  const int nr = (int)min((int64_t)RES_ROWS, (int64_t)n - r0);
  const double* Ar[RES_ROWS];
#pragma unroll
  for (int h = 0; h < RES_ROWS; h++) Ar[h] = A + (size_t)(r0 + min(h, nr - 1)) * n;
  for (int k0 = 0; k0 < nrhs; k0 += RES_MAXR) {
    const int kn = min(RES_MAXR, nrhs - k0);
    double sr[RES_ROWS][RES_MAXR], si[RES_ROWS][RES_MAXR];
#pragma unroll
    for (int h = 0; h < RES_ROWS; h++)
#pragma unroll
      for (int k = 0; k < RES_MAXR; k++) sr[h][k] = si[h][k] = 0.0;
    for (int c0 = 0; c0 < n; c0 += 128) {
      double a[RES_ROWS][4];
#pragma unroll
      for (int h = 0; h < RES_ROWS; h++)
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int c = c0 + lane + 32 * u;
          a[h][u] = c < n ? __ldg(Ar[h] + c) : 0.0;
        }
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int c = c0 + lane + 32 * u;
        if (c >= n) break;
#pragma unroll
        for (int k = 0; k < RES_MAXR; k++) {
          if (k >= kn) break;
          const double2 yv = __ldg(y + (size_t)(k0 + k) * n + c);
#pragma unroll
          for (int h = 0; h < RES_ROWS; h++) {
            sr[h][k] += a[h][u] * yv.x;
            si[h][k] += a[h][u] * yv.y;
          }
        }
      }
    }
#pragma unroll
    for (int h = 0; h < RES_ROWS; h++)
#pragma unroll
      for (int k = 0; k < RES_MAXR; k++) {
        for (int o = 16; o > 0; o >>= 1) {
          sr[h][k] += __shfl_xor_sync(0xffffffffu, sr[h][k], o);
          si[h][k] += __shfl_xor_sync(0xffffffffu, si[h][k], o);
        }
      }
    if (lane == 0) {
#pragma unroll
      for (int h = 0; h < RES_ROWS; h++)
#pragma unroll
        for (int k = 0; k < RES_MAXR; k++) {
          if (h < nr && k < kn) {
            const size_t o = (size_t)(k0 + k) * n + r0 + h;
            r[o] = make_double2(b[o].x - x[o].x + sr[h][k], b[o].y - x[o].y + si[h][k]);
          }
        }
    }
  }
}

// r_v = b_v - x_v + A y_v for NV <= 4 vectors in one pass over A (even n):
// a CTA owns 32 rows (4 per warp); per 256-column tile the NV slices of y are
// staged once in shared memory, and each lane keeps 4 rows x 4 double2 of A in
// flight (8 columns per row), so y is read from L2 once per 32 rows of A.
constexpr int R2_ROWS = 32, R2_TILE = 256;
template <int NV>
__global__ void __launch_bounds__(256, 1) k_residual2(const double* __restrict__ A, int n,
                                                       const double2* __restrict__ y, const double2* __restrict__ b,
                                                       const double2* __restrict__ x, double2* __restrict__ r) {
  __shared__ double2 sy[NV][R2_TILE];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t row0 = (int64_t)blockIdx.x * R2_ROWS + warp * 4;
  const double* Ar[4];
#pragma unroll
  for (int h = 0; h < 4; h++) Ar[h] = A + (size_t)min(row0 + h, (int64_t)n - 1) * n;
  double sr[4][NV], si[4][NV];
#pragma unroll
  for (int h = 0; h < 4; h++)
#pragma unroll
    for (int v = 0; v < NV; v++) sr[h][v] = si[h][v] = 0.0;
  for (int c0 = 0; c0 < n; c0 += R2_TILE) {
    __syncthreads();
#pragma unroll
    for (int v = 0; v < NV; v++) {
      const int c = c0 + threadIdx.x;
      sy[v][threadIdx.x] = c < n ? y[(size_t)v * n + c] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    double2 a[4][4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int c = c0 + 2 * lane + 64 * u;  // c and c + 1 (n even, c even)
#pragma unroll
      for (int h = 0; h < 4; h++)
        a[h][u] = c < n ? __ldcs(reinterpret_cast<const double2*>(Ar[h] + c)) : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int cl = 2 * lane + 64 * u;
#pragma unroll
      for (int v = 0; v < NV; v++) {
        const double2 y0 = sy[v][cl], y1 = sy[v][cl + 1];
#pragma unroll
        for (int h = 0; h < 4; h++) {
          sr[h][v] += a[h][u].x * y0.x + a[h][u].y * y1.x;
          si[h][v] += a[h][u].x * y0.y + a[h][u].y * y1.y;
        }
      }
    }
  }
#pragma unroll
  for (int h = 0; h < 4; h++)
#pragma unroll
    for (int v = 0; v < NV; v++)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        sr[h][v] += __shfl_xor_sync(0xffffffffu, sr[h][v], o);
        si[h][v] += __shfl_xor_sync(0xffffffffu, si[h][v], o);
      }
  if (lane == 0) {
#pragma unroll
    for (int h = 0; h < 4; h++) {
      if (row0 + h >= n) break;
#pragma unroll
      for (int v = 0; v < NV; v++) {
        const size_t o = (size_t)v * n + row0 + h;
        r[o] = make_double2(b[o].x - x[o].x + sr[h][v], b[o].y - x[o].y + si[h][v]);
      }
    }
  }
}

__global__ void k_hadamard(const double2* __restrict__ G, const int32_t* __restrict__ rhs_e, int n,
                           const double2* __restrict__ x, int nrhs, double2* __restrict__ y) {
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (size_t)n * nrhs) return;
  const int k = (int)(tid / n), c = (int)(tid % n);
  const double2 g = G[(size_t)rhs_e[k] * n + c];
  const double2 v = x[tid];
  y[tid] = make_double2(g.x * v.x - g.y * v.y, g.x * v.y + g.y * v.x);
}

__global__ void k_axpy_norm(double2* __restrict__ x, const double2* __restrict__ d, int n, int nrhs,
                            unsigned long long* __restrict__ dmax, unsigned long long* __restrict__ xmax) {
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double ad = 0.0, ax = 0.0;
  int k = 0;
  if (tid < (size_t)n * nrhs) {
    k = (int)(tid / n);
    const double2 dv = d[tid];
    double2 xv = x[tid];
    xv.x += dv.x;
    xv.y += dv.y;
    x[tid] = xv;
    ad = fmax(fabs(dv.x), fabs(dv.y));
    ax = fmax(fabs(xv.x), fabs(xv.y));
  }
  if (tid < (size_t)n * nrhs) {
    // non-negative doubles order like their bit patterns
    atomicMax(&dmax[k], (unsigned long long)__double_as_longlong(ad));
    atomicMax(&xmax[k], (unsigned long long)__double_as_longlong(ax));
  }
}

// On-shell entries after the update: out[k nrows + r] = (|d_k[rows[r]]|, |x_k[rows[r]]|)
__global__ void k_onshell_pick(const double2* __restrict__ x, const double2* __restrict__ d, int n, int nrhs,
                               const int32_t* __restrict__ rows, int nrows, double2* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nrhs * nrows) return;
  const int k = t / nrows, r = t % nrows;
  const size_t i = (size_t)k * n + rows[r];
  out[t] = make_double2(hypot(d[i].x, d[i].y), hypot(x[i].x, x[i].y));
}

}  // namespace

int resolvent_device(const DeviceLayout& L, const double* d_E, int nE, double* d_G, cudaStream_t st) {
  const size_t total = (size_t)L.n * nE;
  if (total == 0) return TT_OK;
  ProfScope prof(TT_PROF_VECTOR, st, 0.0, 16.0 * (double)total);
  k_resolvent<<<ceil_div(total, 256), 256, 0, st>>>(L.Nalpha, L.Nq, L.Np, L.e_off.ptr, L.e_swp.ptr, L.q_WP.ptr, d_E,
                                                    nE, reinterpret_cast<double2*>(d_G));
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

int dresolvent_device(const DeviceLayout& L, const double* d_de, double dE, const double* d_E, int nE, double* d_dG,
                      cudaStream_t st) {
  const size_t total = (size_t)L.n * nE;
  if (total == 0) return TT_OK;
  k_dresolvent<<<ceil_div(total, 256), 256, 0, st>>>(L.Nalpha, L.Nq, L.Np, L.e_off.ptr, L.e_swp.ptr, d_de, L.q_WP.ptr,
                                                     d_E, nE, dE, reinterpret_cast<double2*>(d_dG));
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

int resolvent_device_tables(int Na, int Nq, int Np, const int32_t* e_off, const double* e_swp, const double* q_WP,
                            const double* d_E, int nE, double* d_G, cudaStream_t st) {
  const size_t total = (size_t)Na * Nq * Np * nE;
  if (total == 0) return TT_OK;
  k_resolvent<<<ceil_div(total, 256), 256, 0, st>>>(Na, Nq, Np, e_off, e_swp, q_WP, d_E, nE,
                                                    reinterpret_cast<double2*>(d_G));
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

template <typename T>
int form_L_device(const double* d_A, const double* d_G, int n, T* d_L, cudaStream_t st) {
  const size_t total = (size_t)n * n;
  ProfScope prof(TT_PROF_FORM_L, st, 2.0 * (double)total, (8.0 + sizeof(T)) * (double)total);
  k_form_L<T><<<ceil_div(total, 256), 256, 0, st>>>(d_A, reinterpret_cast<const double2*>(d_G), n, d_L);
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}
template int form_L_device<double2>(const double*, const double*, int, double2*, cudaStream_t);
template int form_L_device<float2>(const double*, const double*, int, float2*, cudaStream_t);

int gather_rhs_device(const double* d_A, int n, const int32_t* d_cols, int nrhs, double* d_b, cudaStream_t st) {
  ProfScope prof(TT_PROF_VECTOR, st, 0.0, 24.0 * (double)n * nrhs);
  k_gather_rhs<<<ceil_div((size_t)n * nrhs, 256), 256, 0, st>>>(d_A, n, d_cols, nrhs, reinterpret_cast<double2*>(d_b));
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

int hadamard_device(const double* d_G, const int32_t* d_rhs_e, int n, const double* d_x, int nrhs, double* d_y,
                    cudaStream_t st) {
  ProfScope prof(TT_PROF_VECTOR, st, 6.0 * (double)n * nrhs, 48.0 * (double)n * nrhs);
  k_hadamard<<<ceil_div((size_t)n * nrhs, 256), 256, 0, st>>>(reinterpret_cast<const double2*>(d_G), d_rhs_e, n,
                                                             reinterpret_cast<const double2*>(d_x), nrhs,
                                                             reinterpret_cast<double2*>(d_y));
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

int residual_multi_device(const double* d_A, int n, const double* d_y, const double* d_b, const double* d_x, int nrhs,
                          double* d_r, cudaStream_t st) {
  if (n % 2 == 0) {
    // one pass over A per group of up to 4 vectors
    ProfScope prof(TT_PROF_RESIDUAL, st, 4.0 * n * (double)n * nrhs, 8.0 * n * (double)n * ((nrhs + 3) / 4));
    const unsigned grid = ceil_div((size_t)n, R2_ROWS);
    for (int v0 = 0; v0 < nrhs; v0 += 4) {
      const int nv = std::min(4, nrhs - v0);
      const size_t o = (size_t)v0 * n;
      const double2* y = reinterpret_cast<const double2*>(d_y) + o;
      const double2* b = reinterpret_cast<const double2*>(d_b) + o;
      const double2* x = reinterpret_cast<const double2*>(d_x) + o;
      double2* r = reinterpret_cast<double2*>(d_r) + o;
      switch (nv) {
        case 1: k_residual2<1><<<grid, 256, 0, st>>>(d_A, n, y, b, x, r); break;
        case 2: k_residual2<2><<<grid, 256, 0, st>>>(d_A, n, y, b, x, r); break;
        case 3: k_residual2<3><<<grid, 256, 0, st>>>(d_A, n, y, b, x, r); break;
        default: k_residual2<4><<<grid, 256, 0, st>>>(d_A, n, y, b, x, r); break;
      }
      count_launch();
      TT_CUDA_TRY(cudaGetLastError());
    }
    return TT_OK;
  }
  ProfScope prof(TT_PROF_RESIDUAL, st, 4.0 * n * (double)n * nrhs,
                 8.0 * n * (double)n * ((nrhs + RES_MAXR - 1) / RES_MAXR));
  k_residual<<<ceil_div(ceil_div((size_t)n, RES_ROWS) * 32, 256), 256, 0, st>>>(
      d_A, n, reinterpret_cast<const double2*>(d_y), reinterpret_cast<const double2*>(d_b),
      reinterpret_cast<const double2*>(d_x), nrhs, reinterpret_cast<double2*>(d_r));
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

int axpy_norms_device(double* d_x, const double* d_d, int n, int nrhs, double* h_ratio, cudaStream_t st,
                      const int32_t* d_rows, int nrows, double* h_elem) {
  if (!d_rows || !h_elem) nrows = 0;
  // [2 nrhs] maxima as ordered bit patterns, then nrhs x nrows (|d|, |x|) pairs
  const size_t words = 2 * (size_t)nrhs + 2 * (size_t)nrhs * nrows;
  DevBuf<unsigned long long> mx;
  TT_TRY(mx.alloc(words));
  TT_CUDA_TRY(cudaMemsetAsync(mx.ptr, 0, sizeof(unsigned long long) * 2 * nrhs, st));
  ProfScope prof(TT_PROF_VECTOR, st, 4.0 * (double)n * nrhs, 48.0 * (double)n * nrhs);
  k_axpy_norm<<<ceil_div((size_t)n * nrhs, 256), 256, 0, st>>>(reinterpret_cast<double2*>(d_x),
                                                              reinterpret_cast<const double2*>(d_d), n, nrhs, mx.ptr,
                                                              mx.ptr + nrhs);
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  if (nrows > 0) {
    k_onshell_pick<<<ceil_div((size_t)nrhs * nrows, 64), 64, 0, st>>>(
        reinterpret_cast<const double2*>(d_x), reinterpret_cast<const double2*>(d_d), n, nrhs, d_rows, nrows,
        reinterpret_cast<double2*>(mx.ptr + 2 * nrhs));
    count_launch();
    TT_CUDA_TRY(cudaGetLastError());
  }
  std::vector<unsigned long long> h(words);
  TT_CUDA_TRY(cudaMemcpyAsync(h.data(), mx.ptr, sizeof(unsigned long long) * words, cudaMemcpyDeviceToHost, st));
  TT_CUDA_TRY(cudaStreamSynchronize(st));
  for (int k = 0; k < nrhs; k++) {
    double dm, xm;
    memcpy(&dm, &h[k], 8);
    memcpy(&xm, &h[nrhs + k], 8);
    h_ratio[k] = xm > 0 ? dm / xm : dm;
  }
  if (nrows > 0) {
    // each on-shell entry's own |dx| / |x|; entries below kOnshellZeroFloor of
    // the largest on-shell |x| of their right-hand side are zero by symmetry
    // up to rounding and are measured against that floor instead
    const double* pr = reinterpret_cast<const double*>(h.data() + 2 * nrhs);
    for (int k = 0; k < nrhs; k++) {
      double big = 0;
      for (int r = 0; r < nrows; r++) big = std::max(big, pr[2 * ((size_t)k * nrows + r) + 1]);
      for (int r = 0; r < nrows; r++) {
        const double dv = pr[2 * ((size_t)k * nrows + r)], xv = pr[2 * ((size_t)k * nrows + r) + 1];
        const double den = std::max(xv, kOnshellZeroFloor * big);
        h_elem[(size_t)k * nrows + r] = den > 0 ? dv / den : dv;
      }
    }
  }
  return TT_OK;
}

int smem_limit_once(const void* kernel, int bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, int> limit;  // (kernel, device) -> limit set so far
  int dev = 0;
  TT_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  int& cur = limit[std::make_pair(kernel, dev)];
  if (bytes <= cur) return TT_OK;  // only ever raised: a launch needing less still fits
  TT_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  cur = bytes;
  return TT_OK;
}

int device_sm_count() {
  static int sms = -1;
  if (sms < 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

}  // namespace tt
