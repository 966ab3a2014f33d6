// Device builder of the sparse wave-packet permutation matrix P123 of one 3N
// channel, in CSR.  Restates calculate_WP_overlap and
// calculate_permutation_elements_for_3N_channel
// (CPP/make_permutation_matrix.cpp:160-255, 324-943) and the cell integral and
// geometric function of CPP/auxiliary.cpp:660-746, 950-1067 as a pipeline of
// kernels:
//
//   1. k_overlap      boolean WP-cell overlap mask over (q',p',q,p)
//   2. k_cell_weights quadrature weights of each overlapping cell on the
//                     (phi, x) mesh: wx wphi cos sin (kmax^2-kmin^2)/(2 z1 z2)
//   3. k_legendre     spharm tables at cos(theta1), cos(theta2) per (phi, x)
//   4. k_gtilde       Gtilde_{alpha' alpha}(phi, x) per bra cell (q',p')
//   5. k_contract     P[cell][pair] = sum_k W[cell][k] Gtilde[pair][k]
//   6. k_row_count / k_row_fill   CSR rows (alpha', q', p'), columns ascending
//
// All geometric decisions (kmin < kmax tests) use explicitly rounded
// intrinsics on host-computed sin/cos tables, so they are bit-identical to the
// reference's host arithmetic.
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>

#include "../host/tt_p123.h"
#include "tt_device.h"
#include "tt_kernels.h"

namespace tt {
namespace {

// std::max / std::min semantics: max(a,b) = (a<b)?b:a, min(a,b) = (b<a)?b:a
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }

// pi1_tilde / pi2_tilde (auxiliary.cpp:453-462), never contracted into FMA
__device__ __forceinline__ double pi1_tilde(double p, double q, double x) {
  double t1 = __dmul_rn(__dmul_rn(0.25, p), p);
  double t2 = __dmul_rn(__dmul_rn(9.0 / 16.0, q), q);
  double t3 = __dmul_rn(__dmul_rn(__dmul_rn(0.75, p), q), x);
  return __dsqrt_rn(__dadd_rn(__dadd_rn(t1, t2), t3));
}
__device__ __forceinline__ double pi2_tilde(double p, double q, double x) {
  double t1 = __dmul_rn(p, p);
  double t2 = __dmul_rn(__dmul_rn(0.25, q), q);
  double t3 = __dmul_rn(__dmul_rn(p, q), x);
  return __dsqrt_rn(__dsub_rn(__dadd_rn(t1, t2), t3));
}

__global__ void k_overlap(const double* __restrict__ pb, const double* __restrict__ qb, int Np, int Nq,
                          const double* __restrict__ x, int Nx, const uint8_t* __restrict__ phi_ok,
                          const double* __restrict__ sinphi, const double* __restrict__ cosphi, int Nphi,
                          uint8_t* __restrict__ mask) {
  const size_t total = (size_t)Nq * Np * Nq * Np;
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= total) return;
  const int p = (int)(tid % Np);
  size_t r = tid / Np;
  const int q = (int)(r % Nq);
  r /= Nq;
  const int pp = (int)(r % Np);
  const int qp = (int)(r / Np);
  const double qp_l = qb[qp], qp_u = qb[qp + 1], pp_l = pb[pp], pp_u = pb[pp + 1];
  const double q_l = qb[q], q_u = qb[q + 1], p_l = pb[p], p_u = pb[p + 1];
  const size_t row = (size_t)qp * Np + pp;
  bool hit = false;
  if (phi_ok[row]) {
    for (int ip = 0; ip < Nphi && !hit; ip++) {
      const double s = sinphi[row * Nphi + ip], c = cosphi[row * Nphi + ip];
      const double kmin = smax(__ddiv_rn(pp_l, s), __ddiv_rn(qp_l, c));
      const double kmax = smin(__ddiv_rn(pp_u, s), __ddiv_rn(qp_u, c));
      if (!(kmin < kmax)) continue;
      for (int ix = 0; ix < Nx; ix++) {
        const double xv = x[ix];
        const double z1 = pi1_tilde(s, c, xv), z2 = pi2_tilde(s, c, xv);
        const double hl = smax(__ddiv_rn(p_l, z1), __ddiv_rn(q_l, z2));
        const double hu = smin(__ddiv_rn(p_u, z1), __ddiv_rn(q_u, z2));
        if (hl < hu) {
          const double kpmin = smax(kmin, hl), kpmax = smin(kmax, hu);
          if (kpmin < kpmax) {
            hit = true;
            break;
          }
        }
      }
    }
  }
  mask[tid] = hit ? 1 : 0;
}

// One block per overlapping cell; threads over the Nphi*Nx mesh (k = iphi*Nx + ix).
__global__ void k_cell_weights(const int32_t* __restrict__ cells, const double* __restrict__ pb,
                               const double* __restrict__ qb, int Np, const double* __restrict__ x,
                               const double* __restrict__ wx, int Nx, const double* __restrict__ sinphi,
                               const double* __restrict__ cosphi, const double* __restrict__ wphi, int Nphi,
                               double* __restrict__ W) {
  const int c = blockIdx.x;
  const int qp = cells[4 * c + 0], pp = cells[4 * c + 1], q = cells[4 * c + 2], p = cells[4 * c + 3];
  const double qp_l = qb[qp], qp_u = qb[qp + 1], pp_l = pb[pp], pp_u = pb[pp + 1];
  const double q_l = qb[q], q_u = qb[q + 1], p_l = pb[p], p_u = pb[p + 1];
  const size_t row = (size_t)qp * Np + pp;
  const int K = Nphi * Nx;
  for (int k = threadIdx.x; k < K; k += blockDim.x) {
    const int ip = k / Nx, ix = k % Nx;
    const double s = sinphi[row * Nphi + ip], co = cosphi[row * Nphi + ip];
    const double xv = x[ix];
    const double z1 = pi1_tilde(s, co, xv), z2 = pi2_tilde(s, co, xv);
    // kmin/kmax over the four bin constraints (auxiliary.cpp:713-717)
    double kmin = __ddiv_rn(pp_l, s);
    kmin = smax(kmin, __ddiv_rn(qp_l, co));
    kmin = smax(kmin, __ddiv_rn(p_l, z1));
    kmin = smax(kmin, __ddiv_rn(q_l, z2));
    double kmax = __ddiv_rn(pp_u, s);
    kmax = smin(kmax, __ddiv_rn(qp_u, co));
    kmax = smin(kmax, __ddiv_rn(p_u, z1));
    kmax = smin(kmax, __ddiv_rn(q_u, z2));
    double w = 0.0;
    if (!(kmin > kmax)) {
      const double a = __dmul_rn(__dmul_rn(__dmul_rn(wx[ix], wphi[row * Nphi + ip]), co), s);
      const double dk = __dsub_rn(__dmul_rn(kmax, kmax), __dmul_rn(kmin, kmin));
      w = __ddiv_rn(__dmul_rn(a, dk), __dmul_rn(__dmul_rn(2.0, z1), z2));
    }
    W[(size_t)c * K + k] = w;
  }
}

__device__ void spharm_row(int lmax, double x, double* out) {
  const double s = sqrt((1.0 - x) * (1.0 + x));
  double ymm = 1.0 / sqrt(4.0 * M_PI);
  for (int m = 0; m <= lmax; m++) {
    if (m > 0) ymm = -sqrt((2.0 * m + 1.0) / (2.0 * m)) * s * ymm;
    out[m * (m + 1) / 2 + m] = ymm;
    if (m + 1 > lmax) continue;
    double ylm1 = ymm;
    double yl = x * sqrt(2.0 * m + 3.0) * ymm;
    out[(m + 1) * (m + 2) / 2 + m] = yl;
    for (int l = m + 2; l <= lmax; l++) {
      const double a = sqrt((4.0 * l * l - 1.0) / ((double)l * l - (double)m * m));
      const double b = sqrt(((double)(l - 1) * (l - 1) - (double)m * m) / (4.0 * (l - 1) * (l - 1) - 1.0));
      const double yn = a * (x * yl - b * ylm1);
      ylm1 = yl;
      yl = yn;
      out[l * (l + 1) / 2 + m] = yl;
    }
  }
}

// spharm tables of cos(theta1) (lmax = max L12) and cos(theta2) (lmax = max l3)
// for a batch of bra rows; make_permutation_matrix.cpp:554-592.
__global__ void k_legendre(int row0, int nrows, const double* __restrict__ x, int Nx,
                           const double* __restrict__ sinphi, const double* __restrict__ cosphi, int Nphi,
                           int maxL, int lenL, int maxl, int lenl, double* __restrict__ plm2,
                           double* __restrict__ plm3) {
  const int K = Nphi * Nx;
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (size_t)nrows * K) return;
  const int b = (int)(tid / K), k = (int)(tid % K);
  const size_t row = (size_t)(row0 + b);
  const int ip = k / Nx, ix = k % Nx;
  const double p = sinphi[row * Nphi + ip], q = cosphi[row * Nphi + ip], xv = x[ix];
  const double pi1 = pi1_tilde(p, q, xv), pi2 = pi2_tilde(p, q, xv);
  double ct1 = -(0.5 * p + 0.75 * q * xv) / pi1;
  double ct2 = (p - 0.5 * q * xv) / pi2;
  ct1 = ct1 > 1 ? 1 : (ct1 < -1 ? -1 : ct1);
  ct2 = ct2 > 1 ? 1 : (ct2 < -1 ? -1 : ct2);
  spharm_row(maxL, ct1, plm2 + tid * lenL);
  spharm_row(maxl, ct2, plm3 + tid * lenl);
}

__global__ void k_gtilde(int nrows, int npairs, int K, int Nx, const int32_t* __restrict__ pair_off,
                         const GTerm* __restrict__ terms, const double* __restrict__ pair_norm,
                         const double* __restrict__ plm1, int lenl, const double* __restrict__ plm2, int lenL,
                         const double* __restrict__ plm3, double* __restrict__ G) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int pr = blockIdx.y;
  const int b = blockIdx.z;
  if (k >= K) return;
  const int ix = k % Nx;
  const double* P1 = plm1 + (size_t)ix * lenl;
  const double* P2 = plm2 + ((size_t)b * K + k) * lenL;
  const double* P3 = plm3 + ((size_t)b * K + k) * lenl;
  double ret = 0.0, fac2 = 0.0;
  const int t0 = pair_off[pr], t1 = pair_off[pr + 1];
  for (int t = t0; t < t1; t++) {
    const GTerm g = terms[t];
    if (g.signs & 8) {
      double v1 = P1[g.i1];
      if (g.signs & 1) v1 = -v1;
      fac2 = g.cgm * v1;
    }
    if (fac2 == 0) continue;
    double v2 = P2[g.i2], v3 = P3[g.i3];
    if (g.signs & 2) v2 = -v2;
    if (g.signs & 4) v3 = -v3;
    ret += g.fac1 * fac2 * g.cg2 * v2 * v3;
  }
  G[((size_t)b * npairs + pr) * K + k] = ret * pair_norm[pr];
}

// P[c][pair] = sum_k W[c][k] G[row(c)][pair][k] for the cells of one bra row.
// Block: 32 cells x 64 pairs, 256 threads, K staged through shared memory.
constexpr int CT_C = 32, CT_P = 64, CT_K = 32;
__global__ void __launch_bounds__(256) k_contract(int row0, const int32_t* __restrict__ row_cell_off,
                                                  int npairs, int K, const double* __restrict__ W,
                                                  const double* __restrict__ G, double* __restrict__ Pv) {
  __shared__ double sW[CT_K][CT_C + 1];
  __shared__ double sG[CT_K][CT_P + 1];
  const int b = blockIdx.y;
  const int row = row0 + b;
  const int c_lo = row_cell_off[row], c_hi = row_cell_off[row + 1];
  const int p0 = blockIdx.x * CT_P;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;  // 16 x 16 threads, each 2 cells x 4 pairs
  const double* Gb = G + (size_t)b * npairs * K;
  for (int cbase = c_lo; cbase < c_hi; cbase += CT_C) {
    double acc[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
    for (int k0 = 0; k0 < K; k0 += CT_K) {
      for (int i = threadIdx.x; i < CT_C * CT_K; i += 256) {
        const int cc = i / CT_K, kk = i % CT_K;
        const int c = cbase + cc, k = k0 + kk;
        sW[kk][cc] = (c < c_hi && k < K) ? W[(size_t)c * K + k] : 0.0;
      }
      for (int i = threadIdx.x; i < CT_P * CT_K; i += 256) {
        const int pp = i / CT_K, kk = i % CT_K;
        const int pr = p0 + pp, k = k0 + kk;
        sG[kk][pp] = (pr < npairs && k < K) ? Gb[(size_t)pr * K + k] : 0.0;
      }
      __syncthreads();
#pragma unroll 8
      for (int kk = 0; kk < CT_K; kk++) {
        const double w0 = sW[kk][ty * 2 + 0], w1 = sW[kk][ty * 2 + 1];
        double g[4];
#pragma unroll
        for (int j = 0; j < 4; j++) g[j] = sG[kk][tx * 4 + j];
#pragma unroll
        for (int j = 0; j < 4; j++) {
          acc[0][j] += w0 * g[j];
          acc[1][j] += w1 * g[j];
        }
      }
      __syncthreads();
    }
    for (int i = 0; i < 2; i++) {
      const int c = cbase + ty * 2 + i;
      if (c >= c_hi) continue;
      for (int j = 0; j < 4; j++) {
        const int pr = p0 + tx * 4 + j;
        if (pr < npairs) Pv[(size_t)c * npairs + pr] = acc[i][j];
      }
    }
  }
}

// One warp per CSR row (alpha', q', p'): entries (alpha, q, p) over the active
// pairs of alpha' (ascending alpha) x the cells of the bra row (ascending q,p).
__global__ void k_row_count(int Na, int Nq, int Np, const int32_t* __restrict__ ap_pair_lo,
                            const int32_t* __restrict__ row_cell_off, int npairs, const double* __restrict__ Pv,
                            int64_t* __restrict__ counts) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) / 32, lane = threadIdx.x % 32;
  const int nrows = Na * Nq * Np;
  if (warp >= nrows) return;
  const int ap = warp / (Nq * Np), brow = warp % (Nq * Np);
  const int pr0 = ap_pair_lo[ap], pr1 = ap_pair_lo[ap + 1];
  const int c0 = row_cell_off[brow], c1 = row_cell_off[brow + 1];
  const int nc = c1 - c0;
  int64_t cnt = 0;
  for (int i = lane; i < (pr1 - pr0) * nc; i += 32) {
    const int pr = pr0 + i / nc, c = c0 + i % nc;
    if (Pv[(size_t)c * npairs + pr] != 0.0) cnt++;
  }
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  if (lane == 0) counts[warp] = cnt;
}

__global__ void k_row_fill(int Na, int Nq, int Np, const int32_t* __restrict__ ap_pair_lo,
                           const int32_t* __restrict__ pair_a, const int32_t* __restrict__ row_cell_off,
                           const int32_t* __restrict__ cells, const double* __restrict__ cell_norm, int npairs,
                           const double* __restrict__ Pv, const int64_t* __restrict__ rowptr,
                           int32_t* __restrict__ col, double* __restrict__ val) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) / 32, lane = threadIdx.x % 32;
  const int nrows = Na * Nq * Np;
  if (warp >= nrows) return;
  const int ap = warp / (Nq * Np), brow = warp % (Nq * Np);
  const int pr0 = ap_pair_lo[ap], pr1 = ap_pair_lo[ap + 1];
  const int c0 = row_cell_off[brow], c1 = row_cell_off[brow + 1];
  const int nc = c1 - c0;
  int64_t pos = rowptr[warp];
  const int total = (pr1 - pr0) * nc;
  for (int base = 0; base < total; base += 32) {
    const int i = base + lane;
    double v = 0.0;
    int pr = 0, c = 0;
    if (i < total) {
      pr = pr0 + i / nc;
      c = c0 + i % nc;
      v = Pv[(size_t)c * npairs + pr];
    }
    const bool nz = (i < total) && (v != 0.0);
    const unsigned bal = __ballot_sync(0xffffffffu, nz);
    if (nz) {
      const int off = __popc(bal & ((1u << lane) - 1u));
      const int a = pair_a[pr];
      const int q = cells[4 * c + 2], p = cells[4 * c + 3];
      col[pos + off] = a * Nq * Np + q * Np + p;
      val[pos + off] = v / cell_norm[c];
    }
    pos += __popc(bal);
  }
}

}  // namespace

int p123_build_device(const P123Tables& t, DeviceCSR& out, cudaStream_t st, P123Stats* stats) {
  const int Np = t.Np, Nq = t.Nq, Na = t.Nalpha, Nphi = t.Nphi, Nx = t.Nx;
  const int K = Nphi * Nx;
  const size_t nrow = (size_t)Nq * Np;
  const int n = Na * Nq * Np;
  if (!t.production_run) {
    set_error("production_run=false is not supported by the device P123 builder");
    return TT_ERR_UNSUPPORTED;
  }
  DevBuf<double> d_pb, d_qb, d_x, d_wx, d_sin, d_cos, d_wphi, d_plm1, d_pnorm;
  DevBuf<uint8_t> d_phi_ok, d_mask;
  TT_TRY(d_pb.upload(t.p_WP, st));
  TT_TRY(d_qb.upload(t.q_WP, st));
  TT_TRY(d_x.upload(t.x, st));
  TT_TRY(d_wx.upload(t.wx, st));
  TT_TRY(d_sin.upload(t.sinphi, st));
  TT_TRY(d_cos.upload(t.cosphi, st));
  TT_TRY(d_wphi.upload(t.wphi, st));
  TT_TRY(d_plm1.upload(t.plm1, st));
  std::vector<uint8_t> phi_ok(nrow);
  for (int qp = 0; qp < Nq; qp++)
    for (int pp = 0; pp < Np; pp++) {
      const double lo = std::atan(t.p_WP[pp] / t.q_WP[qp + 1]);
      const double hi = std::atan(t.p_WP[pp + 1] / t.q_WP[qp]);
      phi_ok[(size_t)qp * Np + pp] = lo < hi ? 1 : 0;
    }
  TT_TRY(d_phi_ok.upload(phi_ok, st));
  const size_t ncell_all = nrow * nrow;
  TT_TRY(d_mask.alloc(ncell_all));
  k_overlap<<<ceil_div(ncell_all, 128), 128, 0, st>>>(d_pb.ptr, d_qb.ptr, Np, Nq, d_x.ptr, Nx, d_phi_ok.ptr,
                                                      d_sin.ptr, d_cos.ptr, Nphi, d_mask.ptr);
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  std::vector<uint8_t> mask(ncell_all);
  TT_CUDA_TRY(cudaMemcpyAsync(mask.data(), d_mask.ptr, ncell_all, cudaMemcpyDeviceToHost, st));
  TT_CUDA_TRY(cudaStreamSynchronize(st));
  // cell list per bra row, (q,p) ascending; WP normalisation per cell
  std::vector<int32_t> cells, row_cell_off(nrow + 1, 0);
  std::vector<double> cell_norm;
  for (size_t r = 0; r < nrow; r++) {
    const int qp = (int)(r / Np), pp = (int)(r % Np);
    for (int q = 0; q < Nq; q++)
      for (int p = 0; p < Np; p++) {
        if (!mask[r * nrow + (size_t)q * Np + p]) continue;
        cells.push_back(qp);
        cells.push_back(pp);
        cells.push_back(q);
        cells.push_back(p);
        const double nw = std::sqrt(t.q_WP[q + 1] - t.q_WP[q]) * std::sqrt(t.p_WP[p + 1] - t.p_WP[p]) *
                          std::sqrt(t.q_WP[qp + 1] - t.q_WP[qp]) * std::sqrt(t.p_WP[pp + 1] - t.p_WP[pp]);
        cell_norm.push_back(nw);
      }
    row_cell_off[r + 1] = (int32_t)(cells.size() / 4);
  }
  const int ncell = (int)(cells.size() / 4);
  const int npairs = (int)t.pair_ap.size();
  if (stats) {
    stats->n_cells = ncell;
    stats->n_pairs = npairs;
  }
  out.n = n;
  TT_TRY(out.rowptr.alloc((size_t)n + 1));
  if (ncell == 0 || npairs == 0) {
    TT_CUDA_TRY(cudaMemsetAsync(out.rowptr.ptr, 0, sizeof(int64_t) * (n + 1), st));
    out.nnz = 0;
    return TT_OK;
  }
  DevBuf<int32_t> d_cells, d_rco, d_pair_off, d_pair_a, d_ap_lo;
  DevBuf<double> d_cnorm, d_W, d_Pv;
  DevBuf<GTerm> d_terms;
  TT_TRY(d_cells.upload(cells, st));
  TT_TRY(d_rco.upload(row_cell_off, st));
  TT_TRY(d_cnorm.upload(cell_norm, st));
  TT_TRY(d_pair_off.upload(t.pair_term_off, st));
  TT_TRY(d_pair_a.upload(t.pair_a, st));
  TT_TRY(d_terms.upload(t.terms, st));
  TT_TRY(d_pnorm.upload(t.pair_norm, st));
  std::vector<int32_t> ap_lo(Na + 1, 0);
  {
    int pr = 0;
    for (int ap = 0; ap < Na; ap++) {
      ap_lo[ap] = pr;
      while (pr < npairs && t.pair_ap[pr] == ap) pr++;
    }
    ap_lo[Na] = npairs;
  }
  TT_TRY(d_ap_lo.upload(ap_lo, st));
  TT_TRY(d_W.alloc((size_t)ncell * K));
  k_cell_weights<<<ncell, 256, 0, st>>>(d_cells.ptr, d_pb.ptr, d_qb.ptr, Np, d_x.ptr, d_wx.ptr, Nx, d_sin.ptr,
                                        d_cos.ptr, d_wphi.ptr, Nphi, d_W.ptr);
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  TT_TRY(d_Pv.alloc((size_t)ncell * npairs));
  // batches of bra rows so that Gtilde stays within ~4 GB
  const size_t g_row_bytes = (size_t)npairs * K * sizeof(double);
  int batch = (int)std::max<size_t>(1, std::min<size_t>(nrow, ((size_t)4 << 30) / std::max<size_t>(1, g_row_bytes)));
  DevBuf<double> d_G, d_plm2, d_plm3;
  TT_TRY(d_G.alloc((size_t)batch * npairs * K));
  TT_TRY(d_plm2.alloc((size_t)batch * K * t.lenL));
  TT_TRY(d_plm3.alloc((size_t)batch * K * t.lenl));
  for (size_t r0 = 0; r0 < nrow; r0 += batch) {
    const int nb = (int)std::min<size_t>(batch, nrow - r0);
    if (row_cell_off[r0 + nb] == row_cell_off[r0]) continue;  // no overlapping cells in this batch
    k_legendre<<<ceil_div((size_t)nb * K, 128), 128, 0, st>>>((int)r0, nb, d_x.ptr, Nx, d_sin.ptr, d_cos.ptr, Nphi,
                                                             t.max_L12, t.lenL, t.max_l3, t.lenl, d_plm2.ptr,
                                                             d_plm3.ptr);
    count_launch();
    TT_CUDA_TRY(cudaGetLastError());
    dim3 gg(ceil_div(K, 128), npairs, nb);
    k_gtilde<<<gg, 128, 0, st>>>(nb, npairs, K, Nx, d_pair_off.ptr, d_terms.ptr, d_pnorm.ptr, d_plm1.ptr, t.lenl,
                                 d_plm2.ptr, t.lenL, d_plm3.ptr, d_G.ptr);
    count_launch();
    TT_CUDA_TRY(cudaGetLastError());
    dim3 gc(ceil_div(npairs, CT_P), nb);
    k_contract<<<gc, 256, 0, st>>>((int)r0, d_rco.ptr, npairs, K, d_W.ptr, d_G.ptr, d_Pv.ptr);
    count_launch();
    TT_CUDA_TRY(cudaGetLastError());
  }
  DevBuf<int64_t> d_counts;
  TT_TRY(d_counts.alloc((size_t)n + 1));
  TT_CUDA_TRY(cudaMemsetAsync(d_counts.ptr + n, 0, sizeof(int64_t), st));
  k_row_count<<<ceil_div((size_t)n * 32, 256), 256, 0, st>>>(Na, Nq, Np, d_ap_lo.ptr, d_rco.ptr, npairs, d_Pv.ptr,
                                                           d_counts.ptr);
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  size_t tmp_bytes = 0;
  TT_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_counts.ptr, out.rowptr.ptr, n + 1, st));
  DevBuf<uint8_t> d_tmp;
  TT_TRY(d_tmp.alloc(tmp_bytes));
  TT_CUDA_TRY(cub::DeviceScan::ExclusiveSum(d_tmp.ptr, tmp_bytes, d_counts.ptr, out.rowptr.ptr, n + 1, st));
  int64_t nnz = 0;
  TT_CUDA_TRY(cudaMemcpyAsync(&nnz, out.rowptr.ptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  TT_CUDA_TRY(cudaStreamSynchronize(st));
  out.nnz = nnz;
  TT_TRY(out.col.alloc((size_t)std::max<int64_t>(nnz, 1)));
  TT_TRY(out.val.alloc((size_t)std::max<int64_t>(nnz, 1)));
  k_row_fill<<<ceil_div((size_t)n * 32, 256), 256, 0, st>>>(Na, Nq, Np, d_ap_lo.ptr, d_pair_a.ptr, d_rco.ptr,
                                                          d_cells.ptr, d_cnorm.ptr, npairs, d_Pv.ptr,
                                                          out.rowptr.ptr, out.col.ptr, out.val.ptr);
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  TT_CUDA_TRY(cudaStreamSynchronize(st));
  return TT_OK;
}

}  // namespace tt
