// Complex128 update C[M x N] -= L[M x K] U[K x N] on the FP64 tensor cores
// (mma.sync m8n8k4 f64, the only FP64 matrix instruction of sm_100a), for the
// trailing and panel updates of the FP64 factorisation.
//
// CTA tile 64 x 128 complex, 8 warps of 32 x 32 (4 x 4 m8n8 tiles), k tiles of
// 16.  L and U are split into re/im planes in shared memory, k-major, with
// padded strides (68 and 132 doubles) so that the fragment loads of a
// half-warp hit 16 distinct even banks.  Per k4 step a warp loads 16 doubles
// of fragments and issues 64 DMMAs:
//   Re += Lr Ur + Li (-Ui),   Im += Lr Ui + Li Ur
// The next k tile is read from global memory into registers while the current
// one is multiplied, then stored into the second shared-memory buffer.
#include <algorithm>

#include "tt_kernels.h"
#include "tt_lu_internal.h"

namespace tt {
namespace dmma {

constexpr int BM = 64, BN = 128, BK = 16;
constexpr int AS = BM + 4;  // shared-memory stride of the L planes [BK][AS]
constexpr int BS = BN + 4;  // and of the U planes [BK][BS]
constexpr int SMEM_BYTES = 2 * (2 * BK * AS + 2 * BK * BS) * 8;  // two buffers

__device__ __forceinline__ void mma884(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(256) k_zgemm_dmma(double2* __restrict__ C, int ldc, const double2* __restrict__ L,
                                                    int ldl, const double2* __restrict__ U, int ldu, int M, int N,
                                                    int K) {
  // two buffers of the re/im planes: the next k tile is stored into one while
  // the other is multiplied, one barrier per k tile
  extern __shared__ double dsm[];
  constexpr int BUF = 2 * BK * AS + 2 * BK * BS;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int gid = lane >> 2, tig = lane & 3;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int wm0 = (warp >> 2) * 32, wn0 = (warp & 3) * 32;

  double accr[4][4][2], acci[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) accr[i][j][0] = accr[i][j][1] = acci[i][j][0] = acci[i][j][1] = 0.0;

  double2 ra[4], rb[8];
  auto load = [&](int k0) {
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int idx = tid + 256 * e, r = idx >> 4, c = idx & 15;
      const int gr = m0 + r, gk = k0 + c;
      ra[e] = (gr < M && gk < K) ? __ldg(&L[(size_t)gr * ldl + gk]) : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const int idx = tid + 256 * e, kr = idx >> 7, c = idx & 127;
      const int gk = k0 + kr, gc = n0 + c;
      rb[e] = (gk < K && gc < N) ? __ldg(&U[(size_t)gk * ldu + gc]) : make_double2(0.0, 0.0);
    }
  };
  auto store = [&](int buf) {
    double* sAr = dsm + buf * BUF;
    double* sAi = sAr + BK * AS;
    double* sBr = sAi + BK * AS;
    double* sBi = sBr + BK * BS;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int idx = tid + 256 * e, r = idx >> 4, c = idx & 15;
      sAr[c * AS + r] = ra[e].x;
      sAi[c * AS + r] = ra[e].y;
    }
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const int idx = tid + 256 * e, kr = idx >> 7, c = idx & 127;
      sBr[kr * BS + c] = rb[e].x;
      sBi[kr * BS + c] = rb[e].y;
    }
  };

  load(0);
  store(0);
  __syncthreads();
  int buf = 0;
  for (int k0 = 0; k0 < K; k0 += BK) {
    const bool more = k0 + BK < K;
    if (more) load(k0 + BK);
    const double* sAr = dsm + buf * BUF;
    const double* sAi = sAr + BK * AS;
    const double* sBr = sAi + BK * AS;
    const double* sBi = sBr + BK * BS;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double ar[4], ai[4], br[4], bi[4], nbi[4];
#pragma unroll
      for (int i = 0; i < 4; i++) {
        ar[i] = sAr[(kk + tig) * AS + wm0 + i * 8 + gid];
        ai[i] = sAi[(kk + tig) * AS + wm0 + i * 8 + gid];
      }
#pragma unroll
      for (int j = 0; j < 4; j++) {
        br[j] = sBr[(kk + tig) * BS + wn0 + j * 8 + gid];
        bi[j] = sBi[(kk + tig) * BS + wn0 + j * 8 + gid];
        nbi[j] = -bi[j];
      }
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
          mma884(accr[i][j], ar[i], br[j]);
          mma884(accr[i][j], ai[i], nbi[j]);
          mma884(acci[i][j], ar[i], bi[j]);
          mma884(acci[i][j], ai[i], br[j]);
        }
    }
    // the other buffer was last read before the previous barrier
    if (more) store(buf ^ 1);
    __syncthreads();
    buf ^= 1;
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int row = m0 + wm0 + i * 8 + gid;
    if (row >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int col = n0 + wn0 + j * 8 + 2 * tig + e;
        if (col < N) {
          double2* p = &C[(size_t)row * ldc + col];
          const double2 v = *p;
          *p = make_double2(v.x - accr[i][j][e], v.y - acci[i][j][e]);
        }
      }
  }
}

}  // namespace dmma

int zgemm_sub_dmma(double2* C, int ldc, const double2* L, int ldl, const double2* U, int ldu, int M, int N, int K,
                   cudaStream_t st) {
  if (M <= 0 || N <= 0 || K <= 0) return TT_OK;
  TT_TRY(smem_limit_once((const void*)dmma::k_zgemm_dmma, dmma::SMEM_BYTES));
  dim3 grid(ceil_div(N, dmma::BN), ceil_div(M, dmma::BM));
  ProfScope prof(TT_PROF_FP64_UPDATE, st, 8.0 * M * N * K, 32.0 * M * N + 16.0 * ((double)M + N) * K);
  dmma::k_zgemm_dmma<<<grid, 256, dmma::SMEM_BYTES, st>>>(C, ldc, L, ldl, U, ldu, M, N, K);
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

}  // namespace tt
