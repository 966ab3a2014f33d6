// The dense kernel matrix of one 3N channel,
//   A = C^T (2 P123) (V C)                      (solve_faddeev.cpp:4-181),
// in one pass over P123 that writes each element of A once.
//
// Index of a state: (alpha, q, p) -> (alpha Nq + q) Np + p.  C and V C are
// block diagonal over the 2N blocks: alpha couples only with the partners of
// its coupling list (itself and at most one other partial wave of the same 2N
// block), and
//   A[(ar,q,pr), (ac,q',pc)] = sum_{ai in cpl(ar)} sum_pi Ct(ar,ai)[pr][pi] T_ai[(q,pi), (q',pc)],
//   T_ai[(q,pi), (q',pc)]     = 2 sum_{aj in cpl(ac)} sum_pj P[(ai,q,pi), (aj,q',pj)] VC[(aj,pj), (ac,pc)].
// The reference forms the product column by column (calculate_PVC_col,
// calculate_CPVC_col); here one CTA owns a row block (ar, q) and a column
// partial wave ac, walks the P123 rows (ai, q, pi) of the coupled ai once over
// the q' range of the coupled aj (sorted columns; each row's start of every
// alpha range is tabulated once per channel), accumulates T for a chunk of q'
// in shared memory, contracts it with Ct and streams the chunk of A out.
// No n x n intermediate: HBM traffic is the A written once plus P123 read
// (twice per coupled pair).
#include <algorithm>
#include <climits>

#include "tt_kernels.h"

namespace tt {
namespace {

constexpr int AB_THREADS = 256;
constexpr int AB_COLS = 64;  // columns of A per chunk: QW = AB_COLS / Np values of q'

__device__ __forceinline__ int64_t first_col_at_least(const int32_t* __restrict__ col, int64_t lo, int64_t hi,
                                                      int32_t key) {
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (col[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// aoff[r * (Na + 1) + a] = first nonzero of row r with column >= a Nq Np,
// relative to rowptr[r], for a = 0 .. Na
__global__ void k_alpha_offsets(int n, int Na, int NqNp, const int64_t* __restrict__ rowptr,
                                const int32_t* __restrict__ col, int32_t* __restrict__ aoff) {
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (size_t)n * (Na + 1)) return;
  const int r = (int)(tid / (Na + 1)), a = (int)(tid % (Na + 1));
  const int64_t lo = rowptr[r], hi = rowptr[r + 1];
  aoff[tid] = (int32_t)(first_col_at_least(col, lo, hi, a * NqNp) - lo);
}

// Shared-memory layout of k_abuild for Np and the staging depth CAP.
struct AbLayout {
  int QW, CW, RT2;
  size_t ct, t, start, end, base, scol, sval, bytes;
  __host__ __device__ AbLayout(int Np, int cap) {
    QW = AB_COLS / Np > 0 ? AB_COLS / Np : 1;
    CW = QW * Np;
    RT2 = 2 * Np * 2;  // (T row, coupled column wave) pairs
    ct = 0;                                          // double [2][Np][Np]
    t = ct + sizeof(double) * 2 * Np * Np;           // double [2 Np][CW]
    start = t + sizeof(double) * 2 * Np * CW;        // int64 [RT2]: cursor
    end = start + sizeof(int64_t) * RT2;             // int64 [RT2]: end of the range
    base = end + sizeof(int64_t) * RT2;              // int64 [RT2]: index of the first staged nonzero
    sval = base + sizeof(int64_t) * RT2;             // double [RT2][CAP]
    scol = sval + sizeof(double) * RT2 * cap;        // int32 [RT2][CAP]
    bytes = scol + sizeof(int32_t) * RT2 * cap;
  }
};

// One CTA per (row block R = ar Nq + q, column partial wave ac).  MT = number
// of 8-row tiles of Np (4 for Np <= 32, 8 for Np <= 64; the 64 chunk columns
// are 8 tiles); CAP nonzeros of every (T row, coupled aj) range are staged in
// shared memory and refilled by the owning warp when a range runs past them.
template <int MT, int CAP>
__global__ void __launch_bounds__(AB_THREADS, 2) k_abuild(int Na, int Nq, int Np, const int64_t* __restrict__ rowptr,
                                                       const int32_t* __restrict__ col,
                                                       const double* __restrict__ val,
                                                       const int32_t* __restrict__ aoff,
                                                       const int32_t* __restrict__ blk,
                                                       const int32_t* __restrict__ part,
                                                       const int32_t* __restrict__ cpl_off,
                                                       const int32_t* __restrict__ cpl,
                                                       const int64_t* __restrict__ blk_off,
                                                       const int32_t* __restrict__ blk_dim,
                                                       const double* __restrict__ Cm,
                                                       const double* __restrict__ VC, double* __restrict__ A) {
  extern __shared__ __align__(16) unsigned char ab_raw[];
  const AbLayout ly(Np, CAP);
  double* sCt = reinterpret_cast<double*>(ab_raw + ly.ct);       // [t][pr][pi]
  double* sT = reinterpret_cast<double*>(ab_raw + ly.t);         // [t Np + pi][c]
  int64_t* sCur = reinterpret_cast<int64_t*>(ab_raw + ly.start);  // [rr 2 + t2]
  int64_t* sEnd = reinterpret_cast<int64_t*>(ab_raw + ly.end);
  int64_t* sBase = reinterpret_cast<int64_t*>(ab_raw + ly.base);
  double* sVal = reinterpret_cast<double*>(ab_raw + ly.sval);    // [rr 2 + t2][CAP]
  int32_t* sCol = reinterpret_cast<int32_t*>(ab_raw + ly.scol);
  const int n = Na * Nq * Np, NqNp = Nq * Np;
  const int QW = ly.QW, CW = ly.CW;
  const int R = blockIdx.x, ac = blockIdx.y;
  const int ar = R / Nq, q = R % Nq;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cr0 = cpl_off[ar], ncr = cpl_off[ar + 1] - cr0;
  const int cc0 = cpl_off[ac], ncc = cpl_off[ac + 1] - cc0;
  const int RT = ncr * Np;  // rows of T
  // Ct(ar, ai)[pr][pi] = C[(part_i, pi), (part_r, pr)] of ar's 2N block
  {
    const int b = blk[ar], dimb = blk_dim[b], part_r = part[ar];
    const double* Cb = Cm + blk_off[b];
    for (int i = tid; i < ncr * Np * Np; i += AB_THREADS) {
      const int t = i / (Np * Np), pr = (i / Np) % Np, pi = i % Np;
      const int ai = cpl[cr0 + t];
      sCt[i] = Cb[(size_t)(part[ai] * Np + pi) * dimb + part_r * Np + pr];
    }
  }
  // the range of every (T row, coupled aj) in its P123 row
  for (int i = tid; i < RT * 2; i += AB_THREADS) {
    const int rr = i >> 1, t2 = i & 1;
    int64_t e0 = 0, e1 = 0;
    if (t2 < ncc) {
      const int ai = cpl[cr0 + rr / Np], pi = rr % Np, aj = cpl[cc0 + t2];
      const int r = (ai * Nq + q) * Np + pi;
      const int64_t rp = rowptr[r];
      e0 = rp + aoff[(size_t)r * (Na + 1) + aj];
      e1 = rp + aoff[(size_t)r * (Na + 1) + aj + 1];
    }
    sCur[i] = e0;
    sEnd[i] = e1;
    sBase[i] = e0;
  }
  __syncthreads();
  // the first CAP nonzeros of every range
  for (int i = tid; i < RT * 2 * CAP; i += AB_THREADS) {
    const int pr2 = i / CAP, k = i % CAP;
    const int64_t e = sBase[pr2] + k;
    const bool in = e < sEnd[pr2];
    sCol[i] = in ? col[e] : INT_MAX;
    sVal[i] = in ? val[e] : 0.0;
  }
  const int bc = blk[ac], dimc = blk_dim[bc], part_c = part[ac];
  const float rNp = 1.0f / (float)Np, hNp = 0.5f / (float)Np;
  const double* VCb = VC + blk_off[bc];
  for (int q0 = 0; q0 < Nq; q0 += QW) {
    const int cw = min(QW, Nq - q0) * Np;  // columns of this chunk
    __syncthreads();
    for (int i = tid; i < RT * CW; i += AB_THREADS) sT[i] = 0.0;
    __syncthreads();
    // ---- T chunk: one warp per T row (warp-private rows: no atomics)
    for (int rr = warp; rr < RT; rr += AB_THREADS / 32) {
      double* Trow = sT + (size_t)rr * CW;
      for (int t2 = 0; t2 < ncc; t2++) {
        const int pr2 = rr * 2 + t2;
        const int aj = cpl[cc0 + t2], part_j = part[aj];
        const double* VCj = VCb + (size_t)part_j * Np * dimc + part_c * Np;  // row pj of VC(aj -> ac): + pj dimc
        const int32_t lim = aj * NqNp + min(q0 + QW, Nq) * Np;  // first column past the chunk
        const int32_t cbase = aj * NqNp + q0 * Np;
        const int64_t e_end = sEnd[pr2];
        int64_t e = sCur[pr2], eb = sBase[pr2];
        while (e < e_end) {
          if (e - eb >= CAP) {
            // past the staged nonzeros: the next CAP of this range
            __syncwarp();
            for (int k = lane; k < CAP; k += 32) {
              const int64_t ek = e + k;
              const bool in = ek < e_end;
              sCol[pr2 * CAP + k] = in ? col[ek] : INT_MAX;
              sVal[pr2 * CAP + k] = in ? val[ek] : 0.0;
            }
            eb = e;
            __syncwarp();
          }
          const int32_t cj = sCol[pr2 * CAP + (int)(e - eb)];
          if (cj >= lim) break;
          const double v = 2.0 * sVal[pr2 * CAP + (int)(e - eb)];
          // rel / Np by a float reciprocal: rel < QW Np <= 64 + Np, so the
          // product's error (< 2^-17) is far below the 0.5 / Np margin
          const int rel = cj - cbase, qq = (int)((float)rel * rNp + hNp), pj = rel - qq * Np;
          const double* vrow = VCj + (size_t)pj * dimc;
          for (int pc = lane; pc < Np; pc += 32) Trow[qq * Np + pc] += v * vrow[pc];
          e++;
        }
        if (lane == 0) {
          sCur[pr2] = e;
          sBase[pr2] = eb;
        }
      }
    }
    __syncthreads();
    // ---- A chunk on the FP64 tensor cores: (Np x RT) Ct times (RT x cw) T as
    // 8 x 8 tiles (mma m8n8k4); warp w owns row tile w % MT and MT column tiles
    {
      const int gid = lane >> 2, tig = lane & 3;
      const int mt = warp % MT, nt0 = (warp / MT) * MT;
      const int row = mt * 8 + gid;
      double acc[MT][2];
#pragma unroll
      for (int j = 0; j < MT; j++) acc[j][0] = acc[j][1] = 0.0;
      for (int k0 = 0; k0 < RT; k0 += 4) {
        const int k = k0 + tig, t = k / Np, pi = k - t * Np;
        const bool kin = k < RT;
        const double a = (kin && row < Np) ? sCt[(t * Np + row) * Np + pi] : 0.0;
#pragma unroll
        for (int j = 0; j < MT; j++) {
          const int col = (nt0 + j) * 8 + gid;
          const double b = (kin && col < CW) ? sT[(size_t)k * CW + col] : 0.0;
          asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                       : "+d"(acc[j][0]), "+d"(acc[j][1])
                       : "d"(a), "d"(b));
        }
      }
      if (row < Np) {
        double* Arow = A + ((size_t)R * Np + row) * n + (size_t)(ac * Nq + q0) * Np;
#pragma unroll
        for (int j = 0; j < MT; j++) {
          const int col = (nt0 + j) * 8 + 2 * tig;
          double* p = Arow + col;
          if (col + 1 < cw && ((uintptr_t)p & 15) == 0) {
            __stcs(reinterpret_cast<double2*>(p), make_double2(acc[j][0], acc[j][1]));
          } else {
            if (col < cw) __stcs(p, acc[j][0]);
            if (col + 1 < cw) __stcs(p + 1, acc[j][1]);
          }
        }
      }
    }
  }
}

}  // namespace

int alpha_offsets_device(const DeviceLayout& L, const DeviceCSR& P, int32_t* d_aoff, cudaStream_t st) {
  const size_t total = (size_t)L.n * (L.Nalpha + 1);
  if (total == 0) return TT_OK;
  k_alpha_offsets<<<ceil_div(total, 256), 256, 0, st>>>(L.n, L.Nalpha, L.Nq * L.Np, P.rowptr.ptr, P.col.ptr, d_aoff);
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

int build_A_device(const DeviceLayout& L, const DeviceCSR& P, const int32_t* d_aoff, double* d_A, cudaStream_t st) {
  const int n = L.n;
  if (n == 0) return TT_OK;
  if (L.Np > 64) {
    set_error("Np_WP > 64 is not supported by the A-build kernel");
    return TT_ERR_UNSUPPORTED;
  }
  // dense contraction 2 k Np n^2 and sparse product 2 k Np nnz flops (k = mean
  // coupled partners); A written once, P123 read once per coupled column wave
  const double kcpl = L.Nalpha ? (double)L.cpl.count / L.Nalpha : 0.0;
  ProfScope prof(TT_PROF_A_BUILD, st, 2.0 * kcpl * L.Np * ((double)P.nnz + (double)n * n),
                 12.0 * kcpl * (double)P.nnz + 8.0 * (double)n * n);
  dim3 grid(L.Nalpha * L.Nq, L.Nalpha);
  if (L.Np <= 32) {
    const size_t smem = AbLayout(L.Np, 32).bytes;
    TT_TRY(smem_limit_once((const void*)k_abuild<4, 32>, (int)smem));
    k_abuild<4, 32><<<grid, AB_THREADS, smem, st>>>(L.Nalpha, L.Nq, L.Np, P.rowptr.ptr, P.col.ptr, P.val.ptr,
                                                    d_aoff, L.blk.ptr, L.part.ptr, L.cpl_off.ptr, L.cpl.ptr,
                                                    L.blk_off.ptr, L.blk_dim.ptr, L.C.ptr, L.VC.ptr, d_A);
  } else {
    const size_t smem = AbLayout(L.Np, 16).bytes;
    TT_TRY(smem_limit_once((const void*)k_abuild<8, 16>, (int)smem));
    k_abuild<8, 16><<<grid, AB_THREADS, smem, st>>>(L.Nalpha, L.Nq, L.Np, P.rowptr.ptr, P.col.ptr, P.val.ptr,
                                                     d_aoff, L.blk.ptr, L.part.ptr, L.cpl_off.ptr, L.cpl.ptr,
                                                     L.blk_off.ptr, L.blk_dim.ptr, L.C.ptr, L.VC.ptr, d_A);
  }
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

}  // namespace tt
