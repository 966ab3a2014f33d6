// Blocked right-looking LU with partial pivoting of the complex Faddeev kernel
// matrix 1 - A G (row-major, in place).  Replaces the LAPACK zgetrf of the
// reference's dense solver (CPP/General_functions/matrix_routines.cpp:73-80).
//
// Outer panels of NB columns (512 for the complex64 / tensor-core path, 128
// for complex128).  Each panel is factored in IB = 32 column sub-panels:
//   k_subpanel_smem  cooperative kernel with each block's rows in shared
//                memory, ONE grid barrier per column: every block posts its
//                best pivot candidate as a packed 64-bit key (atomicMax) and a
//                copy of that row (the owner of the diagonal row posts it too),
//                so after the barrier every block reads the key and the pivot
//                row and the two owners swap their rows without a second
//                barrier (k_subpanel: the same from global memory, for
//                sub-panels too tall for shared memory)
//   k_laswp2     the sub-panel's interchanges on the rest of the panel
//   k_trsm_blk   U = L^{-1} U for the 32-wide unit-lower diagonal block
//   tc_gemm_sub / k_gemm_sub  rank-32 update of the remaining panel columns
// then the panel's interchanges outside the panel, the blocked triangular
// solve for U12 and the trailing update A22 -= L21 U12 (tcgen05 BF16x3 for
// complex64, CUDA-core complex GEMM for complex128).
#include <cooperative_groups.h>

#include <algorithm>
#include <functional>

#include "tc2_pack.cuh"
#include "tt_kernels.h"
#include "tt_lu_internal.h"

namespace cg = cooperative_groups;

namespace tt {
namespace {

template <typename T>
struct Real;
template <>
struct Real<double2> {
  using R = double;
};
template <>
struct Real<float2> {
  using R = float;
};

template <typename T>
__device__ __forceinline__ T cdiv_smith(T a, T b) {
  using R = typename Real<T>::R;
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

constexpr int IB = 32;
constexpr int SP = IB + 1;                     // shared-memory row stride of a staged sub-panel
constexpr size_t kSubpanelSmem = 220 * 1024;  // bound on one block's staged sub-panel rows
constexpr int SP_THREADS = 512;               // threads of the shared-memory sub-panel kernel

template <typename T>
struct PivotScratch {
  double* val;              // [2][G]
  int* idx;                 // [2][G]
  T* row;                   // [2][G][IB]
  T* top;                   // [2][IB]
  unsigned long long* key;  // [n], zero before the factorization: column j's packed pivot
};

// Matrices of equal n factored together: the sub-panel grid is split into B
// equal groups of blocks, group b working on matrix b, all sharing each grid
// barrier (the barrier, not the work, bounds a sub-panel column).
constexpr int kMaxBatch = 4;
template <typename T>
struct SubpanelBatch {
  T* A[kMaxBatch];
  int32_t* ipiv[kMaxBatch];
  unsigned long long* key[kMaxBatch];  // [n] each, zero before the factorization
  int* info;                           // [B]
  int B;
};
// a[i] by predicated selects: a runtime index into a kernel parameter array
// would copy the whole parameter struct to local memory
template <typename P>
__device__ __forceinline__ P batch_pick(const P (&a)[kMaxBatch], int i) {
  P r = a[0];
#pragma unroll
  for (int q = 1; q < kMaxBatch; q++)
    if (i == q) r = a[q];
  return r;
}

// Sub-panel rows [c0, n), columns [c0, c0+w), w <= IB.
template <typename T>
__global__ void __launch_bounds__(256) k_subpanel(T* __restrict__ A, int n, int c0, int w, int32_t* __restrict__ ipiv,
                                                  PivotScratch<T> scr, int* __restrict__ info) {
  cg::grid_group grid = cg::this_grid();
  const int G = gridDim.x;
  const int m = n - c0;
  const int chunk = (m + G - 1) / G;
  const int lo = c0 + blockIdx.x * chunk;
  const int hi = min(n, lo + chunk);
  __shared__ double s_val[256];
  __shared__ int s_idx[256];
  __shared__ T s_prow[IB];
  __shared__ int s_grp[256];
  __shared__ int s_piv;
  __shared__ int s_zero;
  __shared__ int s_win;
  for (int jj = 0; jj < w; jj++) {
    const int j = c0 + jj;  // diagonal row/column
    const int buf = jj & 1;
    // 1. local candidate among own rows >= j
    double best = -1.0;
    int bidx = -1;
    for (int i = max(lo, j) + threadIdx.x; i < hi; i += blockDim.x) {
      const T v = A[(size_t)i * n + j];
      const double a = fabs((double)v.x) + fabs((double)v.y);
      if (a > best || (a == best && i < bidx)) {
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
        const double mv = s_val[threadIdx.x];
        const int mi = s_idx[threadIdx.x];
        if (oi >= 0 && (mi < 0 || o > mv || (o == mv && oi < mi))) {
          s_val[threadIdx.x] = o;
          s_idx[threadIdx.x] = oi;
        }
      }
      __syncthreads();
    }
    const int cand = s_idx[0];
    if (threadIdx.x == 0) {
      scr.val[buf * G + blockIdx.x] = s_val[0];
      scr.idx[buf * G + blockIdx.x] = cand;
    }
    if (cand >= 0 && threadIdx.x < w) scr.row[((size_t)buf * G + blockIdx.x) * IB + threadIdx.x] = A[(size_t)cand * n + c0 + threadIdx.x];
    if (j >= lo && j < hi && threadIdx.x < w) scr.top[buf * IB + threadIdx.x] = A[(size_t)j * n + c0 + threadIdx.x];
    grid.sync();
    // 2. global pivot: every block reduces the G candidates in parallel (same rule everywhere)
    {
      double v = -1.0;
      int vi = -1, vg = -1;
      for (int g = threadIdx.x; g < G; g += blockDim.x) {
        const int ci = scr.idx[buf * G + g];
        if (ci < 0) continue;
        const double cv = scr.val[buf * G + g];
        if (vi < 0 || cv > v || (cv == v && ci < vi)) {
          v = cv;
          vi = ci;
          vg = g;
        }
      }
      s_val[threadIdx.x] = v;
      s_idx[threadIdx.x] = vi;
      s_grp[threadIdx.x] = vg;
      __syncthreads();
      for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
          const double o = s_val[threadIdx.x + s];
          const int oi = s_idx[threadIdx.x + s];
          const double mv = s_val[threadIdx.x];
          const int mi = s_idx[threadIdx.x];
          if (oi >= 0 && (mi < 0 || o > mv || (o == mv && oi < mi))) {
            s_val[threadIdx.x] = o;
            s_idx[threadIdx.x] = oi;
            s_grp[threadIdx.x] = s_grp[threadIdx.x + s];
          }
        }
        __syncthreads();
      }
      if (threadIdx.x == 0) {
        s_piv = s_idx[0];
        s_zero = !(s_val[0] > 0.0);
        if (blockIdx.x == 0) {
          ipiv[j] = s_zero ? j : s_idx[0];
          if (s_zero && *info == 0) *info = j + 1;
        }
        s_win = s_grp[0];
      }
      __syncthreads();
    }
    const int piv = s_piv;
    if (s_zero) {
      __syncthreads();
      continue;
    }
    const int winner = s_win;
    if (threadIdx.x < w) s_prow[threadIdx.x] = scr.row[((size_t)buf * G + winner) * IB + threadIdx.x];
    __syncthreads();
    // 3. the two owners exchange rows j and piv (sub-panel columns only)
    if (piv != j) {
      if (piv >= lo && piv < hi && threadIdx.x < w)
        A[(size_t)piv * n + c0 + threadIdx.x] = scr.top[buf * IB + threadIdx.x];
      if (j >= lo && j < hi && threadIdx.x < w) A[(size_t)j * n + c0 + threadIdx.x] = s_prow[threadIdx.x];
    } else if (j >= lo && j < hi && threadIdx.x < w) {
      A[(size_t)j * n + c0 + threadIdx.x] = s_prow[threadIdx.x];
    }
    __syncthreads();
    // 4. eliminate below the diagonal in own rows
    const T d = s_prow[jj];
    const int r0 = max(lo, j + 1);
    const int ncol = w - jj - 1;
    for (int i = r0 + threadIdx.x; i < hi; i += blockDim.x) {
      T* row = A + (size_t)i * n + c0;
      const T l = cdiv_smith(row[jj], d);
      row[jj] = l;
      for (int c = 1; c <= ncol; c++) {
        const T u = s_prow[jj + c];
        T a = row[jj + c];
        a.x -= l.x * u.x - l.y * u.y;
        a.y -= l.x * u.y + l.y * u.x;
        row[jj + c] = a;
      }
    }
    __syncthreads();
  }
}

// (value, row) pivot candidates: larger |re| + |im| wins, ties go to the lower
// row, as in LAPACK's izamax; row < 0 marks "no candidate"
template <typename V>
__device__ __forceinline__ bool cand_better(V v, int i, V bv, int bi) {
  return i >= 0 && (bi < 0 || v > bv || (v == bv && i < bi));
}
// best of lanes [0, W) into lane 0 (W a power of two <= 32)
template <int W, typename V>
__device__ __forceinline__ void warp_argmax(V& v, int& i) {
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) {
    const V ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int oi = __shfl_xor_sync(0xffffffffu, i, o);
    if (cand_better(ov, oi, v, i)) {
      v = ov;
      i = oi;
    }
  }
}
// A candidate packed so that a larger key is the better candidate: the top 44
// bits of the non-negative double magnitude (exact for FP32 magnitudes;
// complex128 magnitudes that agree to 2^-32 relative count as equal), then
// the complement of the row offset (lower row wins ties).  0 = no candidate.
__device__ __forceinline__ unsigned long long pivot_key(double v, int off) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v) >> 20;
  return (b << 20) | (unsigned long long)(0xFFFFF - off);
}

// Same algorithm with each block's rows of the sub-panel resident in shared
// memory for all w columns: one coalesced load and one store per element.
// Warps own rows and lanes own columns.  One pass per column applies the
// multipliers (times the pivot's reciprocal, as LAPACK's zgetf2 scales),
// updates the remaining columns and tracks the next column's candidate.  The
// pivot is chosen through one 64-bit atomicMax per block on the column's key,
// so after the grid barrier each block reads one word, then the winner's
// published row: one grid barrier, two dependent L2 reads and two block
// barriers per column.  Row offsets below 2^20 - 1 (checked by the caller).
// With a batch, blocks [b Gb, (b+1) Gb) factor matrix b (gridDim.x = B Gb).
// With pk0 < pk1, the sub-panel's interchanges are also applied to the other
// columns [pk0, c0) and [c0 + w, pk1) of its panel after one more grid barrier.
template <typename T>
__global__ void __launch_bounds__(SP_THREADS) k_subpanel_smem(SubpanelBatch<T> bt, int n, int c0, int w, int pk0,
                                                              int pk1, PivotScratch<T> scr) {
  cg::grid_group grid = cg::this_grid();
  extern __shared__ unsigned char sp_raw[];
  T* sA = reinterpret_cast<T*>(sp_raw);  // [chunk][SP]
  using R = typename Real<T>::R;
  constexpr int NW = SP_THREADS / 32;
  const int G = gridDim.x;  // scratch row slots are indexed by the global block
  const int Gb = G / bt.B, grp = blockIdx.x / Gb, cta = blockIdx.x - grp * Gb;
  T* __restrict__ A = batch_pick(bt.A, grp);
  int32_t* __restrict__ ipiv = batch_pick(bt.ipiv, grp);
  unsigned long long* __restrict__ keys = batch_pick(bt.key, grp);
  T* __restrict__ top = scr.top + (size_t)grp * 2 * IB;  // [2][IB] per matrix
  const int m = n - c0;
  const int chunk = (m + Gb - 1) / Gb;
  const int lo = c0 + cta * chunk;
  const int hi = min(n, lo + chunk);
  const int nr = max(0, hi - lo);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __shared__ R s_wv[NW];
  __shared__ int s_wi[NW];
  __shared__ T s_prow[IB];
  __shared__ int s_zero;
  for (int r = warp; r < nr; r += NW)
    if (lane < w) sA[r * SP + lane] = A[(size_t)(lo + r) * n + c0 + lane];
  __syncthreads();
  // this block's candidate for column jc: warp 0 reduces the warps' and posts
  // it, with a copy of the candidate row (and of the diagonal row, if held here)
  auto publish = [&](int jc, R best, int bidx) {
    if (lane == jc) {
      s_wv[warp] = best;
      s_wi[warp] = bidx;
    }
    __syncthreads();
    if (warp == 0) {
      R v = lane < NW ? s_wv[lane] : R(-1);
      int i = lane < NW ? s_wi[lane] : -1;
      warp_argmax<NW>(v, i);
      i = __shfl_sync(0xffffffffu, i, 0);  // lanes >= NW reduced only among themselves
      const int buf = jc & 1, j = c0 + jc;
      if (lane == 0 && i >= 0) atomicMax(&keys[j], pivot_key((double)v, i - c0));
      if (i >= 0 && lane < w) scr.row[((size_t)buf * G + blockIdx.x) * IB + lane] = sA[(i - lo) * SP + lane];
      if (j >= lo && j < hi && lane < w) top[buf * IB + lane] = sA[(j - lo) * SP + lane];
    }
  };
  // candidate of column jc over its rows without an update (first column, or
  // after a zero pivot)
  auto scan = [&](int jc) {
    R best = -1;
    int bidx = -1;
    for (int r = max(0, c0 + jc - lo) + warp; r < nr; r += NW) {
      if (lane == jc) {
        const T v = sA[r * SP + jc];
        const R a = fabs(v.x) + fabs(v.y);
        if (a > best) {
          best = a;
          bidx = lo + r;
        }
      }
    }
    publish(jc, best, bidx);
  };
  scan(0);
  for (int jj = 0; jj < w; jj++) {
    const int j = c0 + jj;
    const int buf = jj & 1;
    grid.sync();
    // warp 0: the column's pivot, then the winner's row and the diagonal row
    if (warp == 0) {
      unsigned long long k = 0;
      if (lane == 0) k = __ldcg(&keys[j]);
      k = __shfl_sync(0xffffffffu, k, 0);
      const bool zero = (k >> 20) == 0;
      const int piv = zero ? j : c0 + (0xFFFFF - (int)(k & 0xFFFFF));
      if (lane == 0) {
        s_zero = zero;
        if (cta == 0) {
          ipiv[j] = piv;
          if (zero && bt.info[grp] == 0) bt.info[grp] = j + 1;
        }
      }
      if (!zero && lane < w) {
        const int owner = grp * Gb + (piv - c0) / chunk;
        const T pr = scr.row[((size_t)buf * G + owner) * IB + lane];
        const T tp = top[buf * IB + lane];
        s_prow[lane] = pr;
        if (piv != j && piv >= lo && piv < hi) sA[(piv - lo) * SP + lane] = tp;
        if (j >= lo && j < hi) sA[(j - lo) * SP + lane] = pr;
      }
    }
    __syncthreads();
    if (s_zero) {
      // singular column: nothing to eliminate; the next column's candidate
      if (jj + 1 < w) scan(jj + 1);
      continue;
    }
    const T d = s_prow[jj];
    T rd;
    rd.x = 1;
    rd.y = 0;
    rd = cdiv_smith(rd, d);
    const T u = lane < w ? s_prow[lane] : T{0, 0};
    const int jn = jj + 1;
    R best = -1;
    int bidx = -1;
    // four rows per warp per iteration, independent, for latency hiding
    constexpr int RU = 4;
    for (int rb = max(0, j + 1 - lo) + warp; rb < nr; rb += NW * RU) {
      T a[RU];
#pragma unroll
      for (int k = 0; k < RU; k++) {
        const int r = rb + k * NW;
        a[k] = (r < nr && lane >= jj && lane < w) ? sA[r * SP + lane] : T{0, 0};  // columns < jj are final
      }
#pragma unroll
      for (int k = 0; k < RU; k++) {
        T p, l;
        p.x = __shfl_sync(0xffffffffu, a[k].x, jj);
        p.y = __shfl_sync(0xffffffffu, a[k].y, jj);
        l.x = p.x * rd.x - p.y * rd.y;
        l.y = p.x * rd.y + p.y * rd.x;
        if (lane == jj) {
          a[k] = l;
        } else {
          a[k].x -= l.x * u.x - l.y * u.y;
          a[k].y -= l.x * u.y + l.y * u.x;
        }
      }
#pragma unroll
      for (int k = 0; k < RU; k++) {
        const int r = rb + k * NW;
        if (r < nr) {
          if (lane >= jj && lane < w) sA[r * SP + lane] = a[k];
          if (lane == jn) {
            const R av = fabs(a[k].x) + fabs(a[k].y);
            if (av > best) {
              best = av;
              bidx = lo + r;
            }
          }
        }
      }
    }
    if (jn < w) publish(jn, best, bidx);
  }
  __syncthreads();
  for (int r = warp; r < nr; r += NW)
    if (lane < w) A[(size_t)(lo + r) * n + c0 + lane] = sA[r * SP + lane];
  if (pk1 - pk0 > w) {
    // every column's pivot is in ipiv once all blocks passed this barrier
    grid.sync();
    const int nl = c0 - pk0, nc = nl + (pk1 - (c0 + w));
    for (int t = cta * SP_THREADS + threadIdx.x; t < nc; t += Gb * SP_THREADS) {
      const int c = t < nl ? pk0 + t : c0 + w + (t - nl);
      for (int jj = 0; jj < w; jj++) {
        const int j = c0 + jj, p = __ldcg(&ipiv[j]);
        if (p != j) {
          const T a = A[(size_t)j * n + c];
          A[(size_t)j * n + c] = A[(size_t)p * n + c];
          A[(size_t)p * n + c] = a;
        }
      }
    }
  }
}

// X = L^{-1} for the w x w unit-lower block L at (r0, r0) of A (ld n),
// w <= INV_MAX, into X[w][w] (row-major, ld w), by recursive doubling:
// k_inv_diag32 inverts the 32 x 32 diagonal blocks (one CTA each), then per
// level s = 64, 128, .. every pair of inverted s/2 blocks is joined,
//   [X11 0; X21 X22] with X21 = -X22 (L21 X11),
// first T = L21 X11, then X21 = -X22 T, one CTA per 32 x 32 tile
// (k_inv_join_t, k_inv_join_x), all pairs of a level in the same two
// launches.  Entries above the diagonal are written as zero.
constexpr int INV_MAX = 512;
template <typename T>
__device__ __forceinline__ void cfma_sub(T& acc, T a, T b) {
  acc.x -= a.x * b.x - a.y * b.y;
  acc.y -= a.x * b.y + a.y * b.x;
}
template <typename T>
__device__ __forceinline__ void cfma_add(T& acc, T a, T b) {
  acc.x += a.x * b.x - a.y * b.y;
  acc.y += a.x * b.y + a.y * b.x;
}

// Matrices whose unit-lower blocks are inverted in the same launches: block
// (blockIdx.y for the diagonal blocks, blockIdx.z / pairs for the joins)
// picks matrix b, whose inverse is X + b w w and join scratch T + b w w / 2.
template <typename T>
struct InvBatch {
  const T* A[4];
};

template <typename T>
__global__ void __launch_bounds__(256) k_inv_diag32(InvBatch<T> ib, int n, int r0, int w, T* __restrict__ X) {
  __shared__ T sL[32][33];
  __shared__ T sX[32][33];
  const T* __restrict__ A = ib.A[blockIdx.y];
  X += (size_t)blockIdx.y * w * w;
  const int i0 = blockIdx.x * 32, hi = min(32, w - i0);
  for (int t = threadIdx.x; t < 32 * 32; t += 256) {
    const int i = t >> 5, j = t & 31;
    T l;
    l.x = 0;
    l.y = 0;
    if (i < hi && j < hi) l = A[(size_t)(r0 + i0 + i) * n + r0 + i0 + j];
    sL[i][j] = l;
  }
  __syncthreads();
  // one warp, lane = column c of the inverse: row i = e_i - sum_{j<i} L[i][j] X[j]
  if (threadIdx.x < 32) {
    const int c = threadIdx.x;
    for (int i = 0; i < hi; i++) {
      T v;
      v.x = (i == c) ? 1 : 0;
      v.y = 0;
      for (int j = c; j < i; j++) cfma_sub(v, sL[i][j], sX[j][c]);
      sX[i][c] = v;
    }
  }
  __syncthreads();
  // the whole 32-row band of X: the diagonal block, zeros elsewhere in the band
  for (int t = threadIdx.x; t < hi * w; t += 256) {
    const int i = t / w, c = t % w;
    T v;
    v.x = 0;
    v.y = 0;
    if (c >= i0 && c - i0 < hi && c - i0 <= i) v = sX[i][c - i0];
    X[(size_t)(i0 + i) * w + c] = v;
  }
}

// Level s: pair p joins the blocks [p s, p s + s/2) and [p s + s/2, p s + s)
// (the second may be shorter at the end of w) in two launches of one CTA per
// 32 x 32 tile (ty: tile row of block 2, tx: tile column of block 1):
//   k_inv_join_t:  Tp = L21 X11          (X11 lower: k from the tile's column)
//   k_inv_join_x:  X21 = -X22 Tp         (X22 lower: m up to the tile's row)
// Tp is the pair's h x h scratch at T + p h h.
template <typename T>
__global__ void __launch_bounds__(256) k_inv_join_t(InvBatch<T> ib, int n, int r0, int w, int s,
                                                    const T* __restrict__ X, T* __restrict__ Tsc) {
  __shared__ T sa[32][33];
  __shared__ T sb[32][33];
  const int h = s / 2;
  const int pairs = (w + s - 1) / s, mb = blockIdx.z / pairs;
  const int p = blockIdx.z - mb * pairs, base = p * s;
  const T* __restrict__ A = ib.A[mb];
  X += (size_t)mb * w * w;
  Tsc += (size_t)mb * w * w / 2;
  const int h2 = min(h, w - base - h);  // rows of the second block
  const int ty = blockIdx.y, tx = blockIdx.x;
  if (h2 <= 0 || ty * 32 >= h2) return;
  const int tid = threadIdx.x, row = tid >> 3, cq = (tid & 7) * 4;
  const int c0 = base + tx * 32;  // columns of X11
  T acc[4];
#pragma unroll
  for (int q = 0; q < 4; q++) acc[q].x = acc[q].y = 0;
  for (int k0 = tx * 32; k0 < h; k0 += 32) {
    __syncthreads();
    for (int t = tid; t < 1024; t += 256) {
      const int i = t >> 5, j = t & 31;
      T a;
      a.x = a.y = 0;
      if (ty * 32 + i < h2) a = A[(size_t)(r0 + base + h + ty * 32 + i) * n + r0 + base + k0 + j];
      sa[i][j] = a;
      sb[i][j] = X[(size_t)(base + k0 + i) * w + c0 + j];
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < 32; kk++) {
      const T a = sa[row][kk];
#pragma unroll
      for (int q = 0; q < 4; q++) cfma_add(acc[q], a, sb[kk][cq + q]);
    }
  }
  if (ty * 32 + row < h2) {
    T* Tp = Tsc + (size_t)p * h * h;
#pragma unroll
    for (int q = 0; q < 4; q++) Tp[(size_t)(ty * 32 + row) * h + tx * 32 + cq + q] = acc[q];
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_inv_join_x(int w, int s, T* __restrict__ X, const T* __restrict__ Tsc) {
  __shared__ T sa[32][33];
  __shared__ T sb[32][33];
  const int h = s / 2;
  const int pairs = (w + s - 1) / s, mb = blockIdx.z / pairs;
  const int p = blockIdx.z - mb * pairs, base = p * s;
  X += (size_t)mb * w * w;
  Tsc += (size_t)mb * w * w / 2;
  const int h2 = min(h, w - base - h);
  const int ty = blockIdx.y, tx = blockIdx.x;
  if (h2 <= 0 || ty * 32 >= h2) return;
  const int tid = threadIdx.x, row = tid >> 3, cq = (tid & 7) * 4;
  const T* Tp = Tsc + (size_t)p * h * h;
  T acc[4];
#pragma unroll
  for (int q = 0; q < 4; q++) acc[q].x = acc[q].y = 0;
  for (int m0 = 0; m0 <= ty * 32; m0 += 32) {
    __syncthreads();
    for (int t = tid; t < 1024; t += 256) {
      const int i = t >> 5, j = t & 31;
      T a, b;
      a.x = a.y = b.x = b.y = 0;
      if (ty * 32 + i < h2 && m0 + j < h2) a = X[(size_t)(base + h + ty * 32 + i) * w + base + h + m0 + j];
      if (m0 + i < h2) b = Tp[(size_t)(m0 + i) * h + tx * 32 + j];
      sa[i][j] = a;
      sb[i][j] = b;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < 32; kk++) {
      const T a = sa[row][kk];
#pragma unroll
      for (int q = 0; q < 4; q++) cfma_sub(acc[q], a, sb[kk][cq + q]);
    }
  }
  if (ty * 32 + row < h2) {
    const int gr = base + h + ty * 32 + row, c0 = base + tx * 32;
#pragma unroll
    for (int q = 0; q < 4; q++) X[(size_t)gr * w + c0 + cq + q] = acc[q];
  }
}

// Interchanges of pivots [p0, p1) applied to columns [a0, a1) and [b0, b1).
template <typename T>
__global__ void k_laswp2(T* __restrict__ A, int n, const int32_t* __restrict__ ipiv, int p0, int p1, int a0, int a1,
                         int b0, int b1) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int na = a1 - a0;
  int c;
  if (t < na) c = a0 + t;
  else if (t - na < b1 - b0) c = b0 + (t - na);
  else return;
  for (int j = p0; j < p1; j++) {
    const int p = ipiv[j];
    if (p != j) {
      const T tmp = A[(size_t)j * n + c];
      A[(size_t)j * n + c] = A[(size_t)p * n + c];
      A[(size_t)p * n + c] = tmp;
    }
  }
}

// X <- L^{-1} X, L the w x w unit-lower block at (r0, r0), X = rows [r0, r0+w) of columns [cb, ce).
// With pack_mode (complex64 only), X is also written as the packed B operand
// of the real-row tensor-core update that follows (w deep, ce - cb columns).
// The matrices of a batch whose same 32-row block is solved in one launch
// (blockIdx.y = matrix); matrix b's operand planes start at WB + b plane.
template <typename T>
struct TrsmBatch {
  T* A[4];
  unsigned char* WB;
  size_t plane;
};

template <typename T>
__global__ void __launch_bounds__(256) k_trsm_blk(TrsmBatch<T> tb, int n, int r0, int w, int cb, int ce,
                                                  int pack_mode) {
  __shared__ T sL[IB][IB + 1];
  __shared__ T sX[IB][33];
  T* __restrict__ A = tb.A[blockIdx.y];
  void* __restrict__ WB = tb.WB ? tb.WB + tb.plane * blockIdx.y : nullptr;
  const int c0 = cb + blockIdx.x * 32;
  for (int t = threadIdx.x; t < w * w; t += blockDim.x) sL[t / w][t % w] = A[(size_t)(r0 + t / w) * n + r0 + t % w];
  for (int t = threadIdx.x; t < w * 32; t += blockDim.x) {
    const int i = t / 32, c = c0 + t % 32;
    T v;
    v.x = 0;
    v.y = 0;
    if (c < ce) v = A[(size_t)(r0 + i) * n + c];
    sX[i][t % 32] = v;
  }
  __syncthreads();
  const int cc = threadIdx.x % 32, grp = threadIdx.x / 32;
  for (int i = 0; i < w; i++) {
    const T xi = sX[i][cc];
    for (int r = i + 1 + grp; r < w; r += 8) {
      const T l = sL[r][i];
      T v = sX[r][cc];
      v.x -= l.x * xi.x - l.y * xi.y;
      v.y -= l.x * xi.y + l.y * xi.x;
      sX[r][cc] = v;
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < w * 32; t += blockDim.x) {
    const int i = t / 32, c = c0 + t % 32;
    if (c < ce) {
      A[(size_t)(r0 + i) * n + c] = sX[i][t % 32];
      if constexpr (sizeof(T) == sizeof(float2)) {
        if (pack_mode) {
          const T v = sX[i][t % 32];
          tc2_pack_b(pack_mode, WB, ce - cb, w, c - cb, i, make_float2(v.x, v.y));
        }
      }
    }
  }
}

// C[M x N] -= L[M x K] U[K x N], complex, leading dimensions ld*; 64 x 64 tiles.
template <typename T>
__global__ void __launch_bounds__(256) k_gemm_sub(T* __restrict__ C, int ldc, const T* __restrict__ L, int ldl,
                                                  const T* __restrict__ U, int ldu, int M, int N, int K) {
  using R = typename Real<T>::R;
  constexpr int BM = 64, BN = 64, BK = 16;
  __shared__ T sA[BK][BM + 1];
  __shared__ T sB[BK][BN + 1];
  const int r0 = blockIdx.y * BM, c0 = blockIdx.x * BN;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  R ar[4][4], ai[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) ar[i][j] = ai[i][j] = 0;
  for (int k0 = 0; k0 < K; k0 += BK) {
    for (int t = threadIdx.x; t < BM * BK; t += 256) {
      const int i = t / BK, q = t % BK;
      T v;
      v.x = 0;
      v.y = 0;
      if (r0 + i < M && k0 + q < K) v = L[(size_t)(r0 + i) * ldl + k0 + q];
      sA[q][i] = v;
    }
    for (int t = threadIdx.x; t < BK * BN; t += 256) {
      const int q = t / BN, j = t % BN;
      T v;
      v.x = 0;
      v.y = 0;
      if (c0 + j < N && k0 + q < K) v = U[(size_t)(k0 + q) * ldu + c0 + j];
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
          ar[i][j] += a[i].x * b[j].x - a[i].y * b[j].y;
          ai[i][j] += a[i].x * b[j].y + a[i].y * b[j].x;
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int r = r0 + ty + 16 * i;
    if (r >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int c = c0 + tx + 16 * j;
      if (c >= N) continue;
      T v = C[(size_t)r * ldc + c];
      v.x -= ar[i][j];
      v.y -= ai[i][j];
      C[(size_t)r * ldc + c] = v;
    }
  }
}

template <typename T>
int gemm_sub(T* C, int ldc, const T* L, int ldl, const T* U, int ldu, int M, int N, int K, cudaStream_t st) {
  if (M <= 0 || N <= 0 || K <= 0) return TT_OK;
  if constexpr (sizeof(T) == sizeof(double2))
    return zgemm_sub_dmma(reinterpret_cast<double2*>(C), ldc, reinterpret_cast<const double2*>(L), ldl,
                          reinterpret_cast<const double2*>(U), ldu, M, N, K, st);
  dim3 grid(ceil_div(N, 64), ceil_div(M, 64));
  ProfScope prof(TT_PROF_SIMT_UPDATE, st, 8.0 * M * N * K, 2.0 * M * N * sizeof(T) + ((double)M + N) * K * sizeof(T));
  k_gemm_sub<T><<<grid, 256, 0, st>>>(C, ldc, L, ldl, U, ldu, M, N, K);
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

template <typename T>
int laswp2(T* A, int n, const int32_t* ipiv, int p0, int p1, int a0, int a1, int b0, int b1, cudaStream_t st) {
  const int cols = std::max(0, a1 - a0) + std::max(0, b1 - b0);
  if (cols <= 0 || p1 <= p0) return TT_OK;
  ProfScope prof(TT_PROF_LASWP, st, 0.0, 4.0 * (p1 - p0) * cols * sizeof(T));
  k_laswp2<T><<<ceil_div(cols, 256), 256, 0, st>>>(A, n, ipiv, p0, p1, a0, std::max(a0, a1), b0, std::max(b0, b1));
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

// X: B w w elements (inverse of matrix b at X + b w w, ld w); Tsc: scratch of
// at least B w w / 2 elements.  B <= 4.
template <typename T>
int inv_unit_lower(const T* const* As, int B, int n, int r0, int w, T* X, T* Tsc, cudaStream_t st) {
  if (w <= 0) return TT_OK;
  InvBatch<T> ib{};
  for (int b = 0; b < B; b++) ib.A[b] = As[b];
  if (w > INV_MAX || w % 32 != 0) {
    set_error("unit-lower inverse of a block of " + std::to_string(w) + " rows (multiples of 32 up to " +
              std::to_string(INV_MAX) + ")");
    return TT_ERR_BADARG;
  }
  ProfScope prof(TT_PROF_PANEL_TRSM, st, 8.0 / 6.0 * w * (double)w * w * B, 2.0 * w * (double)w * sizeof(T) * B);
  k_inv_diag32<T><<<dim3(w / 32, B), 256, 0, st>>>(ib, n, r0, w, X);
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  for (int s = 64; s / 2 < w; s *= 2) {
    const int h = s / 2;
    dim3 grid(h / 32, h / 32, ((w + s - 1) / s) * B);
    k_inv_join_t<T><<<grid, 256, 0, st>>>(ib, n, r0, w, s, X, Tsc);
    count_launch();
    TT_CUDA_TRY(cudaGetLastError());
    k_inv_join_x<T><<<grid, 256, 0, st>>>(w, s, X, Tsc);
    count_launch();
    TT_CUDA_TRY(cudaGetLastError());
  }
  return TT_OK;
}

// the same block of B <= 4 matrices (pack_mode: matrix b's solved rows also
// go to its operand planes at WB + b plane)
template <typename T>
int trsm_blk_batched(T* const* As, int B, int n, int r0, int w, int cb, int ce, cudaStream_t st, int pack_mode = 0,
                     unsigned char* WB = nullptr, size_t plane = 0) {
  if (ce <= cb) return TT_OK;
  ProfScope prof(TT_PROF_PANEL_TRSM, st, 4.0 * w * w * (double)(ce - cb) * B,
                 2.0 * w * (double)(ce - cb) * sizeof(T) * B);
  TrsmBatch<T> tb{};
  for (int b = 0; b < B; b++) tb.A[b] = As[b];
  tb.WB = WB;
  tb.plane = plane;
  k_trsm_blk<T><<<dim3(ceil_div(ce - cb, 32), B), 256, 0, st>>>(tb, n, r0, w, cb, ce, pack_mode);
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

template <typename T>
int trsm_blk(T* A, int n, int r0, int w, int cb, int ce, cudaStream_t st) {
  return trsm_blk_batched<T>(&A, 1, n, r0, w, cb, ce, st);
}

// C -= L U on the tensor cores in the factorisation's product mode when K is
// a multiple of the mode's k-chunk, else on the CUDA cores
template <typename T>
int panel_gemm_sub(int mode, T* C, int ldc, const T* L, int ldl, const T* U, int ldu, int M, int N, int K,
                   cudaStream_t st) {
  if (M <= 0 || N <= 0 || K <= 0) return TT_OK;
  if (mode == TC_LEGACY_BF16X3 && K % 32 == 0)
    return tc_gemm_sub(reinterpret_cast<float2*>(C), ldc, reinterpret_cast<const float2*>(L), ldl,
                       reinterpret_cast<const float2*>(U), ldu, M, N, K, st);
  if ((mode == TC_TF32 || mode == TC_BF16X3) && K % 16 == 0)
    return tc2_gemm_sub(mode, reinterpret_cast<float2*>(C), ldc, reinterpret_cast<const float2*>(L), ldl,
                        reinterpret_cast<const float2*>(U), ldu, M, N, K, st);
  return gemm_sub(C, ldc, L, ldl, U, ldu, M, N, K, st);
}

}  // namespace

template <typename T>
int lu_factor_batched_device(T* const* As, int B, int n, int32_t* const* ipivs, cudaStream_t st, int use_tc,
                             int* info, bool blocked_order, int panel, int inv_block, bool cta_pairs, int mid) {
  const int mode = use_tc;
  const bool tc = mode != 0;
  if (mode < 0 || mode > TC_BF16X3) {
    set_error("unknown tensor-core product mode " + std::to_string(mode));
    return TT_ERR_BADARG;
  }
  if (tc && sizeof(T) != sizeof(float2)) {
    set_error("tensor-core trailing update is only defined for the complex64 factorisation");
    return TT_ERR_UNSUPPORTED;
  }
  if (B < 1 || B > kMaxBatch) {
    set_error("LU batch of " + std::to_string(B) + " matrices (1.." + std::to_string(kMaxBatch) + ")");
    return TT_ERR_BADARG;
  }
  if (panel < 0 || panel > INV_MAX || panel % IB != 0) {
    set_error("panel width " + std::to_string(panel) + " (a multiple of 32 up to 512)");
    return TT_ERR_BADARG;
  }
  if (mid < 0 || mid % IB != 0) {
    set_error("mid-panel width " + std::to_string(mid) + " (0 or a multiple of 32)");
    return TT_ERR_BADARG;
  }
  if (inv_block < 0 || inv_block > INV_MAX || inv_block % IB != 0) {
    set_error("inverse block " + std::to_string(inv_block) + " (a multiple of 32 up to 512)");
    return TT_ERR_BADARG;
  }
  const int IVB = inv_block ? inv_block : INV_MAX;
  // the update kernel's tile shape for this factorisation (restored on return)
  struct PairScope {
    explicit PairScope(bool on) { tc2_set_pairs(on); }
    ~PairScope() { tc2_set_pairs(false); }
  } pair_scope(cta_pairs);
  const int NB = panel ? panel : (sizeof(T) == sizeof(float2)) ? 512 : 128;
  const int G = device_sm_count();
  DevBuf<double> sval;
  DevBuf<int> sidx, d_info;
  DevBuf<T> srow, stop;
  DevBuf<unsigned long long> skey;
  TT_TRY(sval.alloc(2 * (size_t)G));
  TT_TRY(sidx.alloc(2 * (size_t)G));
  TT_TRY(srow.alloc(2 * (size_t)G * IB));
  TT_TRY(stop.alloc(2 * (size_t)kMaxBatch * IB));
  TT_TRY(skey.alloc((size_t)B * n));
  TT_TRY(d_info.alloc(B));
  TT_CUDA_TRY(cudaMemsetAsync(d_info.ptr, 0, sizeof(int) * B, st));
  TT_CUDA_TRY(cudaMemsetAsync(skey.ptr, 0, sizeof(unsigned long long) * B * n, st));
  PivotScratch<T> scr{sval.ptr, sidx.ptr, srow.ptr, stop.ptr, skey.ptr};
  TT_TRY(smem_limit_once((const void*)k_subpanel_smem<T>, (int)kSubpanelSmem));
  // the sub-panel of matrices [b0, b0 + nb) in one cooperative launch
  auto subpanel = [&](int b0, int nb, int j0, int w, int pk0, int pk1, int grid) -> int {
    SubpanelBatch<T> bt{};
    for (int b = 0; b < nb; b++) {
      bt.A[b] = As[b0 + b];
      bt.ipiv[b] = ipivs[b0 + b];
      bt.key[b] = skey.ptr + (size_t)(b0 + b) * n;
    }
    bt.info = d_info.ptr + b0;
    bt.B = nb;
    int nn = n, cc0 = j0, ww = w, p0 = pk0, p1 = pk1;
    void* args[] = {&bt, &nn, &cc0, &ww, &p0, &p1, &scr};
    const size_t chunk = (size_t)(n - j0 + grid / nb - 1) / (grid / nb);
    TT_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_subpanel_smem<T>, dim3(grid), dim3(SP_THREADS), args,
                                            chunk * SP * sizeof(T), st));
    count_launch();
    return TT_OK;
  };
  // pivoted factorisation of columns [j0, j0 + w), w <= IB, rows [j0, n), of all B matrices,
  // with its interchanges applied to the panel's other columns [pk0, j0) and [j0 + w, pk1)
  auto leaf = [&](int j0, int w, int pk0, int pk1) -> int {
    const size_t m = (size_t)(n - j0);
    const int Gb = G / B;
    const bool keyed = m < 0xFFFFF;
    const bool together = B > 1 && keyed && ((m + Gb - 1) / Gb) * SP * sizeof(T) <= kSubpanelSmem;
    const bool alone = keyed && ((m + G - 1) / G) * SP * sizeof(T) <= kSubpanelSmem;
    ProfScope prof(TT_PROF_SUBPANEL, st, 4.0 * m * w * w * B, 2.0 * m * w * sizeof(T) * B);
    if (together) return subpanel(0, B, j0, w, pk0, pk1, Gb * B);
    for (int b = 0; b < B; b++) {
      if (alone) {
        TT_TRY(subpanel(b, 1, j0, w, pk0, pk1, G));
      } else {
        T* Ap = As[b];
        int nn = n, cc0 = j0, ww = w;
        int32_t* ip = ipivs[b];
        int* inf = d_info.ptr + b;
        void* args[] = {&Ap, &nn, &cc0, &ww, &ip, &scr, &inf};
        TT_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_subpanel<T>, dim3(G), dim3(256), args, 0, st));
        count_launch();
        TT_TRY(laswp2(As[b], n, ipivs[b], j0, j0 + w, pk0, j0, j0 + w, pk1, st));
      }
    }
    return TT_OK;
  };
  // split of a block of h rows or columns: the largest multiple of IB not above h / 2, at least IB
  auto half = [](int h) { return std::max(IB, (h / 2) / IB * IB); };
  // the tensor-core modes solve a block row with the explicit inverse of its
  // unit-lower block: X = L^{-1} once, then U = X A in one product
  const bool inv_solve = (mode == TC_TF32 || mode == TC_BF16X3);
  DevBuf<T> Xinv, Tinv;
  if (inv_solve) {
    const size_t wmax = (size_t)std::min(NB, IVB);
    TT_TRY(Xinv.alloc(wmax * wmax * B));
    TT_TRY(Tinv.alloc(wmax * wmax * B / 2));
  }
  // rows [r0, r0 + h) of columns [cb, ce) <- L^{-1} of them, L the unit-lower h x h block at (r0, r0):
  // halves recursively, so that most of the work is one update of depth h / 2
  std::function<int(T*, int, int, int, int)> trsm_rec = [&](T* A, int r0, int h, int cb, int ce) -> int {
    if (h <= IB) return trsm_blk(A, n, r0, h, cb, ce, st);
    if (inv_solve && h % 32 == 0 && h <= IVB) {
      const T* A1 = A;
      TT_TRY(inv_unit_lower(&A1, 1, n, r0, h, Xinv.ptr, Tinv.ptr, st));
      return tc2_gemm_sub(mode, reinterpret_cast<float2*>(A) + (size_t)r0 * n + cb, n,
                          reinterpret_cast<const float2*>(Xinv.ptr), h,
                          reinterpret_cast<const float2*>(A) + (size_t)r0 * n + cb, n, h, ce - cb, h, st, 1);
    }
    const int h1 = half(h);
    TT_TRY(trsm_rec(A, r0, h1, cb, ce));
    TT_TRY(panel_gemm_sub(mode, A + (size_t)(r0 + h1) * n + cb, n, A + (size_t)(r0 + h1) * n + r0, n,
                          A + (size_t)r0 * n + cb, n, h - h1, ce - cb, h1, st));
    return trsm_rec(A, r0 + h1, h - h1, cb, ce);
  };
  // trsm_rec of the same block in all B matrices: one set of inverse launches
  // for all of them when the block is solved through its explicit inverse
  auto trsm_all = [&](int r0, int h, int cb, int ce) -> int {
    if (!(inv_solve && h > IB && h % 32 == 0 && h <= IVB)) {
      for (int b = 0; b < B; b++) TT_TRY(trsm_rec(As[b], r0, h, cb, ce));
      return TT_OK;
    }
    const T* Ac[kMaxBatch];
    for (int b = 0; b < B; b++) Ac[b] = As[b];
    TT_TRY(inv_unit_lower(Ac, B, n, r0, h, Xinv.ptr, Tinv.ptr, st));
    float2* Cs[kMaxBatch];
    const float2* Ls[kMaxBatch];
    const float2* Us[kMaxBatch];
    for (int b = 0; b < B; b++) {
      Cs[b] = reinterpret_cast<float2*>(As[b]) + (size_t)r0 * n + cb;
      Ls[b] = reinterpret_cast<const float2*>(Xinv.ptr + (size_t)b * h * h);
      Us[b] = Cs[b];
    }
    return tc2_gemm_sub_batched(mode, B, Cs, n, Ls, h, Us, n, h, ce - cb, h, st, 1);
  };
  // C -= L U at the same offsets of all B matrices (row/column offsets of C,
  // L and U given as (row, col) pairs): one batched tensor-core launch in the
  // real-row modes, else one update per matrix
  auto gemm_all = [&](int cr, int cc, int lr, int lc, int ur, int uc, int M, int N, int K) -> int {
    if (M <= 0 || N <= 0 || K <= 0) return TT_OK;
    if ((mode == TC_TF32 || mode == TC_BF16X3) && K % 16 == 0) {
      float2* Cs[kMaxBatch];
      const float2* Ls[kMaxBatch];
      const float2* Us[kMaxBatch];
      for (int b = 0; b < B; b++) {
        float2* A = reinterpret_cast<float2*>(As[b]);
        Cs[b] = A + (size_t)cr * n + cc;
        Ls[b] = A + (size_t)lr * n + lc;
        Us[b] = A + (size_t)ur * n + uc;
      }
      return tc2_gemm_sub_batched(mode, B, Cs, n, Ls, n, Us, n, M, N, K, st);
    }
    for (int b = 0; b < B; b++) {
      T* A = As[b];
      TT_TRY(panel_gemm_sub(mode, A + (size_t)cr * n + cc, n, A + (size_t)lr * n + lc, n, A + (size_t)ur * n + uc, n,
                            M, N, K, st));
    }
    return TT_OK;
  };
  // columns [c0, c0 + w) of the panel [k, k + kb) factored by recursive halving:
  // left half, its U block and the update of the right half (depth w / 2), right half
  std::function<int(int, int, int, int)> factor_cols = [&](int k, int kb, int c0, int w) -> int {
    if (w <= IB) {
      return leaf(c0, w, k, k + kb);
    }
    const int h = half(w);
    TT_TRY(factor_cols(k, kb, c0, h));
    for (int b = 0; b < B; b++) {
      T* A = As[b];
      TT_TRY(trsm_rec(A, c0, h, c0 + h, c0 + w));
      TT_TRY(panel_gemm_sub(mode, A + (size_t)(c0 + h) * n + (c0 + h), n, A + (size_t)(c0 + h) * n + c0, n,
                            A + (size_t)c0 * n + (c0 + h), n, n - c0 - h, w - h, h, st));
    }
    return factor_cols(k, kb, c0 + h, w - h);
  };
  const bool blocked = blocked_order || mode == TC_LEGACY_BF16X3;
  for (int k = 0; k < n; k += NB) {
    const int kb = std::min(NB, n - k);
    const int rest = n - k - kb;
    if (!blocked) {
      TT_TRY(factor_cols(k, kb, k, kb));
      for (int b = 0; b < B; b++) {
        T* A = As[b];
        // ---- interchanges outside the panel, U12 = L11^{-1} A12, trailing update
        TT_TRY(laswp2(A, n, ipivs[b], k, k + kb, 0, k, k + kb, n, st));
        if (rest <= 0) continue;
        TT_TRY(trsm_rec(A, k, kb, k + kb, n));
        if (tc)
          TT_TRY(tc2_gemm_sub(mode, reinterpret_cast<float2*>(A) + (size_t)(k + kb) * n + (k + kb), n,
                              reinterpret_cast<const float2*>(A) + (size_t)(k + kb) * n + k, n,
                              reinterpret_cast<const float2*>(A) + (size_t)k * n + (k + kb), n, rest, rest, kb, st));
        else
          TT_TRY(gemm_sub(A + (size_t)(k + kb) * n + (k + kb), n, A + (size_t)(k + kb) * n + k, n,
                          A + (size_t)k * n + (k + kb), n, rest, rest, kb, st));
      }
      continue;
    }
    // ---- panel [k, k+kb) in mid-panels of MB columns (MB = kb: one level),
    // each in sub-panels of IB columns updated within the mid-panel, then the
    // mid-panel's U block row and the update of the panel's columns right of it
    const int MB = (mid > 0 && mid < kb) ? mid : kb;
    for (int m0 = k; m0 < k + kb; m0 += MB) {
      const int mw = std::min(MB, k + kb - m0);
      for (int j0 = m0; j0 < m0 + mw; j0 += IB) {
        const int w = std::min(IB, m0 + mw - j0);
        TT_TRY(leaf(j0, w, k, k + kb));
        const int right = m0 + mw - (j0 + w);
        if (right > 0 && inv_solve && w % 16 == 0) {
          // the solved block rows are written straight into the update's
          // operand planes, then one update for all matrices
          int ws = TT_OK;
          unsigned char* WB = static_cast<unsigned char*>(tc2_b_workspace(mode, right, w, &ws, B));
          TT_TRY(ws);
          const size_t plane = tc2_b_plane_bytes(mode, right, w);
          float2* Cs[kMaxBatch];
          const float2* Ls[kMaxBatch];
          const float2* Us[kMaxBatch];
          TT_TRY(trsm_blk_batched<T>(As, B, n, j0, w, j0 + w, m0 + mw, st, mode, WB, plane));
          for (int b = 0; b < B; b++) {
            float2* A = reinterpret_cast<float2*>(As[b]);
            Cs[b] = A + (size_t)(j0 + w) * n + (j0 + w);
            Ls[b] = A + (size_t)(j0 + w) * n + j0;
            Us[b] = A + (size_t)j0 * n + (j0 + w);
          }
          TT_TRY(tc2_gemm_sub_batched(mode, B, Cs, n, Ls, n, Us, n, n - j0 - w, right, w, st, 0, true));
        } else if (right > 0) {
          for (int b = 0; b < B; b++) {
            T* A = As[b];
            TT_TRY(trsm_blk(A, n, j0, w, j0 + w, m0 + mw, st));
            TT_TRY(panel_gemm_sub(mode, A + (size_t)(j0 + w) * n + (j0 + w), n, A + (size_t)(j0 + w) * n + j0, n,
                                  A + (size_t)j0 * n + (j0 + w), n, n - j0 - w, right, w, st));
          }
        }
      }
      const int right_out = k + kb - (m0 + mw);
      if (right_out > 0) {
        TT_TRY(trsm_all(m0, mw, m0 + mw, k + kb));
        TT_TRY(gemm_all(m0 + mw, m0 + mw, m0 + mw, m0, m0, m0 + mw, n - m0 - mw, right_out, mw));
      }
    }
    // ---- interchanges outside the panel; U12 = L11^{-1} A12 with the
    // explicit inverse in the tensor-core modes (all matrices together)
    for (int b = 0; b < B; b++) TT_TRY(laswp2(As[b], n, ipivs[b], k, k + kb, 0, k, k + kb, n, st));
    if (rest > 0 && inv_solve) TT_TRY(trsm_all(k, kb, k + kb, n));
    for (int b = 0; b < B; b++) {
      T* A = As[b];
      if (rest <= 0) continue;
      // ---- U12 blocked by IB without tensor cores
      if (!inv_solve) for (int i0 = k; i0 < k + kb; i0 += IB) {
        const int wi = std::min(IB, k + kb - i0);
        TT_TRY(trsm_blk(A, n, i0, wi, k + kb, n, st));
        const int below = k + kb - (i0 + wi);
        if (below > 0)
          TT_TRY(panel_gemm_sub(mode, A + (size_t)(i0 + wi) * n + (k + kb), n, A + (size_t)(i0 + wi) * n + i0, n,
                                A + (size_t)i0 * n + (k + kb), n, below, rest, wi, st));
      }
      // ---- trailing update (the real-row modes: below, all matrices in one launch)
      if (mode == TC_LEGACY_BF16X3)
        TT_TRY(lu_update_tc(reinterpret_cast<float2*>(A), n, k, kb, st));
      else if (!tc)
        TT_TRY(gemm_sub(A + (size_t)(k + kb) * n + (k + kb), n, A + (size_t)(k + kb) * n + k, n,
                        A + (size_t)k * n + (k + kb), n, rest, rest, kb, st));
    }
    if (rest > 0 && (mode == TC_TF32 || mode == TC_BF16X3))
      TT_TRY(gemm_all(k + kb, k + kb, k + kb, k, k, k + kb, rest, rest, kb));
  }
  if (mode == TC_LEGACY_BF16X3) TT_TRY(tc_check_error(st));
  if (mode == TC_TF32 || mode == TC_BF16X3) TT_TRY(tc2_check_error(st));
  if (info) {
    TT_CUDA_TRY(cudaMemcpyAsync(info, d_info.ptr, sizeof(int) * B, cudaMemcpyDeviceToHost, st));
    TT_CUDA_TRY(cudaStreamSynchronize(st));
  }
  return TT_OK;
}
template int lu_factor_batched_device<double2>(double2* const*, int, int, int32_t* const*, cudaStream_t, int, int*,
                                               bool, int, int, bool, int);
template int lu_factor_batched_device<float2>(float2* const*, int, int, int32_t* const*, cudaStream_t, int, int*,
                                              bool, int, int, bool, int);

template <typename T>
int lu_factor_device(T* A, int n, int32_t* ipiv, cudaStream_t st, int use_tc, int* info) {
  return lu_factor_batched_device<T>(&A, 1, n, &ipiv, st, use_tc, info);
}
template int lu_factor_device<double2>(double2*, int, int32_t*, cudaStream_t, int, int*);
template int lu_factor_device<float2>(float2*, int, int32_t*, cudaStream_t, int, int*);

}  // namespace tt
