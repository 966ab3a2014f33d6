// Triangular solves with the LU factor of lu_factor.cu (the zgetrs half of the
// reference's LAPACK solve, General_functions/matrix_routines.cpp:73-80), for a
// few right-hand sides at a time: forward substitution with the unit lower
// factor and back substitution with the upper factor.
//
// The factor is read once per substitution, as a stream: after each
// factorisation the 64 x 64 diagonal blocks of L and U are inverted (one CTA
// per block, in shared memory) and multiplied into the neighbouring
// off-diagonal block; each substitution is then one cooperative kernel with
// one grid barrier per block column (k_trsv).

#include <cooperative_groups.h>

#include <algorithm>
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

constexpr int TSB = 64;       // diagonal block of the substitution (both element types)
constexpr int TLD = TSB + 1;  // padded shared-memory row of a 64 x 64 tile

template <typename T>
__device__ __forceinline__ T cmul(T a, T b) {
  T r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename T>
__device__ __forceinline__ T crecip(T b) {
  using R = typename CT<T>::R;
  // Smith's algorithm for 1 / b
  T r;
  if (fabs((double)b.x) >= fabs((double)b.y)) {
    const R t = b.y / b.x, d = b.x + b.y * t;
    r.x = R(1) / d;
    r.y = -t / d;
  } else {
    const R t = b.x / b.y, d = b.y + b.x * t;
    r.x = t / d;
    r.y = R(-1) / d;
  }
  return r;
}

__global__ void k_permute(const double2* __restrict__ b, const int32_t* __restrict__ perm, int n, int nrhs,
                          double2* __restrict__ x) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)n * nrhs) return;
  const int k = (int)(t / n), i = (int)(t % n);
  x[t] = b[(size_t)k * n + perm[i]];
}

// x[perm[i]] = w[i]: the row interchanges applied backwards (transposed solves)
__global__ void k_permute_inv(const double2* __restrict__ w, const int32_t* __restrict__ perm, int n, int nrhs,
                              double2* __restrict__ x) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)n * nrhs) return;
  const int k = (int)(t / n), i = (int)(t % n);
  x[(size_t)k * n + perm[i]] = w[t];
}

// ---------------------------------------------------------------------------
// Inverses of the diagonal blocks: inv[b] (64 x 64, row-major) of the lower
// (UPPER = false) or upper (UPPER = true) triangle of block b of the factor,
// with a unit diagonal (UNIT) or the stored one.  The factor of L U keeps the
// unit lower and the upper triangle; its transpose (for transposed solves)
// keeps the non-unit lower and the unit upper triangle.  Rows and columns past
// n are the identity.  In place in shared memory, right-looking, row j being
// final when step j starts:
// lower, j ascending: row j is scaled by 1/D[j][j], then
// X[r][c] -= L[r][j] X[j][c] for r > j, c <= j;
// upper, j descending: row j is scaled by 1/D[j][j], then
// X[r][c] -= U[r][j] X[j][c] for r < j, c >= j.
template <typename T, bool UPPER, bool UNIT>
__global__ void __launch_bounds__(512) k_inv_diag(const T* __restrict__ LU, int n, T* __restrict__ inv) {
  extern __shared__ unsigned char ism[];
  T* M = reinterpret_cast<T*>(ism);  // [TSB][TLD]
  __shared__ T col[TSB];
  const int b = blockIdx.x, r0 = b * TSB, bs = min(TSB, n - r0);
  const T zero = {0, 0}, one = {1, 0};
  // stored entries of the triangle (the diagonal only when it is not unit)
  auto stored = [](int r, int c) { return UPPER ? (UNIT ? c > r : c >= r) : (UNIT ? c < r : c <= r); };
  for (int t = threadIdx.x; t < TSB * TSB; t += blockDim.x) {
    const int r = t / TSB, c = t % TSB;
    T v = (r == c) ? one : zero;
    if (r < bs && c < bs && stored(r, c)) v = LU[(size_t)(r0 + r) * n + r0 + c];
    M[r * TLD + c] = v;
  }
  __syncthreads();
  if (!UPPER) {
    for (int j = 0; j < bs; j++) {
      T d = one;
      if (!UNIT) {
        d = crecip(M[j * TLD + j]);
        __syncthreads();
        for (int c = threadIdx.x; c < j; c += blockDim.x) M[j * TLD + c] = cmul(M[j * TLD + c], d);
        if (threadIdx.x == 0) M[j * TLD + j] = d;
      }
      for (int r = j + 1 + threadIdx.x; r < bs; r += blockDim.x) col[r] = M[r * TLD + j];
      __syncthreads();
      const int w = j + 1, cnt = (bs - 1 - j) * w;
      for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
        const int r = j + 1 + t / w, c = t % w;
        const T l = col[r];
        if (c == j) {
          const T p = cmul(l, d);
          M[r * TLD + j] = T{-p.x, -p.y};
        } else {
          const T p = cmul(l, M[j * TLD + c]);
          T v = M[r * TLD + c];
          v.x -= p.x;
          v.y -= p.y;
          M[r * TLD + c] = v;
        }
      }
      __syncthreads();
    }
  } else {
    for (int j = bs - 1; j >= 0; j--) {
      T d = one;
      if (!UNIT) {
        d = crecip(M[j * TLD + j]);
        __syncthreads();
        for (int c = j + 1 + threadIdx.x; c < bs; c += blockDim.x) M[j * TLD + c] = cmul(M[j * TLD + c], d);
        if (threadIdx.x == 0) M[j * TLD + j] = d;
      }
      for (int r = threadIdx.x; r < j; r += blockDim.x) col[r] = M[r * TLD + j];
      __syncthreads();
      const int w = bs - j, cnt = j * w;
      for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
        const int r = t / w, c = j + t % w;
        const T u = col[r];
        if (c == j) {
          const T p = cmul(u, d);
          M[r * TLD + j] = T{-p.x, -p.y};
        } else {
          const T p = cmul(u, M[j * TLD + c]);
          T v = M[r * TLD + c];
          v.x -= p.x;
          v.y -= p.y;
          M[r * TLD + c] = v;
        }
      }
      __syncthreads();
    }
  }
  T* out = inv + (size_t)b * TSB * TSB;
  for (int t = threadIdx.x; t < TSB * TSB; t += blockDim.x) {
    const int r = t / TSB, c = t % TSB;
    const bool keep = r < bs && c < bs && (UPPER ? c >= r : c <= r);
    out[t] = keep ? M[r * TLD + c] : ((r == c) ? one : zero);
  }
}

// M[b] = inv[b] LU[b, prev(b)] for the blocks after the first in sweep order
// (prev = b-1 forward, b+1 backward): the product that carries the solved
// previous block into block b, so that x_b = inv[b] x_b - M[b] x_prev.
template <typename T, bool UPPER>
__global__ void __launch_bounds__(512) k_prev_mul(const T* __restrict__ LU, int n, const T* __restrict__ inv,
                                                  T* __restrict__ Mo) {
  extern __shared__ unsigned char psm[];
  T* sI = reinterpret_cast<T*>(psm);  // [TSB][TLD]
  T* sT = sI + TSB * TLD;             // [TSB][TLD]
  const int nb = (n + TSB - 1) / TSB, b = blockIdx.x;
  const int prev = UPPER ? b + 1 : b - 1;
  if (prev < 0 || prev >= nb) return;
  const int r0 = b * TSB, rows = min(TSB, n - r0), c0 = prev * TSB, cols = min(TSB, n - c0);
  for (int t = threadIdx.x; t < TSB * TSB; t += blockDim.x) {
    const int r = t / TSB, c = t % TSB;
    sI[r * TLD + c] = inv[(size_t)b * TSB * TSB + t];
    sT[r * TLD + c] = (r < rows && c < cols) ? LU[(size_t)(r0 + r) * n + c0 + c] : T{0, 0};
  }
  __syncthreads();
  for (int t = threadIdx.x; t < TSB * TSB; t += blockDim.x) {
    const int r = t / TSB, c = t % TSB;
    T acc = {0, 0};
    for (int u = 0; u < TSB; u++) {
      const T p = cmul(sI[r * TLD + u], sT[u * TLD + c]);
      acc.x += p.x;
      acc.y += p.y;
    }
    Mo[(size_t)b * TSB * TSB + t] = acc;
  }
}

// ---------------------------------------------------------------------------
// One substitution (forward with L when !UPPER, backward with U when UPPER)
// for kn <= RHS right-hand sides x[k][n], cooperative, one grid barrier per
// block column.  Blocks are visited in sweep order q = 0, 1, .. (block q for
// the forward sweep, block nb-1-q for the backward one).  Arithmetic is in the
// factor's precision (FP32 for the complex64 factor, whose solves only feed the
// FP64-residual refinement; FP64 for the complex128 factor); x stays complex128.
//  - CTA 0 owns the serial chain: at step s it solves block q = s+1,
//    x_{s+1} = inv[s+1] x_{s+1} - M[s+1] x_s, one 64 x 128 product with both
//    tiles already in shared memory (cp.async issued a step ahead, during the
//    barrier), and writes the solved block to x.
//  - Blocks q >= 2 are owned round-robin by CTAs 1..G-1, which keep their rows
//    of x in shared memory for the whole sweep: at step s every owner applies
//    block column s to its unsolved blocks (q >= s+2) and publishes block s+2
//    to x, which CTA 0 reads at the next step.  Eight lanes share a row (four
//    rows per warp) against x_s staged in shared memory, and the next owned
//    tile is loaded while the current one is applied.  x is never read-modify-written in global
//    memory.
constexpr int RHS = 4;
constexpr int TRSV_THREADS = 512;

__device__ __forceinline__ void cp_async_elem(void* smem, const void* gmem, int bytes) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  if (bytes == 16)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// 64 x 64 block b of a [nb][64][64] array into dst[TSB][TLD]; no commit
template <typename T>
__device__ __forceinline__ void tile_async(const T* __restrict__ src, int b, T* dst) {
  for (int t = threadIdx.x; t < TSB * TSB; t += blockDim.x)
    cp_async_elem(&dst[(t / TSB) * TLD + t % TSB], src + (size_t)b * TSB * TSB + t, sizeof(T));
}

// reduce 16 values over the 32 lanes of a warp: a butterfly that halves the
// values each round (8+4+2+1 shuffles) and a final pair sum; value lane >> 1
// ends complete in lanes 2i and 2i+1
template <typename C>
__device__ __forceinline__ C butterfly16(C (&acc)[16], int lane) {
#pragma unroll
  for (int o = 16, m = 8; m >= 1; o >>= 1, m >>= 1) {
    const bool up = (lane & o) != 0;
#pragma unroll
    for (int j = 0; j < m; j++) {
      const C send = up ? acc[j] : acc[j + m];
      const C keep = up ? acc[j + m] : acc[j];
      acc[j] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
  }
  return acc[0] + __shfl_xor_sync(0xffffffffu, acc[0], 1);
}

// Up to kMaxSweeps factors swept in one cooperative launch: the grid splits
// into B equal groups, each with its own lead CTA and owners, sharing every
// grid barrier.
constexpr int kMaxSweeps = 4;
template <typename T>
struct TrsvBatch {
  const T* LU[kMaxSweeps];
  const T* inv[kMaxSweeps];
  const T* Mp[kMaxSweeps];
  double2* x[kMaxSweeps];
  int B;
};

template <typename T, bool UPPER>
__global__ void __launch_bounds__(TRSV_THREADS, 1) k_trsv(TrsvBatch<T> bt, int n, int kn, int own_max) {
  const int Gb = gridDim.x / bt.B, grp = blockIdx.x / Gb, local = blockIdx.x - grp * Gb;
  const T* __restrict__ LU = bt.LU[grp];
  const T* __restrict__ inv = bt.inv[grp];
  const T* __restrict__ Mp = bt.Mp[grp];
  double2* __restrict__ x = bt.x[grp];
  using C = typename CT<T>::R;
  constexpr int TILE = TSB * TLD;
  cg::grid_group grid = cg::this_grid();
  extern __shared__ __align__(16) unsigned char tsm[];
  T* tI = reinterpret_cast<T*>(tsm);                         // CTA 0: inverse tile
  T* tM = tI + TILE;                                         // CTA 0: M tile
  T* xo = reinterpret_cast<T*>(tsm + 2 * TILE * sizeof(T));  // owners: [own_max][RHS][TSB]
  __shared__ T xs[RHS][TSB];   // CTA 0: solved block of this step
  __shared__ T bsh[RHS][TSB];  // CTA 0: published rows of the block being solved
  __shared__ T ysh[RHS][TSB];  // CTA 0: its solution
  const int nb = (n + TSB - 1) / TSB;
  const int G = Gb;  // this factor's CTAs, >= 2
  const bool lead = local == 0;
  auto blk = [&](int q) { return UPPER ? nb - 1 - q : q; };
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  auto ld_x = [&](int k, int r) -> T {
    const double2 v = x[(size_t)k * n + r];
    return T{(C)v.x, (C)v.y};
  };
  // CTA 0: out = tI . bsh - tM . xs for rows warp*4 .. +3 (two pairs), lanes
  // over the columns lane and lane+32, to ysh and to x rows [r0, r0+rows)
  auto lead_solve = [&](int r0, int rows) {
#pragma unroll
    for (int hp = 0; hp < 2; hp++) {
      C acc[16];
#pragma unroll
      for (int hh = 0; hh < 2; hh++) {
        const int r = warp * 4 + hp * 2 + hh;
        const T i0 = tI[r * TLD + lane], i1 = tI[r * TLD + lane + 32];
        const T m0 = tM[r * TLD + lane], m1 = tM[r * TLD + lane + 32];
#pragma unroll
        for (int k = 0; k < RHS; k++) {
          C sr = 0, si = 0;
          if (k < kn) {
            const T b0 = bsh[k][lane], b1 = bsh[k][lane + 32], y0 = xs[k][lane], y1 = xs[k][lane + 32];
            sr = i0.x * b0.x - i0.y * b0.y + i1.x * b1.x - i1.y * b1.y -
                 (m0.x * y0.x - m0.y * y0.y + m1.x * y1.x - m1.y * y1.y);
            si = i0.x * b0.y + i0.y * b0.x + i1.x * b1.y + i1.y * b1.x -
                 (m0.x * y0.y + m0.y * y0.x + m1.x * y1.y + m1.y * y1.x);
          }
          acc[(hh * RHS + k) * 2 + 0] = sr;
          acc[(hh * RHS + k) * 2 + 1] = si;
        }
      }
      const C v = butterfly16<C>(acc, lane);
      const int idx = lane >> 1, hh = idx >> 3, k = (idx >> 1) & 3, part = idx & 1;
      const int r = warp * 4 + hp * 2 + hh;
      if ((lane & 1) == 0 && k < kn) {
        reinterpret_cast<C*>(&ysh[k][r])[part] = v;
        if (r < rows) reinterpret_cast<double*>(x + (size_t)k * n + r0 + r)[part] = (double)v;
      }

    }
  };

  // owners: slots j of block q = 2 + me + j (G-1)
  const int me = local - 1;
  auto first_slot = [&](int s) { return s > me ? (s - me + (G - 1) - 1) / (G - 1) : 0; };
  auto live = [&](int j) { return j < own_max && 2 + me + j * (G - 1) < nb; };

  if (lead) {
    // first block: x_0 = inv[0] x_0
    tile_async<T>(inv, blk(0), tI);
    cp_async_commit();
    const int r0 = blk(0) * TSB, bsz = min(TSB, n - r0);
    for (int e = t; e < TSB * RHS; e += blockDim.x) {
      const int k = e / TSB, r = e % TSB;
      bsh[k][r] = (k < kn && r < bsz) ? ld_x(k, r0 + r) : T{0, 0};
      xs[k][r] = T{0, 0};
    }
    for (int e = t; e < TILE; e += blockDim.x) tM[e] = T{0, 0};
    cp_async_wait_all();
    __syncthreads();
    lead_solve(r0, bsz);
    __syncthreads();
    for (int e = t; e < TSB * RHS; e += blockDim.x) xs[e / TSB][e % TSB] = ysh[e / TSB][e % TSB];
    if (nb > 1) {
      tile_async<T>(inv, blk(1), tI);
      tile_async<T>(Mp, blk(1), tM);
      cp_async_commit();
    }
  } else {
    for (int j = 0; j < own_max; j++) {
      const int q = 2 + me + j * (G - 1);
      const int r0 = q < nb ? blk(q) * TSB : 0, bsz = q < nb ? min(TSB, n - r0) : 0;
      for (int e = t; e < TSB * RHS; e += blockDim.x) {
        const int k = e / TSB, r = e % TSB;
        xo[((size_t)j * RHS + k) * TSB + r] = (k < kn && r < bsz) ? ld_x(k, r0 + r) : T{0, 0};
      }
    }
  }
  grid.sync();
  for (int s = 0; s + 1 < nb; s++) {
    const int c0 = blk(s) * TSB, csz = min(TSB, n - c0);
    if (lead) {
      const int nr0 = blk(s + 1) * TSB, nsz = min(TSB, n - nr0);
      for (int e = t; e < TSB * RHS; e += blockDim.x) {
        const int k = e / TSB, r = e % TSB;
        bsh[k][r] = (k < kn && r < nsz) ? ld_x(k, nr0 + r) : T{0, 0};
      }
      cp_async_wait_all();
      __syncthreads();
      lead_solve(nr0, nsz);
      __syncthreads();
      for (int e = t; e < TSB * RHS; e += blockDim.x) xs[e / TSB][e % TSB] = ysh[e / TSB][e % TSB];
      if (s + 2 < nb) {
        tile_async<T>(inv, blk(s + 2), tI);
        tile_async<T>(Mp, blk(s + 2), tM);
        cp_async_commit();
      }
    } else {
      for (int e = t; e < TSB * RHS; e += blockDim.x) {
        const int k = e / TSB, r = e % TSB;
        xs[k][r] = (k < kn && r < csz) ? ld_x(k, c0 + r) : T{0, 0};
      }
      __syncthreads();
      // 8 lanes per row, 4 rows per warp: x_s from shared memory, the next
      // owned tile loaded while this one is applied
      const int sub = lane >> 3, sl = lane & 7, row = warp * 4 + sub;
      T a[8], an[8];
      auto load8 = [&](int j, T(&dst)[8]) {
        const int r = blk(2 + me + j * (G - 1)) * TSB + row;
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const int c = sl + 8 * u;
          dst[u] = (r < n && c < csz) ? LU[(size_t)r * n + c0 + c] : T{0, 0};
        }
      };
      // complex128 tiles are not double-buffered: two would not fit in registers
      constexpr bool PF = sizeof(T) == sizeof(float2);
      const int j0 = first_slot(s);
      if (PF && live(j0)) load8(j0, a);
      for (int j = j0; live(j); j++) {
        const bool more = PF && live(j + 1);
        if (more) load8(j + 1, an);
        if (!PF) load8(j, a);
#pragma unroll
        for (int k = 0; k < RHS; k++) {
          if (k >= kn) break;
          C sr = 0, si = 0;
#pragma unroll
          for (int u = 0; u < 8; u++) {
            const T v = xs[k][sl + 8 * u];
            sr += a[u].x * v.x - a[u].y * v.y;
            si += a[u].x * v.y + a[u].y * v.x;
          }
#pragma unroll
          for (int o = 4; o > 0; o >>= 1) {
            sr += __shfl_xor_sync(0xffffffffu, sr, o);
            si += __shfl_xor_sync(0xffffffffu, si, o);
          }
          if (sl == 0) {
            T& d = xo[((size_t)j * RHS + k) * TSB + row];
            d.x -= sr;
            d.y -= si;
          }
        }
        if (more) {
#pragma unroll
          for (int u = 0; u < 8; u++) a[u] = an[u];
        }
      }
      // publish block s+2 if owned here
      const int qp = s + 2;
      if (qp < nb && (qp - 2) % (G - 1) == me) {
        __syncthreads();
        const int j = (qp - 2) / (G - 1), r0 = blk(qp) * TSB, bsz = min(TSB, n - r0);
        for (int e = t; e < TSB * RHS; e += blockDim.x) {
          const int k = e / TSB, r = e % TSB;
          if (k < kn && r < bsz) {
            const T v = xo[((size_t)j * RHS + k) * TSB + r];
            x[(size_t)k * n + r0 + r] = make_double2((double)v.x, (double)v.y);
          }
        }
      }
    }
    grid.sync();
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
int lu_trsv_prepare(const T* d_LU, int n, TrsvBlocks<T>& blk, cudaStream_t st, bool transposed) {
  const int nb = (n + TSB - 1) / TSB;
  const size_t need = (size_t)nb * TSB * TSB;
  if (blk.invL.count < need) {
    TT_TRY(blk.invL.alloc(need));
    TT_TRY(blk.invU.alloc(need));
    TT_TRY(blk.mL.alloc(need));
    TT_TRY(blk.mU.alloc(need));
  }
  blk.n = n;
  ProfScope prof(TT_PROF_SUBST_PREP, st, 0.0, 2.0 * (double)n * TSB * sizeof(T));
  const size_t smem = (size_t)TSB * TLD * sizeof(T);
  TT_TRY(smem_limit_once((const void*)k_inv_diag<T, false, true>, (int)(smem)));
  TT_TRY(smem_limit_once((const void*)k_inv_diag<T, true, false>, (int)(smem)));
  TT_TRY(smem_limit_once((const void*)k_inv_diag<T, false, false>, (int)(smem)));
  TT_TRY(smem_limit_once((const void*)k_inv_diag<T, true, true>, (int)(smem)));
  TT_TRY(smem_limit_once((const void*)k_prev_mul<T, false>, (int)(2 * smem)));
  TT_TRY(smem_limit_once((const void*)k_prev_mul<T, true>, (int)(2 * smem)));
  if (!transposed) {
    k_inv_diag<T, false, true><<<nb, 512, smem, st>>>(d_LU, n, blk.invL.ptr);
    count_launch();
    k_inv_diag<T, true, false><<<nb, 512, smem, st>>>(d_LU, n, blk.invU.ptr);
    count_launch();
  } else {
    k_inv_diag<T, false, false><<<nb, 512, smem, st>>>(d_LU, n, blk.invL.ptr);
    count_launch();
    k_inv_diag<T, true, true><<<nb, 512, smem, st>>>(d_LU, n, blk.invU.ptr);
    count_launch();
  }
  k_prev_mul<T, false><<<nb, 512, 2 * smem, st>>>(d_LU, n, blk.invL.ptr, blk.mL.ptr);
  count_launch();
  k_prev_mul<T, true><<<nb, 512, 2 * smem, st>>>(d_LU, n, blk.invU.ptr, blk.mU.ptr);
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}
template int lu_trsv_prepare<double2>(const double2*, int, TrsvBlocks<double2>&, cudaStream_t, bool);
template int lu_trsv_prepare<float2>(const float2*, int, TrsvBlocks<float2>&, cudaStream_t, bool);

// forward then backward substitution sweeps over x_b [k][n] in place for the
// B factors of a batch (one cooperative launch per sweep for all of them)
template <typename T>
int trsv_sweeps_batched(int B, const T* const* d_LU, int n, const TrsvBlocks<T>* const* blk, double2* const* x,
                        int nrhs, cudaStream_t st) {
  if (B < 1 || B > kMaxSweeps) {
    set_error("substitution batch of " + std::to_string(B) + " factors (1.." + std::to_string(kMaxSweeps) + ")");
    return TT_ERR_BADARG;
  }
  for (int b = 0; b < B; b++)
    if (blk[b]->n != n || !blk[b]->invL.ptr) {
      set_error("triangular solve called without the inverted diagonal blocks of this factor");
      return TT_ERR_BADARG;
    }
  const int Gb = std::max(2, device_sm_count() / B);
  const int nb = (n + TSB - 1) / TSB;
  int own_max = std::max(1, (nb - 2 + (Gb - 1) - 1) / (Gb - 1));
  const size_t smem = (size_t)2 * TSB * TLD * sizeof(T) + (size_t)own_max * RHS * TSB * sizeof(T);
  constexpr size_t kMaxSmem = 212 * 1024;  // + up to 12 KB static, within the 227 KB per CTA
  if (smem > kMaxSmem) {
    if (B > 1) {
      // fewer owners per factor would not hold their rows: one factor at a time
      for (int b = 0; b < B; b++) TT_TRY(trsv_sweeps_batched<T>(1, d_LU + b, n, blk + b, x + b, nrhs, st));
      return TT_OK;
    }
    set_error("triangular solve: n = " + std::to_string(n) + " needs " + std::to_string(smem) +
              " bytes of shared memory per CTA (limit " + std::to_string(kMaxSmem) + ")");
    return TT_ERR_UNSUPPORTED;
  }
  TT_TRY(smem_limit_once((const void*)k_trsv<T, false>, (int)kMaxSmem));
  TT_TRY(smem_limit_once((const void*)k_trsv<T, true>, (int)kMaxSmem));
  for (int k0 = 0; k0 < nrhs; k0 += RHS) {
    int kn = std::min(RHS, nrhs - k0);
    TrsvBatch<T> bl{}, bu{};
    bl.B = bu.B = B;
    for (int b = 0; b < B; b++) {
      bl.LU[b] = bu.LU[b] = d_LU[b];
      bl.inv[b] = blk[b]->invL.ptr;
      bu.inv[b] = blk[b]->invU.ptr;
      bl.Mp[b] = blk[b]->mL.ptr;
      bu.Mp[b] = blk[b]->mU.ptr;
      bl.x[b] = bu.x[b] = x[b] + (size_t)k0 * n;
    }
    int nn = n;
    void* argsL[] = {&bl, &nn, &kn, &own_max};
    TT_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_trsv<T, false>, dim3(Gb * B), dim3(TRSV_THREADS), argsL, smem,
                                            st));
    count_launch();
    void* argsU[] = {&bu, &nn, &kn, &own_max};
    TT_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_trsv<T, true>, dim3(Gb * B), dim3(TRSV_THREADS), argsU, smem,
                                            st));
    count_launch();
  }
  return TT_OK;
}

template <typename T>
int trsv_sweeps(const T* d_LU, int n, const TrsvBlocks<T>& blk, double2* x, int nrhs, cudaStream_t st) {
  const TrsvBlocks<T>* pb = &blk;
  return trsv_sweeps_batched<T>(1, &d_LU, n, &pb, &x, nrhs, st);
}

template <typename T>
int lu_solve_batched_device(int B, const T* const* d_LU, int n, const TrsvBlocks<T>* const* blk,
                            const int32_t* const* d_perm, double* const* d_x, double* d_tmp, int nrhs,
                            cudaStream_t st) {
  if (n <= 0 || nrhs <= 0 || B <= 0) return TT_OK;
  ProfScope prof(TT_PROF_TRSV, st, 8.0 * n * (double)n * nrhs * B, (double)n * n * sizeof(T) * B);
  double2* xs[kMaxSweeps];
  for (int b = 0; b < B; b++) {
    TT_CUDA_TRY(cudaMemcpyAsync(d_tmp, d_x[b], sizeof(double2) * (size_t)n * nrhs, cudaMemcpyDeviceToDevice, st));
    xs[b] = reinterpret_cast<double2*>(d_x[b]);
    k_permute<<<ceil_div((size_t)n * nrhs, 256), 256, 0, st>>>(reinterpret_cast<const double2*>(d_tmp), d_perm[b],
                                                              n, nrhs, xs[b]);
    count_launch();
    TT_CUDA_TRY(cudaGetLastError());
  }
  return trsv_sweeps_batched<T>(B, d_LU, n, blk, xs, nrhs, st);
}
template int lu_solve_batched_device<float2>(int, const float2* const*, int, const TrsvBlocks<float2>* const*,
                                             const int32_t* const*, double* const*, double*, int, cudaStream_t);

template <typename T>
int lu_solve_device(const T* d_LU, int n, const TrsvBlocks<T>& blk, const int32_t* d_perm, double* d_x,
                    double* d_tmp, int nrhs, cudaStream_t st) {
  if (n <= 0 || nrhs <= 0) return TT_OK;
  ProfScope prof(TT_PROF_TRSV, st, 8.0 * n * (double)n * nrhs, (double)n * n * sizeof(T));
  TT_CUDA_TRY(cudaMemcpyAsync(d_tmp, d_x, sizeof(double2) * (size_t)n * nrhs, cudaMemcpyDeviceToDevice, st));
  double2* x = reinterpret_cast<double2*>(d_x);
  k_permute<<<ceil_div((size_t)n * nrhs, 256), 256, 0, st>>>(reinterpret_cast<const double2*>(d_tmp), d_perm, n,
                                                            nrhs, x);
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return trsv_sweeps<T>(d_LU, n, blk, x, nrhs, st);
}

template <typename T>
int lu_solve_transposed_device(const T* d_LUt, int n, const TrsvBlocks<T>& blkT, const int32_t* d_perm, double* d_x,
                               double* d_tmp, int nrhs, cudaStream_t st) {
  if (n <= 0 || nrhs <= 0) return TT_OK;
  ProfScope prof(TT_PROF_TRSV, st, 8.0 * n * (double)n * nrhs, (double)n * n * sizeof(T));
  double2* x = reinterpret_cast<double2*>(d_x);
  TT_TRY(trsv_sweeps<T>(d_LUt, n, blkT, x, nrhs, st));
  TT_CUDA_TRY(cudaMemcpyAsync(d_tmp, d_x, sizeof(double2) * (size_t)n * nrhs, cudaMemcpyDeviceToDevice, st));
  k_permute_inv<<<ceil_div((size_t)n * nrhs, 256), 256, 0, st>>>(reinterpret_cast<const double2*>(d_tmp), d_perm, n,
                                                                nrhs, x);
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}
template int lu_solve_transposed_device<double2>(const double2*, int, const TrsvBlocks<double2>&, const int32_t*,
                                                 double*, double*, int, cudaStream_t);
template int lu_solve_transposed_device<float2>(const float2*, int, const TrsvBlocks<float2>&, const int32_t*,
                                                double*, double*, int, cudaStream_t);
template int lu_solve_device<double2>(const double2*, int, const TrsvBlocks<double2>&, const int32_t*, double*,
                                      double*, int, cudaStream_t);
template int lu_solve_device<float2>(const float2*, int, const TrsvBlocks<float2>&, const int32_t*, double*,
                                     double*, int, cudaStream_t);

}  // namespace tt
