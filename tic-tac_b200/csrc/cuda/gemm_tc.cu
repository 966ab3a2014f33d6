// Tensor-core trailing update of the complex64 LU on sm_100a:
//
//   C[M x N] -= L[M x K] U[K x N]     (complex, C row-major complex64 in place)
//
// Each complex factor is split into bf16 hi/lo parts (x = hi + lo), and the
// product is accumulated in FP32 in tensor memory as
//   Re += Lr.Ur - Li.Ui ,  Im += Lr.Ui + Li.Ur
// with every real product taken as hi.hi + hi.lo + lo.hi (BF16x3), i.e. 12
// tcgen05.mma (kind::f16, M=128, N=128, K=16) per 16-deep k step; the
// negative terms use the instruction descriptor's negate-A bit.
//
// Kernel organisation (one CTA per SM, persistent over 128 x 128 output tiles):
//   warp 0      TMA producer: cp.async.bulk.tensor loads of the bf16 parts of
//               L (4 x 8 KB) and U^T (4 x 8 KB) per 32-deep k chunk into a
//               3-stage ring of 64B-swizzled shared memory
//   warp 1      MMA issuer (one elected thread), accumulators double-buffered
//               in TMEM (2 x (128 Re + 128 Im) columns = all 512)
//   warps 2..9  epilogue: tcgen05.ld of a 32-row x 16-column accumulator
//               slice, staged through swizzled shared memory, then a
//               coalesced C -= acc read-modify-write
// Every mbarrier wait is bounded in time; on expiry the kernel records an
// error code, drains its own copies in flight, frees TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>

#include "tt_kernels.h"
#include "tt_lu_internal.h"

namespace tt {
namespace tc {

constexpr int BM = 128;           // rows per tile (MMA M)
constexpr int BN = 128;           // complex columns per tile (MMA N)
constexpr int KC = 32;            // k elements per chunk (64 B of bf16 = one swizzle row)
constexpr int STAGES = 3;
constexpr int A_PART_BYTES = BM * KC * 2;  // 8 KB
constexpr int B_PART_BYTES = BN * KC * 2;  // 8 KB
constexpr int STAGE_BYTES = 4 * A_PART_BYTES + 4 * B_PART_BYTES;  // 64 KB
constexpr int TMEM_COLS = 512;    // 2 accumulators x (BN re + BN im)
constexpr int EPI_WARPS = 8;
constexpr int NUM_THREADS = 64 + 32 * EPI_WARPS;  // producer, MMA, epilogue
constexpr int EPI_STAGE_BYTES = 32 * 16 * 8;      // 32 rows x 16 complex per epilogue warp
constexpr uint64_t WAIT_NS = 2000000000ull;  // 2 s bound on any single wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: false if the phase did not complete within WAIT_NS or another
// role of this launch already reported an error.
__device__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, int code) {
  const uint64_t t0 = now_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (*(volatile int*)err != 0) return false;
    if (now_ns() - t0 > WAIT_NS) {
      atomicCAS(err, 0, code);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::
          "r"(smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// K-major, 64B-swizzled operand: rows of 64 B, 8-row atoms 512 B apart.
__device__ __forceinline__ uint64_t sw64_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);  // start address
  d |= (uint64_t)1 << 16;                    // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(512 >> 4) << 32;           // stride byte offset: next 8-row atom
  d |= (uint64_t)1 << 46;                    // descriptor version for tcgen05
  d |= (uint64_t)4 << 61;                    // SWIZZLE_64B
  return d;
}

// kind::f16 instruction descriptor: D f32, A/B bf16, K-major, M=128, N=128.
__host__ __device__ constexpr uint32_t idesc_bf16(bool negA) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((negA ? 1u : 0u) << 13) | ((uint32_t)(BN >> 3) << 17) |
         ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                     uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

struct TileSched {
  int tiles_m, tiles_n, group;
  __device__ void coords(int t, int& tm, int& tn) const {
    // bands of `group` row tiles swept across all column tiles (keeps a
    // band of L rows and the current U^T columns resident in L2)
    const int per_group = group * tiles_n;
    const int g = t / per_group;
    const int first_m = g * group;
    const int gm = min(group, tiles_m - first_m);
    const int r = t % per_group;
    tm = first_m + r % gm;
    tn = r / gm;
  }
};

// K = 64 * kchunks complex depth.  WA: [M][4K] bf16 (parts re_hi, re_lo,
// im_hi, im_lo of L), WB: [N][4K] bf16 (same parts of U, transposed).
__global__ void __launch_bounds__(NUM_THREADS, 1)
    k_lu_update_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, float2* __restrict__ C,
                   int ldc, int M, int N, int K, int* err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  float2* epi_stage = (float2*)(smem + STAGES * STAGE_BYTES);
  uint64_t* full = (uint64_t*)(smem + STAGES * STAGE_BYTES + EPI_WARPS * EPI_STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* acc_full = empty + STAGES;
  uint64_t* acc_empty = acc_full + 2;
  uint32_t* tmem_base_slot = (uint32_t*)(acc_empty + 2);

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int kchunks = K / KC;
  TileSched sched{(M + BM - 1) / BM, (N + BN - 1) / BN, 16};
  const int ntiles = sched.tiles_m * sched.tiles_n;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], EPI_WARPS);  // one arrival per epilogue warp
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_base_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_base_slot;

  if (warp == 0) {
    // ---------------- TMA producer
    if (lane == 0) {
      int it = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        int tm, tn;
        sched.coords(t, tm, tn);
        for (int kc = 0; kc < kchunks && ok; kc++, it++) {
          const int s = it % STAGES;
          const uint32_t ph = (uint32_t)(it / STAGES) & 1u;
          if (it >= STAGES && !mbar_wait(&empty[s], ph ^ 1u, err, 1)) {
            ok = false;
            break;
          }
          unsigned char* st = smem + s * STAGE_BYTES;
          mbar_expect_tx(&full[s], STAGE_BYTES);
#pragma unroll
          for (int p = 0; p < 4; p++) tma_load_2d(st + p * A_PART_BYTES, &tmA, &full[s], p * K + kc * KC, tm * BM);
#pragma unroll
          for (int p = 0; p < 4; p++)
            tma_load_2d(st + 4 * A_PART_BYTES + p * B_PART_BYTES, &tmB, &full[s], p * K + kc * KC, tn * BN);
        }
      }
      // drain: wait (bounded) until every issued load has landed before exit
      for (int j = (it > STAGES ? it - STAGES : 0); j < it; j++)
        mbar_wait(&full[j % STAGES], (uint32_t)(j / STAGES) & 1u, err, 5);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer
    if (lane == 0) {
      // term table: (A part, B part, negate) for Re then Im
      const int ta[12] = {0, 0, 1, 2, 2, 3, 0, 0, 1, 2, 2, 3};
      const int tb[12] = {0, 1, 0, 2, 3, 2, 2, 3, 2, 0, 1, 0};
      const uint32_t id_pos = idesc_bf16(false), id_neg = idesc_bf16(true);
      int it = 0, local = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, local++) {
        const int ab = local & 1;
        const uint32_t aph = (uint32_t)(local >> 1) & 1u;
        if (local >= 2 && !mbar_wait(&acc_empty[ab], aph ^ 1u, err, 2)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d_re = tmem_base + ab * (2 * BN);
        const uint32_t d_im = d_re + BN;
        for (int kc = 0; kc < kchunks; kc++, it++) {
          const int s = it % STAGES;
          const uint32_t ph = (uint32_t)(it / STAGES) & 1u;
          if (!mbar_wait(&full[s], ph, err, 3)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a0 = smem_u32(smem + s * STAGE_BYTES);
          const uint32_t b0 = a0 + 4 * A_PART_BYTES;
#pragma unroll
          for (int ks = 0; ks < KC / 16; ks++) {
#pragma unroll
            for (int q = 0; q < 12; q++) {
              const uint64_t ad = sw64_desc(a0 + ta[q] * A_PART_BYTES + ks * 32);
              const uint64_t bd = sw64_desc(b0 + tb[q] * B_PART_BYTES + ks * 32);
              const bool first = (kc == 0 && ks == 0 && (q == 0 || q == 6));
              const bool neg = (q >= 3 && q < 6);
              umma(q < 6 ? d_re : d_im, ad, bd, neg ? id_neg : id_pos, first ? 0u : 1u);
            }
          }
          umma_commit(&empty[s]);  // stage reusable once these MMAs completed
        }
        if (!ok) break;
        umma_commit(&acc_full[ab]);
      }
    }
  } else {
    // ---------------- epilogue (warps 2..9): warp w reads TMEM lane quarter
    // w % 4 (the hardware lane-access rule) and column half (w - 2) / 4
    const int quarter = warp & 3;
    const int half = (warp - 2) >> 2;
    float2* stage = epi_stage + (size_t)(warp - 2) * (32 * 16);
    int local = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, local++) {
      int tm, tn;
      sched.coords(t, tm, tn);
      const int ab = local & 1;
      const uint32_t aph = (uint32_t)(local >> 1) & 1u;
      if (!mbar_wait(&acc_full[ab], aph, err, 4)) break;
      tc_fence_after();
      const uint32_t lane_addr = tmem_base + ((uint32_t)(quarter * 32) << 16) + ab * (2 * BN);
      const int row0 = tm * BM + quarter * 32;
#pragma unroll 1
      for (int cc = 0; cc < BN / 2; cc += 16) {
        const int col = half * (BN / 2) + cc;
        float re[16], im[16];
        tmem_ld16(lane_addr + col, re);
        tmem_ld16(lane_addr + BN + col, im);
        // stage this thread's row (row = lane) with an XOR swizzle on the column
#pragma unroll
        for (int j = 0; j < 16; j++) stage[lane * 16 + (j ^ (lane & 15))] = make_float2(re[j], im[j]);
        __syncwarp();
        // coalesced read-modify-write: two rows of 16 complex per instruction
        const int gcol0 = tn * BN + col;
        float2 cv[16];
#pragma unroll
        for (int i = 0; i < 16; i++) {
          const int idx = i * 32 + lane, r = idx >> 4, c = idx & 15;
          const int grow = row0 + r, gcol = gcol0 + c;
          cv[i] = (grow < M && gcol < N) ? C[(size_t)grow * ldc + gcol] : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int i = 0; i < 16; i++) {
          const int idx = i * 32 + lane, r = idx >> 4, c = idx & 15;
          const int grow = row0 + r, gcol = gcol0 + c;
          const float2 a = stage[r * 16 + (c ^ (r & 15))];
          if (grow < M && gcol < N) C[(size_t)grow * ldc + gcol] = make_float2(cv[i].x - a.x, cv[i].y - a.y);
        }
        __syncwarp();
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[ab]);
    }
  }
  __syncwarp();
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS));
  }
}

// Split of the trailing-update factors into bf16 hi/lo parts.
//   WA[i][p*K + kk] from L[i][kk] (rows i of the panel below the diagonal block)
//   WB[j][p*K + kk] from U[kk][j] (transposed)
__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

__global__ void k_split_L(const float2* __restrict__ A, int lda, int M, int K, __nv_bfloat16* __restrict__ WA) {
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (size_t)M * K) return;
  const int i = (int)(tid / K), kk = (int)(tid % K);
  const float2 v = A[(size_t)i * lda + kk];
  __nv_bfloat16 h, l;
  __nv_bfloat16* w = WA + (size_t)i * 4 * K + kk;
  split_bf16(v.x, h, l);
  w[0] = h;
  w[K] = l;
  split_bf16(v.y, h, l);
  w[2 * K] = h;
  w[3 * K] = l;
}

__global__ void k_split_U(const float2* __restrict__ A, int lda, int K, int N, __nv_bfloat16* __restrict__ WB) {
  __shared__ float2 tile[32][33];
  const int j0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;  // 32 x 8
  for (int r = ty; r < 32; r += 8) {
    const int kk = k0 + r, j = j0 + tx;
    float2 v = make_float2(0.f, 0.f);
    if (kk < K && j < N) v = A[(size_t)kk * lda + j];
    tile[r][tx] = v;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int j = j0 + r, kk = k0 + tx;
    if (j < N && kk < K) {
      const float2 v = tile[tx][r];
      __nv_bfloat16 h, l;
      __nv_bfloat16* w = WB + (size_t)j * 4 * K + kk;
      split_bf16(v.x, h, l);
      w[0] = h;
      w[K] = l;
      split_bf16(v.y, h, l);
      w[2 * K] = h;
      w[3 * K] = l;
    }
  }
}

}  // namespace tc

namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

// 2D bf16 tensor [rows][cols] row-major, box = 32 cols (64 B) x box_rows, 64B swizzle.
int make_map(CUtensorMap* map, void* base, uint64_t rows, uint64_t cols, uint32_t box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) {
    set_error("cuTensorMapEncodeTiled is not available from the driver");
    return TT_ERR_CUDA;
  }
  const cuuint64_t dims[2] = {cols, rows};
  const cuuint64_t strides[1] = {cols * 2};
  const cuuint32_t box[2] = {tc::KC, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed with code " + std::to_string((int)r));
    return TT_ERR_CUDA;
  }
  return TT_OK;
}

struct TCWorkspace {
  DevBuf<__nv_bfloat16> WA, WB;
  DevBuf<int> err;
  size_t capA = 0, capB = 0;
};

TCWorkspace& workspace() {
  static thread_local TCWorkspace ws;
  return ws;
}

}  // namespace

int tc_gemm_sub(float2* C, int ldc, const float2* L, int ldl, const float2* U, int ldu, int M, int N, int K,
                cudaStream_t st) {
  if (M <= 0 || N <= 0 || K <= 0) return TT_OK;
  if (K % tc::KC != 0) {
    set_error("tensor-core update needs K to be a multiple of 32");
    return TT_ERR_BADARG;
  }
  TCWorkspace& ws = workspace();
  const size_t needA = (size_t)M * 4 * K, needB = (size_t)N * 4 * K;
  if (needA > ws.capA) {
    TT_TRY(ws.WA.alloc(needA));
    ws.capA = needA;
  }
  if (needB > ws.capB) {
    TT_TRY(ws.WB.alloc(needB));
    ws.capB = needB;
  }
  if (!ws.err.ptr) {
    TT_TRY(ws.err.alloc(1));
    TT_CUDA_TRY(cudaMemsetAsync(ws.err.ptr, 0, sizeof(int), st));
  }
  {
    ProfScope prof(TT_PROF_OPERANDS, st, 0.0, 16.0 * ((double)M + N) * K);
    tc::k_split_L<<<ceil_div((size_t)M * K, 256), 256, 0, st>>>(L, ldl, M, K, ws.WA.ptr);
    count_launch();
    TT_CUDA_TRY(cudaGetLastError());
    dim3 gs(ceil_div(N, 32), ceil_div(K, 32));
    tc::k_split_U<<<gs, 256, 0, st>>>(U, ldu, K, N, ws.WB.ptr);
    count_launch();
    TT_CUDA_TRY(cudaGetLastError());
  }
  CUtensorMap mA, mB;
  TT_TRY(make_map(&mA, ws.WA.ptr, (uint64_t)M, (uint64_t)4 * K, tc::BM));
  TT_TRY(make_map(&mB, ws.WB.ptr, (uint64_t)N, (uint64_t)4 * K, tc::BN));
  const size_t smem = (size_t)tc::STAGES * tc::STAGE_BYTES + tc::EPI_WARPS * tc::EPI_STAGE_BYTES + 1024 + 128;
  TT_TRY(smem_limit_once((const void*)tc::k_lu_update_tc, (int)smem));
  const int tiles = ((M + tc::BM - 1) / tc::BM) * ((N + tc::BN - 1) / tc::BN);
  const int grid = std::min(tiles, device_sm_count());
  {
    ProfScope prof(K >= 256 ? TT_PROF_TC_UPDATE : TT_PROF_TC_PANEL, st, 8.0 * M * N * K,
                   16.0 * M * N + 8.0 * ((double)M + N) * K);
    tc::k_lu_update_tc<<<grid, tc::NUM_THREADS, smem, st>>>(mA, mB, C, ldc, M, N, K, ws.err.ptr);
  }
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

int tc_check_error(cudaStream_t st) {
  TCWorkspace& ws = workspace();
  if (!ws.err.ptr) return TT_OK;
  int h = 0;
  TT_CUDA_TRY(cudaMemcpyAsync(&h, ws.err.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
  TT_CUDA_TRY(cudaStreamSynchronize(st));
  if (h != 0) {
    TT_CUDA_TRY(cudaMemsetAsync(ws.err.ptr, 0, sizeof(int), st));
    set_error("tensor-core update timed out waiting on a pipeline barrier (code " + std::to_string(h) + ")");
    return TT_ERR_CUDA;
  }
  return TT_OK;
}

int lu_update_tc(float2* A, int n, int k, int nb, cudaStream_t st) {
  const int r0 = k + nb;
  const int m = n - r0;
  if (m <= 0) return TT_OK;
  return tc_gemm_sub(A + (size_t)r0 * n + r0, n, A + (size_t)r0 * n + k, n, A + (size_t)k * n + r0, n, m, m, nb, st);
}

}  // namespace tt
