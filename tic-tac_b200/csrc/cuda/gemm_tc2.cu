// Tensor-core trailing update of the complex64 LU on sm_100a, real-row form:
//
//   C[M x N] -= L[M x K] U[K x N]     (complex, C row-major complex64 in place)
//
// A complex row of L, read as 2K reals [Lr0, Li0, Lr1, Li1, ...], times the two
// real rows that column j of U gives,
//   re-row j: [Ur0j, -Ui0j, Ur1j, -Ui1j, ...]   im-row j: [Ui0j, Ur0j, Ui1j, Ur1j, ...]
// is Re(LU)_ij and Im(LU)_ij.  So one real product of depth 2K with N = 256
// B rows (128 re-rows, then the 128 im-rows of the same columns) produces a
// 128 x 128 complex tile in one tcgen05.mma per k step, the re and im halves
// of the accumulator landing in TMEM columns [0,128) and [128,256).  Against
// four separate real products this reads each L tile from shared memory once
// per k step instead of twice.
//
// Two operand precisions:
//   TF32    one kind::tf32 product (K = 8 per instruction); L is read by TMA
//           straight from the matrix (the tensor core uses the top 19 bits of
//           each fp32), U's rows are packed rounded to tf32 (cvt.rna)
//   BF16X3  x = hi + lo in bf16, hi.hi + hi.lo + lo.hi (kind::f16, K = 16);
//           L and U rows packed into hi/lo planes
// Accumulation in FP32 in TMEM, double-buffered (2 x 256 columns).
//
// Kernel organisation (one CTA per SM, persistent over 128 x 128 tiles):
//   warp 0      TMA producer into a 4-stage ring (16 complex k per stage)
//   warp 1      MMA issuer (one elected thread)
//   warps 2..9  epilogue: C of the tile's first column chunk is loaded while
//               the accumulator fills; per 16-column chunk the C loads are
//               issued before the tcgen05.ld of the accumulator slice, then a
//               coalesced C -= acc store
// Every mbarrier wait is bounded in time; on expiry the kernel records an
// error code, drains its own copies in flight, frees TMEM and returns.
// Every TMA copy here lands in the shared memory of the CTA that issues it.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>
#include <cstring>

#include "tc2_pack.cuh"
#include "tt_kernels.h"
#include "tt_lu_internal.h"

namespace tt {
namespace tc2 {

constexpr int BM = 128;         // rows per tile (MMA M)
constexpr int BN = 128;         // complex columns per tile (MMA N = 2 BN real rows of B)
constexpr int KCC = 16;         // complex k per stage = 32 real k
constexpr int STAGES = 4;
constexpr int TMEM_COLS = 512;  // 2 accumulators x (BN re + BN im)
constexpr int EPI_WARPS = 8;
constexpr int NUM_THREADS = 64 + 32 * EPI_WARPS;
constexpr int EPI_STAGE_BYTES = 32 * 16 * 8;
constexpr uint64_t WAIT_NS = 2000000000ull;

// Per-mode layout of one stage.  TF32: 32 real k in fp32 = 128 B rows,
// SWIZZLE_128B.  BF16X3: 32 real k in bf16 = 64 B rows, SWIZZLE_64B, hi and lo
// planes.  Every tile below is a multiple of 1 KB, so 1 KB alignment holds.
template <int MODE>
struct Cfg;
template <>
struct Cfg<TC_TF32> {
  static constexpr int ROW_BYTES = 128;
  static constexpr int PARTS = 1;
  static constexpr int A_TILE = BM * ROW_BYTES;            // 16 KB
  static constexpr int B_TILE = 2 * BN * ROW_BYTES;        // 32 KB (re-rows then im-rows)
  static constexpr int STAGE = PARTS * (A_TILE + B_TILE);  // 48 KB
  static constexpr int KSTEPS = 4;                         // k8 steps of 32 B per stage
  static constexpr int TERMS = 1;
  static constexpr uint32_t SBO = 1024;                    // 8-row swizzle atom
  static constexpr uint64_t LAYOUT = 2;                    // SWIZZLE_128B
};
template <>
struct Cfg<TC_BF16X3> {
  static constexpr int ROW_BYTES = 64;
  static constexpr int PARTS = 2;
  static constexpr int A_TILE = BM * ROW_BYTES;            // 8 KB per part
  static constexpr int B_TILE = 2 * BN * ROW_BYTES;        // 16 KB per part
  static constexpr int STAGE = PARTS * (A_TILE + B_TILE);  // 48 KB
  static constexpr int KSTEPS = 2;                         // k16 steps of 32 B per stage
  static constexpr int TERMS = 3;                          // hi.hi, hi.lo, lo.hi
  static constexpr uint32_t SBO = 512;
  static constexpr uint64_t LAYOUT = 4;                    // SWIZZLE_64B
};

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
// try_wait with a suspend-time hint: the waiting thread sleeps until the phase
// completes or about SUSPEND_NS pass, instead of spinning on issue slots that
// the MMA-issuing warp shares
constexpr uint32_t SUSPEND_NS = 20000;
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(SUSPEND_NS)
      : "memory");
  return ok != 0;
}
// Bounded wait: false if the phase did not complete within WAIT_NS or another
// role of this launch already reported an error.
__device__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, int code) {
  if (mbar_try_wait(bar, parity)) return true;
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

// K-major swizzled operand descriptor (tcgen05 shared-memory matrix descriptor).
template <int MODE>
__device__ __forceinline__ uint64_t op_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);    // start address
  d |= (uint64_t)1 << 16;                      // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(Cfg<MODE>::SBO >> 4) << 32;  // stride byte offset: next 8-row atom
  d |= (uint64_t)1 << 46;                      // descriptor version for tcgen05
  d |= Cfg<MODE>::LAYOUT << 61;
  return d;
}

// Instruction descriptor: D f32, A/B tf32 (2) or bf16 (1), K-major, M = 128, N = 256.
template <int MODE>
__host__ __device__ constexpr uint32_t idesc() {
  constexpr uint32_t ab = (MODE == TC_TF32) ? 2u : 1u;
  return (1u << 4) | (ab << 7) | (ab << 10) | ((uint32_t)((2 * BN) >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

template <int MODE>
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  const uint32_t z = 0;
  constexpr uint32_t id = idesc<MODE>();
  if constexpr (MODE == TC_TF32) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(id), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(id), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
  }
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
    // bands of `group` row tiles swept across all column tiles (keeps a band
    // of L rows and the current U columns resident in L2)
    const int per_group = group * tiles_n;
    const int g = t / per_group;
    const int first_m = g * group;
    const int gm = min(group, tiles_m - first_m);
    const int r = t % per_group;
    tm = first_m + r % gm;
    tn = r / gm;
  }
};

// C loads of one 16-column chunk of a 32-row slice: cv[i] = C[row0 + r][gcol0 + c], idx = i*32 + lane.
__device__ __forceinline__ void load_c_chunk(const float2* __restrict__ C, int ldc, int M, int N, int row0, int gcol0,
                                             int lane, float2 (&cv)[16]) {
#pragma unroll
  for (int i = 0; i < 16; i++) {
    const int idx = i * 32 + lane, r = idx >> 4, c = idx & 15;
    const int grow = row0 + r, gcol = gcol0 + c;
    cv[i] = (grow < M && gcol < N) ? __ldcs(&C[(size_t)grow * ldc + gcol]) : make_float2(0.f, 0.f);
  }
}

// Up to kBatch products of the same shape in one launch: matrix b's L is read
// through A[b], its U planes are rows [b PARTS 2N, (b + 1) PARTS 2N) of the B
// operand, its output is C[b]; the tiles of all of them share the persistent
// grid (tile t of matrix t / tiles-per-matrix).
constexpr int kBatch = 4;
struct Ops {
  CUtensorMap A[kBatch];
  float2* C[kBatch];
  int nb;
};

// tmA: L as [rows][2K] reals (TF32: the matrix itself or a packed copy; BF16X3:
// hi plane rows [0, M), lo plane rows [a_plane, a_plane + M)).  tmB: U as
// [2N][2K] reals per plane (re-rows [0, N), im-rows [N, 2N); BF16X3: lo plane
// at row offset 2N).  K complex depth, a multiple of KCC.
template <int MODE>
__global__ void __launch_bounds__(NUM_THREADS, 1)
    k_lu_update_tc2(const __grid_constant__ Ops ops, const __grid_constant__ CUtensorMap tmB, int ldc, int M, int N,
                    int K, int a_plane, int store, int* err) {
  using CF = Cfg<MODE>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  float2* epi_stage = (float2*)(smem + STAGES * CF::STAGE);
  uint64_t* full = (uint64_t*)(smem + STAGES * CF::STAGE + EPI_WARPS * EPI_STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* acc_full = empty + STAGES;
  uint64_t* acc_empty = acc_full + 2;
  uint32_t* tmem_base_slot = (uint32_t*)(acc_empty + 2);

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int kchunks = K / KCC;
  TileSched sched{(M + BM - 1) / BM, (N + BN - 1) / BN, 16};
  const int per = sched.tiles_m * sched.tiles_n, ntiles = per * ops.nb;

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
        const int mb = t / per;
        sched.coords(t - mb * per, tm, tn);
        const int brow = mb * CF::PARTS * 2 * N;
        for (int kc = 0; kc < kchunks && ok; kc++, it++) {
          const int s = it % STAGES;
          const uint32_t ph = (uint32_t)(it / STAGES) & 1u;
          if (it >= STAGES && !mbar_wait(&empty[s], ph ^ 1u, err, 1)) {
            ok = false;
            break;
          }
          unsigned char* st = smem + s * CF::STAGE;
          mbar_expect_tx(&full[s], CF::STAGE);
          const int x = kc * 2 * KCC;  // real k offset: 32 reals per stage
#pragma unroll
          for (int p = 0; p < CF::PARTS; p++) {
            unsigned char* a = st + p * (CF::A_TILE + CF::B_TILE);
            tma_load_2d(a, &ops.A[mb], &full[s], x, p * a_plane + tm * BM);
            tma_load_2d(a + CF::A_TILE, &tmB, &full[s], x, brow + p * 2 * N + tn * BN);
            tma_load_2d(a + CF::A_TILE + CF::B_TILE / 2, &tmB, &full[s], x, brow + p * 2 * N + N + tn * BN);
          }
        }
      }
      // drain: wait (bounded) until every issued load has landed before exit
      for (int j = (it > STAGES ? it - STAGES : 0); j < it; j++)
        mbar_wait(&full[j % STAGES], (uint32_t)(j / STAGES) & 1u, err, 5);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer
    if (lane == 0) {
      // BF16X3 terms (A plane, B plane): hi.hi, hi.lo, lo.hi
      const int ta[3] = {0, 0, 1};
      const int tb[3] = {0, 1, 0};
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
        const uint32_t d = tmem_base + ab * (2 * BN);
        for (int kc = 0; kc < kchunks; kc++, it++) {
          const int s = it % STAGES;
          const uint32_t ph = (uint32_t)(it / STAGES) & 1u;
          if (!mbar_wait(&full[s], ph, err, 3)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t s0 = smem_u32(smem + s * CF::STAGE);
#pragma unroll
          for (int ks = 0; ks < CF::KSTEPS; ks++) {
#pragma unroll
            for (int q = 0; q < CF::TERMS; q++) {
              const uint32_t a0 = s0 + ta[q] * (CF::A_TILE + CF::B_TILE);
              const uint32_t b0 = s0 + tb[q] * (CF::A_TILE + CF::B_TILE) + CF::A_TILE;
              const uint64_t ad = op_desc<MODE>(a0 + ks * 32);
              const uint64_t bd = op_desc<MODE>(b0 + ks * 32);
              umma<MODE>(d, ad, bd, (kc == 0 && ks == 0 && q == 0) ? 0u : 1u);
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
      const int mb = t / per;
      sched.coords(t - mb * per, tm, tn);
      float2* __restrict__ C = ops.C[mb];
      const int ab = local & 1;
      const uint32_t aph = (uint32_t)(local >> 1) & 1u;
      const int row0 = tm * BM + quarter * 32;
      float2 cv[16];
      // the first chunk's C is fetched while the accumulator fills (store: C = acc, nothing to fetch)
      if (!store) load_c_chunk(C, ldc, M, N, row0, tn * BN + half * (BN / 2), lane, cv);
      if (!mbar_wait(&acc_full[ab], aph, err, 4)) break;
      tc_fence_after();
      const uint32_t lane_addr = tmem_base + ((uint32_t)(quarter * 32) << 16) + ab * (2 * BN);
#pragma unroll 1
      for (int cc = 0; cc < BN / 2; cc += 16) {
        const int col = half * (BN / 2) + cc;
        const int gcol0 = tn * BN + col;
        if (cc > 0 && !store) load_c_chunk(C, ldc, M, N, row0, gcol0, lane, cv);
        float re[16], im[16];
        tmem_ld16(lane_addr + col, re);
        tmem_ld16(lane_addr + BN + col, im);
        // stage this thread's row (row = lane) with an XOR swizzle on the column
#pragma unroll
        for (int j = 0; j < 16; j++) stage[lane * 16 + (j ^ (lane & 15))] = make_float2(re[j], im[j]);
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 16; i++) {
          const int idx = i * 32 + lane, r = idx >> 4, c = idx & 15;
          const int grow = row0 + r, gcol = gcol0 + c;
          const float2 a = stage[r * 16 + (c ^ (r & 15))];
          if (grow < M && gcol < N)
            C[(size_t)grow * ldc + gcol] = store ? a : make_float2(cv[i].x - a.x, cv[i].y - a.y);
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

// ---- CTA pairs (cta_group::2)
//
// Two CTAs of a cluster compute a 256 x 128 complex tile: each holds its 128
// L rows (A) and one half of the 256 real B rows, the first CTA the re-rows and
// the second the im-rows, and the first CTA issues one M = 256, N = 256 MMA per
// k step that reads both halves of A and of B from the two shared memories; the
// accumulator rows of each CTA land in its own TMEM (re in columns [0,128), im
// in [128,256), as in the single-CTA kernel).  Per CTA a stage is a 128-row A
// tile and 128 B rows, a third less operand traffic per flop than the single
// CTA's 128 + 256 rows, and five stages fit instead of four.
//
// Barriers: both CTAs' copies of a stage complete on the first CTA's full[s]
// (expect_tx of both CTAs' bytes there); the MMA's commit arrives on empty[s]
// of both CTAs; acc_full is committed to both; each CTA's epilogue warps arrive
// on the first CTA's acc_empty.  Each copy lands in its issuing CTA only.
template <int MODE>
struct PairCfg {
  static constexpr int A_TILE = Cfg<MODE>::A_TILE;            // 128 rows
  static constexpr int B_CTA = Cfg<MODE>::B_TILE / 2;         // 128 of the 256 real B rows
  static constexpr int PART = A_TILE + B_CTA;
  static constexpr int STAGE = Cfg<MODE>::PARTS * PART;       // 32 KB
  static constexpr int STAGES = 5;
};

template <int MODE>
__host__ __device__ constexpr uint32_t idesc_pair() {
  constexpr uint32_t ab = (MODE == TC_TF32) ? 2u : 1u;
  return (1u << 4) | (ab << 7) | (ab << 10) | ((uint32_t)((2 * BN) >> 3) << 17) | ((uint32_t)((2 * BM) >> 4) << 24);
}

template <int MODE>
__device__ __forceinline__ void umma_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  const uint32_t z = 0;
  constexpr uint32_t id = idesc_pair<MODE>();
  if constexpr (MODE == TC_TF32) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8, %9, %10, %11, %12}, p;\n\t}" ::"r"(
            tmem_d),
        "l"(adesc), "l"(bdesc), "r"(id), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z), "r"(z), "r"(z), "r"(z),
        "r"(z));
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8, %9, %10, %11, %12}, p;\n\t}" ::"r"(
            tmem_d),
        "l"(adesc), "l"(bdesc), "r"(id), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z), "r"(z), "r"(z), "r"(z),
        "r"(z));
  }
}
// commit of the pair's MMAs: one arrival on the barrier at this offset in both CTAs
__device__ __forceinline__ void umma_commit_pair(uint64_t* bar) {
  const uint16_t both = 3;
  asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::
                   "r"(smem_u32(bar)),
               "h"(both)
               : "memory");
}
// shared::cluster address of this CTA's variable at `p` in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t cluster_addr(const void* p, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
  return r;
}
__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_bar) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_bar) : "memory");
}
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// 2D tile copy into this CTA's shared memory completing on an mbarrier of the
// pair's first CTA (cluster address); one destination CTA
__device__ __forceinline__ void tma_load_2d_pair(void* dst, const CUtensorMap* map, uint32_t cluster_bar, int x,
                                                 int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], "
      "[%2];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(cluster_bar), "r"(x), "r"(y)
      : "memory");
}

template <int MODE>
__global__ void __launch_bounds__(NUM_THREADS, 1)
    k_lu_update_tc2_pair(const __grid_constant__ Ops ops, const __grid_constant__ CUtensorMap tmB, int ldc, int M,
                         int N, int K, int a_plane, int store, int* err) {
  using CF = Cfg<MODE>;
  using PC = PairCfg<MODE>;
  constexpr int STAGES_P = PC::STAGES;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  float2* epi_stage = (float2*)(smem + STAGES_P * PC::STAGE);
  uint64_t* full = (uint64_t*)(smem + STAGES_P * PC::STAGE + EPI_WARPS * EPI_STAGE_BYTES);
  uint64_t* empty = full + STAGES_P;
  uint64_t* acc_full = empty + STAGES_P;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* fin = acc_empty + 2;  // completion of every MMA the first CTA issued
  uint32_t* tmem_base_slot = (uint32_t*)(fin + 1);

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  uint32_t rank;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
  const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
  const bool lead = rank == 0;
  const int kchunks = K / KCC;
  TileSched sched{(M + 2 * BM - 1) / (2 * BM), (N + BN - 1) / BN, 8};
  const int per = sched.tiles_m * sched.tiles_n, ntiles = per * ops.nb;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES_P; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 2 * EPI_WARPS);  // one arrival per epilogue warp of both CTAs
    }
    mbar_init(fin, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_base_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  // both CTAs' barriers exist before either signals the other
  tc_fence_before();
  cluster_sync();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_base_slot;

  if (warp == 0) {
    // ---------------- TMA producer (both CTAs)
    if (lane == 0) {
      int it = 0;
      bool ok = true;
      for (int t = pair; t < ntiles && ok; t += npairs) {
        int tm, tn;
        const int mb = t / per;
        sched.coords(t - mb * per, tm, tn);
        const int brow = mb * CF::PARTS * 2 * N;
        for (int kc = 0; kc < kchunks && ok; kc++, it++) {
          const int s = it % STAGES_P;
          const uint32_t ph = (uint32_t)(it / STAGES_P) & 1u;
          if (it >= STAGES_P && !mbar_wait(&empty[s], ph ^ 1u, err, 1)) {
            ok = false;
            break;
          }
          unsigned char* st = smem + s * PC::STAGE;
          if (lead) mbar_expect_tx(&full[s], 2 * PC::STAGE);
          const uint32_t bar = cluster_addr(&full[s], 0);
          const int x = kc * 2 * KCC;
#pragma unroll
          for (int p = 0; p < CF::PARTS; p++) {
            unsigned char* a = st + p * PC::PART;
            tma_load_2d_pair(a, &ops.A[mb], bar, x, p * a_plane + tm * 2 * BM + (int)rank * BM);
            tma_load_2d_pair(a + PC::A_TILE, &tmB, bar, x, brow + p * 2 * N + (int)rank * N + tn * BN);
          }
        }
      }
      // the first CTA waits (bounded) until every issued copy of both CTAs has
      // landed; the second is held by the closing cluster barrier meanwhile
      if (lead)
        for (int j = (it > STAGES_P ? it - STAGES_P : 0); j < it; j++)
          mbar_wait(&full[j % STAGES_P], (uint32_t)(j / STAGES_P) & 1u, err, 5);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer (first CTA only)
    if (lead && lane == 0) {
      const int ta[3] = {0, 0, 1};
      const int tb[3] = {0, 1, 0};
      int it = 0, local = 0;
      bool ok = true;
      for (int t = pair; t < ntiles && ok; t += npairs, local++) {
        const int ab = local & 1;
        const uint32_t aph = (uint32_t)(local >> 1) & 1u;
        if (local >= 2 && !mbar_wait(&acc_empty[ab], aph ^ 1u, err, 2)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem_base + ab * (2 * BN);
        for (int kc = 0; kc < kchunks; kc++, it++) {
          const int s = it % STAGES_P;
          const uint32_t ph = (uint32_t)(it / STAGES_P) & 1u;
          if (!mbar_wait(&full[s], ph, err, 3)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t s0 = smem_u32(smem + s * PC::STAGE);
#pragma unroll
          for (int ks = 0; ks < CF::KSTEPS; ks++) {
#pragma unroll
            for (int q = 0; q < CF::TERMS; q++) {
              const uint32_t a0 = s0 + ta[q] * PC::PART;
              const uint32_t b0 = s0 + tb[q] * PC::PART + PC::A_TILE;
              umma_pair<MODE>(d, op_desc<MODE>(a0 + ks * 32), op_desc<MODE>(b0 + ks * 32),
                              (kc == 0 && ks == 0 && q == 0) ? 0u : 1u);
            }
          }
          umma_commit_pair(&empty[s]);
        }
        if (!ok) break;
        umma_commit_pair(&acc_full[ab]);
      }
      // no MMA may still read the second CTA's shared memory when the pair
      // leaves (also after an early exit)
      umma_commit_pair(fin);
      mbar_wait(fin, 0, err, 6);
    }
  } else {
    // ---------------- epilogue (warps 2..9 of both CTAs): this CTA's 128 rows
    const int quarter = warp & 3;
    const int half = (warp - 2) >> 2;
    float2* stage = epi_stage + (size_t)(warp - 2) * (32 * 16);
    const uint32_t lead_acc_empty[2] = {cluster_addr(&acc_empty[0], 0), cluster_addr(&acc_empty[1], 0)};
    int local = 0;
    for (int t = pair; t < ntiles; t += npairs, local++) {
      int tm, tn;
      const int mb = t / per;
      sched.coords(t - mb * per, tm, tn);
      float2* __restrict__ C = ops.C[mb];
      const int ab = local & 1;
      const uint32_t aph = (uint32_t)(local >> 1) & 1u;
      const int row0 = tm * 2 * BM + (int)rank * BM + quarter * 32;
      float2 cv[16];
      if (!store) load_c_chunk(C, ldc, M, N, row0, tn * BN + half * (BN / 2), lane, cv);
      if (!mbar_wait(&acc_full[ab], aph, err, 4)) break;
      tc_fence_after();
      const uint32_t lane_addr = tmem_base + ((uint32_t)(quarter * 32) << 16) + ab * (2 * BN);
#pragma unroll 1
      for (int cc = 0; cc < BN / 2; cc += 16) {
        const int col = half * (BN / 2) + cc;
        const int gcol0 = tn * BN + col;
        if (cc > 0 && !store) load_c_chunk(C, ldc, M, N, row0, gcol0, lane, cv);
        float re[16], im[16];
        tmem_ld16(lane_addr + col, re);
        tmem_ld16(lane_addr + BN + col, im);
#pragma unroll
        for (int j = 0; j < 16; j++) stage[lane * 16 + (j ^ (lane & 15))] = make_float2(re[j], im[j]);
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 16; i++) {
          const int idx = i * 32 + lane, r = idx >> 4, c = idx & 15;
          const int grow = row0 + r, gcol = gcol0 + c;
          const float2 a = stage[r * 16 + (c ^ (r & 15))];
          if (grow < M && gcol < N)
            C[(size_t)grow * ldc + gcol] = store ? a : make_float2(cv[i].x - a.x, cv[i].y - a.y);
        }
        __syncwarp();
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_remote(lead_acc_empty[ab]);
    }
  }
  __syncwarp();
  // neither CTA leaves while the other may still read its shared memory or
  // signal its barriers
  tc_fence_before();
  cluster_sync();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS));
  }
}

// ---- operand packing

// L rows as [M][2K] reals.  TF32: one fp32 plane (used when the matrix itself
// cannot be read by TMA); BF16X3: hi plane rows [0, M), lo plane [M, 2M).
template <int MODE>
__global__ void k_pack_A(const float2* __restrict__ L, int ldl, int M, int K, void* __restrict__ WA) {
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (size_t)M * K) return;
  const int i = (int)(tid / K), kk = (int)(tid % K);
  const float2 v = L[(size_t)i * ldl + kk];
  if constexpr (MODE == TC_TF32) {
    reinterpret_cast<float2*>(WA)[(size_t)i * K + kk] = v;
  } else {
    __nv_bfloat162* w = reinterpret_cast<__nv_bfloat162*>(WA);
    const __nv_bfloat162 hi = __floats2bfloat162_rn(v.x, v.y);
    const float2 hf = __bfloat1622float2(hi);
    w[(size_t)i * K + kk] = hi;
    w[(size_t)M * K + (size_t)i * K + kk] = __floats2bfloat162_rn(v.x - hf.x, v.y - hf.y);
  }
}

// Column j of U as its re-row [Ur, -Ui, ...] (row j) and im-row [Ui, Ur, ...]
// (row N + j) of a [2N][2K] real plane; BF16X3 adds the lo plane at row 2N.
template <int MODE>
__global__ void k_pack_B(const float2* __restrict__ U, int ldu, int K, int N, void* __restrict__ WB) {
  __shared__ float2 tile[32][33];
  const int j0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;  // 32 x 8
  for (int r = ty; r < 32; r += 8) {
    const int kk = k0 + r, j = j0 + tx;
    float2 v = make_float2(0.f, 0.f);
    if (kk < K && j < N) v = U[(size_t)kk * ldu + j];
    tile[r][tx] = v;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int j = j0 + r, kk = k0 + tx;
    if (j < N && kk < K) {
      const float2 v = tile[tx][r];
      tc2_pack_b(MODE, WB, N, K, j, kk, v);
    }
  }
}

}  // namespace tc2

namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn2() {
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

// 2D real tensor [rows][cols] with row pitch `pitch_bytes`, box = one swizzle
// row (32 reals) x box_rows.
int make_map2(CUtensorMap* map, int mode, void* base, uint64_t rows, uint64_t cols, uint64_t pitch_bytes,
              uint32_t box_rows) {
  EncodeTiledFn fn = encode_fn2();
  if (!fn) {
    set_error("cuTensorMapEncodeTiled is not available from the driver");
    return TT_ERR_CUDA;
  }
  const bool tf32 = mode == TC_TF32;
  const cuuint64_t dims[2] = {cols, rows};
  const cuuint64_t strides[1] = {pitch_bytes};
  const cuuint32_t box[2] = {32, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(map, tf32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        tf32 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed with code " + std::to_string((int)r));
    return TT_ERR_CUDA;
  }
  return TT_OK;
}

struct TC2Workspace {
  DevBuf<unsigned char> WA, WB;
  DevBuf<int> err;
};

// CTA-pair kernel for updates of more than 128 rows (tc2_set_pairs)
thread_local bool g_tc2_pairs = false;

int current_device_index() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}

TC2Workspace& workspace2() {
  static thread_local TC2Workspace ws;
  return ws;
}

template <int MODE>
int launch_tc2(int nb, float2* const* C, int ldc, const float2* const* L, int ldl, const float2* const* U, int ldu,
               int M, int N, int K, cudaStream_t st, int store, bool prepacked) {
  using CF = tc2::Cfg<MODE>;
  if (nb < 1 || nb > tc2::kBatch) {
    set_error("tensor-core update batch of " + std::to_string(nb) + " products (1.." + std::to_string(tc2::kBatch) +
              ")");
    return TT_ERR_BADARG;
  }
  TC2Workspace& ws = workspace2();
  const size_t esz = (MODE == TC_TF32) ? 4 : 2;
  // the matrix itself is the TF32 A operand when TMA can address it: 16-byte
  // aligned base and row pitch (the panel's x offsets are multiples of 32 reals)
  bool direct_A = MODE == TC_TF32 && ((size_t)ldl * 8 % 16 == 0);
  for (int b = 0; b < nb; b++) direct_A = direct_A && ((uintptr_t)L[b] % 16 == 0);
  const size_t planeA = (size_t)CF::PARTS * M * 2 * K * esz, planeB = (size_t)CF::PARTS * 2 * N * 2 * K * esz;
  const size_t needA = direct_A ? 0 : planeA * nb;
  const size_t needB = planeB * nb;
  if (needA > ws.WA.count) TT_TRY(ws.WA.alloc(needA));
  if (needB > ws.WB.count) {
    if (prepacked) {
      set_error("tensor-core update: prepacked operand planes larger than the workspace");
      return TT_ERR_BADARG;
    }
    TT_TRY(ws.WB.alloc(needB));
  }
  if (!ws.err.ptr) {
    TT_TRY(ws.err.alloc(1));
    TT_CUDA_TRY(cudaMemsetAsync(ws.err.ptr, 0, sizeof(int), st));
  }
  {
    ProfScope prof(TT_PROF_OPERANDS, st, 0.0,
                   nb * (8.0 * (direct_A ? 0.0 : (double)M) * K + (double)(needA / nb) +
                         (prepacked ? 0.0 : 8.0 * N * K + (double)planeB)));
    for (int b = 0; b < nb; b++) {
      if (!direct_A) {
        tc2::k_pack_A<MODE><<<ceil_div((size_t)M * K, 256), 256, 0, st>>>(L[b], ldl, M, K, ws.WA.ptr + planeA * b);
        count_launch();
        TT_CUDA_TRY(cudaGetLastError());
      }
      if (!prepacked) {
        dim3 gs(ceil_div(N, 32), ceil_div(K, 32));
        tc2::k_pack_B<MODE><<<gs, 256, 0, st>>>(U[b], ldu, K, N, ws.WB.ptr + planeB * b);
        count_launch();
        TT_CUDA_TRY(cudaGetLastError());
      }
    }
  }
  tc2::Ops ops;
  std::memset(&ops, 0, sizeof(ops));
  ops.nb = nb;
  for (int b = 0; b < nb; b++) {
    ops.C[b] = C[b];
    if (direct_A)
      TT_TRY(make_map2(&ops.A[b], MODE, const_cast<float2*>(L[b]), (uint64_t)M, (uint64_t)2 * K, (uint64_t)ldl * 8,
                       tc2::BM));
    else
      TT_TRY(make_map2(&ops.A[b], MODE, ws.WA.ptr + planeA * b, (uint64_t)CF::PARTS * M, (uint64_t)2 * K,
                       (uint64_t)2 * K * esz, tc2::BM));
  }
  CUtensorMap mB;
  TT_TRY(make_map2(&mB, MODE, ws.WB.ptr, (uint64_t)nb * CF::PARTS * 2 * N, (uint64_t)2 * K, (uint64_t)2 * K * esz,
                   tc2::BN));
  ProfScope prof(K >= 256 ? TT_PROF_TC_UPDATE : TT_PROF_TC_PANEL, st, 8.0 * M * N * K * nb,
                 nb * (16.0 * M * N + 8.0 * ((double)M + N) * K));
  if (g_tc2_pairs && M > tc2::BM) {
    // CTA pairs on 256-row tiles, as many pairs as can be resident at once
    using PC = tc2::PairCfg<MODE>;
    const size_t smem = (size_t)PC::STAGES * PC::STAGE + tc2::EPI_WARPS * tc2::EPI_STAGE_BYTES + 1024 + 128;
    const void* kfn = (const void*)tc2::k_lu_update_tc2_pair<MODE>;
    TT_TRY(smem_limit_once(kfn, (int)smem));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(tc2::NUM_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    static int max_pairs[2][16] = {};
    int& mp = max_pairs[MODE == TC_TF32 ? 0 : 1][current_device_index() & 15];
    if (mp == 0) {
      cfg.gridDim = dim3(2 * (device_sm_count() / 2));
      int clusters = 0;
      TT_CUDA_TRY(cudaOccupancyMaxActiveClusters(&clusters, kfn, &cfg));
      mp = std::max(1, clusters);
    }
    const int tiles = nb * ((M + 2 * tc2::BM - 1) / (2 * tc2::BM)) * ((N + tc2::BN - 1) / tc2::BN);
    cfg.gridDim = dim3(2 * std::min(tiles, mp));
    TT_CUDA_TRY(cudaLaunchKernelEx(&cfg, tc2::k_lu_update_tc2_pair<MODE>, ops, mB, ldc, M, N, K, M, store,
                                   ws.err.ptr));
  } else {
    const size_t smem = (size_t)tc2::STAGES * CF::STAGE + tc2::EPI_WARPS * tc2::EPI_STAGE_BYTES + 1024 + 128;
    TT_TRY(smem_limit_once((const void*)tc2::k_lu_update_tc2<MODE>, (int)smem));
    const int tiles = nb * ((M + tc2::BM - 1) / tc2::BM) * ((N + tc2::BN - 1) / tc2::BN);
    const int grid = std::min(tiles, device_sm_count());
    tc2::k_lu_update_tc2<MODE><<<grid, tc2::NUM_THREADS, smem, st>>>(ops, mB, ldc, M, N, K, M, store, ws.err.ptr);
  }
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  return TT_OK;
}

}  // namespace

void tc2_set_pairs(bool on) { g_tc2_pairs = on; }

size_t tc2_b_plane_bytes(int mode, int N, int K) {
  const size_t esz = (mode == TC_TF32) ? 4 : 2, parts = (mode == TC_TF32) ? 1 : 2;
  return parts * 2 * (size_t)N * 2 * K * esz;
}

void* tc2_b_workspace(int mode, int N, int K, int* status, int nb) {
  TC2Workspace& ws = workspace2();
  const size_t esz = (mode == TC_TF32) ? 4 : 2, parts = (mode == TC_TF32) ? 1 : 2;
  const size_t need = parts * 2 * (size_t)N * 2 * K * esz * nb;
  *status = TT_OK;
  if (need > ws.WB.count) *status = ws.WB.alloc(need);
  return *status == TT_OK ? ws.WB.ptr : nullptr;
}

int tc2_gemm_sub(int mode, float2* C, int ldc, const float2* L, int ldl, const float2* U, int ldu, int M, int N, int K,
                 cudaStream_t st, int store, bool prepacked) {
  if (M <= 0 || N <= 0 || K <= 0) return TT_OK;
  if (K % tc2::KCC != 0) {
    set_error("tensor-core update needs K to be a multiple of 16");
    return TT_ERR_BADARG;
  }
  return tc2_gemm_sub_batched(mode, 1, &C, ldc, &L, ldl, &U, ldu, M, N, K, st, store, prepacked);
}

int tc2_gemm_sub_batched(int mode, int nb, float2* const* C, int ldc, const float2* const* L, int ldl,
                         const float2* const* U, int ldu, int M, int N, int K, cudaStream_t st, int store,
                         bool prepacked) {
  if (M <= 0 || N <= 0 || K <= 0 || nb <= 0) return TT_OK;
  if (K % tc2::KCC != 0) {
    set_error("tensor-core update needs K to be a multiple of 16");
    return TT_ERR_BADARG;
  }
  if (mode == TC_TF32) return launch_tc2<TC_TF32>(nb, C, ldc, L, ldl, U, ldu, M, N, K, st, store, prepacked);
  if (mode == TC_BF16X3) return launch_tc2<TC_BF16X3>(nb, C, ldc, L, ldl, U, ldu, M, N, K, st, store, prepacked);
  set_error("unknown tensor-core product mode " + std::to_string(mode));
  return TT_ERR_BADARG;
}

int tc2_check_error(cudaStream_t st) {
  TC2Workspace& ws = workspace2();
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

}  // namespace tt
