// Operand layout of the real-row tensor-core update (gemm_tc2.cu), shared by
// the kernels that write it: column j of U (K x N, complex) becomes the re-row
// j [Ur, -Ui, ...] and the im-row N + j [Ui, Ur, ...] of a [2N][2K] real plane;
// TF32 rounds to tf32 (cvt.rna), BF16X3 stores hi and lo planes (lo at 2N rows).
#pragma once
#include <cuda_bf16.h>

#include "tt_lu_internal.h"

namespace tt {

__device__ __forceinline__ float tc2_round_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// U[kk][j] = v into the packed plane(s) WB of an N-column, K-deep operand
__device__ __forceinline__ void tc2_pack_b(int mode, void* __restrict__ WB, int N, int K, int j, int kk, float2 v) {
  const size_t re_at = (size_t)j * K + kk, im_at = (size_t)(N + j) * K + kk;  // in pairs of reals
  if (mode == TC_TF32) {
    float2* w = reinterpret_cast<float2*>(WB);
    const float ur = tc2_round_tf32(v.x), ui = tc2_round_tf32(v.y);
    w[re_at] = make_float2(ur, -ui);
    w[im_at] = make_float2(ui, ur);
  } else {
    __nv_bfloat162* w = reinterpret_cast<__nv_bfloat162*>(WB);
    const size_t lo = (size_t)2 * N * K;
    const __nv_bfloat162 hre = __floats2bfloat162_rn(v.x, -v.y);
    const __nv_bfloat162 him = __floats2bfloat162_rn(v.y, v.x);
    const float2 fre = __bfloat1622float2(hre), fim = __bfloat1622float2(him);
    w[re_at] = hre;
    w[im_at] = him;
    w[lo + re_at] = __floats2bfloat162_rn(v.x - fre.x, -v.y - fre.y);
    w[lo + im_at] = __floats2bfloat162_rn(v.y - fim.x, v.x - fim.y);
  }
}

}  // namespace tt
