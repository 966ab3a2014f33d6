// Internal hooks between the LU driver and the tensor-core trailing update.
#pragma once
#include <cuda_runtime.h>

#include "tt_device.h"

namespace tt {

// A22 -= L21 U12 for the complex64 factorisation on tcgen05 tensor cores with
// a BF16x3 split (gemm_tc.cu).
int lu_update_tc(float2* A, int n, int k, int nb, cudaStream_t st);

// Reports (and clears) a barrier timeout recorded by the tensor-core kernel.
int tc_check_error(cudaStream_t st);

// Product modes of the complex64 factorisation's updates (the use_tensor_cores
// argument of lu_factor_batched_device); 0 = CUDA-core FP32 updates.
constexpr int TC_LEGACY_BF16X3 = 1;  // gemm_tc.cu: four real products, N = 128, BF16x3 (12 MMAs per k16)
constexpr int TC_TF32 = 2;           // gemm_tc2.cu: real-row form, N = 256, one tf32 product
constexpr int TC_BF16X3 = 3;         // gemm_tc2.cu: real-row form, N = 256, BF16x3 (3 MMAs per k16)
// C[M x N] -= L[M x K] U[K x N] in the real-row form (gemm_tc2.cu), K % 16 == 0;
// store != 0: C = L U (C is not read; it may be U's own storage, which is
// packed before the product, but must not overlap L).
// prepacked: U's operand planes are already in the workspace (tc2_b_workspace).
int tc2_gemm_sub(int mode, float2* C, int ldc, const float2* L, int ldl, const float2* U, int ldu, int M, int N, int K,
                 cudaStream_t st, int store = 0, bool prepacked = false);
// Updates of more than 128 rows on CTA pairs (cta_group::2, 256-row tiles) on
// this host thread's next tc2_gemm_sub calls.
void tc2_set_pairs(bool on);
// The same for nb <= 4 products of one shape in one launch (the tiles of all
// of them share the persistent grid): C[b] -= L[b] U[b].
int tc2_gemm_sub_batched(int mode, int nb, float2* const* C, int ldc, const float2* const* L, int ldl,
                         const float2* const* U, int ldu, int M, int N, int K, cudaStream_t st, int store = 0,
                         bool prepacked = false);
// The B-operand workspace of tc2_gemm_sub(_batched), grown to nb N-column,
// K-deep operands; product b's planes start nb-th of the way in (b times the
// size of one operand's planes).
void* tc2_b_workspace(int mode, int N, int K, int* status, int nb = 1);
// Bytes of one N-column, K-deep operand's planes in that workspace.
size_t tc2_b_plane_bytes(int mode, int N, int K);
int tc2_check_error(cudaStream_t st);
// C[M x N] -= L[M x K] U[K x N], complex128, on the FP64 tensor cores (zgemm_dmma.cu).
int zgemm_sub_dmma(double2* C, int ldc, const double2* L, int ldl, const double2* U, int ldu, int M, int N, int K,
                   cudaStream_t st);
// C[M x N] -= L[M x K] U[K x N], complex64 row-major operands, K % 64 == 0.
int tc_gemm_sub(float2* C, int ldc, const float2* L, int ldl, const float2* U, int ldu, int M, int N, int K,
                cudaStream_t st);

inline int lu_update_tc(double2*, int, int, int, cudaStream_t) {
  set_error("tensor-core trailing update is only defined for the complex64 factorisation");
  return TT_ERR_UNSUPPORTED;
}

}  // namespace tt
