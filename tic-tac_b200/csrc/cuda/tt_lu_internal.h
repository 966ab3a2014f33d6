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
// C[M x N] -= L[M x K] U[K x N], complex64 row-major operands, K % 64 == 0.
int tc_gemm_sub(float2* C, int ldc, const float2* L, int ldl, const float2* U, int ldu, int M, int N, int K,
                cudaStream_t st);

inline int lu_update_tc(double2*, int, int, int, cudaStream_t) {
  set_error("tensor-core trailing update is only defined for the complex64 factorisation");
  return TT_ERR_UNSUPPORTED;
}

}  // namespace tt
