// P123 handed over in the reference's CSC form (values, int row indices,
// size_t column pointers; CPP/main.cpp:230-243 builds it) turned into the
// device CSR the A build reads (columns ascending within a row), on the GPU:
// column ids are expanded from the pointers, the (row, position) pairs are
// sorted by row with a stable radix sort (so the column order of the CSC
// sequence is kept inside each row), values and columns gathered, and the
// row pointers made by a histogram and a scan.

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "tt_kernels.h"

namespace tt {
namespace {

// col[e] = c for colptr[c] <= e < colptr[c+1]; warp per column
__global__ void k_expand_cols(const uint64_t* __restrict__ colptr, int n, int32_t* __restrict__ col) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int c = (int)warp;
  for (uint64_t e = colptr[c] + lane; e < colptr[c + 1]; e += 32) col[e] = c;
}

__global__ void k_iota(int64_t m, int32_t* __restrict__ idx) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < m) idx[t] = (int32_t)t;
}

__global__ void k_row_hist(const int32_t* __restrict__ row, int64_t m, int64_t* __restrict__ counts) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < m) atomicAdd(reinterpret_cast<unsigned long long*>(&counts[row[t]]), 1ull);
}

__global__ void k_gather_csr(const int32_t* __restrict__ perm, const int32_t* __restrict__ col_csc,
                             const double* __restrict__ val_csc, int64_t m, int32_t* __restrict__ col,
                             double* __restrict__ val) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m) return;
  const int32_t p = perm[t];
  col[t] = col_csc[p];
  val[t] = val_csc[p];
}

__global__ void k_check_rows(const int32_t* __restrict__ row, int64_t m, int n, int* __restrict__ bad) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < m && (row[t] < 0 || row[t] >= n)) atomicExch(bad, 1);
}

}  // namespace

int csc_to_csr_device(const double* h_val, const int32_t* h_row, const uint64_t* h_colptr, int64_t nnz, int n,
                      DeviceCSR& out, cudaStream_t st) {
  out.n = n;
  out.nnz = nnz;
  TT_TRY(out.rowptr.alloc((size_t)n + 1));
  if (nnz <= 0) {
    TT_CUDA_TRY(cudaMemsetAsync(out.rowptr.ptr, 0, sizeof(int64_t) * ((size_t)n + 1), st));
    return TT_OK;
  }
  if (nnz > INT32_MAX) {
    set_error("P123 with more than 2^31 nonzeros in one channel is not supported by the CSR conversion");
    return TT_ERR_UNSUPPORTED;
  }
  const size_t m = (size_t)nnz;
  DevBuf<double> val_csc;
  DevBuf<int32_t> row_csc, col_csc, row_sorted, idx, perm;
  DevBuf<uint64_t> colptr;
  DevBuf<int> bad;
  TT_TRY(val_csc.upload(h_val, m, st));
  TT_TRY(row_csc.upload(h_row, m, st));
  TT_TRY(colptr.upload(h_colptr, (size_t)n + 1, st));
  TT_TRY(bad.alloc(1));
  TT_CUDA_TRY(cudaMemsetAsync(bad.ptr, 0, sizeof(int), st));
  k_check_rows<<<ceil_div(m, 256), 256, 0, st>>>(row_csc.ptr, (int64_t)m, n, bad.ptr);
  count_launch();
  int h_bad = 0;
  TT_CUDA_TRY(cudaMemcpyAsync(&h_bad, bad.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
  TT_CUDA_TRY(cudaStreamSynchronize(st));
  if (h_bad) {
    set_error("P123 row index out of range");
    return TT_ERR_BADARG;
  }
  TT_TRY(col_csc.alloc(m));
  k_expand_cols<<<ceil_div((size_t)n * 32, 256), 256, 0, st>>>(colptr.ptr, n, col_csc.ptr);
  count_launch();
  TT_TRY(idx.alloc(m));
  k_iota<<<ceil_div(m, 256), 256, 0, st>>>((int64_t)m, idx.ptr);
  count_launch();
  // stable sort of positions by row
  TT_TRY(row_sorted.alloc(m));
  TT_TRY(perm.alloc(m));
  int end_bit = 1;
  while ((1ll << end_bit) < (long long)n) end_bit++;
  size_t tmp_bytes = 0;
  TT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, row_csc.ptr, row_sorted.ptr, idx.ptr, perm.ptr,
                                              (int)m, 0, end_bit, st));
  DevBuf<uint8_t> tmp;
  TT_TRY(tmp.alloc(tmp_bytes));
  TT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp.ptr, tmp_bytes, row_csc.ptr, row_sorted.ptr, idx.ptr, perm.ptr,
                                              (int)m, 0, end_bit, st));
  count_launch();
  TT_TRY(out.col.alloc(m));
  TT_TRY(out.val.alloc(m));
  k_gather_csr<<<ceil_div(m, 256), 256, 0, st>>>(perm.ptr, col_csc.ptr, val_csc.ptr, (int64_t)m, out.col.ptr,
                                                 out.val.ptr);
  count_launch();
  // row pointers: histogram of the rows, exclusive scan over n+1 entries
  DevBuf<int64_t> counts;
  TT_TRY(counts.alloc((size_t)n + 1));
  TT_CUDA_TRY(cudaMemsetAsync(counts.ptr, 0, sizeof(int64_t) * ((size_t)n + 1), st));
  k_row_hist<<<ceil_div(m, 256), 256, 0, st>>>(row_csc.ptr, (int64_t)m, counts.ptr);
  count_launch();
  size_t scan_bytes = 0;
  TT_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, counts.ptr, out.rowptr.ptr, n + 1, st));
  DevBuf<uint8_t> scan_tmp;
  TT_TRY(scan_tmp.alloc(scan_bytes));
  TT_CUDA_TRY(cub::DeviceScan::ExclusiveSum(scan_tmp.ptr, scan_bytes, counts.ptr, out.rowptr.ptr, n + 1, st));
  count_launch();
  TT_CUDA_TRY(cudaGetLastError());
  TT_CUDA_TRY(cudaStreamSynchronize(st));
  return TT_OK;
}

}  // namespace tt
