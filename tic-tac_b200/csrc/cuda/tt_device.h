// Shared device-side utilities: error propagation, RAII device buffers.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "tictac_b200.h"  // status codes

namespace tt {

void set_error(const std::string& msg);
const char* last_error();

// Count of kernels this library has launched (reported by tt_kernel_launches).
void count_launch();

// Optional per-kernel-class timing, off unless tt_profile_begin() was called:
// a ProfScope brackets its launches with CUDA events on the launching stream
// and books the scope's algorithmic flops and bytes (TT_PROF_* classes).
struct ProfScope {
  ProfScope(int kernel_class, cudaStream_t st, double flops, double bytes);
  ~ProfScope();
  ProfScope(const ProfScope&) = delete;
  ProfScope& operator=(const ProfScope&) = delete;

 private:
  int cls_ = -1;
  long ev0_ = -1;
  cudaStream_t st_ = nullptr;
  double flops_ = 0, bytes_ = 0;
};

#define TT_CUDA_TRY(expr)                                                                   \
  do {                                                                                      \
    cudaError_t _e = (expr);                                                                \
    if (_e != cudaSuccess) {                                                                \
      ::tt::set_error(std::string(#expr) + " failed: " + cudaGetErrorString(_e) + " at " + \
                      __FILE__ + ":" + std::to_string(__LINE__));                           \
      return (_e == cudaErrorMemoryAllocation) ? TT_ERR_NOMEM : TT_ERR_CUDA;   \
    }                                                                                       \
  } while (0)

#define TT_TRY(expr)                 \
  do {                               \
    int _s = (expr);                 \
    if (_s != TT_OK) return _s; \
  } while (0)

// Large device blocks (at least kCacheMinBytes) that a DevBuf releases are
// kept for reuse instead of going back to the driver, where cudaMalloc and
// cudaFree of tens of GB take 5-35 ms each.  A cached block serves a request
// of at most its size and at least two thirds of it.  Releasing a block waits
// for the device, as cudaFree does, so a block is idle when it is handed out
// again.  When an allocation would otherwise fail, cached blocks are freed
// one at a time, the longest-held first, until it succeeds; device_cache_trim(),
// tt_run_destroy and tt_release_cached_device_memory free all of them.
constexpr size_t kCacheMinBytes = size_t(256) << 20;
void* device_cache_take(size_t bytes, size_t* capacity);
void device_cache_give(void* p, size_t capacity);
size_t device_cache_bytes();  // cached on the current device
size_t device_cache_evict_one();  // frees the longest-held block; its bytes (0: none)
void device_cache_trim();     // frees the current device's cached blocks

// Owning device buffer.  alloc() reports NOMEM through the status path instead
// of faulting.
template <typename T>
struct DevBuf {
  T* ptr = nullptr;
  size_t count = 0;
  size_t cap = 0;  // bytes of the underlying block
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : ptr(o.ptr), count(o.count), cap(o.cap) {
    o.ptr = nullptr;
    o.count = 0;
    o.cap = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      ptr = o.ptr;
      count = o.count;
      cap = o.cap;
      o.ptr = nullptr;
      o.count = 0;
      o.cap = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void release() {
    if (ptr) {
      if (cap >= kCacheMinBytes) device_cache_give(ptr, cap);
      else cudaFree(ptr);
    }
    ptr = nullptr;
    count = 0;
    cap = 0;
  }
  int alloc(size_t n) {
    release();
    if (n == 0) return TT_OK;
    const size_t bytes = n * sizeof(T);
    if (bytes >= kCacheMinBytes) {
      size_t c = 0;
      if (void* p = device_cache_take(bytes, &c)) {
        ptr = static_cast<T*>(p);
        count = n;
        cap = c;
        return TT_OK;
      }
    }
    cudaError_t e = cudaMalloc((void**)&ptr, bytes);
    while (e == cudaErrorMemoryAllocation && device_cache_evict_one() > 0) {
      cudaGetLastError();
      e = cudaMalloc((void**)&ptr, bytes);
    }
    if (e != cudaSuccess) {
      ptr = nullptr;
      cudaGetLastError();
      set_error("device allocation of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
      return e == cudaErrorMemoryAllocation ? TT_ERR_NOMEM : TT_ERR_CUDA;
    }
    count = n;
    cap = bytes;
    return TT_OK;
  }
  int upload(const T* h, size_t n, cudaStream_t s) {
    TT_TRY(alloc(n));
    if (n) TT_CUDA_TRY(cudaMemcpyAsync(ptr, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
    return TT_OK;
  }
  int upload(const std::vector<T>& v, cudaStream_t s) { return upload(v.data(), v.size(), s); }
};

// Device CSR matrix (rows sorted, columns ascending within a row).
struct DeviceCSR {
  int n = 0;
  int64_t nnz = 0;
  DevBuf<int64_t> rowptr;
  DevBuf<int32_t> col;
  DevBuf<double> val;
};

inline unsigned ceil_div(size_t a, size_t b) { return (unsigned)((a + b - 1) / b); }

// Raises a kernel's dynamic shared-memory limit on the current device to at
// least `bytes` (never lowers it): function attributes are per device.
int smem_limit_once(const void* kernel, int bytes);

}  // namespace tt
