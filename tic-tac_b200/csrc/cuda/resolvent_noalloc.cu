// Resolvent into device memory the caller owns, with no device allocation.
//
// The tables the resolvent kernel reads (per-alpha offsets, SWP energy
// boundaries, q grid, energies) are staged in one file-scope device array of
// TT_RESOLVENT_NOALLOC_SCRATCH_BYTES instead of buffers allocated per call.
// Its address is looked up once per device (cudaGetSymbolAddress, with that
// device current); that first lookup also loads this module on the device.
// Nothing in the scratch has to start at zero: each call rewrites every table
// it reads, on the caller's stream, before the kernel that reads it.  Calls
// that overlap in time on one device (different streams or host threads)
// share the one array and race; calls on one stream are ordered by it.
//
// The tables are assembled on the host in one static staging buffer and
// copied with one cudaMemcpyAsync.  A copy from pageable memory may still be
// reading its source after the call returns, so each copy records an event
// and the next call waits for it before it rewrites the staging buffer.
#include <mutex>

#include "../host/tt_solver.h"
#include "tt_device.h"
#include "tt_kernels.h"

namespace tt {
namespace {

constexpr size_t kScratchBytes = TT_RESOLVENT_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_resolvent_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices];
// host image of the tables, shared by all calls (under g_mu)
alignas(256) unsigned char g_stage[kScratchBytes];
// the last copy out of g_stage, and its device; waited for before g_stage is rewritten
cudaEvent_t g_stage_copied[kMaxDevices];
int g_stage_dev = -1;

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

int scratch_address(void** out) {
  int dev = -1;
  TT_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device ordinal " + std::to_string(dev) + " is beyond the " + std::to_string(kMaxDevices) +
              " devices the static resolvent scratch is tracked for");
    return TT_ERR_UNSUPPORTED;
  }
  if (!g_stage_copied[dev]) {
    const cudaError_t e = cudaEventCreateWithFlags(&g_stage_copied[dev], cudaEventDisableTiming);
    if (e != cudaSuccess) {
      g_stage_copied[dev] = nullptr;
      set_error(std::string("creating the staging event on device ") + std::to_string(dev) + " failed: " +
                cudaGetErrorString(e));
      return TT_ERR_CUDA;
    }
  }
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_resolvent_scratch);
    if (e != cudaSuccess || !p) {
      set_error(std::string("cudaGetSymbolAddress of the static resolvent scratch failed on device ") +
                std::to_string(dev) + ": " + cudaGetErrorString(e));
      return TT_ERR_CUDA;
    }
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return TT_OK;
}

}  // namespace

int resolvent_noalloc(const RunParams& rp, const PWChannel& ch, int Np, int Nq, int n_unco, int n_coup,
                      const double* e_unco, const double* e_coup, const double* q_WP, const double* E, int nE,
                      double* d_G, cudaStream_t st) {
  const size_t n_eu = (size_t)(Np + 1) * n_unco, n_ec = (size_t)2 * (Np + 1) * n_coup;
  const size_t off_e_off = 0;
  const size_t off_swp = align256(off_e_off + sizeof(int32_t) * (size_t)ch.Nalpha);
  const size_t off_q = align256(off_swp + sizeof(double) * (n_eu + n_ec));
  const size_t off_E = align256(off_q + sizeof(double) * (size_t)(Nq + 1));
  const size_t bytes = off_E + sizeof(double) * (size_t)nE;
  if (bytes > kScratchBytes) {
    set_error("the resolvent tables need " + std::to_string(bytes) + " bytes (" + std::to_string(ch.Nalpha) +
              " partial waves, " + std::to_string(n_eu + n_ec) + " SWP energies, Nq=" + std::to_string(Nq) +
              ", " + std::to_string(nE) + " energies); the static scratch holds " + std::to_string(kScratchBytes));
    return TT_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  void* base = nullptr;
  TT_TRY(scratch_address(&base));
  int dev = 0;
  TT_CUDA_TRY(cudaGetDevice(&dev));
  // the previous call's copy must have read the staging buffer before it is rewritten
  if (g_stage_dev >= 0) {
    int cur = dev;
    if (g_stage_dev != cur) TT_CUDA_TRY(cudaSetDevice(g_stage_dev));
    const cudaError_t e = cudaEventSynchronize(g_stage_copied[g_stage_dev]);
    if (g_stage_dev != cur) TT_CUDA_TRY(cudaSetDevice(cur));
    TT_CUDA_TRY(e);
  }
  std::string err;
  if (!channel_energy_offsets(rp, ch, Np, n_unco, n_coup, reinterpret_cast<int32_t*>(g_stage + off_e_off), &err)) {
    set_error(err);
    return TT_ERR_BADARG;
  }
  double* swp = reinterpret_cast<double*>(g_stage + off_swp);
  for (size_t i = 0; i < n_eu; i++) swp[i] = e_unco[i];
  for (size_t i = 0; i < n_ec; i++) swp[n_eu + i] = e_coup[i];
  double* q = reinterpret_cast<double*>(g_stage + off_q);
  for (int i = 0; i <= Nq; i++) q[i] = q_WP[i];
  double* e = reinterpret_cast<double*>(g_stage + off_E);
  for (int i = 0; i < nE; i++) e[i] = E[i];
  TT_CUDA_TRY(cudaMemcpyAsync(base, g_stage, bytes, cudaMemcpyHostToDevice, st));
  TT_CUDA_TRY(cudaEventRecord(g_stage_copied[dev], st));
  g_stage_dev = dev;
  unsigned char* d = static_cast<unsigned char*>(base);
  return resolvent_device_tables(ch.Nalpha, Nq, Np, reinterpret_cast<const int32_t*>(d + off_e_off),
                                 reinterpret_cast<const double*>(d + off_swp),
                                 reinterpret_cast<const double*>(d + off_q), reinterpret_cast<const double*>(d + off_E),
                                 nE, d_G, st);
}

}  // namespace tt
