// Per-kernel-class event timing behind tt_profile_begin / end / read.
#include <mutex>
#include <vector>

#include "../cuda/tt_device.h"

namespace tt {
namespace {

struct Record {
  int cls;
  long ev0, ev1;
  double flops, bytes;
};

struct ProfState {
  std::mutex mu;
  bool on = false;
  unsigned long long mask = ~0ull;  // classes recorded while on
  std::vector<cudaEvent_t> pool;  // reused across regions
  size_t used = 0;
  std::vector<Record> recs;
  tt_kernel_profile result[TT_PROF_COUNT] = {};
};

ProfState& state() {
  static ProfState s;
  return s;
}

// next free event of the pool (created on first use); -1 if creation fails
long take_event(ProfState& s) {
  if (s.used == s.pool.size()) {
    cudaEvent_t e;
    if (cudaEventCreateWithFlags(&e, cudaEventDefault) != cudaSuccess) return -1;
    s.pool.push_back(e);
  }
  return (long)s.used++;
}

}  // namespace

ProfScope::ProfScope(int kernel_class, cudaStream_t st, double flops, double bytes) {
  ProfState& s = state();
  if (!s.on || !((s.mask >> kernel_class) & 1ull)) return;
  std::lock_guard<std::mutex> lock(s.mu);
  if (!s.on) return;
  const long e = take_event(s);
  if (e < 0 || cudaEventRecord(s.pool[e], st) != cudaSuccess) return;
  cls_ = kernel_class;
  ev0_ = e;
  st_ = st;
  flops_ = flops;
  bytes_ = bytes;
}

ProfScope::~ProfScope() {
  if (cls_ < 0) return;
  ProfState& s = state();
  std::lock_guard<std::mutex> lock(s.mu);
  if (!s.on) return;
  const long e = take_event(s);
  if (e < 0 || cudaEventRecord(s.pool[e], st_) != cudaSuccess) return;
  s.recs.push_back(Record{cls_, ev0_, e, flops_, bytes_});
}

}  // namespace tt

using namespace tt;

extern "C" {

int tt_profile_select(unsigned long long class_mask) {
  ProfState& s = state();
  std::lock_guard<std::mutex> lock(s.mu);
  s.mask = class_mask;
  return TT_OK;
}

int tt_profile_begin(void) {
  ProfState& s = state();
  std::lock_guard<std::mutex> lock(s.mu);
  s.used = 0;
  s.recs.clear();
  for (auto& r : s.result) r = tt_kernel_profile{};
  s.on = true;
  return TT_OK;
}

int tt_profile_end(void) {
  ProfState& s = state();
  std::lock_guard<std::mutex> lock(s.mu);
  s.on = false;
  for (const Record& r : s.recs) {
    if (cudaEventSynchronize(s.pool[r.ev1]) != cudaSuccess) {
      set_error("event synchronisation failed while reading kernel timings");
      return TT_ERR_CUDA;
    }
    float ms = 0;
    if (cudaEventElapsedTime(&ms, s.pool[r.ev0], s.pool[r.ev1]) != cudaSuccess) {
      set_error("event timing failed while reading kernel timings");
      return TT_ERR_CUDA;
    }
    tt_kernel_profile& o = s.result[r.cls];
    o.launches++;
    o.ms += ms;
    o.flops += r.flops;
    o.bytes += r.bytes;
  }
  s.recs.clear();
  return TT_OK;
}

int tt_profile_read(int kernel_class, tt_kernel_profile* out) {
  if (kernel_class < 0 || kernel_class >= TT_PROF_COUNT || !out) {
    set_error("kernel class out of range or null output");
    return TT_ERR_BADARG;
  }
  ProfState& s = state();
  std::lock_guard<std::mutex> lock(s.mu);
  *out = s.result[kernel_class];
  return TT_OK;
}

}  // extern "C"
