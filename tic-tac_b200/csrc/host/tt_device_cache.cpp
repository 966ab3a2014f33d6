// Cache of large device blocks behind DevBuf (see tt_device.h).
#include <algorithm>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "../cuda/tt_device.h"

namespace tt {
namespace {

// never destroyed: buffers with static storage duration release into the
// cache during exit
std::mutex& cache_mu() {
  static std::mutex* m = new std::mutex;
  return *m;
}
std::map<int, std::vector<std::pair<void*, size_t>>>& cache() {  // device -> (block, bytes)
  static auto* c = new std::map<int, std::vector<std::pair<void*, size_t>>>;
  return *c;
}

int current_device() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}

}  // namespace

void* device_cache_take(size_t bytes, size_t* capacity) {
  std::lock_guard<std::mutex> lk(cache_mu());
  auto& v = cache()[current_device()];
  int best = -1;
  for (int i = 0; i < (int)v.size(); i++) {
    const size_t c = v[i].second;
    if (c >= bytes && 2 * c <= 3 * bytes && (best < 0 || c < v[best].second)) best = i;
  }
  if (best < 0) return nullptr;
  void* p = v[best].first;
  *capacity = v[best].second;
  v.erase(v.begin() + best);
  return p;
}

void device_cache_give(void* p, size_t capacity) {
  // the block may still be in use by queued work: wait, as cudaFree would
  cudaDeviceSynchronize();
  std::lock_guard<std::mutex> lk(cache_mu());
  cache()[current_device()].emplace_back(p, capacity);
}

size_t device_cache_bytes() {
  std::lock_guard<std::mutex> lk(cache_mu());
  size_t s = 0;
  for (const auto& b : cache()[current_device()]) s += b.second;
  return s;
}

size_t device_cache_evict_one() {
  std::pair<void*, size_t> b{nullptr, 0};
  {
    std::lock_guard<std::mutex> lk(cache_mu());
    auto& v = cache()[current_device()];
    if (v.empty()) return 0;
    b = v.front();  // the block released longest ago
    v.erase(v.begin());
  }
  cudaFree(b.first);
  return b.second;
}

void device_cache_trim() {
  std::vector<std::pair<void*, size_t>> v;
  {
    std::lock_guard<std::mutex> lk(cache_mu());
    v.swap(cache()[current_device()]);
  }
  for (const auto& b : v) cudaFree(b.first);
}

}  // namespace tt
