// Host plumbing of the C ABI: error text, launch counter, version, SM-count grid sizing.
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "pt_common.cuh"

namespace pt {

static thread_local std::string g_last_error;
static std::atomic<uint64_t> g_launches{0};

pt_status fail(pt_status s, const std::string& msg)
{
  g_last_error = msg;
  return s;
}

pt_status cuda_status(cudaError_t e, const char* what)
{
  if (e == cudaSuccess) return PT_OK;
  std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();  // allocation failures are not sticky; clear them
    return fail(PT_OOM, m);
  }
  return fail(PT_CUDA_ERROR, m);
}

void count_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int sm_count()
{
  static std::mutex mu;
  static std::vector<int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  std::lock_guard<std::mutex> lk(mu);
  if ((int)cache.size() <= dev) cache.resize(dev + 1, 0);
  if (cache[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cache[dev] = n;
  }
  return cache[dev];
}

int grid_for(uint64_t items, int block, int blocks_per_sm)
{
  uint64_t need = (items + (uint64_t)block - 1) / (uint64_t)block;
  uint64_t cap = (uint64_t)sm_count() * (uint64_t)blocks_per_sm;
  uint64_t g = need < cap ? need : cap;
  return g == 0 ? 1 : (int)g;
}

}  // namespace pt

extern "C" {

const char* pt_last_error_message(void) { return pt::g_last_error.c_str(); }
int pt_version(void) { return 100; }
uint64_t pt_kernel_launch_count(void) { return pt::g_launches.load(std::memory_order_relaxed); }

}  // extern "C"
