// pool.cpp — the per-GPU memory pool behind every device block of the
// library (see pool.h).
#include "pool.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>
#include <mutex>

#include "../../include/hprqp.h"
#include "common.cuh"

namespace hprqp {
namespace {

constexpr int kMaxDevices = 64;

struct DevPool {
  cudaMemPool_t pool = nullptr;
  cudaStream_t st = nullptr;  // allocations and frees are ordered on it
};

std::mutex g_mu;
DevPool g_pools[kMaxDevices];

// The pool of device `dev` (created on first use, with `dev` current).
DevPool* pool_of(int dev) {
  if (dev < 0 || dev >= kMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lk(g_mu);
  DevPool& d = g_pools[dev];
  if (d.pool) return &d;
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  if (cudaMemPoolCreate(&d.pool, &props) != cudaSuccess) {
    d.pool = nullptr;
    return nullptr;
  }
  uint64_t keep = ~0ull;  // keep everything; an allocation that fails trims and retries
  if (const char* e = std::getenv("HPRQP_POOL_KEEP_MB")) keep = (uint64_t)std::strtoull(e, nullptr, 10) << 20;
  cudaMemPoolSetAttribute(d.pool, cudaMemPoolAttrReleaseThreshold, &keep);
  if (cudaStreamCreateWithFlags(&d.st, cudaStreamNonBlocking) != cudaSuccess) {
    cudaMemPoolDestroy(d.pool);
    d.pool = nullptr;
    d.st = nullptr;
    return nullptr;
  }
  return &d;
}

}  // namespace

void* pool_alloc(size_t bytes) {
  int dev = 0;
  HPRQP_CUDA(cudaGetDevice(&dev));
  DevPool* d = pool_of(dev);
  if (!d) throw Error(HPRQP_E_CUDA, "cannot create the device memory pool");
  void* p = nullptr;
  const size_t b = bytes < 16 ? 16 : bytes;
  if (cudaMallocFromPoolAsync(&p, b, d->pool, d->st) != cudaSuccess) {
    // out of memory: return the pool's unused reserve to the driver, then retry once
    cudaGetLastError();
    cudaStreamSynchronize(d->st);
    cudaMemPoolTrimTo(d->pool, 0);
    HPRQP_CUDA(cudaMallocFromPoolAsync(&p, b, d->pool, d->st));
  }
  HPRQP_CUDA(cudaStreamSynchronize(d->st));
  return p;
}

void pool_free(std::vector<void*>& blocks, int dev) {
  if (blocks.empty()) return;
  int cur = -1;
  cudaGetDevice(&cur);
  if (dev >= 0 && dev != cur) cudaSetDevice(dev);
  DevPool* d = pool_of(dev >= 0 ? dev : cur);
  cudaDeviceSynchronize();
  for (void* p : blocks)
    if (d) cudaFreeAsync(p, d->st);
  if (d) cudaStreamSynchronize(d->st);
  blocks.clear();
  if (dev >= 0 && dev != cur && cur >= 0) cudaSetDevice(cur);
}

namespace {
std::mutex g_pin_mu;
std::vector<std::pair<size_t, void*>> g_pinned;  // free pinned buffers by size
}  // namespace

void* pinned_take(size_t bytes) {
  {
    std::lock_guard<std::mutex> lk(g_pin_mu);
    for (size_t i = 0; i < g_pinned.size(); ++i)
      if (g_pinned[i].first == bytes) {
        void* p = g_pinned[i].second;
        g_pinned.erase(g_pinned.begin() + (long)i);
        return p;
      }
  }
  void* p = nullptr;
  HPRQP_CUDA(cudaMallocHost(&p, bytes));
  return p;
}

void pinned_give(void* p, size_t bytes) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(g_pin_mu);
  g_pinned.emplace_back(bytes, p);
}

void* PoolBlocks::get(size_t bytes) {
  if (dev < 0) HPRQP_CUDA(cudaGetDevice(&dev));
  void* p = pool_alloc(bytes);
  blocks.push_back(p);
  return p;
}

}  // namespace hprqp
