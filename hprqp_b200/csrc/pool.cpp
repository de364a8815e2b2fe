// pool.cpp — the per-GPU memory pool behind every device block of the
// library (see pool.h).
#include "pool.h"

#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <unordered_map>

#include <sys/mman.h>

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

namespace {
struct HostBlock {
  size_t size;
  bool pinned;  // registered with the driver: copies DMA from / to it directly
  bool live;
};
std::mutex g_host_mu;
std::map<char*, HostBlock> g_host_blocks;  // every block, handed out or kept
std::multimap<size_t, char*> g_host_free;  // kept blocks by size
size_t g_host_kept = 0;
size_t host_keep_limit() {
  static const size_t lim = [] {
    size_t mb = 4096;
    if (const char* e = std::getenv("HPRQP_HOST_KEEP_MB")) mb = (size_t)std::strtoull(e, nullptr, 10);
    return mb << 20;
  }();
  return lim;
}
bool host_pin_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("HPRQP_HOST_PIN");
    return !(e && e[0] == '0');
  }();
  return on;
}
constexpr size_t kHostPage = size_t(2) << 20;
}  // namespace

void* host_take(size_t bytes) {
  const size_t want = (std::max<size_t>(bytes, 1) + kHostPage - 1) / kHostPage * kHostPage;
  {
    std::lock_guard<std::mutex> lk(g_host_mu);
    auto it = g_host_free.lower_bound(want);
    if (it != g_host_free.end() && it->first <= want + want / 4) {
      char* p = it->second;
      g_host_kept -= it->first;
      g_host_free.erase(it);
      g_host_blocks[p].live = true;
      return p;
    }
  }
  char* p = static_cast<char*>(std::aligned_alloc(kHostPage, want));
  if (!p) throw std::bad_alloc();
  madvise(p, want, MADV_HUGEPAGE);  // a hint: without transparent huge pages the pages stay 4 KiB
  // registration faults the pages in once (measured 3 ms per 100 MB with
  // huge pages) and lets copies run at the link's rate (55 against 20 GB/s
  // through the pinned chunks); without a device it fails and the block
  // stays pageable
  bool pinned = false;
  if (host_pin_enabled()) {
    pinned = cudaHostRegister(p, want, cudaHostRegisterPortable) == cudaSuccess;
    if (!pinned) cudaGetLastError();
  }
  std::lock_guard<std::mutex> lk(g_host_mu);
  g_host_blocks[p] = HostBlock{want, pinned, true};
  return p;
}

void host_give(void* ptr) {
  if (!ptr) return;
  char* p = static_cast<char*>(ptr);
  std::unique_lock<std::mutex> lk(g_host_mu);
  auto it = g_host_blocks.find(p);
  if (it == g_host_blocks.end() || !it->second.live) return;  // not a block of ours
  const HostBlock b = it->second;
  if (g_host_kept + b.size > host_keep_limit()) {
    g_host_blocks.erase(it);
    lk.unlock();
    if (b.pinned) cudaHostUnregister(p);
    std::free(p);
    return;
  }
  it->second.live = false;
  g_host_kept += b.size;
  g_host_free.emplace(b.size, p);
}

bool host_pinned(const void* ptr, size_t bytes) {
  const char* p = static_cast<const char*>(ptr);
  std::lock_guard<std::mutex> lk(g_host_mu);
  auto it = g_host_blocks.upper_bound(const_cast<char*>(p));
  if (it == g_host_blocks.begin()) return false;
  --it;
  return it->second.pinned && it->second.live && p + bytes <= it->first + it->second.size;
}

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

void h2d_staged(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  constexpr size_t kChunk = 8u << 20;
  // small (the driver stages pageable memory before returning), or from a
  // registered host block: one DMA, done before `src` may change
  const bool pinned = host_pinned(src, bytes);
  if (bytes < (1u << 20) || pinned) {
    if (bytes) HPRQP_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    if (bytes && pinned) HPRQP_CUDA(cudaStreamSynchronize(st));
    return;
  }
  char* buf[2] = {(char*)pinned_take(kChunk), (char*)pinned_take(kChunk)};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  bool used[2] = {false, false};
  try {
    for (int b = 0; b < 2; ++b) HPRQP_CUDA(cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming));
    const char* s = (const char*)src;
    char* d = (char*)dst;
    int b = 0;
    for (size_t off = 0; off < bytes; off += kChunk, b ^= 1) {
      const size_t len = std::min(kChunk, bytes - off);
      if (used[b]) HPRQP_CUDA(cudaEventSynchronize(ev[b]));  // the chunk's previous DMA has read it
      const int nt = std::max(1, std::min(16, omp_get_max_threads()));
#pragma omp parallel for schedule(static) num_threads(nt)
      for (int t = 0; t < nt; ++t) {
        const size_t a = len * (size_t)t / (size_t)nt, e = len * (size_t)(t + 1) / (size_t)nt;
        if (e > a) std::memcpy(buf[b] + a, s + off + a, e - a);
      }
      HPRQP_CUDA(cudaMemcpyAsync(d + off, buf[b], len, cudaMemcpyHostToDevice, st));
      HPRQP_CUDA(cudaEventRecord(ev[b], st));
      used[b] = true;
    }
    for (int k = 0; k < 2; ++k)
      if (used[k]) HPRQP_CUDA(cudaEventSynchronize(ev[k]));  // the chunks go back to the free list
  } catch (...) {
    for (int k = 0; k < 2; ++k)
      if (ev[k]) {
        cudaEventSynchronize(ev[k]);
        cudaEventDestroy(ev[k]);
      }
    pinned_give(buf[0], kChunk);
    pinned_give(buf[1], kChunk);
    throw;
  }
  for (int k = 0; k < 2; ++k) cudaEventDestroy(ev[k]);
  pinned_give(buf[0], kChunk);
  pinned_give(buf[1], kChunk);
}

void d2h_staged(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  constexpr size_t kChunk = 8u << 20;
  if (bytes < (1u << 20) || host_pinned(dst, bytes)) {  // small, or a registered host block: one DMA
    if (bytes) {
      HPRQP_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
      HPRQP_CUDA(cudaStreamSynchronize(st));
    }
    return;
  }
  char* buf[2] = {(char*)pinned_take(kChunk), (char*)pinned_take(kChunk)};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  auto out = [&](int b, size_t off, size_t len) {  // pinned chunk b -> dst + off
    const int nt = std::max(1, std::min(16, omp_get_max_threads()));
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int t = 0; t < nt; ++t) {
      const size_t a = len * (size_t)t / (size_t)nt, e = len * (size_t)(t + 1) / (size_t)nt;
      if (e > a) std::memcpy((char*)dst + off + a, buf[b] + a, e - a);
    }
  };
  try {
    for (int b = 0; b < 2; ++b) HPRQP_CUDA(cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming));
    size_t prev_off = 0, prev_len = 0;
    int b = 0;
    for (size_t off = 0; off < bytes; off += kChunk, b ^= 1) {
      const size_t len = std::min(kChunk, bytes - off);
      HPRQP_CUDA(cudaMemcpyAsync(buf[b], (const char*)src + off, len, cudaMemcpyDeviceToHost, st));
      HPRQP_CUDA(cudaEventRecord(ev[b], st));
      if (prev_len) {  // the previous chunk, whose DMA was enqueued before this one
        HPRQP_CUDA(cudaEventSynchronize(ev[b ^ 1]));
        out(b ^ 1, prev_off, prev_len);
      }
      prev_off = off;
      prev_len = len;
    }
    HPRQP_CUDA(cudaEventSynchronize(ev[b ^ 1]));
    out(b ^ 1, prev_off, prev_len);
  } catch (...) {
    for (int k = 0; k < 2; ++k)
      if (ev[k]) {
        cudaEventSynchronize(ev[k]);
        cudaEventDestroy(ev[k]);
      }
    pinned_give(buf[0], kChunk);
    pinned_give(buf[1], kChunk);
    throw;
  }
  for (int k = 0; k < 2; ++k) cudaEventDestroy(ev[k]);
  pinned_give(buf[0], kChunk);
  pinned_give(buf[1], kChunk);
}

void* PoolBlocks::get(size_t bytes) {
  if (dev < 0) HPRQP_CUDA(cudaGetDevice(&dev));
  void* p = pool_alloc(bytes);
  blocks.push_back(p);
  return p;
}

}  // namespace hprqp
