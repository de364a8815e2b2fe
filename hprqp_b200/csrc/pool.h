// pool.h — device memory of the library's engines and batches.
//
// Every device block the library owns comes from one stream-ordered memory
// pool per GPU (cudaMemPoolCreate), whose release threshold keeps freed
// memory mapped for the process: a handle that is destroyed and a new one
// built for the next problem (the load -> solve -> destroy cycle of a caller
// that solves many problems) reuse the physical pages instead of paying
// cudaMalloc / cudaFree (page mapping, unmapping and an implicit device
// synchronisation) for every block.  The pool keeps what it has reserved
// (at most the peak of the blocks in use at once); an allocation that finds
// the device full first returns the pool's unused reserve to the driver and
// retries.  HPRQP_POOL_KEEP_MB caps the reserve kept across frees instead.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

namespace hprqp {

// A block of `bytes` (at least 16) on the current device, usable on any
// stream once this returns.  Throws Error(HPRQP_E_CUDA) when out of memory.
void* pool_alloc(size_t bytes);

// Return blocks allocated on device `dev`.  Waits for the device first (no
// kernel of ours may still use them), never throws; clears the list.
void pool_free(std::vector<void*>& blocks, int dev);

// Pinned host buffers, kept for the process once allocated: a handle's
// scalar mirror is taken from this list and given back at destroy, since
// cudaFreeHost synchronises the device and measured up to a second here.
void* pinned_take(size_t bytes);
void pinned_give(void* p, size_t bytes);

// Host blocks for the library's large host arrays: 2 MiB-aligned, advised
// for transparent huge pages, registered with the driver (page-locked, so
// that copies to and from them run as one DMA at the link's rate), and kept
// by the process once given back, so that the arrays of the next problem
// (the load -> solve -> destroy cycle) reuse pages that are mapped, faulted
// in and registered already.  A request takes the smallest kept block of at
// least its size and at most 1.25 times it, else maps a new one.  At most
// HPRQP_HOST_KEEP_MB (default 4096) MiB of free blocks are kept; the rest go
// back to the system.  HPRQP_HOST_PIN=0 leaves new blocks pageable.  Throws
// std::bad_alloc when out of memory.
void* host_take(size_t bytes);
void host_give(void* p);
// Whether [p, p + bytes) lies in one registered block handed out by host_take.
bool host_pinned(const void* p, size_t bytes);

// Host -> device copy of `bytes` from pageable memory, enqueued on `st`:
// copies of 1 MiB and more go through two pinned 8 MiB chunks, each filled
// by the host threads while the other one's DMA runs (a plain copy from
// pageable memory is staged by one thread); from a registered host block
// (host_pinned) the copy is one DMA.  `src` may be reused on return; the
// copy completes in stream order.
void h2d_staged(void* dst, const void* src, size_t bytes, cudaStream_t st);
// Device -> host copy of `bytes` into pageable memory, the mirror image: the
// DMA of each 8 MiB chunk into a pinned buffer runs while the host threads
// copy the previous chunk out (one DMA into a registered host block).
// Synchronous: `dst` holds the data on return.
void d2h_staged(void* dst, const void* src, size_t bytes, cudaStream_t st);

// Owner of a list of pool blocks of one device, freed together.
struct PoolBlocks {
  std::vector<void*> blocks;
  int dev = -1;
  void* get(size_t bytes);
  ~PoolBlocks() { pool_free(blocks, dev); }
};

}  // namespace hprqp
