// kernels.cuh — sm_100a kernels of the HPR-QP iteration engine.
//
// Every iteration pass is ONE kernel: a CSR row product (TPR threads per
// row, shuffle-reduced) whose per-row epilogue applies the projection /
// prox / Halpern update of the reference's fused update kernels
// (src/kernels.jl:261-1426).  The epilogues follow the reference CPU loops
// (src/kernels.jl:2115-2832) expression by expression; `fma` stands where
// the reference writes `muladd`.  Epilogue arithmetic is FP64; `V` is the
// storage type of vectors and matrix values (double, or float in the FP32
// phase); the Halpern anchors (last_*) are stored as V in the engines
// (every value they take is a V iterate) and as FP64 in the batch engines.
//
// Reductions (KKT residuals, M-norm, sigma statistics, power method) are
// single-pass: per-CTA shuffle/shared reduction, per-CTA partials, and the
// last CTA to finish (atomic ticket) folds the partials in a fixed order, so
// results are deterministic and stay on the device.
#pragma once

#include <type_traits>
#include <utility>

#include "common.cuh"

namespace hprqp {

// ---------------------------------------------------------------------------
// Row sources: what the per-row accumulator is
// ---------------------------------------------------------------------------
template <typename V, typename X>
struct CsrSrc {  // (M x)_row with M in CSR
  const int* __restrict__ ptr;
  const int* __restrict__ col;
  const V* __restrict__ val;
  const X* __restrict__ x;
  template <int TPR, typename Acc>
  __device__ __forceinline__ Acc dot(int row, int lane) const {
    const int b = __ldg(ptr + row), e = __ldg(ptr + row + 1);
    Acc s = Acc(0);
#pragma unroll 4
    for (int k = b + lane; k < e; k += TPR) s = fma((Acc)__ldg(val + k), (Acc)__ldg(x + __ldg(col + k)), s);
    return group_sum<TPR>(s);
  }
};

template <typename V, typename X>
struct SellSrc {  // (M x)_row with M in SELL-32, one thread per row
  const int* __restrict__ sptr;
  const int* __restrict__ ptr;
  const int* __restrict__ col;
  const V* __restrict__ val;
  const X* __restrict__ x;
  template <int TPR, typename Acc>
  __device__ __forceinline__ Acc dot(int row, int) const {
    const int len = __ldg(ptr + row + 1) - __ldg(ptr + row);
    const int base = __ldg(sptr + (row >> 5)) + (row & 31);
    Acc s = Acc(0);
#pragma unroll 4
    for (int k = 0; k < len; ++k)
      s = fma((Acc)__ldg(val + base + 32 * k), (Acc)__ldg(x + __ldg(col + base + 32 * k)), s);
    return s;
  }
};

template <typename V, typename X>
struct EllSrc {  // (M x)_row with M in ELL (width w, column-major), one thread per row
  const int* __restrict__ col;
  const V* __restrict__ val;
  const X* __restrict__ x;
  int rows, w;
  template <int TPR, typename Acc>
  __device__ __forceinline__ Acc dot(int row, int) const {
    Acc s = Acc(0);
    const int* c = col + row;
    const V* v = val + row;
#pragma unroll 4
    for (int k = 0; k < w; ++k) s = fma((Acc)__ldg(v + (size_t)k * rows), (Acc)__ldg(x + __ldg(c + (size_t)k * rows)), s);
    return s;
  }
};

template <typename V>
struct VecSrc {  // precomputed product (operator Q)
  const V* __restrict__ v;
  template <int TPR, typename Acc>
  __device__ __forceinline__ Acc dot(int row, int) const { return (Acc)v[row]; }
};

struct ZeroSrc {
  template <int TPR, typename Acc>
  __device__ __forceinline__ Acc dot(int, int) const { return Acc(0); }
};

__device__ __forceinline__ double clampd(double v, double lo, double hi) { return fmin(fmax(v, lo), hi); }

// ---------------------------------------------------------------------------
// Generic row kernels
// ---------------------------------------------------------------------------
// Epilogue operand prefetch: an epilogue may declare prefetch(i, level)
// naming the vectors its row i reads; level 1 = into L1, 2 = into L2.
template <typename E, typename = void>
struct HasPrefetch : std::false_type {};
template <typename E>
struct HasPrefetch<E, std::void_t<decltype(std::declval<const E&>().prefetch(0, 1))>> : std::true_type {};

__device__ __forceinline__ void pf_line(const void* p, int level) {
  if (level == 1) asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
  else asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}
template <typename... P>
__device__ __forceinline__ void pf_rows(int i, int level, const P*... p) {
  (pf_line(p + i, level), ...);
}

template <int TPR, typename Acc, typename Src, typename Epi>
__global__ void __launch_bounds__(kBlock) k_row_pass(int nrows, Src src, Epi epi, int pf = 0) {
  pdl_enter();
  const long long g = (long long)blockIdx.x * kBlock + threadIdx.x;
  const int row = (int)(g / TPR);
  if (row >= nrows) return;  // whole row groups leave together
  const int lane = threadIdx.x & (TPR - 1);
  // the epilogue's own operands do not depend on the row's product: ask for
  // them before the dependent col -> x gathers, so their latency overlaps
  if constexpr (HasPrefetch<Epi>::value)
    if (pf && lane == 0) epi.prefetch(row, pf);
  const Acc acc = src.template dot<TPR, Acc>(row, lane);
  if (lane == 0) epi(row, acc);
}

// An epilogue may split off `Pre pre(i)`: the operands of row i that are
// constant over a solve (problem data written at set-up), and take them back
// in operator()(i, acc, pre).  k_ell_pass loads them before it waits on the
// previous kernel.
template <typename E, typename = void>
struct HasPre : std::false_type {};
template <typename E>
struct HasPre<E, std::void_t<typename E::Pre>> : std::true_type {};

// ELL pass (one thread per row, width w <= WMAX) whose constant loads come
// before the wait on the previous kernel.  Passes are launched with
// programmatic dependent launch: CTAs of this pass become resident while the
// previous pass drains, and here they already stream their rows' column
// indices and values (constant over a solve) and the epilogue's constant
// operands; only the gathers of the input vector and the epilogue's other
// operands wait for the previous pass's writes.  Same products, same order
// of summation as EllSrc::dot.
template <int WMAX, typename Acc, typename V, typename X, typename Epi>
__global__ void __launch_bounds__(kBlock) k_ell_pass(int nrows, EllSrc<V, X> src, Epi epi, int with_pre) {
  const int row = blockIdx.x * kBlock + threadIdx.x;
  const bool live = row < nrows;
  int c[WMAX];
  V v[WMAX];
  if (live) {
#pragma unroll
    for (int k = 0; k < WMAX; ++k)
      if (k < src.w) {
        c[k] = __ldg(src.col + (size_t)k * src.rows + row);
        v[k] = __ldg(src.val + (size_t)k * src.rows + row);
      }
  }
  if constexpr (HasPre<Epi>::value) {
    typename Epi::Pre pre{};
    if (live && with_pre) pre = epi.pre(row);
    pdl_enter();
    if (!live) return;
    Acc s = Acc(0);
#pragma unroll
    for (int k = 0; k < WMAX; ++k)
      if (k < src.w) s = fma((Acc)v[k], (Acc)__ldg(src.x + c[k]), s);
    if (!with_pre) pre = epi.pre(row);
    epi(row, s, pre);
  } else {
    pdl_enter();
    if (!live) return;
    Acc s = Acc(0);
#pragma unroll
    for (int k = 0; k < WMAX; ++k)
      if (k < src.w) s = fma((Acc)v[k], (Acc)__ldg(src.x + c[k]), s);
    epi(row, s);
  }
}

// Row-split pass (DCsr::split): one warp per piece of a row, pieces in the
// order of the schedule (heaviest first, so the long rows of a heavy-tailed
// matrix start at once instead of finishing last).  A whole row runs its
// epilogue at once; the pieces of a split row store their partial sums, and
// the last one to arrive (atomic counter) folds them in piece order, resets
// the counter and runs the epilogue, so results do not depend on timing.
template <typename Acc, typename V, typename X, typename Epi>
__global__ void __launch_bounds__(kBlock) k_split_pass(int npieces, const int4* __restrict__ pieces,
                                                       const int* __restrict__ ptr, const int* __restrict__ col,
                                                       const V* __restrict__ val, const X* __restrict__ x,
                                                       const int2* __restrict__ srow, int T,
                                                       double* __restrict__ part, unsigned* __restrict__ cnt,
                                                       Epi epi) {
  const int wid = (int)((blockIdx.x * kBlock + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  int4 pc = make_int4(0, 0, 0, -1);
  if (wid < npieces) pc = __ldg(pieces + wid);  // the schedule is constant: before the wait
  pdl_enter();
  if (wid >= npieces) return;
  Acc s = Acc(0);
#pragma unroll 4
  for (int k = pc.y + lane; k < pc.z; k += 32) s = fma((Acc)__ldg(val + k), (Acc)__ldg(x + __ldg(col + k)), s);
  s = group_sum<32>(s);
  if (lane != 0) return;
  if (pc.w < 0) {
    epi(pc.x, s);
    return;
  }
  const int2 sr = __ldg(srow + pc.w);
  const int j = (pc.y - __ldg(ptr + pc.x)) / T;
  part[sr.x + j] = (double)s;
  __threadfence();
  const unsigned arrived = atomicAdd(cnt + pc.w, 1u);
  if (arrived == (unsigned)(sr.y - 1)) {
    __threadfence();
    Acc t = Acc(0);
    for (int q = 0; q < sr.y; ++q) t += (Acc)__ldcg(part + sr.x + q);
    cnt[pc.w] = 0u;
    epi(pc.x, t);
  }
}

// ---------------------------------------------------------------------------
// Staged pass (DCsr::stage): the input vector's column block sits in shared
// memory, so the gathers cost a shared-memory access (a few bank conflicts)
// instead of one L1 wavefront per lane; the matrix streams as 16-byte
// loads of 8 16-bit columns and 8 values per lane.
// ---------------------------------------------------------------------------
template <typename V>
struct StageView {
  int rows, cols, bw, nblk;
  const uint16_t* __restrict__ col;
  const V* __restrict__ val;
  const int2* __restrict__ wt;    // per 32-chunk warp tile {first slot, segment-head mask}
  const int4* __restrict__ tile;  // {first warp tile, chunks, first row, end row}
  const int4* __restrict__ item;  // per CTA {block, first tile, end tile, 0}
  const int* __restrict__ srow;   // nblk x (rows + 1): first slot of each row
  double* __restrict__ part;      // nblk x rows block sums (nblk > 1)
  unsigned* __restrict__ cnt;     // per-row arrivals (nblk > 1)
};

// Chunk c = 32 g + l (lane l of warp tile g) of the staged copy in registers:
// 8 16-bit columns (two per word; the 32 chunks of a warp tile are 512
// contiguous bytes) and 8 values, stored lane-interleaved in 16-byte slices
// (slice q of the 32 lanes contiguous), so every load of a warp reads 512
// contiguous bytes.
template <typename V>
struct StageChunk {
  uint4 c;
  V v[8];
};

template <typename V>
__device__ __forceinline__ void stage_load(StageChunk<V>& k, const uint16_t* __restrict__ col,
                                           const V* __restrict__ val, int64_t g, int l) {
  k.c = __ldg(reinterpret_cast<const uint4*>(col) + g * 32 + l);
  if constexpr (sizeof(V) == 4) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(val) + (g * 2 + 0) * 32 + l);
    const float4 b = __ldg(reinterpret_cast<const float4*>(val) + (g * 2 + 1) * 32 + l);
    k.v[0] = a.x; k.v[1] = a.y; k.v[2] = a.z; k.v[3] = a.w; k.v[4] = b.x; k.v[5] = b.y; k.v[6] = b.z; k.v[7] = b.w;
  } else {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double2 a = __ldg(reinterpret_cast<const double2*>(val) + (g * 4 + q) * 32 + l);
      k.v[2 * q] = a.x;
      k.v[2 * q + 1] = a.y;
    }
  }
}

// Bulk prefetch of warp tile g (its 512 bytes of columns and 256 values)
// into L2: the loads of the warp's next step then wait for L2, not HBM, and
// no register holds the data in flight.
template <typename V>
__device__ __forceinline__ void stage_prefetch(const uint16_t* col, const V* val, int64_t g) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(col + g * 256), "r"(512u) : "memory");
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(val + g * 256), "r"((unsigned)(256 * sizeof(V)))
               : "memory");
}

// Sum of the chunk's 8 products val[k] * xs[col[k]], in entry order.
template <typename Acc, typename V, typename X>
__device__ __forceinline__ Acc stage_dot(const StageChunk<V>& k, const X* xs) {
  const unsigned idx[4] = {k.c.x, k.c.y, k.c.z, k.c.w};
  Acc s = Acc(0);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    s = fma((Acc)k.v[2 * q], (Acc)xs[idx[q] & 0xffffu], s);
    s = fma((Acc)k.v[2 * q + 1], (Acc)xs[idx[q] >> 16], s);
  }
  return s;
}

// Row r's sum over block b: the epilogue at once with one block; else the
// block sum is stored and the last block to arrive folds the sums in block
// order, resets the row's counter and runs the epilogue.
template <typename Acc, typename V, typename Epi>
__device__ __forceinline__ void stage_finish(const StageView<V>& s, int b, int r, Acc v, const Epi& epi) {
  if (s.nblk == 1) {
    epi(r, v);
    return;
  }
  s.part[(size_t)b * s.rows + r] = (double)v;
  __threadfence();
  const unsigned a = atomicAdd(s.cnt + r, 1u);
  if (a == (unsigned)(s.nblk - 1)) {
    __threadfence();
    Acc t = Acc(0);
    for (int q = 0; q < s.nblk; ++q) t += (Acc)__ldcg(s.part + (size_t)q * s.rows + r);
    s.cnt[r] = 0u;
    epi(r, t);
  }
}

// Threads of a staged-pass CTA (32 warps), and warp tiles a warp keeps in
// flight: two in FP32; one in FP64, whose chunks take twice the registers
// (two with 24 warps and 80 registers measured slower).
template <typename V>
__host__ __device__ constexpr int stage_block() { return 1024; }
template <typename V>
__host__ __device__ constexpr int stage_unroll() { return sizeof(V) == 8 ? 1 : 2; }

// One CTA per SM (one wave).  CTA i stages block b = item[i].x of the input
// into shared memory and runs its tiles [item.y, item.z) one after another,
// each in two phases.  Phase 1: a tile's chunks [C0, C1) (C0 = 32 x its
// first warp tile) are cut into warp tiles of 32 chunks; warp k takes warp
// tiles k, k + NW, ... (two at a time in FP32, their loads in flight
// together); lane l sums chunk l, and a segmented scan over the warp tile's
// segment heads (row starts, and lane 0 where a row continues from the
// previous warp tile) leaves each segment's sum in its last lane, which
// stores it in the segment's shared-memory slot.
// Phase 2: one thread per row of the tile (consecutive rows, so the
// epilogue's accesses coalesce) folds the row's slots in order and finishes
// the row.  Every lane but the tile's last warp tile's tail has a chunk, no
// epilogue latency stalls the streaming phase, and every sum runs in a fixed
// order.  The first tile's first loads (constant data) are issued before the
// wait on the previous kernel, and every step prefetches the warp's next
// step into L2.
template <typename Acc, typename V, typename X, typename Epi>
__global__ void __launch_bounds__(stage_block<V>(), 1) k_stage_pass(StageView<V> s, const X* __restrict__ x, Epi epi) {
  extern __shared__ __align__(16) unsigned char stage_smem[];
  Acc* sums = reinterpret_cast<Acc*>(stage_smem);
  X* xs = reinterpret_cast<X*>(stage_smem + kStageSlots * sizeof(Acc));
  constexpr int NT = stage_block<V>(), NW = NT / 32;
  constexpr int U = stage_unroll<V>();  // warp tiles per step
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int4 it = __ldg(s.item + blockIdx.x);  // the schedule and the matrix are constant: before the wait
  const int b = it.x;
  const int* srow = s.srow + (size_t)b * (s.rows + 1);
  int t = it.y;
  int4 tl = make_int4(0, 0, 0, 0);
  int C0 = 0, C1 = 0, k = warp;
  StageChunk<V> ck[U];
  int2 d[U];
  auto load_step = [&]() {  // warp tiles k + u NW of tile tl; the next step's into L2
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int wt = k + u * NW;
      d[u] = C0 + 32 * wt < C1 ? __ldg(s.wt + tl.x + wt) : make_int2(0, 0);
      if (C0 + 32 * wt + lane < C1) stage_load(ck[u], s.col, s.val, (int64_t)tl.x + wt, lane);
    }
    if (lane == 0) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int wt = k + (U + u) * NW;
        if (C0 + 32 * wt < C1) stage_prefetch(s.col, s.val, (int64_t)tl.x + wt);
      }
    }
  };
  if (t < it.z) {
    tl = __ldg(s.tile + t);
    C0 = 32 * tl.x;
    C1 = C0 + tl.y;
    load_step();
  }
  pdl_enter();
  const int c0 = b * s.bw;
  const int len = min(s.bw, s.cols - c0);
  const X* src = x + c0;
  if ((reinterpret_cast<uintptr_t>(src) & 15u) == 0) {
    constexpr int P = 16 / (int)sizeof(X);
    const int nv = len / P;
    for (int q = threadIdx.x; q < nv; q += NT)
      reinterpret_cast<uint4*>(xs)[q] = __ldg(reinterpret_cast<const uint4*>(src) + q);
    for (int q = nv * P + threadIdx.x; q < len; q += NT) xs[q] = __ldg(src + q);
  } else {
    for (int q = threadIdx.x; q < len; q += NT) xs[q] = __ldg(src + q);
  }
  __syncthreads();
  for (; t < it.z;) {
    const int slot0 = __ldg(srow + tl.z);
    const int nwt = (C1 - C0 + 31) / 32;
    while (k < nwt) {
      Acc v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {  // every gather before any slot store
        v[u] = C0 + 32 * (k + u * NW) + lane < C1 ? stage_dot<Acc>(ck[u], xs) : Acc(0);
      }
      unsigned f[U], heads[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        heads[u] = (unsigned)d[u].y;  // bit l: chunk l starts a segment
        f[u] = (heads[u] >> lane) & 1u;  // my segment's head is inside the lanes summed so far
      }
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const Acc o = __shfl_up_sync(0xffffffffu, v[u], off);
          const unsigned fo = __shfl_up_sync(0xffffffffu, f[u], off);
          if (lane >= off) {
            if (!f[u]) v[u] += o;
            f[u] |= fo;
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int base = 32 * (k + u * NW);
        const int last = min(31, C1 - C0 - base - 1);  // (negative: no such warp tile)
        if (lane <= last && (lane == last || ((heads[u] >> (lane + 1)) & 1u)))
          sums[d[u].x - slot0 + __popc(heads[u] & (0xffffffffu >> (31 - lane))) - 1] = v[u];
      }
      k += U * NW;
      if (k < nwt) load_step();
    }
    __syncthreads();
    for (int r = tl.z + (int)threadIdx.x; r < tl.w; r += NT) {
      const int a = __ldg(srow + r) - slot0, e = __ldg(srow + r + 1) - slot0;
      Acc acc = sums[a];
      for (int q = a + 1; q < e; ++q) acc += sums[q];
      stage_finish(s, b, r, acc, epi);
    }
    __syncthreads();  // the slots are the next tile's
    if (++t < it.z) {
      tl = __ldg(s.tile + t);
      C0 = 32 * tl.x;
      C1 = C0 + tl.y;
      k = warp;
      load_step();
    }
  }
}

// Block reduction of K slots; MaxMask bit k selects max (else sum).
// Result valid in thread 0.
template <int K, unsigned MaxMask>
__device__ __forceinline__ void block_reduce(double (&r)[K]) {
  __shared__ double sh[K][kBlock / 32];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double v = r[k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double o = __shfl_down_sync(0xffffffffu, v, off);
      v = ((MaxMask >> k) & 1u) ? fmax(v, o) : v + o;
    }
    if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double v = threadIdx.x < kBlock / 32 ? sh[k][threadIdx.x] : (((MaxMask >> k) & 1u) ? 0.0 : 0.0);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double o = __shfl_down_sync(0xffffffffu, v, off);
        v = ((MaxMask >> k) & 1u) ? fmax(v, o) : v + o;
      }
      r[k] = v;
    }
  }
  __syncthreads();
}

constexpr int kMaxReduceGrid = 1184;   // default cap of reduction grids: 8 CTAs per SM on 148 SMs
constexpr int kReduceGridLimit = 8192;  // largest cap the engine's partials buffers hold

// Grid of a grid-stride reduction: the fewest CTAs (<= kMaxReduceGrid) that
// give every thread the same number of row groups, so the last sweep is not
// left to a fraction of the threads.
inline int reduce_grid(long long nrows, int tpr, int max_grid = kMaxReduceGrid) {
  const long long threads = (nrows > 0 ? nrows : 1) * tpr;
  const long long cap = (long long)max_grid * kBlock;
  const long long per = (threads + cap - 1) / cap;           // row groups per thread
  const long long grid = (threads + (long long)kBlock * per - 1) / ((long long)kBlock * per);
  return (int)(grid < 1 ? 1 : grid);
}

struct ReduceWs {  // partials (one K-vector per CTA) + ticket counter
  double* partials;
  unsigned* counter;
};

struct NoFin {
  template <int K>
  __device__ __forceinline__ void operator()(const double (&)[K]) const {}
};

// Fold per-CTA partials in the last CTA; write K results to out, then let
// `fin` (thread 0 of the last CTA) derive further scalars from them.
template <int K, unsigned MaxMask, typename Fin = NoFin>
__device__ __forceinline__ void grid_finish(double (&r)[K], ReduceWs ws, double* out, Fin fin = Fin()) {
  __shared__ bool am_last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) ws.partials[(size_t)blockIdx.x * K + k] = r[k];
    __threadfence();
    const unsigned t = atomicAdd(ws.counter, 1u);
    am_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; ++k) acc[k] = 0.0;
  // the partials are read in batches of kFold CTAs per thread, all loads of
  // a batch issued before any is consumed; they are still combined in
  // increasing CTA order, so the result does not depend on the batching
  constexpr int kFold = 4;
  for (int b0 = threadIdx.x; b0 < (int)gridDim.x; b0 += kFold * kBlock) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double v[kFold];
#pragma unroll
      for (int q = 0; q < kFold; ++q) {
        const int b = b0 + q * kBlock;
        v[q] = b < (int)gridDim.x ? __ldcg(ws.partials + (size_t)b * K + k) : 0.0;
      }
#pragma unroll
      for (int q = 0; q < kFold; ++q)
        if (b0 + q * kBlock < (int)gridDim.x) acc[k] = ((MaxMask >> k) & 1u) ? fmax(acc[k], v[q]) : acc[k] + v[q];
    }
  }
  block_reduce<K, MaxMask>(acc);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) out[k] = acc[k];
    fin(acc);
    *ws.counter = 0u;
  }
}

// Row product + epilogue that also contributes to K reduction slots.
// Grid-stride over rows; the grid is capped so the partials stay small.
template <int TPR, int K, unsigned MaxMask, typename Acc, typename Src, typename Epi, typename Fin = NoFin>
__global__ void __launch_bounds__(kBlock) k_row_reduce(int nrows, Src src, Epi epi, ReduceWs ws,
                                                       double* out, Fin fin = Fin()) {
  pdl_enter();
  double r[K];
#pragma unroll
  for (int k = 0; k < K; ++k) r[k] = 0.0;
  const int lane = threadIdx.x & (TPR - 1);
  const int rows_per_grid = (int)(gridDim.x * (kBlock / TPR));
  for (int row = (int)((blockIdx.x * kBlock + threadIdx.x) / TPR); row < nrows; row += rows_per_grid) {
    const Acc acc = src.template dot<TPR, Acc>(row, lane);
    if (lane == 0) epi(row, acc, r);
  }
  block_reduce<K, MaxMask>(r);
  grid_finish<K, MaxMask, Fin>(r, ws, out, fin);
}

// The same fused product + reduction for an ELL matrix with R rows per
// thread in flight (rows r0 + q * stride, so a warp's loads stay
// coalesced): the col -> x gathers of R rows overlap instead of running one
// row after another as in the grid-stride loop above.
template <int R, int K, unsigned MaxMask, typename Acc, typename V, typename X, typename Epi, typename Fin = NoFin>
__global__ void __launch_bounds__(kBlock) k_ell_reduce(int nrows, EllSrc<V, X> src, Epi epi, ReduceWs ws,
                                                       double* out, Fin fin = Fin()) {
  pdl_enter();
  double r[K];
#pragma unroll
  for (int k = 0; k < K; ++k) r[k] = 0.0;
  const int stride = (int)(gridDim.x * kBlock);
  for (int r0 = (int)(blockIdx.x * kBlock + threadIdx.x); r0 < nrows; r0 += R * stride) {
    Acc acc[R];
#pragma unroll
    for (int q = 0; q < R; ++q) acc[q] = Acc(0);
    for (int k = 0; k < src.w; ++k) {
      const int* c = src.col + (size_t)k * src.rows;
      const V* v = src.val + (size_t)k * src.rows;
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int row = r0 + q * stride;
        if (row < nrows) acc[q] = fma((Acc)__ldg(v + row), (Acc)__ldg(src.x + __ldg(c + row)), acc[q]);
      }
    }
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int row = r0 + q * stride;
      if (row < nrows) epi(row, acc[q], r);
    }
  }
  block_reduce<K, MaxMask>(r);
  grid_finish<K, MaxMask, Fin>(r, ws, out, fin);
}

// ---------------------------------------------------------------------------
// Epilogues of the iteration passes
// ---------------------------------------------------------------------------

// Plain product: y = scale * (M x)
template <typename V>
struct EpiStore {
  V* __restrict__ y;
  double scale;
  __device__ __forceinline__ void operator()(int i, double acc) const { y[i] = (V)(scale * acc); }
  __device__ __forceinline__ void operator()(int i, float acc) const { y[i] = (V)(scale * (double)acc); }
};

// QP step 1: Qw = Q w fused with update_zxw1_cpu! (src/kernels.jl:2301-2397)
template <typename V, bool Full, bool Diag, typename AV = double>
struct EpiZxw1 {
  V *Qw, *x, *x_hat, *w_bar, *dx, *x_bar, *z_bar;
  const V *ATy, *c, *l, *u, *w, *fact1, *fact2;
  const AV* last_x;
  double sigma, f1s, f2s, h1, h2;
  __device__ __forceinline__ void prefetch(int i, int lv) const {
    pf_rows(i, lv, x, w, ATy, c, l, u, last_x);
    if (Diag) pf_rows(i, lv, fact1, fact2);
  }
  struct Pre {
    V c, l, u;
  };
  __device__ __forceinline__ Pre pre(int i) const { return Pre{c[i], l[i], u[i]}; }
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A acc) const { (*this)(i, acc, pre(i)); }
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A acc, const Pre& p) const {
    const double qw = (double)acc;
    Qw[i] = (V)qw;
    const double x_i = x[i], w_i = w[i];
    const double tmp = -qw + (double)ATy[i] - (double)p.c;
    const double z_raw = x_i + sigma * tmp;
    const double xb = clampd(z_raw, p.l, p.u);
    const double xh = 2.0 * xb - x_i;
    const double xn = fma(h2, xh, h1 * (double)last_x[i]);
    const double wb = Diag ? fma((double)fact1[i], w_i, (double)fact2[i] * xh) : fma(f1s, w_i, f2s * xh);
    if (Full) {
      dx[i] = (V)(xb - x_i);
      x_bar[i] = (V)xb;
      z_bar[i] = (V)((xb - z_raw) / sigma);
    }
    x[i] = (V)xn;
    x_hat[i] = (V)xh;
    w_bar[i] = (V)wb;
  }
};

// QP step 2: tempv = x_hat + sigma (Qw - Q w_bar)  (update_y_cpu!, kernels.jl:2690-2694)
template <typename V>
struct EpiTempv {
  V* tempv;
  const V *x_hat, *Qw;
  double sigma;
  __device__ __forceinline__ void prefetch(int i, int lv) const { pf_rows(i, lv, x_hat, Qw); }
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A acc) const {
    tempv[i] = (V)((double)x_hat[i] + sigma * ((double)Qw[i] - (double)acc));
  }
};

// y step: A*v fused with update_y_cpu! / unified_update_y_cpu! /
// unified_update_y_noQ_cpu! (src/kernels.jl:2242-2298, 2582-2658, 2682-2743).
// YbarAlways: the QP / noC loops write y_bar in partial steps too, the LP
// loop only in full steps.
template <typename V, bool Full, bool YbarAlways, typename AV = double>
struct EpiY {
  V *y, *y_bar, *s, *dy;
  const V *AL, *AU;
  const AV* last_y;
  double f1, f2, h1, h2;
  __device__ __forceinline__ void prefetch(int i, int lv) const { pf_rows(i, lv, (const V*)y, AL, AU, last_y); }
  struct Pre {
    V al, au;
  };
  __device__ __forceinline__ Pre pre(int i) const { return Pre{AL[i], AU[i]}; }
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A acc) const { (*this)(i, acc, pre(i)); }
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A acc, const Pre& p) const {
    const double yi = y[i];
    const double s_raw = (double)acc - f1 * yi;
    const double s_proj = clampd(s_raw, p.al, p.au);
    const double yb = f2 * (s_proj - s_raw);
    const double yh = 2.0 * yb - yi;
    const double yn = fma(h2, yh, h1 * (double)last_y[i]);
    if (Full) {
      s[i] = (V)s_proj;
      dy[i] = (V)(yb - yi);
    }
    if (Full || YbarAlways) y_bar[i] = (V)yb;
    y[i] = (V)yn;
  }
};

// QP step 4: A'y_bar fused with update_w2_cpu! (src/kernels.jl:2747-2832)
template <typename V, bool Full, bool Diag, typename AV = double>
struct EpiW2 {
  V *w, *ATy, *w_bar, *dw, *ATdy, *ATy_bar;
  const V* fact;
  const AV *last_w, *last_ATy;
  double fs, h1, h2;
  __device__ __forceinline__ void prefetch(int i, int lv) const {
    pf_rows(i, lv, (const V*)w, (const V*)ATy, (const V*)w_bar, last_w, last_ATy);
    if (Diag) pf_rows(i, lv, fact);
  }
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A acc) const {
    const double atyb = (double)acc;
    const double w_i = w[i], aty = ATy[i];
    const double f = Diag ? (double)fact[i] : fs;
    const double wbn = (double)w_bar[i] + f * (atyb - aty);
    const double wn = h1 * (double)last_w[i] + h2 * (2.0 * wbn - w_i);
    const double atyn = h1 * (double)last_ATy[i] + h2 * (2.0 * atyb - aty);
    w[i] = (V)wn;
    ATy[i] = (V)atyn;
    if (Full) {
      w_bar[i] = (V)wbn;
      dw[i] = (V)(wbn - w_i);
      ATdy[i] = (V)(atyb - aty);
      ATy_bar[i] = (V)atyb;
    }
  }
};

// QP-noC step 1: A'y fused with unified_update_zxw_cpu! (kernels.jl:2117-2223)
template <typename V, bool Full, bool Diag, typename AV = double>
struct EpiZxwNoC {
  V *x, *x_hat, *w_bar, *w, *dx, *x_bar, *z_bar, *dw;
  const V *Qw, *c, *l, *u, *fact1, *fact2;
  const AV *last_x, *last_w;
  double sigma, f1s, f2s, h1, h2;
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A acc) const {
    const double x_i = x[i], w_i = w[i];
    const double tmp = -(double)Qw[i] + (double)acc - (double)c[i];
    const double z_raw = x_i + sigma * tmp;
    const double xb = clampd(z_raw, l[i], u[i]);
    const double xh = 2.0 * xb - x_i;
    const double xn = fma(h2, xh, h1 * (double)last_x[i]);
    const double wb = Diag ? fma((double)fact1[i], w_i, (double)fact2[i] * xh) : fma(f1s, w_i, f2s * xh);
    const double wh = 2.0 * wb - w_i;
    const double wn = fma(h2, wh, h1 * (double)last_w[i]);
    if (Full) {
      dx[i] = (V)(xb - x_i);
      x_bar[i] = (V)xb;
      z_bar[i] = (V)((xb - z_raw) / sigma);
      dw[i] = (V)(wb - w_i);
    }
    x[i] = (V)xn;
    x_hat[i] = (V)xh;
    w_bar[i] = (V)wb;
    w[i] = (V)wn;
  }
};

// QP-noC step 2: Q w_bar; Halpern-averaged Qw and tempv (kernels.jl:2226-2237)
template <typename V, bool Full, typename AV = double>
struct EpiTempvNoC {
  V *Qw, *tempv, *Qw_bar;
  const V* x_hat;
  const AV* last_Qw;
  double sigma, h1, h2;
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A acc) const {
    const double qwb = (double)acc, qw = Qw[i];
    const double qwh = 2.0 * qwb - qw;
    Qw[i] = (V)fma(h2, qwh, h1 * (double)last_Qw[i]);
    tempv[i] = (V)((double)x_hat[i] + sigma * (qw - qwb));
    if (Full) Qw_bar[i] = (V)qwb;
  }
};

// LP step 1: A'y fused with unified_update_zx_cpu! (kernels.jl:2504-2578)
template <typename V, bool Full, typename AV = double>
struct EpiZxLP {
  V *x, *x_hat, *dx, *x_bar, *z_bar;
  const V *c, *l, *u;
  const AV* last_x;
  double sigma, h1, h2;
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A acc) const {
    const double x_i = x[i];
    const double z_raw = x_i + sigma * ((double)acc - (double)c[i]);
    const double xb = clampd(z_raw, l[i], u[i]);
    const double xh = 2.0 * xb - x_i;
    const double xn = fma(h2, xh, h1 * (double)last_x[i]);
    if (Full) {
      dx[i] = (V)(xb - x_i);
      x_bar[i] = (V)xb;
      z_bar[i] = (V)((xb - z_raw) / sigma);
    }
    x[i] = (V)xn;
    x_hat[i] = (V)xh;
  }
};

// LASSO: A_d'(A_d w) fused with update_zxw_LASSO_cpu! (kernels.jl:2400-2496)
template <typename V, bool Full, typename AV = double>
struct EpiLasso {
  V *x, *x_hat, *w_bar, *w, *dx, *x_bar, *z_bar, *dw;
  const V* c;
  const AV *last_x, *last_w;
  double sigma, lam, f1s, f2s, h1, h2;
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A acc) const {
    const double x_i = x[i], w_i = w[i];
    const double tmp = -(double)acc + 0.0 - (double)c[i];  // A'y == 0 (m = 0)
    const double z_raw = x_i + sigma * tmp;
    const double shrink = fmax(fabs(z_raw) - lam * sigma, 0.0);
    const double xb = copysign(shrink, z_raw);
    const double xh = 2.0 * xb - x_i;
    const double xn = fma(h2, xh, h1 * (double)last_x[i]);
    const double wb = fma(f1s, w_i, f2s * xh);
    const double wn = fma(h2, 2.0 * wb - w_i, h1 * (double)last_w[i]);
    if (Full) {
      dx[i] = (V)(xb - x_i);
      x_bar[i] = (V)xb;
      z_bar[i] = (V)((xb - z_raw) / sigma);
      dw[i] = (V)(wb - w_i);
    }
    x[i] = (V)xn;
    x_hat[i] = (V)xh;
    w_bar[i] = (V)wb;
    w[i] = (V)wn;
  }
};

// ---------------------------------------------------------------------------
// Reduction epilogues
// ---------------------------------------------------------------------------

// compute_residuals! n-part (algorithm.jl:55-79, kernels.jl:132-148,
// algorithm.jl:127-133): acc = (A' y_bar)_i.
// slots: 0 c'x  1 x'Qx  2 z'x  3 |lam x|_1  4 |Rd|inf  5 |A'y s|inf  6 |Qx s|inf  7 bound viol
template <typename V>
struct EpiResN {
  const V *x_bar, *Qx, *c, *z_bar, *col_norm, *l, *u;
  double lam, c_scale, b_scale;
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A acc, double (&r)[8]) const {
    const double xb = x_bar[i], qx = Qx[i], ci = c[i], zb = z_bar[i];
    const double aty = (double)acc;
    const double f = (double)col_norm[i] * c_scale;
    r[0] += ci * xb;
    r[1] += xb * qx;
    r[2] += zb * xb;
    r[3] += fabs(lam * xb);
    r[4] = fmax(r[4], fabs((qx + ci - aty - zb) * f));
    r[5] = fmax(r[5], fabs(aty * f));
    r[6] = fmax(r[6], fabs(qx * f));
    const double viol = fmax((double)l[i] - xb, 0.0) + fmax(xb - (double)u[i], 0.0);
    r[7] = fmax(r[7], fabs(viol * (b_scale / (double)col_norm[i])));
  }
};
constexpr unsigned kResNMax = (1u << 4) | (1u << 5) | (1u << 6) | (1u << 7);

// compute_residuals! m-part (algorithm.jl:62,82-85, kernels.jl:172-194):
// acc = (A x_bar)_i.  slots: 0 y's  1 |Rp|inf  2 |Ax s|inf
template <typename V>
struct EpiResM {
  const V *y_bar, *s, *AL, *AU, *row_norm;
  double b_scale;
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A acc, double (&r)[3]) const {
    const double ax = (double)acc;
    const double corr = clampd(ax, AL[i], AU[i]) - ax;
    const double f = (double)row_norm[i] * b_scale;
    r[0] += (double)y_bar[i] * (double)s[i];
    r[1] = fmax(r[1], fabs(corr * f));
    r[2] = fmax(r[2], fabs(ax * f));
  }
};
constexpr unsigned kResMMax = (1u << 1) | (1u << 2);

// compute_M_norm! n-part (algorithm.jl:689-739).  slots:
// 0 dx.dx 1 dQw.dx 2 dQw.ATdy 3 ATdy.dx 4 (ATdy*fact_M).QATdy 5 ATdy.QATdy 6 dQw.dQw 7 dw.dQw
template <typename V>
struct EpiMnormN {
  const V *dx, *dQw, *ATdy, *QATdy, *fact_M, *dw;
  bool has_m;
  __device__ __forceinline__ void operator()(int i, double, double (&r)[8]) const {
    const double ddx = dx[i], dqw = dQw[i], ddw = dw[i];
    r[0] += ddx * ddx;
    r[1] += dqw * ddx;
    if (has_m) {
      const double at = ATdy[i], qat = QATdy[i];
      r[2] += dqw * at;
      r[3] += at * ddx;
      r[4] += (at * (double)fact_M[i]) * qat;
      r[5] += at * qat;
    }
    r[6] += dqw * dqw;
    r[7] += ddw * dqw;
  }
  __device__ __forceinline__ void operator()(int i, float a, double (&r)[8]) const { (*this)(i, (double)a, r); }
};

// sum of squares of an m-vector (dy.dy)
template <typename V>
struct EpiSumSq {
  const V* v;
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A, double (&r)[1]) const {
    const double t = v[i];
    r[0] += t * t;
  }
};

// update_sigma! statistics (algorithm.jl:344-371). slots:
// 0 dx.dx 1 dQw.ATdy 2 dQw.dQw 3 dw.dQw 4 ATdy.QATdy
template <typename V>
struct EpiSigmaN {
  const V *dx, *dQw, *ATdy, *QATdy, *dw;
  bool has_m;
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A, double (&r)[5]) const {
    const double ddx = dx[i], dqw = dQw[i], ddw = dw[i];
    r[0] += ddx * ddx;
    if (has_m) {
      const double at = ATdy[i];
      r[1] += dqw * at;
      r[4] += at * (double)QATdy[i];
    }
    r[2] += dqw * dqw;
    r[3] += ddw * dqw;
  }
};

// Power method, fused: acc is (M z_cur)_i (scale_acc: divide by ||z_cur||,
// i.e. the product of the normalised q = z_cur/||z_cur||) or already the
// product of q.  Stores z_next and accumulates 0 q.z_next  1 z_next.z_next
// 2 q.q, so ||z_next - lambda q||^2 = zz - 2 lambda^2 + lambda^2 qq needs no
// second pass (power_iteration_A/Q, src/utils.jl:1352-1372).
template <typename V>
struct EpiPowerFused {
  const V* zc;
  V* zn;
  const double* zz;
  bool scale_acc;
  const double* inv_norm = nullptr;  // 1/||z_cur|| formed once by the previous step, or null
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A acc, double (&r)[3]) const {
    const double inv = inv_norm ? *inv_norm : 1.0 / sqrt(*zz);
    const double v = scale_acc ? (double)acc * inv : (double)acc;
    if (zn) zn[i] = (V)v;
    const double q = (double)zc[i] * inv;
    r[0] += q * v;
    r[1] += v * v;
    r[2] += q * q;
  }
};

// y = (M x) / ||x||, the norm read from the device
template <typename V>
struct EpiStoreInvNorm {
  V* y;
  const double* zz;
  const double* inv_norm = nullptr;  // 1/||x|| formed once, or null
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A acc) const {
    y[i] = inv_norm ? (V)((double)acc * *inv_norm) : (V)((double)acc / sqrt(*zz));
  }
};

// Last-CTA step of a power iteration: log (lambda, err) for iteration k.
struct PowerFin {
  double* log;
  int k;
  double* inv_out = nullptr;  // also store 1/||z_next|| for the next step's rows
  __device__ __forceinline__ void operator()(const double (&a)[3]) const {
    const double lam = a[0], zz = a[1], qq = a[2];
    const double rr = fmax(zz - 2.0 * lam * lam + lam * lam * qq, 0.0);
    log[2 * k] = lam;
    log[2 * k + 1] = sqrt(rr) / (sqrt(zz) + lam);
    if (inv_out) *inv_out = 1.0 / sqrt(zz);
  }
  template <int K>
  __device__ __forceinline__ void operator()(const double (&)[K]) const {}
};

// The A A' power step carried in n-space on the Gram matrix G = A'A.  With
// q_k = z_k / ||z_k|| the reference's iterate, w_k = A' q_k, and
// u_k = G w_{k-1} kept unnormalised (w_k = u_k / ||z_k||):
//   z_{k+1} = A w_k,  lambda_k = q_k . z_{k+1} = ||w_k||^2,
//   ||z_{k+1}||^2 = w_k . G w_k,  ||z_{k+1} - lambda_k q_k||^2 = ||z_{k+1}||^2 - lambda_k^2,
// i.e. the same (lambda, err) sequence with one sweep of G per step.
// Row i: u_{k+1,i} = (G u_k)_i / ||z_k||; sums 0: w.u_{k+1}, 1: w.w.  The
// state is kept in FP64 whatever G's type: ||z||^2 - lambda^2 cancels to
// ~4e-8 lambda^2 at the 1e-4 stopping test, and FP32 rounding of u would
// move that difference by several per cent (the stop by up to ~100 steps).
template <typename V>
struct EpiGramPower {
  const V* uc;
  V* un;
  const double* inv_norm;  // 1 / ||z_k||
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A acc, double (&r)[2]) const {
    const double s = *inv_norm;
    const double v = (double)acc * s;
    un[i] = (V)v;
    const double w = (double)uc[i] * s;
    r[0] += w * v;
    r[1] += w * w;
  }
};

// Last-CTA step of a Gram power step: log (lambda, err) for iteration k and
// store 1/||z_{k+1}|| for the next step's rows
struct GramPowerFin {
  double* log;
  int k;
  double* inv_out;
  __device__ __forceinline__ void operator()(const double (&a)[2]) const {
    const double zz = a[0], lam = a[1];
    const double rr = fmax(zz - lam * lam, 0.0);
    log[2 * k] = lam;
    log[2 * k + 1] = sqrt(rr) / (sqrt(zz) + lam);
    *inv_out = 1.0 / sqrt(zz);
  }
  template <int K>
  __device__ __forceinline__ void operator()(const double (&)[K]) const {}
};

// The power method's start vector on the device: element i takes outputs 2i
// and 2i + 1 of the splitmix64 stream from state 1 (output k mixes
// 1 + (k + 1) * 0x9E3779B97F4A7C15, so every element is independent) through
// Box-Muller, plus 1e-8: the host power_start_vector values up to the last
// bit of log / cos / sqrt.
__device__ __forceinline__ uint64_t splitmix_at(uint64_t k) {
  uint64_t v = 1ull + (k + 1ull) * 0x9E3779B97F4A7C15ULL;
  v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ULL;
  v = (v ^ (v >> 27)) * 0x94D049BB133111EBULL;
  return v ^ (v >> 31);
}
template <typename V>
__global__ void __launch_bounds__(kBlock) k_start_vector(int64_t len, V* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x;
  if (i >= len) return;
  const double u1 = ((double)(splitmix_at(2 * (uint64_t)i) >> 11) + 1.0) * 0x1.0p-53;
  const double u2 = (double)(splitmix_at(2 * (uint64_t)i + 1) >> 11) * 0x1.0p-53;
  out[i] = (V)(sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2) + 1e-8);
}

// The same for B instances concatenated at offsets off[0..B] (instance k's
// own stream in [off[k], off[k+1]); zeros past off[B])
template <typename V>
__global__ void __launch_bounds__(kBlock) k_start_vector_seg(int B, const int64_t* __restrict__ off, int64_t total,
                                                             V* __restrict__ out) {
  const int64_t j = (int64_t)blockIdx.x * kBlock + threadIdx.x;
  if (j >= total) return;
  if (j >= off[B]) {
    out[j] = (V)0;
    return;
  }
  int lo = 0, hi = B;  // off[lo] <= j < off[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= j) lo = mid;
    else hi = mid;
  }
  const uint64_t i = (uint64_t)(j - off[lo]);
  const double u1 = ((double)(splitmix_at(2 * i) >> 11) + 1.0) * 0x1.0p-53;
  const double u2 = (double)(splitmix_at(2 * i + 1) >> 11) * 0x1.0p-53;
  out[j] = (V)(sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2) + 1e-8);
}

// ---------------------------------------------------------------------------
// Power steps with the fold once per chunk.  The chains run unnormalised
// (y_{k+1} = M y_k) and every step only writes its per-CTA dot products;
// one fold per chunk of steps turns them into each step's (lambda, err)
// with scale-invariant formulas and renormalises the state.
//   Q chain (q_k = y_k / ||y_k||, z_{k+1} = Q q_k):
//     a = y_k . y_{k+1}, b = y_k . y_k, c = y_{k+1} . y_{k+1}
//     lambda_k = a / b, ||z_{k+1}||^2 = c / b, ||z_{k+1} - lambda q_k||^2 = c / b - lambda^2
//   Gram chain (w_k = s_k u_k with s_0 = 1 at the chunk start, s_k = 1 / sqrt(a_{k-1})):
//     a = u_k . u_{k+1}, b = u_k . u_k
//     lambda_k = s_k^2 b, ||z_{k+1}||^2 = s_k^2 a
// Both states are FP64 (an unnormalised chain grows or shrinks by about
// lambda per step between renormalisations); b is taken from the stored
// y_k, so each step's sums describe the same vectors and ||z||^2 >= lambda^2
// holds up to FP64 rounding.  A total that is not finite and positive
// (a state out of FP64 range) logs NaN, and the host then reruns the
// method with the per-step fold.
// ---------------------------------------------------------------------------
template <int TPR, int K, typename Acc, typename Src, typename Epi>
__global__ void __launch_bounds__(kBlock) k_row_partials(int nrows, Src src, Epi epi, double* __restrict__ partials) {
  pdl_enter();
  double r[K];
#pragma unroll
  for (int k = 0; k < K; ++k) r[k] = 0.0;
  const int lane = threadIdx.x & (TPR - 1);
  const int rows_per_grid = (int)(gridDim.x * (kBlock / TPR));
  for (int row = (int)((blockIdx.x * kBlock + threadIdx.x) / TPR); row < nrows; row += rows_per_grid) {
    const Acc acc = src.template dot<TPR, Acc>(row, lane);
    if (lane == 0) epi(row, acc, r);
  }
  block_reduce<K, 0u>(r);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) partials[(size_t)blockIdx.x * K + k] = r[k];
  }
}

// The same over a SELL-32 matrix, one thread per row, with the matrix
// entries of the thread's first R rows (up to WMAX entries each: row
// lengths, slice offsets, column indices, values; constant over a solve)
// loaded before the wait on the previous kernel, so a CTA made resident
// while the previous step drains already holds them.  Rows past R or entries
// past WMAX are read after the wait.  Summation order as SellSrc::dot.
template <int R, int WMAX, int K, typename Acc, typename V, typename X, typename Epi>
__global__ void __launch_bounds__(kBlock) k_sell_partials(int nrows, SellSrc<V, X> src, Epi epi,
                                                          double* __restrict__ partials) {
  double r[K];
#pragma unroll
  for (int k = 0; k < K; ++k) r[k] = 0.0;
  const int stride = (int)(gridDim.x * kBlock);
  const int row0 = (int)(blockIdx.x * kBlock + threadIdx.x);
  int len[R], base[R], c[R][WMAX];
  V v[R][WMAX];
#pragma unroll
  for (int q = 0; q < R; ++q) {
    const int row = row0 + q * stride;
    len[q] = 0;
    base[q] = 0;
    if (row < nrows) {
      len[q] = __ldg(src.ptr + row + 1) - __ldg(src.ptr + row);
      base[q] = __ldg(src.sptr + (row >> 5)) + (row & 31);
#pragma unroll
      for (int k = 0; k < WMAX; ++k)
        if (k < len[q]) {
          c[q][k] = __ldg(src.col + base[q] + 32 * k);
          v[q][k] = __ldg(src.val + base[q] + 32 * k);
        }
    }
  }
  pdl_enter();
  // every preloaded row's gathers first, then the sums and epilogues: the
  // epilogues' stores must not keep the next row's loads waiting
  Acc g[R][WMAX];
#pragma unroll
  for (int q = 0; q < R; ++q)
#pragma unroll
    for (int k = 0; k < WMAX; ++k) g[q][k] = (k < len[q]) ? (Acc)__ldg(src.x + c[q][k]) : Acc(0);
#pragma unroll
  for (int q = 0; q < R; ++q) {
    const int row = row0 + q * stride;
    if (row < nrows) {
      Acc s = Acc(0);
#pragma unroll
      for (int k = 0; k < WMAX; ++k)
        if (k < len[q]) s = fma((Acc)v[q][k], g[q][k], s);
      for (int k = WMAX; k < len[q]; ++k)
        s = fma((Acc)__ldg(src.val + base[q] + 32 * k), (Acc)__ldg(src.x + __ldg(src.col + base[q] + 32 * k)), s);
      epi(row, s, r);
    }
  }
  for (int row = row0 + R * stride; row < nrows; row += stride) {
    const Acc acc = src.template dot<1, Acc>(row, 0);
    epi(row, acc, r);
  }
  block_reduce<K, 0u>(r);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) partials[(size_t)blockIdx.x * K + k] = r[k];
  }
}

template <typename V>
struct EpiPowRaw {  // Q chain: y_{k+1} = Q y_k; sums a, b, c
  const V* yc;
  V* yn;
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A acc, double (&r)[3]) const {
    const double v = (double)acc;
    yn[i] = (V)v;
    const double y = (double)yc[i];
    r[0] += y * v;
    r[1] += y * y;
    r[2] += v * v;
  }
};

struct EpiGramRaw {  // Gram chain: u_{k+1} = G u_k; sums a, b
  const double* uc;
  double* un;
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A acc, double (&r)[2]) const {
    const double v = (double)acc;
    un[i] = v;
    const double u = uc[i];
    r[0] += u * v;
    r[1] += u * u;
  }
};

// One chain's chunk of steps for the fold: its per-step partials
// (steps x nblk x K), its totals (steps x K), its log (lambda, err per
// step), the state to renormalise, and the kind (0 = Gram, 1 = Q).
struct PowChunkChain {
  const double* partials;
  double* totals;
  double* log;
  int nblk, K, steps, kind;
  double* state64;   // Gram state
  double* stateQ64;  // Q state
  int64_t len;
  double* scale_out;  // the renormalisation factor of the chunk's last state
};

// Fold: CTA (step, chain) sums that step's per-CTA partials in CTA order.
static __global__ void __launch_bounds__(kBlock) k_pow_chunk_fold(PowChunkChain c0, PowChunkChain c1) {
  pdl_enter();  // the chunk's last steps must be complete
  const PowChunkChain& c = blockIdx.y == 0 ? c0 : c1;
  const int k = blockIdx.x;
  if (k >= c.steps || c.nblk == 0) return;
  double acc[3] = {0.0, 0.0, 0.0};
  const double* p = c.partials + (size_t)k * c.nblk * c.K;
  for (int b = threadIdx.x; b < c.nblk; b += kBlock)
    for (int q = 0; q < c.K; ++q) acc[q] += __ldcg(p + (size_t)b * c.K + q);
  block_reduce<3, 0u>(acc);
  if (threadIdx.x == 0)
    for (int q = 0; q < c.K; ++q) c.totals[k * 3 + q] = acc[q];
}

// A step's totals are usable when finite and positive (a state that left
// FP64 range gives inf or 0).
__device__ __forceinline__ bool pow_totals_ok(const double* t, int kind) {
  return isfinite(t[0]) && isfinite(t[1]) && t[0] > 0.0 && t[1] > 0.0 &&
         (kind == 0 || (isfinite(t[2]) && t[2] > 0.0));
}

// the chunk's (lambda, err) recurrence from its totals `tot` (steps x 3)
__device__ __forceinline__ void pow_chunk_log(const PowChunkChain& c, const double* tot) {
  double s2 = 1.0;  // s_k^2 of the Gram chain (1 at the chunk start)
  for (int k = 0; k < c.steps; ++k) {
    const double* t = tot + k * 3;
    if (!pow_totals_ok(t, c.kind)) {
      c.log[2 * k] = c.log[2 * k + 1] = nan("");
      continue;
    }
    double lam, zz;
    if (c.kind == 0) {
      lam = s2 * t[1];
      zz = s2 * t[0];
      s2 = 1.0 / t[0];
    } else {
      lam = t[0] / t[1];
      zz = t[2] / t[1];
    }
    c.log[2 * k] = lam;
    c.log[2 * k + 1] = sqrt(fmax(zz - lam * lam, 0.0)) / (sqrt(zz) + lam);
  }
}

// CTA 0 writes the chunk's log (its totals staged in shared memory first,
// so the recurrence does not wait on one load per step); every CTA
// renormalises its slice of the last state by the factor that the last
// step's totals give (Gram: 1 / sqrt(u_k . u_{k+1}), the s of the next
// chunk's start; Q: 1 / ||y||), 1 when those totals are not usable.
static __global__ void __launch_bounds__(kBlock) k_pow_chunk_finish(PowChunkChain c0, PowChunkChain c1) {
  pdl_enter();  // the fold must be complete
  const PowChunkChain& c = blockIdx.y == 0 ? c0 : c1;
  if (c.steps == 0 || c.steps > 32) return;
  __shared__ double s_tot[32 * 3];
  __shared__ double s_scale;
  if (blockIdx.x == 0)
    for (int q = threadIdx.x; q < c.steps * 3; q += kBlock) s_tot[q] = c.totals[q];
  __syncthreads();
  if (threadIdx.x == 0) {
    if (blockIdx.x == 0) pow_chunk_log(c, s_tot);
    const double* tl = c.totals + (c.steps - 1) * 3;
    double sc = 1.0;
    if (pow_totals_ok(tl, c.kind)) sc = c.kind == 0 ? sqrt(1.0 / tl[0]) : 1.0 / sqrt(tl[2]);
    s_scale = sc;
    if (blockIdx.x == 0 && c.scale_out) *c.scale_out = sc;
  }
  __syncthreads();
  const double sc = s_scale;
  for (int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x; i < c.len; i += (int64_t)gridDim.x * kBlock) {
    if (c.state64) c.state64[i] *= sc;
    if (c.stateQ64) c.stateQ64[i] *= sc;
  }
}

// 1/sqrt of a reduced sum of squares (the start vector's norm)
struct InvNormFin {
  double* inv_out;
  __device__ __forceinline__ void operator()(const double (&a)[1]) const { *inv_out = 1.0 / sqrt(a[0]); }
  template <int K>
  __device__ __forceinline__ void operator()(const double (&)[K]) const {}
};

// Power method partial sums: 0 q.z  1 z.z   (q = zold/||zold||)
template <typename V>
struct EpiPowerDot {
  const V *q, *z;
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A, double (&r)[2]) const {
    const double zi = z[i];
    r[0] += (double)q[i] * zi;
    r[1] += zi * zi;
  }
};

// ---------------------------------------------------------------------------
// Element-wise kernels
// ---------------------------------------------------------------------------
template <typename F>
__global__ void __launch_bounds__(kBlock) k_elementwise(int len, F f) {
  pdl_enter();
  const int i = blockIdx.x * kBlock + threadIdx.x;
  if (i < len) f(i);
}

}  // namespace hprqp
