// power.cuh — the power method (src/utils.jl:1335-1461) as ONE persistent
// cooperative kernel.
//
// The power method is a chain of small dependent products (the 700x700 grid
// QP needs ~2,800 A A' steps of ~23 MB each in FP32, all of it L2-resident
// after the first step), so a launch per product leaves it bound by launch
// gaps and reduction tails.  Here every CTA stays resident for the whole
// method: a step is one or two grid-stride sweeps over a matrix, separated
// by a software grid barrier, and the three dot products of a step (q.v,
// v.v, q.q) are folded by EVERY CTA from the per-CTA partials in the same
// fixed order, so all CTAs derive bit-identical lambda / err / ||z|| and
// take the same stop decision without another barrier.
//
// Two chains run in the same phases: chain 0 (A A': t = A' z/||z||, then
// z' = A t; two phases per step) and chain 1 (sparse Q: z' = Q z/||z||, one
// phase per step; or the LASSO operator L'L, two phases per step).  A chain
// stops at the first step with err < tol (that step's lambda is returned),
// or after max_it steps.
//
// Every barrier wait is bounded (poll count and %globaltimer); a CTA that
// gives up raises `status`, which every other CTA checks while it waits, so
// the whole grid returns and the host reports the error.
#pragma once

#include "kernels.cuh"

namespace hprqp {

constexpr int kPowBlock = 512;
constexpr int kPowMaxGrid = 1024;  // partials buffer capacity (CTAs)
constexpr int kPowIlp = 4;         // ELL rows per thread in flight
constexpr unsigned long long kPowBarrierNs = 2000000000ull;  // 2 s per barrier wait
constexpr unsigned kPowMaxPolls = 1u << 26;

template <typename V>
struct PowChain {
  int kind = 0;  // 0 off; 1: z' = M1 z/||z|| (M1 symmetric); 2: t = M1 z/||z||, z' = M2 t
  DCsr<V> M1, M2;
  V* z0 = nullptr;  // z ping-pongs between z0 and z1
  V* z1 = nullptr;
  V* t = nullptr;
  const double* zz0 = nullptr;  // ||z_0||^2 on the device
};

template <typename V>
struct PowArgs {
  PowChain<V> ch[2];
  double tol;
  int max_it;
  double* partials;  // [2 (phase parity)][2 (chain)][gridDim.x][3]
  unsigned* bar;     // barrier arrivals; bar[32] the released phase (both zeroed before the launch)
  int* status;       // 0, or 1 once a barrier wait gave up
  double* out;       // [c*4 + 0] lambda, [c*4 + 1] stop step (or -1), [c*4 + 2] steps; [8] status
};

__device__ __forceinline__ unsigned long long pow_clock_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned pow_ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid barrier: arrivals count up monotonically on `bar` (target = gridDim.x
// * phase number, so it needs no reset between phases); the CTA whose
// arrival completes the phase publishes the phase number on `flag` (its own
// 128-byte line), and the others poll that flag with a backoff instead of
// the counter the arrivals are still updating.  Returns false when this CTA
// gave up (time or poll limit, or another CTA's abort).
__device__ __forceinline__ bool pow_barrier(unsigned* bar, unsigned* flag, unsigned phase_no, unsigned target,
                                            int* status) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(bar, 1u);
    int ok = 1;
    if (prev == target - 1u) {
      __threadfence();  // every arrival (and the partials fenced before it) precedes the release
      asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(flag), "r"(phase_no) : "memory");
    } else {
      const unsigned long long t0 = pow_clock_ns();
      unsigned backoff = 32;
      for (unsigned polls = 0;; ++polls) {
        if (pow_ld_acquire(flag) >= phase_no) break;
        if ((polls & 63u) == 63u) {
          if (*(volatile int*)status != 0 || pow_clock_ns() - t0 > kPowBarrierNs || polls > kPowMaxPolls) {
            atomicExch(status, 1);
            ok = 0;
            break;
          }
        }
        __nanosleep(backoff);
        if (backoff < 256) backoff <<= 1;
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Sum K slots over the CTA; the result is returned to EVERY thread.
template <int K>
__device__ __forceinline__ void pow_block_sum(double (&r)[K]) {
  __shared__ double sh[K][kPowBlock / 32];
  __shared__ double res[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double v = r[k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double v = threadIdx.x < kPowBlock / 32 ? sh[k][threadIdx.x] : 0.0;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
      if (threadIdx.x == 0) res[k] = v;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) r[k] = res[k];
  __syncthreads();
}

// Row sources of the persistent kernel.  The matrix is read-only for the
// kernel's lifetime (read-only cache path); the vector x was written by
// other CTAs in an earlier phase of the same launch, so it is read through
// L2 (ld.global.cg), never through the non-coherent path.
template <typename V>
struct PowCsrSrc {
  const int* __restrict__ ptr;
  const int* __restrict__ col;
  const V* __restrict__ val;
  const V* x;
  template <int TPR, typename Acc>
  __device__ __forceinline__ Acc dot(int row, int lane) const {
    const int b = __ldg(ptr + row), e = __ldg(ptr + row + 1);
    Acc s = Acc(0);
#pragma unroll 4
    for (int k = b + lane; k < e; k += TPR) s = fma((Acc)__ldg(val + k), (Acc)__ldcg(x + __ldg(col + k)), s);
    return group_sum<TPR>(s);
  }
};

template <typename V>
struct PowSellSrc {
  const int* __restrict__ sptr;
  const int* __restrict__ ptr;
  const int* __restrict__ col;
  const V* __restrict__ val;
  const V* x;
  template <typename Acc>
  __device__ __forceinline__ Acc dot(int row) const {
    const int len = __ldg(ptr + row + 1) - __ldg(ptr + row);
    const int base = __ldg(sptr + (row >> 5)) + (row & 31);
    Acc s = Acc(0);
#pragma unroll 4
    for (int k = 0; k < len; ++k)
      s = fma((Acc)__ldg(val + base + 32 * k), (Acc)__ldcg(x + __ldg(col + base + 32 * k)), s);
    return s;
  }
};

// Grid-stride sweep of M x over M's row schedule; f(row, acc) per row.
template <int TPR, typename Acc, typename V, typename F>
__device__ __forceinline__ void pow_sweep_csr(const DCsr<V>& M, const V* x, long long gtid, long long gthreads,
                                              F& f) {
  const PowCsrSrc<V> src{M.ptr, M.col, M.val, x};
  const int lane = (int)(threadIdx.x & (TPR - 1));
  const long long stride = gthreads / TPR;
  for (long long row = gtid / TPR; row < M.rows; row += stride) {
    const Acc acc = src.template dot<TPR, Acc>((int)row, lane);
    if (lane == 0) f((int)row, acc);
  }
}

template <typename Acc, typename V, typename F>
__device__ __forceinline__ void pow_sweep(const DCsr<V>& M, const V* x, long long gtid, long long gthreads, F& f) {
  if (M.ell) {
    // ELL: kPowIlp rows per thread in flight (rows r0 + q * gthreads, so a
    // warp's loads stay coalesced), no row pointers to wait for
    const long long rows = M.rows;
    for (long long r0 = gtid; r0 < rows; r0 += kPowIlp * gthreads) {
      Acc acc[kPowIlp];
#pragma unroll
      for (int q = 0; q < kPowIlp; ++q) acc[q] = Acc(0);
      for (int k = 0; k < M.ell_w; ++k) {
        const int* c = M.ecol + (size_t)k * rows;
        const V* v = M.evalv + (size_t)k * rows;
#pragma unroll
        for (int q = 0; q < kPowIlp; ++q) {
          const long long row = r0 + q * gthreads;
          if (row < rows) acc[q] = fma((Acc)__ldg(v + row), (Acc)__ldcg(x + __ldg(c + row)), acc[q]);
        }
      }
#pragma unroll
      for (int q = 0; q < kPowIlp; ++q) {
        const long long row = r0 + q * gthreads;
        if (row < rows) f((int)row, acc[q]);
      }
    }
    return;
  }
  if (M.sell) {
    const PowSellSrc<V> src{M.sptr, M.ptr, M.scol, M.sval, x};
    for (long long row = gtid; row < M.rows; row += gthreads) f((int)row, src.template dot<Acc>((int)row));
    return;
  }
  switch (M.tpr) {
    case 1: pow_sweep_csr<1, Acc>(M, x, gtid, gthreads, f); break;
    case 2: pow_sweep_csr<2, Acc>(M, x, gtid, gthreads, f); break;
    case 4: pow_sweep_csr<4, Acc>(M, x, gtid, gthreads, f); break;
    case 8: pow_sweep_csr<8, Acc>(M, x, gtid, gthreads, f); break;
    case 16: pow_sweep_csr<16, Acc>(M, x, gtid, gthreads, f); break;
    default: pow_sweep_csr<32, Acc>(M, x, gtid, gthreads, f); break;
  }
}

template <typename V>
__global__ void __launch_bounds__(kPowBlock, 2) k_power_persistent(PowArgs<V> a) {
  const long long gtid = (long long)blockIdx.x * kPowBlock + threadIdx.x;
  const long long gthreads = (long long)gridDim.x * kPowBlock;
  const int G = (int)gridDim.x;
  // chain state: identical in every CTA
  double zz[2], lam[2] = {0.0, 0.0};
  int cur[2] = {0, 0}, steps[2] = {0, 0}, found[2] = {-1, -1};
  bool done[2];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    done[c] = a.ch[c].kind == 0;
    zz[c] = done[c] ? 1.0 : *a.ch[c].zz0;
  }
  bool ok = true;
  for (unsigned phase = 0; !(done[0] && done[1]); ++phase) {
    bool dot[2] = {false, false};
    double r[2][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      if (done[c]) continue;
      const PowChain<V>& C = a.ch[c];
      const double inv = 1.0 / sqrt(zz[c]);
      const V* zc = cur[c] ? C.z1 : C.z0;
      V* zn = cur[c] ? C.z0 : C.z1;
      double* rc = r[c];
      if (C.kind == 2 && (phase & 1u) == 0) {  // t = M1 z / ||z||
        V* t = C.t;
        const double nrm = sqrt(zz[c]);
        auto f = [&](int i, V acc) { t[i] = (V)((double)acc / nrm); };
        pow_sweep<V>(C.M1, zc, gtid, gthreads, f);
      } else {  // z' = M2 t (kind 2) or M1 z / ||z|| (kind 1), and the dots
        const bool scale = C.kind == 1;
        auto f = [&](int i, double acc) {
          const double v = scale ? acc * inv : acc;
          zn[i] = (V)v;
          const double q = (double)__ldcg(zc + i) * inv;
          rc[0] += q * v;
          rc[1] += v * v;
          rc[2] += q * q;
        };
        if (C.kind == 1) pow_sweep<double>(C.M1, zc, gtid, gthreads, f);
        else pow_sweep<double>(C.M2, C.t, gtid, gthreads, f);
        dot[c] = true;
      }
    }
    double* part = a.partials + (size_t)(phase & 1u) * 2 * G * 3;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      if (!dot[c]) continue;
      pow_block_sum<3>(r[c]);
      if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) part[((size_t)c * G + blockIdx.x) * 3 + k] = r[c][k];
      }
    }
    if (!pow_barrier(a.bar, a.bar + 32, phase + 1u, (unsigned)G * (phase + 1u), a.status)) {
      ok = false;
      break;
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      if (!dot[c]) continue;
      double s[3] = {0.0, 0.0, 0.0};
      for (int b = threadIdx.x; b < G; b += kPowBlock) {
#pragma unroll
        for (int k = 0; k < 3; ++k) s[k] += __ldcg(part + ((size_t)c * G + b) * 3 + k);
      }
      pow_block_sum<3>(s);
      // s = (q.v, v.v, q.q): lambda = q.v, err = ||v - lambda q|| / (||v|| + lambda)
      const double l = s[0], vv = s[1], qq = s[2];
      const double rr = fmax(vv - 2.0 * l * l + l * l * qq, 0.0);
      const double err = sqrt(rr) / (sqrt(vv) + l);
      lam[c] = l;
      zz[c] = vv;
      cur[c] ^= 1;
      steps[c] += 1;
      if (err < a.tol) {
        found[c] = steps[c];
        done[c] = true;
      } else if (steps[c] >= a.max_it) {
        done[c] = true;
      }
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      a.out[c * 4 + 0] = lam[c];
      a.out[c * 4 + 1] = (double)found[c];
      a.out[c * 4 + 2] = (double)steps[c];
      a.out[c * 4 + 3] = (double)(cur[c]);
    }
    a.out[8] = ok ? (double)*(volatile int*)a.status : 1.0;
  }
}

}  // namespace hprqp
