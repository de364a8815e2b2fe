// qap_gemm.cuh — the QAP operator's dense products on the CUDA cores
// (src/Q_operators/QAP_operator.jl:52-75), for one instance or a batch of
// instances of uneven size concatenated in one array.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace hprqp {

// Q operator on the CUDA cores, shared-memory tiled: one CTA computes a
// 64 x 64 tile of one instance's output (blockIdx.x = instance,
// blockIdx.y = tile), each thread a 4 x 4 block.  The products of one
// output are one GEMM over the segments of a concatenated K dimension,
//   TMP_k = A_k X_k                                   (one segment)
//   Y_k / 2 = TMP_k B_k + (-S_k) X_k + (-X_k) T_k     (three segments),
// staged 16 at a time (each segment padded to a multiple of 16 with zeros),
// into ONE accumulator per output: 32 registers of FP64 accumulators keep
// three CTAs of 256 threads resident per SM.  The next chunk's operands are
// loaded into registers while the current one is multiplied.  Sums run
// over the segments in order and over l in increasing order within each.
constexpr int kQT = 64;   // output tile
constexpr int kQK = 16;   // K chunk
constexpr int kQMaxTiles = 4;  // tiles per side: n_k <= 256 on this path

template <typename V, int NS>
struct QapSegs {  // segment s: L[s] (i, l) * sign[s] times R[s] (l, j), column-major n_k x n_k each
  const V* L[NS];
  const V* R[NS];
  V sign[NS];
};

// Shared layout: L tile as Ls[l][i], R tile as Rs[l][j] with rows padded
// to kQT + 2 elements (stores of consecutive l land in different banks;
// rows stay 16-byte aligned).  Thread (ty, tx) owns rows {2ty, 2ty+1,
// 32+2ty, 32+2ty+1} and the same four columns from tx, so each operand
// pair is one 16-byte load and a warp's loads of R cover 16 consecutive
// pairs: no bank conflicts.
constexpr int kQRow = kQT + 2;

template <typename V, int NS>
__global__ void __launch_bounds__(256, 3) k_qap_gemm(const int* qn, const int64_t* off, const unsigned char* on,
                                                     QapSegs<V, NS> sg, V out_scale, V* Y) {
  __shared__ __align__(16) V Ls[kQK][kQT];
  __shared__ __align__(16) V Rs[kQK][kQRow];
  const int k = blockIdx.x;
  if (!on[k]) return;
  const int n = qn[k];
  const int nt = (n + kQT - 1) / kQT;
  if ((int)blockIdx.y >= nt * nt) return;
  const int i0 = (blockIdx.y % nt) * kQT, j0 = (blockIdx.y / nt) * kQT;
  const int64_t o = off[k];
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  const int nch = (n + kQK - 1) / kQK;  // chunks per segment
  const int total = NS * nch;
  // this thread's 4 + 4 staging slots (64 x 16 tiles, 256 threads)
  V lv[4], rv[4];
  auto fetch = [&](int c) {
    const int sgi = c / nch, l0 = (c - sgi * nch) * kQK;
    // a select instead of an indexed read keeps the segment table out of local memory
    const V* Lp = sg.L[0];
    const V* Rp = sg.R[0];
    V sgn = sg.sign[0];
#pragma unroll
    for (int t = 1; t < NS; ++t)
      if (sgi == t) {
        Lp = sg.L[t];
        Rp = sg.R[t];
        sgn = sg.sign[t];
      }
    Lp += o;
    Rp += o;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + 256 * q;
      const int ii = e & (kQT - 1), ll = e >> 6;  // L(i, l): consecutive threads, consecutive i
      const int gi = i0 + ii, gl = l0 + ll;
      lv[q] = (gi < n && gl < n) ? sgn * Lp[gi + (int64_t)gl * n] : V(0);
      const int rl = e & (kQK - 1), jj = e >> 4;  // R(l, j): consecutive threads, consecutive l
      const int rgl = l0 + rl, gj = j0 + jj;
      rv[q] = (rgl < n && gj < n) ? Rp[rgl + (int64_t)gj * n] : V(0);
    }
  };
  V acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = V(0);
  fetch(0);
  for (int c = 0; c < total; ++c) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + 256 * q;
      Ls[e >> 6][e & (kQT - 1)] = lv[q];
      Rs[e & (kQK - 1)][e >> 4] = rv[q];
    }
    __syncthreads();
    if (c + 1 < total) fetch(c + 1);  // in flight during the FMAs below
#pragma unroll
    for (int ll = 0; ll < kQK; ++ll) {
      V a[4], b[4];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        // elements 2ty, 2ty+1 (h = 0) and 32+2ty, 32+2ty+1 (h = 1): one 16-byte load each
        if constexpr (sizeof(V) == 8) {
          const double2 av = *reinterpret_cast<const double2*>(&Ls[ll][32 * h + 2 * ty]);
          const double2 bv = *reinterpret_cast<const double2*>(&Rs[ll][32 * h + 2 * tx]);
          a[2 * h] = av.x;
          a[2 * h + 1] = av.y;
          b[2 * h] = bv.x;
          b[2 * h + 1] = bv.y;
        } else {
          const float2 av = *reinterpret_cast<const float2*>(&Ls[ll][32 * h + 2 * ty]);
          const float2 bv = *reinterpret_cast<const float2*>(&Rs[ll][32 * h + 2 * tx]);
          a[2 * h] = av.x;
          a[2 * h + 1] = av.y;
          b[2 * h] = bv.x;
          b[2 * h + 1] = bv.y;
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = fma(a[u], b[v], acc[u][v]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int i = i0 + 32 * (u >> 1) + 2 * ty + (u & 1), j = j0 + 32 * (v >> 1) + 2 * tx + (v & 1);
      if (i < n && j < n) Y[o + i + (int64_t)j * n] = out_scale * acc[u][v];
    }
}

}  // namespace hprqp
