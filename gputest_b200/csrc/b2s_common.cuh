// Shared device helpers of the B200 SIMPLEC kernels: launch geometry, deterministic
// reductions and the grid-wide context of the cooperative (persistent) kernels.
//
// Determinism: every reduction is two-pass with a fixed order (warp xor-shuffle tree, then
// warps in index order, then blocks in index order). No floating-point atomics anywhere, so
// results do not depend on scheduling, and in a cooperative kernel every block computes
// bit-identical scalars, which keeps the control flow around grid.sync() uniform.
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "b2simplec.h"

namespace cg = cooperative_groups;

namespace b2s {

constexpr int kThreads = 256;        // ordinary kernels
constexpr int kCoopThreads = 1024;   // cooperative kernels: one block per SM
constexpr int kMaxCoopBlocks = 1184; // 148 SMs x 8
constexpr int kWarps = kCoopThreads / 32;
constexpr int kBicgVectors = 11;  // work vectors per right-hand side of the Jacobi-BiCGSTAB kernel

__host__ __device__ inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

inline unsigned grid_for(int64_t n, int threads = kThreads) {
  int64_t g = cdiv(n > 0 ? n : 1, threads);
  return (unsigned)(g > 2147483647 ? 2147483647 : g);
}

// Deterministic warp sum (xor tree: every lane ends with the same value).
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Sum NQ per-thread values over the block; result valid in out[0..NQ) for all threads after
// the call. smem must hold (blockDim.x/32)*NQ doubles plus NQ doubles.
template <int NQ>
__device__ __forceinline__ void block_sum(const double (&v)[NQ], double* smem, double (&out)[NQ]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double s = warp_sum(v[q]);
    if (lane == 0) smem[warp * NQ + q] = s;
  }
  __syncthreads();
  // warp w sums quantities w, w + nw, ... over the warp partials by a shuffle tree
  for (int q = warp; q < NQ; q += nw) {
    double s = lane < nw ? smem[lane * NQ + q] : 0.0;
    s = warp_sum(s);
    if (lane == 0) smem[nw * NQ + q] = s;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NQ; ++q) out[q] = smem[nw * NQ + q];
  __syncthreads();
}

// Block partial sums of NQ values, quantity-major: block b writes part[q*gridDim.x + b].
template <int NQ>
__device__ __forceinline__ void block_partials(const double (&v)[NQ], double* smem, double* part) {
  double out[NQ];
  block_sum<NQ>(v, smem, out);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) part[(int64_t)q * gridDim.x + blockIdx.x] = out[q];
  }
}

// Fixed-order total of quantity q over nb block partials (quantity-major layout), by one warp.
// Each lane adds its partials b = lane, lane + 32, ... in that order; they are loaded eight at a
// time as one straight-line block, so a lane's loads are in flight together instead of one
// after another (the totals follow a grid barrier, on the critical path of every reduction).
__device__ __forceinline__ double warp_total(const double* part, int nb, int nq, int q) {
  const int lane = threadIdx.x & 31;
  const double* pq = part + (int64_t)q * nb;
  double s = 0.0;
  for (int b = lane; b < nb; b += 32 * 8) {
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = (b + 32 * u < nb) ? pq[b + 32 * u] : 0.0;
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (b + 32 * u < nb) s += v[u];
  }
  (void)nq;
  return warp_sum(s);
}

// Totals of nq partial sums (nb blocks each); every thread of the block gets tot[0..nq).
// Warp w reduces quantities w, w + nwarps, ... so the totals' loads are in flight together.
// smem must hold nq doubles.
__device__ __forceinline__ void grid_totals(const double* part, int nb, int nq, double* smem) {
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int q = warp; q < nq; q += nw) {
    double t = warp_total(part, nb, nq, q);
    if ((threadIdx.x & 31) == 0) smem[q] = t;
  }
  __syncthreads();
}

__device__ __forceinline__ bool finite(double x) { return isfinite(x); }

// Load of data that no thread writes while the kernel runs (matrix values, index arrays,
// Jacobi inverses) through the read-only data path. Used by the AMG-PCG, where it measured
// faster on the 524k duct; never for a vector the kernel writes.
template <class T>
__device__ __forceinline__ T ldro(const T* p) {
  return __ldg(p);
}

}  // namespace b2s

// Checks launch errors and maps them to the ABI's status codes.
#define B2S_LAUNCH_CHECK()                                  \
  do {                                                      \
    cudaError_t _e = cudaGetLastError();                    \
    if (_e != cudaSuccess) return B2S_ERR_LAUNCH;           \
  } while (0)
