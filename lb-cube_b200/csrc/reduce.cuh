// Deterministic FP64 block reductions for the statistics epilogues.
//
// Every block writes one partial per quantity; a second pass (one cluster of
// blocks, stats.cu / diag.cu) sums the partials in a fixed order. No atomics,
// so the result is identical from run to run for a given domain.
#pragma once

#include "common.cuh"

namespace lbcube {

// Number of FP64 sums the reactive statistics carry per block:
// sum C_A, sum C_B, sum C_A^2, sum C_B^2, sum C_A C_B (lattice_io.hpp:266-271).
constexpr int kStatSums = 5;

// Sums v[0..N) over the block (every thread must call it; the block is a
// whole number of warps, at most kThreads threads) and writes the block's
// totals to out[0..N) from thread 0. Fixed reduction tree.
template <int N>
__device__ __forceinline__ void block_sum_to(double (&v)[N], double* out) {
  __shared__ double part[kThreads / 32][N];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] += __shfl_down_sync(0xffffffffu, v[k], off);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < N; ++k) part[warp][k] = v[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int warps = (int)(blockDim.x >> 5);
#pragma unroll
    for (int k = 0; k < N; ++k) {
      double s = part[0][k];
      for (int w = 1; w < warps; ++w) s += part[w][k];
      out[k] = s;
    }
  }
}

// Sums v[0..N) over the warp (all 32 lanes must call it); lane 0 ends with
// the totals. Fixed reduction tree, no block barrier.
template <int N>
__device__ __forceinline__ void warp_sum(double (&v)[N]) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] += __shfl_down_sync(0xffffffffu, v[k], off);
  }
}

// Index of this warp's accumulation slot: kThreads / 32 slots per block.
__device__ __forceinline__ long long warp_slot() {
  return (long long)block_linear() * (kThreads / 32) + (long long)(threadIdx.x >> 5);
}

// The same for a launch over some planes of a field (plane_of): blocks indexed
// by their absolute plane, so launches over different planes of one field use
// disjoint slots (the same slots as one launch over every plane).
__device__ __forceinline__ long long warp_slot(const Grid& g) {
  return ((long long)plane_of(g) * gridDim.x + blockIdx.x) * (kThreads / 32) +
         (long long)(threadIdx.x >> 5);
}

}  // namespace lbcube
