// Fluid diagnostics on the device: the per-cell terms of log_diagnostics
// (include/lattice_io.hpp:182-234) and the blow-up test of the TGV driver
// (src/turbulent_tgv_3d.cpp:150-173, :302-316), reduced per block.
//
// Per cell, in the population precision Real and in the reference's order:
//   (rho, u) = compute_macro_state(f),  s2 = u.u,  ke = (0.5 rho) s2,
//   speed = sqrt(s2).
// Per block, four FP64 partials: sum rho, sum ke, the number of cells whose
// speed is not finite, and max speed over the cells whose speed is not NaN
// (std::max(m, speed) in the reference keeps m when speed is NaN, and takes an
// infinite speed). The sums are FP64 where the reference accumulates in Real;
// the max and the count are exact.
#pragma once

#include "collide.cuh"
#include "common.cuh"

namespace lbcube {

// Partials per block: sum rho, sum ke, non-finite cells, max speed.
constexpr int kDiagPartials = 4;
// Values written by the finalize pass.
constexpr int kDiagOut = 5;

struct DiagAcc {
  double mass = 0.0, ke = 0.0, nonfinite = 0.0, vmax = 0.0;
};

template <class L, class Real>
__device__ __forceinline__ void diag_cell(const Real (&f)[L::Q], DiagAcc& a) {
  Real rho, u[L::D];
  macro_state<L>(f, rho, u);
  const Real s2 = u_dot_u<L>(u);
  const Real ke = Real(0.5) * rho * s2;
  const Real speed = sqrt(s2);
  a.mass += (double)rho;
  a.ke += (double)ke;
  if (!isfinite(speed)) a.nonfinite += 1.0;
  a.vmax = fmax(a.vmax, (double)speed);  // fmax drops a NaN operand
}

// Reduces the block's accumulators (every thread of the block calls it; the
// block is a whole number of warps, at most kThreads threads) and writes the
// block's four partials from thread 0. Fixed reduction tree.
__device__ __forceinline__ void diag_block_to(DiagAcc a, double* out) {
  __shared__ double part[kThreads / 32][kDiagPartials];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    a.mass += __shfl_down_sync(0xffffffffu, a.mass, off);
    a.ke += __shfl_down_sync(0xffffffffu, a.ke, off);
    a.nonfinite += __shfl_down_sync(0xffffffffu, a.nonfinite, off);
    a.vmax = fmax(a.vmax, __shfl_down_sync(0xffffffffu, a.vmax, off));
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    part[warp][0] = a.mass;
    part[warp][1] = a.ke;
    part[warp][2] = a.nonfinite;
    part[warp][3] = a.vmax;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int warps = (int)(blockDim.x >> 5);
    double m = part[0][0], k = part[0][1], n = part[0][2], v = part[0][3];
    for (int w = 1; w < warps; ++w) {
      m += part[w][0];
      k += part[w][1];
      n += part[w][2];
      v = fmax(v, part[w][3]);
    }
    out[0] = m;
    out[1] = k;
    out[2] = n;
    out[3] = v;
  }
}

// Second pass (diag.cu): adds `count` block partials in a fixed order and
// writes out[0..5) = total mass, total kinetic energy, max speed, number of
// non-finite cells, and the blow-up flag 1.0 / 0.0 (a non-finite speed, or max
// speed > speed_limit: the test of turbulent_tgv_3d.cpp:305-306).
cudaError_t launch_diag_finalize(const double* partials, long long count, double speed_limit,
                                 double* out, cudaStream_t s);

}  // namespace lbcube
