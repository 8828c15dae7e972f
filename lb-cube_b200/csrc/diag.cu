// Device-resident fluid diagnostics and blow-up guard.
//
// Replaces the host loops of log_diagnostics (include/lattice_io.hpp:182-234)
// and compute_max_velocity (src/turbulent_tgv_3d.cpp:150-173), which need the
// whole population field copied to the host (src/main.cpp:595-606). Pass 1
// reads the Q populations of every cell once (one cell per thread, coalesced
// rows) and writes per-block partials; pass 2 (one cluster of blocks) adds them
// in a fixed order. The host reads five doubles instead of Q values per cell. The fused
// form, one collide-stream step that also reduces the diagnostics of the state
// it writes, is lbm_step_diagnostics_async (fluid_step.cu).
#include <cooperative_groups.h>

#include "collide.cuh"
#include "common.cuh"
#include "diag.cuh"
#include "../../include/lbcube_b200.h"

namespace lbcube {

template <class L, class Real>
__global__ void __launch_bounds__(kThreads)
    diag_partials_kernel(const Real* __restrict__ f, Grid g, double* __restrict__ partials) {
  pdl_enter();
  int x, y, z;
  DiagAcc acc;
  if (cell_of(g, x, y, z)) {
    const size_t plane = (size_t)g.plane;
    const int cell = (z * g.ny + y) * g.nx + x;
    Real v[L::Q];
    static_for<L::Q>([&](auto I) { v[LB_I(I)] = __ldg(f + plane * LB_I(I) + cell); });
    diag_cell<L>(v, acc);
  }
  diag_block_to(acc, partials + block_linear() * kDiagPartials);
}

constexpr int kDiagFinalThreads = 1024;
// Blocks of the second pass: one thread-block cluster, each block taking every
// kDiagFinalBlocks-th run of kDiagFinalThreads partials; the blocks' totals
// meet in rank order through distributed shared memory (a fixed order).
#ifndef LBCUBE_FINAL_BLOCKS
#define LBCUBE_FINAL_BLOCKS 8
#endif
constexpr int kDiagFinalBlocks = LBCUBE_FINAL_BLOCKS;

__global__ void __cluster_dims__(kDiagFinalBlocks, 1, 1) __launch_bounds__(kDiagFinalThreads)
    diag_finalize_kernel(const double* __restrict__ partials, long long count,
                         double speed_limit, double* __restrict__ out) {
  __shared__ double sh[kDiagFinalThreads][kDiagPartials];
  pdl_enter();
  double m = 0.0, k = 0.0, n = 0.0, v = 0.0;
  for (long long b = (long long)blockIdx.x * kDiagFinalThreads + threadIdx.x; b < count;
       b += (long long)kDiagFinalBlocks * kDiagFinalThreads) {
    m += partials[b * kDiagPartials + 0];
    k += partials[b * kDiagPartials + 1];
    n += partials[b * kDiagPartials + 2];
    v = fmax(v, partials[b * kDiagPartials + 3]);
  }
  sh[threadIdx.x][0] = m;
  sh[threadIdx.x][1] = k;
  sh[threadIdx.x][2] = n;
  sh[threadIdx.x][3] = v;
  __syncthreads();
  for (int stride = kDiagFinalThreads / 2; stride > 0; stride >>= 1) {
    if ((int)threadIdx.x < stride) {
      sh[threadIdx.x][0] += sh[threadIdx.x + stride][0];
      sh[threadIdx.x][1] += sh[threadIdx.x + stride][1];
      sh[threadIdx.x][2] += sh[threadIdx.x + stride][2];
      sh[threadIdx.x][3] = fmax(sh[threadIdx.x][3], sh[threadIdx.x + stride][3]);
    }
    __syncthreads();
  }
  bool holder = threadIdx.x == 0;
  double tot[kDiagPartials] = {sh[0][0], sh[0][1], sh[0][2], sh[0][3]};
  if constexpr (kDiagFinalBlocks > 1) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    cluster.sync();
    holder = holder && cluster.block_rank() == 0;
    if (holder) {
      for (unsigned int r = 1; r < (unsigned int)kDiagFinalBlocks; ++r) {
        const double* remote = cluster.map_shared_rank(&sh[0][0], r);
        tot[0] += remote[0];
        tot[1] += remote[1];
        tot[2] += remote[2];
        tot[3] = fmax(tot[3], remote[3]);
      }
    }
    cluster.sync();
  }
  if (holder) {
    const double vmax = tot[3], nonfinite = tot[2];
    out[0] = tot[0];
    out[1] = tot[1];
    out[2] = vmax;
    out[3] = nonfinite;
    out[4] = (nonfinite > 0.0 || vmax > speed_limit) ? 1.0 : 0.0;
  }
}

cudaError_t launch_diag_finalize(const double* partials, long long count, double speed_limit,
                                 double* out, cudaStream_t s) {
  // programmatic dependent launches (the diagnostics kernels open with pdl_enter)
  return launch_pdl(diag_finalize_kernel, dim3(kDiagFinalBlocks), dim3(kDiagFinalThreads), 0, s, partials,
                    count, speed_limit, out);
}

template <class L, class Real>
cudaError_t launch_diagnostics(const void* vf, size_t nx, size_t ny, size_t nz, double speed_limit,
                               double* partials, size_t pbytes, double* out, cudaStream_t s) {
  const Real* f = static_cast<const Real*>(vf);
  Grid g;
  cudaError_t err = validate_domain(f == nullptr || partials == nullptr || out == nullptr, 1, 1, 1,
                                    L::D, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  const size_t need = (size_t)g.blocks() * kDiagPartials * sizeof(double);
  if (pbytes < need) return cudaErrorInvalidValue;
  const Span reads[1] = {{f, (size_t)L::Q * g.plane * sizeof(Real)}};
  const Span writes[2] = {{partials, need}, {out, kDiagOut * sizeof(double)}};
  if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  err = launch_pdl(diag_partials_kernel<L, Real>, grid_dims(g), dim3(block_dims(g)), 0, s, f, g, partials);
  if (err != cudaSuccess) return err;
  return launch_diag_finalize(partials, g.blocks(), speed_limit, out, s);
}

template <class Real>
cudaError_t diagnostics_by_lattice(int lattice, const void* f, size_t nx, size_t ny, size_t nz,
                                   double speed_limit, double* partials, size_t pbytes,
                                   double* out, cudaStream_t s) {
  switch (lattice) {
    case kD2Q9: return launch_diagnostics<D2Q9, Real>(f, nx, ny, nz, speed_limit, partials, pbytes, out, s);
    case kD3Q19: return launch_diagnostics<D3Q19, Real>(f, nx, ny, nz, speed_limit, partials, pbytes, out, s);
    case kD3Q27: return launch_diagnostics<D3Q27, Real>(f, nx, ny, nz, speed_limit, partials, pbytes, out, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace lbcube

using namespace lbcube;

extern "C" size_t lbm_diagnostics_partials_bytes(int lattice, size_t x_extent, size_t y_extent,
                                                 size_t z_extent) {
  Grid g;
  const int dims = lattice == LBM_D2Q9 || lattice == LBM_D2Q5 ? 2 : 3;
  if (validate_domain(false, 1, 1, 1, dims, x_extent, y_extent, z_extent, g) != cudaSuccess)
    return 0;
  return (size_t)g.blocks() * kDiagPartials * sizeof(double);
}

extern "C" int lbm_fluid_diagnostics_async(int lattice, int precision, const void* populations,
                                           size_t x_extent, size_t y_extent, size_t z_extent,
                                           double speed_limit, double* partials,
                                           size_t partials_bytes, double* diagnostics,
                                           void* stream) {
  const cudaStream_t s = as_stream(stream);
  if (precision == LBM_FLOAT)
    return (int)diagnostics_by_lattice<float>(lattice, populations, x_extent, y_extent, z_extent,
                                              speed_limit, partials, partials_bytes, diagnostics, s);
  if (precision == LBM_DOUBLE)
    return (int)diagnostics_by_lattice<double>(lattice, populations, x_extent, y_extent, z_extent,
                                               speed_limit, partials, partials_bytes, diagnostics,
                                               s);
  return (int)cudaErrorInvalidValue;
}
