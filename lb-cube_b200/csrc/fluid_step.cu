// Fused pull-scheme collide-stream step for D2Q9 / D3Q19 / D3Q27 fluids:
// launchers and C-ABI entry points.
//
// Replaces launch_step_gpu (src/lattice_cuda.cu:476-520). The kernels are the
// one-cell-per-thread step (step_cell.cuh) and the vectorised step
// (stream_vec.cuh); kUseVec picks between them per lattice, operator and
// precision.
#include "collide.cuh"
#include "common.cuh"
#include "diag.cuh"
#include "step_cell.cuh"
#include "stream_vec.cuh"
#include "../../include/lbcube_b200.h"

namespace lbcube {

template <class L, class Real, int CT>
cudaError_t launch_fluid_step(const Real* cur, Real* nxt, size_t nx, size_t ny, size_t nz,
                              Real omega, unsigned bx, unsigned by, unsigned bz,
                              cudaStream_t stream) {
  Grid g;
  cudaError_t err =
      validate_domain(cur == nullptr || nxt == nullptr, bx, by, bz, L::D, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  const size_t bytes = (size_t)L::Q * (size_t)g.plane * sizeof(Real);
  const Span reads[1] = {{cur, bytes}};
  const Span writes[1] = {{nxt, bytes}};
  if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  const Real omega_minus = CT == kTRT ? trt_omega_minus<Real>(omega) : Real(0);
  if constexpr (kUseVec<L, Real, CT>) {
    using S = NativeStorage<Real, kVecCells<L, Real>>;
    if (vec_eligible<S>(g, cur, nxt)) {
      const VecGrid vg = make_vec_grid(g, S::V);
      launch_vec_step<L, S, CT>(vg, vec_grid_dims(vg), vec_block_threads(vg), stream, cur, nxt,
                                omega, omega_minus, typename S::Params{});
      return cudaGetLastError();
    }
  }
  if constexpr (kUsePlanes<L, Real, CT>)
    return launch_pdl(fluid_step_planes_kernel<L, Real, CT>, grid_dims(g), dim3(block_dims(g)), 0, stream,
                      planes_of<const Real, L::Q>(cur, g), planes_of<Real, L::Q>(nxt, g), g, omega,
                      omega_minus);
  return launch_pdl(fluid_step_kernel<L, Real, CT, false>, grid_dims(g), dim3(block_dims(g)), 0, stream,
                    cur, nxt, g, omega, omega_minus, (double*)nullptr);
}

// One step plus the diagnostics of the state it writes (diag.cuh): the
// kernel writes one partial per block, the finalize pass reduces them.
template <class L, class Real, int CT>
cudaError_t launch_fluid_step_diag(const Real* cur, Real* nxt, size_t nx, size_t ny, size_t nz,
                                   Real omega, double speed_limit, double* partials,
                                   size_t pbytes, double* out, cudaStream_t stream) {
  Grid g;
  cudaError_t err = validate_domain(cur == nullptr || nxt == nullptr || partials == nullptr ||
                                        out == nullptr,
                                    1, 1, 1, L::D, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  const size_t need = (size_t)g.blocks() * kDiagPartials * sizeof(double);
  if (pbytes < need) return cudaErrorInvalidValue;
  const size_t bytes = (size_t)L::Q * (size_t)g.plane * sizeof(Real);
  const Span reads[1] = {{cur, bytes}};
  const Span writes[3] = {{nxt, bytes}, {partials, need}, {out, kDiagOut * sizeof(double)}};
  if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  const Real omega_minus = CT == kTRT ? trt_omega_minus<Real>(omega) : Real(0);
  long long count = -1;
  if constexpr (kUseVec<L, Real, CT>) {
    using S = NativeStorage<Real, kVecCells<L, Real>>;
    if (vec_eligible<S>(g, cur, nxt)) {
      const VecGrid vg = make_vec_grid(g, S::V);
      const dim3 grid = vec_grid_dims(vg);
      count = (long long)grid.x * grid.y;  // <= g.blocks(): a vector block spans >= one row block
      err = launch_pdl(fluid_step_vec_kernel<L, S, CT, true, false>, grid, dim3(vec_block_threads(vg)), 0,
                       stream, cur, nxt, vg, omega, omega_minus, typename S::Params{}, partials,
                       SlabArgs<Real>{});
    }
  }
  if (count < 0) {
    count = g.blocks();
    err = launch_pdl(fluid_step_kernel<L, Real, CT, true>, grid_dims(g), dim3(block_dims(g)), 0, stream, cur,
                     nxt, g, omega, omega_minus, partials);
  }
  if (err != cudaSuccess) return err;
  return launch_diag_finalize(partials, count, speed_limit, out, stream);
}

template <class Real, int CT>
cudaError_t diag_dispatch_lattice(int lattice, const void* cur, void* nxt, size_t nx, size_t ny,
                                  size_t nz, double omega, double speed_limit, double* partials,
                                  size_t pbytes, double* out, cudaStream_t s) {
  const Real* c = static_cast<const Real*>(cur);
  Real* n = static_cast<Real*>(nxt);
  const Real w = Real(omega);
  switch (lattice) {
    case kD2Q9: return launch_fluid_step_diag<D2Q9, Real, CT>(c, n, nx, ny, nz, w, speed_limit, partials, pbytes, out, s);
    case kD3Q19: return launch_fluid_step_diag<D3Q19, Real, CT>(c, n, nx, ny, nz, w, speed_limit, partials, pbytes, out, s);
    case kD3Q27: return launch_fluid_step_diag<D3Q27, Real, CT>(c, n, nx, ny, nz, w, speed_limit, partials, pbytes, out, s);
    default: return cudaErrorInvalidValue;
  }
}

template <class Real>
cudaError_t diag_dispatch_collision(int lattice, int collision, const void* cur, void* nxt,
                                    size_t nx, size_t ny, size_t nz, double omega,
                                    double speed_limit, double* partials, size_t pbytes,
                                    double* out, cudaStream_t s) {
  switch (collision) {
    case kBGK: return diag_dispatch_lattice<Real, kBGK>(lattice, cur, nxt, nx, ny, nz, omega, speed_limit, partials, pbytes, out, s);
    case kTRT: return diag_dispatch_lattice<Real, kTRT>(lattice, cur, nxt, nx, ny, nz, omega, speed_limit, partials, pbytes, out, s);
    case kMRT: return diag_dispatch_lattice<Real, kMRT>(lattice, cur, nxt, nx, ny, nz, omega, speed_limit, partials, pbytes, out, s);
    case kRLBM: return diag_dispatch_lattice<Real, kRLBM>(lattice, cur, nxt, nx, ny, nz, omega, speed_limit, partials, pbytes, out, s);
    default: return cudaErrorInvalidValue;
  }
}

template <class Real, int CT>
cudaError_t dispatch_lattice(int lattice, const void* cur, void* nxt, size_t nx, size_t ny,
                             size_t nz, double omega, cudaStream_t s) {
  const Real* c = static_cast<const Real*>(cur);
  Real* n = static_cast<Real*>(nxt);
  switch (lattice) {
    case kD2Q9: return launch_fluid_step<D2Q9, Real, CT>(c, n, nx, ny, nz, Real(omega), 1, 1, 1, s);
    case kD3Q19: return launch_fluid_step<D3Q19, Real, CT>(c, n, nx, ny, nz, Real(omega), 1, 1, 1, s);
    case kD3Q27: return launch_fluid_step<D3Q27, Real, CT>(c, n, nx, ny, nz, Real(omega), 1, 1, 1, s);
    default: return cudaErrorInvalidValue;
  }
}

template <class Real>
cudaError_t dispatch_collision(int lattice, int collision, const void* cur, void* nxt, size_t nx,
                               size_t ny, size_t nz, double omega, cudaStream_t s) {
  switch (collision) {
    case kBGK: return dispatch_lattice<Real, kBGK>(lattice, cur, nxt, nx, ny, nz, omega, s);
    case kTRT: return dispatch_lattice<Real, kTRT>(lattice, cur, nxt, nx, ny, nz, omega, s);
    case kMRT: return dispatch_lattice<Real, kMRT>(lattice, cur, nxt, nx, ny, nz, omega, s);
    case kRLBM: return dispatch_lattice<Real, kRLBM>(lattice, cur, nxt, nx, ny, nz, omega, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace lbcube

using namespace lbcube;

#define LBCUBE_STEP_SYMBOL(lat, LAT, real, op, OP)                                                \
  extern "C" int lbm_launch_step_gpu_##lat##_##real##_##op(                                     \
      const real* current_populations, real* next_populations, size_t x_extent,                 \
      size_t y_extent, size_t z_extent, real omega, unsigned block_x, unsigned block_y,         \
      unsigned block_z) {                                                                       \
    return (int)launch_fluid_step<LAT, real, OP>(current_populations, next_populations,        \
                                                 x_extent, y_extent, z_extent, omega, block_x, \
                                                 block_y, block_z, (cudaStream_t)0);            \
  }

#define LBCUBE_STEP_OPS(lat, LAT, real)              \
  LBCUBE_STEP_SYMBOL(lat, LAT, real, bgk, kBGK)      \
  LBCUBE_STEP_SYMBOL(lat, LAT, real, trt, kTRT)      \
  LBCUBE_STEP_SYMBOL(lat, LAT, real, mrt, kMRT)      \
  LBCUBE_STEP_SYMBOL(lat, LAT, real, rlbm, kRLBM)

LBCUBE_STEP_OPS(d2q9, D2Q9, float)
LBCUBE_STEP_OPS(d2q9, D2Q9, double)
LBCUBE_STEP_OPS(d3q19, D3Q19, float)
LBCUBE_STEP_OPS(d3q19, D3Q19, double)
LBCUBE_STEP_OPS(d3q27, D3Q27, float)
LBCUBE_STEP_OPS(d3q27, D3Q27, double)

extern "C" int lbm_step_async(int lattice, int precision, int collision,
                              const void* current_populations, void* next_populations,
                              size_t x_extent, size_t y_extent, size_t z_extent, double omega,
                              void* stream) {
  const cudaStream_t s = as_stream(stream);
  if (precision == LBM_FLOAT)
    return (int)dispatch_collision<float>(lattice, collision, current_populations,
                                          next_populations, x_extent, y_extent, z_extent, omega, s);
  if (precision == LBM_DOUBLE)
    return (int)dispatch_collision<double>(lattice, collision, current_populations,
                                           next_populations, x_extent, y_extent, z_extent, omega,
                                           s);
  return (int)cudaErrorInvalidValue;
}

extern "C" int lbm_step_diagnostics_async(int lattice, int precision, int collision,
                                          const void* current_populations,
                                          void* next_populations, size_t x_extent,
                                          size_t y_extent, size_t z_extent, double omega,
                                          double speed_limit, double* partials,
                                          size_t partials_bytes, double* diagnostics,
                                          void* stream) {
  const cudaStream_t s = as_stream(stream);
  if (precision == LBM_FLOAT)
    return (int)diag_dispatch_collision<float>(lattice, collision, current_populations,
                                               next_populations, x_extent, y_extent, z_extent,
                                               omega, speed_limit, partials, partials_bytes,
                                               diagnostics, s);
  if (precision == LBM_DOUBLE)
    return (int)diag_dispatch_collision<double>(lattice, collision, current_populations,
                                                next_populations, x_extent, y_extent, z_extent,
                                                omega, speed_limit, partials, partials_bytes,
                                                diagnostics, s);
  return (int)cudaErrorInvalidValue;
}
