// Equilibrium initialisation on the device: per cell, the equilibrium of the
// given density (or concentration) and velocity, evaluated exactly as
// compute_equilibrium (include/lattice_physics.hpp:267-290) and
// compute_scalar_equilibrium (:643-659) do on the host in every reference
// driver and test (e.g. tests/test_validation.cpp:41-56,
// src/turbulent_tgv_3d.cpp:87-106). Inputs are rho[N] and u[D*N]
// (component-major) in the population precision.
#include "collide.cuh"
#include "common.cuh"
#include "../../include/lbcube_b200.h"

namespace lbcube {

template <class L, class Real, bool SCALAR>
__global__ void __launch_bounds__(kThreads)
    init_equilibrium_kernel(const Real* __restrict__ rho, const Real* __restrict__ u,
                            Real* __restrict__ out, Grid g) {
  int x, y, z;
  if (!cell_of(g, x, y, z)) return;
  const size_t plane = (size_t)g.plane;
  const int cell = (z * g.ny + y) * g.nx + x;
  const Real r = rho[cell];
  Real uu[L::D];
  static_for<L::D>([&](auto D) { uu[LB_I(D)] = u[plane * LB_I(D) + cell]; });
  if constexpr (SCALAR) {
    static_for<L::Q>([&](auto I) { out[plane * LB_I(I) + cell] = geq<L, LB_I(I)>(r, uu); });
  } else {
    const Real usq = u_dot_u<L>(uu);
    static_for<L::Q>([&](auto I) {
      out[plane * LB_I(I) + cell] = feq<L, LB_I(I)>(r, uu, usq);
    });
  }
}

template <class L, class Real, bool SCALAR>
cudaError_t launch_init(const void* rho, const void* u, void* out, size_t nx, size_t ny, size_t nz,
                        cudaStream_t s) {
  Grid g;
  cudaError_t err = validate_domain(rho == nullptr || u == nullptr || out == nullptr, 1, 1, 1,
                                    L::D, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  const Span reads[2] = {{rho, (size_t)g.plane * sizeof(Real)},
                         {u, (size_t)L::D * g.plane * sizeof(Real)}};
  const Span writes[1] = {{out, (size_t)L::Q * g.plane * sizeof(Real)}};
  if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  init_equilibrium_kernel<L, Real, SCALAR><<<grid_dims(g), block_dims(g), 0, s>>>(
      static_cast<const Real*>(rho), static_cast<const Real*>(u), static_cast<Real*>(out), g);
  return cudaGetLastError();
}

template <class Real>
cudaError_t init_by_lattice(int lattice, const void* rho, const void* u, void* out, size_t nx,
                            size_t ny, size_t nz, cudaStream_t s) {
  switch (lattice) {
    case kD2Q9: return launch_init<D2Q9, Real, false>(rho, u, out, nx, ny, nz, s);
    case kD3Q19: return launch_init<D3Q19, Real, false>(rho, u, out, nx, ny, nz, s);
    case kD3Q27: return launch_init<D3Q27, Real, false>(rho, u, out, nx, ny, nz, s);
    case kD2Q5: return launch_init<D2Q5, Real, true>(rho, u, out, nx, ny, nz, s);
    case kD3Q7: return launch_init<D3Q7, Real, true>(rho, u, out, nx, ny, nz, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace lbcube

using namespace lbcube;

extern "C" int lbm_init_equilibrium_async(int lattice, int precision, const void* rho,
                                          const void* u, void* populations, size_t x_extent,
                                          size_t y_extent, size_t z_extent, void* stream) {
  const cudaStream_t s = as_stream(stream);
  if (precision == LBM_FLOAT)
    return (int)init_by_lattice<float>(lattice, rho, u, populations, x_extent, y_extent, z_extent,
                                       s);
  if (precision == LBM_DOUBLE)
    return (int)init_by_lattice<double>(lattice, rho, u, populations, x_extent, y_extent,
                                        z_extent, s);
  return (int)cudaErrorInvalidValue;
}
