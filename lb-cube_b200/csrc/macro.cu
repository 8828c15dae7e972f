// Macroscopic fields on the device, for output: the quantities the VTK writer
// of the reference reconstructs on the host from a full population copy
// (write_vtk, include/lattice_io.hpp:386-451, via macro_at :78-85):
// density, velocity and |u| per cell, in the population precision and the
// reference's evaluation order (compute_macro_state, lattice_physics.hpp:227-249;
// |u| = sqrt(u.u), :199-204). For D2Q5 / D3Q7 the density slot receives the
// concentration (compute_concentration, :618-627). The host then copies
// (2 + D) values per cell instead of Q.
#include "cells.cuh"
#include "collide.cuh"
#include "common.cuh"
#include "../../include/lbcube_b200.h"

namespace lbcube {

template <class L, class Real>
__global__ void __launch_bounds__(kThreads)
    macro_fields_kernel(const Real* __restrict__ f, Grid g, Real* __restrict__ rho,
                        Real* __restrict__ u, Real* __restrict__ speed) {
  int x, y, z;
  if (!cell_of(g, x, y, z)) return;
  const int cell = (z * g.ny + y) * g.nx + x;
  const size_t plane = (size_t)g.plane;
  Real v[L::Q];
  load_cell<L>(f, g, cell, v);
  if constexpr (L::Q <= 7) {
    if (rho != nullptr) rho[cell] = concentration<L>(v);
  } else {
    Real r, uu[L::D];
    macro_state<L>(v, r, uu);
    if (rho != nullptr) rho[cell] = r;
    if (u != nullptr) static_for<L::D>([&](auto D) { u[plane * LB_I(D) + cell] = uu[LB_I(D)]; });
    if (speed != nullptr) speed[cell] = sqrt(u_dot_u<L>(uu));
  }
}

template <class L, class Real>
cudaError_t launch_macro(const void* vf, size_t nx, size_t ny, size_t nz, void* rho, void* u,
                         void* speed, cudaStream_t s) {
  Grid g;
  cudaError_t err = validate_domain(vf == nullptr, 1, 1, 1, L::D, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  if (L::Q <= 7 && (u != nullptr || speed != nullptr)) return cudaErrorInvalidValue;
  if (rho == nullptr && u == nullptr && speed == nullptr) return cudaErrorInvalidValue;
  const size_t n = (size_t)g.plane * sizeof(Real);
  const Span reads[1] = {{vf, (size_t)L::Q * n}};
  const Span writes[3] = {{rho, rho ? n : 0}, {u, u ? (size_t)L::D * n : 0}, {speed, speed ? n : 0}};
  if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  macro_fields_kernel<L, Real><<<grid_dims(g), block_dims(g), 0, s>>>(
      static_cast<const Real*>(vf), g, static_cast<Real*>(rho), static_cast<Real*>(u),
      static_cast<Real*>(speed));
  return cudaGetLastError();
}

template <class Real>
cudaError_t macro_by_lattice(int lattice, const void* f, size_t nx, size_t ny, size_t nz, void* rho,
                             void* u, void* speed, cudaStream_t s) {
  switch (lattice) {
    case kD2Q9: return launch_macro<D2Q9, Real>(f, nx, ny, nz, rho, u, speed, s);
    case kD3Q19: return launch_macro<D3Q19, Real>(f, nx, ny, nz, rho, u, speed, s);
    case kD3Q27: return launch_macro<D3Q27, Real>(f, nx, ny, nz, rho, u, speed, s);
    case kD2Q5: return launch_macro<D2Q5, Real>(f, nx, ny, nz, rho, u, speed, s);
    case kD3Q7: return launch_macro<D3Q7, Real>(f, nx, ny, nz, rho, u, speed, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace lbcube

using namespace lbcube;

extern "C" int lbm_macro_fields_async(int lattice, int precision, const void* populations,
                                      size_t x_extent, size_t y_extent, size_t z_extent,
                                      void* density, void* velocity, void* speed, void* stream) {
  const cudaStream_t s = as_stream(stream);
  if (precision == LBM_FLOAT)
    return (int)macro_by_lattice<float>(lattice, populations, x_extent, y_extent, z_extent, density,
                                        velocity, speed, s);
  if (precision == LBM_DOUBLE)
    return (int)macro_by_lattice<double>(lattice, populations, x_extent, y_extent, z_extent, density,
                                         velocity, speed, s);
  return (int)cudaErrorInvalidValue;
}
