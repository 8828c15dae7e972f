// Per-cell access helpers shared by the scalar, reaction and adjoint kernels:
// periodic neighbours, pull gathers and whole-cell loads and stores of a
// [Q, Z, Y, X] population field.
#pragma once

#include "collide.cuh"
#include "common.cuh"

namespace lbcube {

struct Neighbours {
  int xm, xp, ym, yp, zm, zp;
};

__device__ __forceinline__ Neighbours neighbours(const Grid& g, int x, int y, int z) {
  Neighbours n;
  n.xm = x == 0 ? g.nx - 1 : x - 1;
  n.xp = x == g.nx - 1 ? 0 : x + 1;
  n.ym = y == 0 ? g.ny - 1 : y - 1;
  n.yp = y == g.ny - 1 ? 0 : y + 1;
  n.zm = z == 0 ? g.nz - 1 : z - 1;
  n.zp = z == g.nz - 1 ? 0 : z + 1;
  return n;
}

// Pull-gather of all Q populations of lattice L at (x, y, z) (lattice_core.hpp:70-78).
template <class L, class Real>
__device__ __forceinline__ void gather(const Real* __restrict__ cur, const Grid& g,
                                       const Neighbours& n, int x, int y, int z,
                                       Real (&f)[L::Q]) {
  const size_t plane = (size_t)g.plane;
  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
    const int sx = cx == 0 ? x : (cx > 0 ? n.xm : n.xp);
    const int sy = cy == 0 ? y : (cy > 0 ? n.ym : n.yp);
    const int sz = cz == 0 ? z : (cz > 0 ? n.zm : n.zp);
    f[i] = __ldg(cur + plane * i + ((sz * g.ny + sy) * g.nx + sx));
  });
}

// All Q populations of the cell itself.
template <class L, class Real>
__device__ __forceinline__ void load_cell(const Real* __restrict__ cur, const Grid& g, int cell,
                                          Real (&f)[L::Q]) {
  const size_t plane = (size_t)g.plane;
  static_for<L::Q>([&](auto I) { f[LB_I(I)] = __ldg(cur + plane * LB_I(I) + cell); });
}

template <class L, class Real>
__device__ __forceinline__ void store_cell(Real* __restrict__ out, const Grid& g, int cell,
                                           const Real (&f)[L::Q]) {
  const size_t plane = (size_t)g.plane;
  static_for<L::Q>([&](auto I) { out[plane * LB_I(I) + cell] = f[LB_I(I)]; });
}

// Fluid velocity at a cell from its populations (compute_macro_state).
template <class FL, class Real>
__device__ __forceinline__ void fluid_velocity(const Real (&f)[FL::Q], Real (&u)[FL::D]) {
  Real rho;
  macro_state<FL>(f, rho, u);
}

}  // namespace lbcube
