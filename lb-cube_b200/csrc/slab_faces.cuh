// Face buffers of a z-slab of the coupled fluid + A + B -> C state, and the
// three ways a slab kernel touches them. No reference counterpart: LB-Cube
// steps one periodic box on one device.
//
// A rank owns planes [0, nz) of a box cut along z (slab.cu holds the fluid
// alone). One face buffer per side holds, per crossing population in
// ascending i, an ny x nx plane: first the fluid's (5 of 19 for D3Q19, 9 of 27
// for D3Q27), then species A's and B's (1 of 7 each for D3Q7).
// * gather_slab (forward pull): populations with c_z = +1 at plane 0 come
//   from halo_lo (the lower neighbour's top-plane sends), c_z = -1 at plane
//   nz - 1 from halo_hi; everything else from the slab's own planes.
// * send_slab (forward): the populations of a face cell that leave the slab,
//   at the cell's own (x, y).
// * scatter_slab (adjoint): the adjoint of a pull is a scatter to the pull
//   sources; a source outside the slab (c_z = +1 at plane 0, c_z = -1 at plane
//   nz - 1) goes to send_lo / send_hi at the source's (x, y), and the
//   neighbour writes it into its own plane nz - 1 / 0 (the only writer of
//   those entries: no other cell pulls them from inside that slab).
// The exchange is the same in both directions: halo_lo(r) <- send_hi(r - 1),
// halo_hi(r) <- send_lo(r + 1).
#pragma once

#include "cells.cuh"
#include "common.cuh"
#include "lattices.cuh"

namespace lbcube {

template <class L>
__host__ __device__ constexpr int face_planes() {
  return zcount_of<L>();
}
template <class FL>
__host__ __device__ constexpr int coupled_face_planes() {
  using SL = typename ScalarOf<FL>::type;
  return face_planes<FL>() + 2 * face_planes<SL>();
}

// Pull-gather with the slab's halos in place of the periodic z wrap.
template <class L, class Real>
__device__ __forceinline__ void gather_slab(const Real* __restrict__ cur, const Grid& g,
                                            const Neighbours& n, int x, int y, int z,
                                            const Real* __restrict__ halo_lo,
                                            const Real* __restrict__ halo_hi, Real (&f)[L::Q]) {
  const size_t plane = (size_t)g.plane;
  const size_t n2 = (size_t)g.ny * g.nx;
  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
    const int sx = cx == 0 ? x : (cx > 0 ? n.xm : n.xp);
    const int sy = cy == 0 ? y : (cy > 0 ? n.ym : n.yp);
    const size_t row = (size_t)sy * g.nx + sx;
    if constexpr (cz > 0) {
      f[i] = z == 0 ? __ldg(halo_lo + zslot_of<L>(i) * n2 + row)
                    : __ldg(cur + plane * i + (size_t)(z - 1) * n2 + row);
    } else if constexpr (cz < 0) {
      f[i] = z == g.nz - 1 ? __ldg(halo_hi + zslot_of<L>(i) * n2 + row)
                           : __ldg(cur + plane * i + (size_t)(z + 1) * n2 + row);
    } else {
      f[i] = __ldg(cur + plane * i + (size_t)z * n2 + row);
    }
  });
}

// Stores the populations of a face cell that leave the slab.
template <class L, class Real>
__device__ __forceinline__ void send_slab(const Grid& g, int x, int y, int z, const Real (&f)[L::Q],
                                          Real* __restrict__ send_lo, Real* __restrict__ send_hi) {
  const size_t n2 = (size_t)g.ny * g.nx;
  const size_t row = (size_t)y * g.nx + x;
  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr int cz = L::c[i][2];
    if constexpr (cz > 0) {
      if (z == g.nz - 1) send_hi[zslot_of<L>(i) * n2 + row] = f[i];
    } else if constexpr (cz < 0) {
      if (z == 0) send_lo[zslot_of<L>(i) * n2 + row] = f[i];
    }
  });
}

// lam[j](x - c_j) = mu[j] for every j, with the sources outside the slab sent
// to the neighbour instead of wrapped.
template <class L, class Real>
__device__ __forceinline__ void scatter_slab(Real* __restrict__ lam, const Grid& g,
                                             const Neighbours& n, int x, int y, int z,
                                             const Real (&mu)[L::Q], Real* __restrict__ send_lo,
                                             Real* __restrict__ send_hi) {
  const size_t plane = (size_t)g.plane;
  const size_t n2 = (size_t)g.ny * g.nx;
  static_for<L::Q>([&](auto I) {
    constexpr int j = LB_I(I);
    constexpr int cx = L::c[j][0], cy = L::c[j][1], cz = L::c[j][2];
    const int tx = cx == 0 ? x : (cx > 0 ? n.xm : n.xp);
    const int ty = cy == 0 ? y : (cy > 0 ? n.ym : n.yp);
    const size_t row = (size_t)ty * g.nx + tx;
    if constexpr (cz > 0) {
      if (z == 0) send_lo[zslot_of<L>(j) * n2 + row] = mu[j];
      else lam[plane * j + (size_t)(z - 1) * n2 + row] = mu[j];
    } else if constexpr (cz < 0) {
      if (z == g.nz - 1) send_hi[zslot_of<L>(j) * n2 + row] = mu[j];
      else lam[plane * j + (size_t)(z + 1) * n2 + row] = mu[j];
    } else {
      lam[plane * j + (size_t)z * n2 + row] = mu[j];
    }
  });
}

// The neighbour's scatter sends of one face cell into the slab's own
// adjoint field: c_z = -1 populations of plane 0 from recv_lo, c_z = +1 of
// plane nz - 1 from recv_hi (side 0: plane 0, side 1: plane nz - 1).
template <class L, class Real>
__device__ __forceinline__ void unscatter_slab(Real* __restrict__ lam, const Grid& g, int side,
                                               size_t row, const Real* __restrict__ recv_lo,
                                               const Real* __restrict__ recv_hi) {
  const size_t plane = (size_t)g.plane;
  const size_t n2 = (size_t)g.ny * g.nx;
  static_for<L::Q>([&](auto I) {
    constexpr int j = LB_I(I);
    constexpr int cz = L::c[j][2];
    if constexpr (cz < 0) {
      if (side == 0) lam[plane * j + row] = recv_lo[zslot_of<L>(j) * n2 + row];
    } else if constexpr (cz > 0) {
      if (side == 1) lam[plane * j + (size_t)(g.nz - 1) * n2 + row] = recv_hi[zslot_of<L>(j) * n2 + row];
    }
  });
}

}  // namespace lbcube
