// Vectorised coupled fluid + A + B -> C step: the fused step of adr.cu
// (fluid_reaction_kernel) and adr_shifted.cu on V x-adjacent cells per thread,
// with the row words and warp shuffles of the vectorised fluid step
// (stream_vec.cuh). The per-cell arithmetic is the one-cell kernels': the
// fluid collision, the velocity of the post-collision populations, and
// react_pair (collide.cuh) on the pulled scalars.
#pragma once

#include "collide.cuh"
#include "common.cuh"
#include "stream_vec.cuh"

namespace lbcube {

// SF: fluid storage policy, SS: scalar storage policy (same V and compute
// type). UOUT: also store the advecting velocity, u_out[d * N + cell].
template <class FL, class SF, class SS, int CT, bool UOUT>
__global__ void __launch_bounds__(kThreads)
    fluid_reaction_vec_kernel(const typename SF::elem* __restrict__ cur_f,
                              typename SF::elem* __restrict__ nxt_f,
                              const typename SS::elem* __restrict__ cur_a,
                              typename SS::elem* __restrict__ nxt_a,
                              const typename SS::elem* __restrict__ cur_b,
                              typename SS::elem* __restrict__ nxt_b, VecGrid vg,
                              typename SF::compute omega, typename SF::compute omega_minus,
                              typename SF::compute omega_c, typename SF::compute k,
                              typename SF::Params pf, typename SS::Params ps,
                              typename SF::compute* __restrict__ u_out) {
  using SL = typename ScalarOf<FL>::type;
  using R = typename SF::compute;
  static_assert(SS::V == SF::V, "fluid and scalars move the same cells per thread");
  constexpr int V = SF::V;
  const Grid& g = vg.g;
  const int yb = blockIdx.x / vg.xblocks;
  const int xb = blockIdx.x - yb * vg.xblocks;
  const int x0 = (xb * vg.tx + (int)(threadIdx.x % vg.tx)) * V;
  const int y = yb * vg.ty + (int)(threadIdx.x / vg.tx);
  const int z = blockIdx.y;
  const bool active = x0 < g.nx && y < g.ny;
  const int yy = y < g.ny ? y : 0;
  R u[V][FL::D];
  {
    R f[V][FL::Q];
    gather_vec<FL, SF>(cur_f, g, x0, yy, z, active, pf, f);
    if (active) {
#pragma unroll
      for (int j = 0; j < V; ++j) {
        SF::template collide_cell<FL, CT>(f[j], omega, omega_minus, pf);
        SF::template velocity<FL>(f[j], pf, u[j]);
      }
      store_vec<FL, SF>(nxt_f, g, x0, y, z, pf, f);
    }
  }
  R a[V][SL::Q], b[V][SL::Q];
  gather_vec<SL, SS>(cur_a, g, x0, yy, z, active, ps, a);
  gather_vec<SL, SS>(cur_b, g, x0, yy, z, active, ps, b);
  if (!active) return;
#pragma unroll
  for (int j = 0; j < V; ++j) react_pair<SL>(a[j], b[j], u[j], omega_c, k);
  store_vec<SL, SS>(nxt_a, g, x0, y, z, ps, a);
  store_vec<SL, SS>(nxt_b, g, x0, y, z, ps, b);
  if constexpr (UOUT) {
    const size_t plane = (size_t)g.plane;
    const size_t cell = (size_t)(z * g.ny + y) * g.nx + x0;
#pragma unroll
    for (int j = 0; j < V; ++j)
      static_for<FL::D>([&](auto D) { u_out[plane * LB_I(D) + cell + j] = u[j][LB_I(D)]; });
  }
}

// Whether every buffer of a coupled step is aligned for the words of V cells.
template <class SF, class SS>
inline bool coupled_vec_eligible(const Grid& g, const void* cf, const void* nf, const void* ca,
                                 const void* na, const void* cb, const void* nb) {
  return vec_eligible<SF>(g, cf, nf) && vec_eligible<SS>(g, ca, na) && vec_eligible<SS>(g, cb, nb);
}

}  // namespace lbcube
