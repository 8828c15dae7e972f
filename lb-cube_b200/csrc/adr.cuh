// Internal entry of adr.cu shared with the reactive adjoint.
#pragma once

#include "common.cuh"

namespace lbcube {

// One fused fluid + A + B -> C step (BGK, TRT or MRT) that also stores the
// advecting velocity (the fluid velocity of the new state) into u_out [D, N].
template <class FL, class Real>
cudaError_t fluid_reaction_with_velocity(int collision, const Real* cur_f, Real* nxt_f,
                                         const Real* cur_a, Real* nxt_a, const Real* cur_b,
                                         Real* nxt_b, Real* u_out, const Grid& g, Real omega,
                                         Real omega_c, Real k, cudaStream_t s);

// The same step on a z-slab (all planes; halos and sends as
// lbm_fluid_reaction_slab_async); u_out may be null.
template <class FL, class Real>
cudaError_t fluid_reaction_slab_with_velocity(int collision, const Real* cur_f, Real* nxt_f,
                                              const Real* cur_a, Real* nxt_a, const Real* cur_b,
                                              Real* nxt_b, Real* u_out, const Grid& g, Real omega,
                                              Real omega_c, Real k, const Real* halo_lo,
                                              const Real* halo_hi, Real* send_lo, Real* send_hi,
                                              cudaStream_t s);

}  // namespace lbcube
