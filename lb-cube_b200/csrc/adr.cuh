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

}  // namespace lbcube
