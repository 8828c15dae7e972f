// The coupled fluid + A + B -> C step on shifted 16-bit populations
// (adr_shifted.cu), shared with the reactive adjoint.
#pragma once

#include "common.cuh"

namespace lbcube {

// One coupled step with the fluid, A and B stored as 16-bit codes of format
// FMT (fluid shifted by rho0, scalars by c0); u_out (optional, FP32 [D, N])
// receives the advecting velocity; partials (optional) the FP64 statistics.
template <class FL, int FMT>
cudaError_t fluid_reaction_shifted(int collision, const unsigned short* cur_f,
                                   unsigned short* nxt_f, const unsigned short* cur_a,
                                   unsigned short* nxt_a, const unsigned short* cur_b,
                                   unsigned short* nxt_b, float* u_out, double* partials,
                                   const Grid& g, float omega, float omega_c, float k, float rho0,
                                   float c0, cudaStream_t s);

// The same step on a z-slab (D3Q19 / D3Q27): every plane, the pulls across the
// faces from halo buffers of codes and the leaving codes into send buffers
// (layout of slab_faces.cuh); u_out may be null; no statistics.
template <class FL, int FMT>
cudaError_t fluid_reaction_shifted_slab(int collision, const unsigned short* cur_f,
                                        unsigned short* nxt_f, const unsigned short* cur_a,
                                        unsigned short* nxt_a, const unsigned short* cur_b,
                                        unsigned short* nxt_b, float* u_out, const Grid& g,
                                        float omega, float omega_c, float k, float rho0, float c0,
                                        const unsigned short* halo_lo, const unsigned short* halo_hi,
                                        unsigned short* send_lo, unsigned short* send_hi,
                                        cudaStream_t s);

}  // namespace lbcube
