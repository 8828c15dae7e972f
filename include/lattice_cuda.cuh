#pragma once
/*
 * lattice_cuda.cuh -- drop-in replacement for LB-Cube's CUDA launcher header
 * (include/lattice_cuda.cuh of the reference), backed by the B200 engine.
 *
 * Put this directory before the reference's include/ directory on the include
 * path and link against liblbcube_b200.so instead of the lbm::cuda static
 * library (CMakeLists.txt:39-75). The launcher templates keep the reference's
 * signatures, default arguments and return codes (cuh:179-319), so callers
 * such as src/main.cpp and src/simulate_reaction.cpp compile unchanged. Each
 * template forwards to the matching extern "C" symbol of lbcube_b200.h; the
 * kernels are the engine's own, so the reference's __global__ kernel
 * declarations (cuh:56-157, only reachable from nvcc-compiled callers) are
 * not provided.
 *
 * Plain C++ (g++ or nvcc); needs cuda_runtime.h for dim3 and cudaError_t.
 */

#include <cuda_runtime.h>

#include <concepts>
#include <cstddef>
#include <type_traits>

#include "lattice_memory.hpp"
#include "lattice_mrt.hpp"
#include "lattice_physics.hpp"
#include "lattice_traits.hpp"
#include "lbcube_b200.h"

namespace lbm {

#ifndef LB_CUBE_COLLISION_TYPE_DEFINED
#define LB_CUBE_COLLISION_TYPE_DEFINED
/** Compile-time collision operator selection (reference cuh:24-42). */
enum class CollisionType {
    BGK,
    TRT,
    MRT,
    RLBM
};
#endif

/** Default block hint, dim3{16, 8, 1} (reference cuh:52-54). Validated, then ignored. */
inline dim3 default_cuda_block_size() noexcept {
    return dim3{16, 8, 1};
}

namespace b200 {

template <typename T>
inline constexpr bool always_false_v = false;

#define LBCUBE_STEP_CASE(LAT, lat, REAL, real, OP, op)                                       \
    if constexpr (std::is_same_v<L, LAT> && std::is_same_v<R, REAL> &&                       \
                  CT == CollisionType::OP) {                                                 \
        return static_cast<cudaError_t>(lbm_launch_step_gpu_##lat##_##real##_##op(           \
            cur, next, x, y, z, omega, block.x, block.y, block.z));                          \
    } else

#define LBCUBE_STEP_OPS(LAT, lat, REAL, real)                                                \
    LBCUBE_STEP_CASE(LAT, lat, REAL, real, BGK, bgk)                                         \
    LBCUBE_STEP_CASE(LAT, lat, REAL, real, TRT, trt)                                         \
    LBCUBE_STEP_CASE(LAT, lat, REAL, real, MRT, mrt)                                         \
    LBCUBE_STEP_CASE(LAT, lat, REAL, real, RLBM, rlbm)

template <typename L, typename R, CollisionType CT>
inline cudaError_t step(const R* cur, R* next, std::size_t x, std::size_t y, std::size_t z,
                        R omega, dim3 block) {
    LBCUBE_STEP_OPS(D2Q9, d2q9, float, float)
    LBCUBE_STEP_OPS(D2Q9, d2q9, double, double)
    LBCUBE_STEP_OPS(D3Q19, d3q19, float, float)
    LBCUBE_STEP_OPS(D3Q19, d3q19, double, double)
    LBCUBE_STEP_OPS(D3Q27, d3q27, float, float)
    LBCUBE_STEP_OPS(D3Q27, d3q27, double, double)
    {
        static_assert(always_false_v<L>, "no engine instantiation for this lattice/precision");
        return cudaErrorInvalidValue;
    }
}
#undef LBCUBE_STEP_OPS
#undef LBCUBE_STEP_CASE

#define LBCUBE_PAIR_CASE(FLAT, fl, sl, REAL, real)                                            \
    if constexpr (std::is_same_v<FL, FLAT> && std::is_same_v<R, REAL>) {                     \
        return static_cast<cudaError_t>(CALL(fl, sl, real));                                 \
    } else

#define LBCUBE_PAIRS                                                                          \
    LBCUBE_PAIR_CASE(D2Q9, d2q9, d2q5, float, float)                                          \
    LBCUBE_PAIR_CASE(D2Q9, d2q9, d2q5, double, double)                                        \
    LBCUBE_PAIR_CASE(D3Q19, d3q19, d3q7, float, float)                                        \
    LBCUBE_PAIR_CASE(D3Q19, d3q19, d3q7, double, double)                                      \
    LBCUBE_PAIR_CASE(D3Q27, d3q27, d3q7, float, float)                                        \
    LBCUBE_PAIR_CASE(D3Q27, d3q27, d3q7, double, double)

template <typename FL, typename SL, typename R>
inline cudaError_t scalar_step(const R* cs, R* ns, const R* cf, std::size_t x, std::size_t y,
                               std::size_t z, R omega_c, R source, dim3 block) {
    static_assert(std::is_same_v<SL, typename std::conditional_t<FL::D == 2, D2Q5, D3Q7>>,
                  "the engine pairs D2Q9 with D2Q5 and D3Q19/D3Q27 with D3Q7");
#define CALL(fl, sl, real) \
    lbm_launch_scalar_step_gpu_##fl##_##sl##_##real(cs, ns, cf, x, y, z, omega_c, source, block.x, block.y, block.z)
    LBCUBE_PAIRS
#undef CALL
    {
        static_assert(always_false_v<FL>, "no engine instantiation for this lattice pair");
        return cudaErrorInvalidValue;
    }
}

template <typename FL, typename SL, typename R>
inline cudaError_t reaction_ab(const R* ca, R* na, const R* cb, R* nb, const R* cf,
                               std::size_t x, std::size_t y, std::size_t z, R omega_c, R k,
                               dim3 block) {
    static_assert(std::is_same_v<SL, typename std::conditional_t<FL::D == 2, D2Q5, D3Q7>>,
                  "the engine pairs D2Q9 with D2Q5 and D3Q19/D3Q27 with D3Q7");
#define CALL(fl, sl, real) \
    lbm_launch_reaction_ab_gpu_##fl##_##sl##_##real(ca, na, cb, nb, cf, x, y, z, omega_c, k, block.x, block.y, block.z)
    LBCUBE_PAIRS
#undef CALL
    {
        static_assert(always_false_v<FL>, "no engine instantiation for this lattice pair");
        return cudaErrorInvalidValue;
    }
}
#undef LBCUBE_PAIRS
#undef LBCUBE_PAIR_CASE

}  // namespace b200

/** Fused pull collide-stream step (reference cuh:179-190). */
template <
    IsLatticeModel Lattice,
    std::floating_point Real,
    CollisionType CT = CollisionType::BGK>
inline cudaError_t launch_step_gpu(
    const Real* current_populations,
    Real* next_populations,
    std::size_t x_extent,
    std::size_t y_extent,
    std::size_t z_extent,
    Real omega,
    dim3 block = default_cuda_block_size()) {
    return b200::step<Lattice, Real, CT>(
        current_populations, next_populations, x_extent, y_extent, z_extent, omega, block);
}

/** Passive-scalar advection-diffusion step (reference cuh:209-222). */
template <
    IsLatticeModel FluidLattice,
    IsLatticeModel ScalarLattice,
    std::floating_point Real>
inline cudaError_t launch_scalar_step_gpu(
    const Real* current_scalar,
    Real* next_scalar,
    const Real* current_fluid,
    std::size_t x_extent,
    std::size_t y_extent,
    std::size_t z_extent,
    Real omega_c,
    Real source_term = Real{},
    dim3 block = default_cuda_block_size()) {
    static_assert(FluidLattice::D == ScalarLattice::D);
    return b200::scalar_step<FluidLattice, ScalarLattice, Real>(
        current_scalar, next_scalar, current_fluid, x_extent, y_extent, z_extent, omega_c,
        source_term, block);
}

/** Scalar step with extents from host memory objects (reference cuh:243-255, cu:716-747). */
template <
    IsLatticeModel FluidLattice,
    IsLatticeModel ScalarLattice,
    std::floating_point Real>
inline cudaError_t launch_scalar_step_gpu(
    const LatticeMemory<ScalarLattice, Real>& scalar_mem,
    const LatticeMemory<FluidLattice, Real>& fluid_mem,
    const Real* current_scalar,
    Real* next_scalar,
    const Real* current_fluid,
    Real omega_c,
    Real source_term = Real{},
    dim3 block = default_cuda_block_size()) {
    static_assert(FluidLattice::D == ScalarLattice::D);
    if (scalar_mem.x_extent() != fluid_mem.x_extent() ||
        scalar_mem.y_extent() != fluid_mem.y_extent() ||
        scalar_mem.z_extent() != fluid_mem.z_extent()) {
        return cudaErrorInvalidValue;
    }
    return launch_scalar_step_gpu<FluidLattice, ScalarLattice, Real>(
        current_scalar, next_scalar, current_fluid, scalar_mem.x_extent(),
        scalar_mem.y_extent(), scalar_mem.z_extent(), omega_c, source_term, block);
}

/** Fused A + B -> C advection-diffusion-reaction step (reference cuh:276-291). */
template <
    IsLatticeModel FluidLattice,
    IsLatticeModel ScalarLattice,
    std::floating_point Real>
inline cudaError_t launch_reaction_AB_gpu(
    const Real* current_a,
    Real* next_a,
    const Real* current_b,
    Real* next_b,
    const Real* current_fluid,
    std::size_t x_extent,
    std::size_t y_extent,
    std::size_t z_extent,
    Real omega_c,
    Real k_react,
    dim3 block = default_cuda_block_size()) {
    static_assert(FluidLattice::D == ScalarLattice::D);
    return b200::reaction_ab<FluidLattice, ScalarLattice, Real>(
        current_a, next_a, current_b, next_b, current_fluid, x_extent, y_extent, z_extent,
        omega_c, k_react, block);
}

/** Step with extents from a host LatticeMemory (reference cuh:310-319, cu:680-698). */
template <
    IsLatticeModel Lattice,
    std::floating_point Real,
    CollisionType CT = CollisionType::BGK>
inline cudaError_t launch_step_gpu(
    const LatticeMemory<Lattice, Real>& mem,
    const Real* current_populations,
    Real* next_populations,
    Real omega,
    dim3 block = default_cuda_block_size()) {
    return launch_step_gpu<Lattice, Real, CT>(
        current_populations, next_populations, mem.x_extent(), mem.y_extent(), mem.z_extent(),
        omega, block);
}

}  // namespace lbm
