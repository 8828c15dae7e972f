/*
 * lbcube_b200.h -- C ABI of the B200 lattice Boltzmann engine.
 *
 * Drop-in boundary for LB-Cube's CUDA backend (include/lattice_cuda.cuh and
 * src/lattice_cuda.cu, the lbm::cuda static library of CMakeLists.txt:39-75).
 * Every symbol takes plain device pointers and element counts; no CUDA or
 * C++ types cross the boundary. Populations are unpadded [Q, Z, Y, X] arrays
 * with X fastest (include/lattice_memory.hpp:55-102), owned by the caller.
 * The launchers never allocate, copy or free, and never synchronise.
 *
 * Return values are cudaError_t codes (0 = cudaSuccess). The reference's
 * validation order is kept (src/lattice_cuda.cu:488-519):
 *   1. a null pointer                     -> 17 cudaErrorInvalidDevicePointer
 *   2. a zero block dimension             ->  9 cudaErrorInvalidConfiguration
 *   3. (2D lattices: z and block.z := 1)
 *   4. a zero extent                      ->  1 cudaErrorInvalidValue
 *   5. otherwise the launch status (cudaGetLastError after the launch).
 * Two checks are added, both returning 1 cudaErrorInvalidValue: a read
 * buffer that overlaps a write buffer (the reference would race), and a
 * domain with more than 2^31 - 1 cells (the kernels index a population
 * plane with 32-bit offsets). The block arguments are validated as above but
 * otherwise ignored: the kernels choose their own tiling.
 *
 * Launchers without a `stream` argument run on the legacy default stream,
 * like the reference. The *_async extensions take a cudaStream_t passed as
 * void* and cover the same kernels plus the engine's additions.
 *
 * Enum codes used by the extensions:
 *   lattice   LBM_D2Q9 0, LBM_D3Q19 1, LBM_D3Q27 2, LBM_D2Q5 3, LBM_D3Q7 4
 *   precision LBM_FLOAT 0, LBM_DOUBLE 1
 *   collision LBM_BGK 0, LBM_TRT 1, LBM_MRT 2, LBM_RLBM 3
 *   16-bit storage format LBM_F16S 2, LBM_BF16S 3, LBM_E3M12S 4, LBM_Q15S 5
 */
#ifndef LBCUBE_B200_H
#define LBCUBE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { LBM_D2Q9 = 0, LBM_D3Q19 = 1, LBM_D3Q27 = 2, LBM_D2Q5 = 3, LBM_D3Q7 = 4 };
enum { LBM_FLOAT = 0, LBM_DOUBLE = 1 };
enum { LBM_BGK = 0, LBM_TRT = 1, LBM_MRT = 2, LBM_RLBM = 3 };
enum { LBM_F16S = 2, LBM_BF16S = 3, LBM_E3M12S = 4, LBM_Q15S = 5 };
enum { LBM_NATIVE = 0 }; /* population storage in the stated precision */

/* ---------------------------------------------------------------------------
 * Fused pull collide-stream step, one symbol per instantiation. Each replaces
 *   template <L, Real, CT> cudaError_t lbm::launch_step_gpu(
 *       const Real* current, Real* next, size_t x, size_t y, size_t z,
 *       Real omega, dim3 block = {16, 8, 1})
 * declared at include/lattice_cuda.cuh:179-190, defined at
 * src/lattice_cuda.cu:476-520 and instantiated at :808-858. The
 * LatticeMemory overload (cuh:310-319, cu:680-698) forwards here with the
 * memory object's extents.
 * omega is the BGK relaxation frequency, the TRT even frequency (odd one from
 * Lambda = 1/4, lattice_physics.hpp:336-344), the MRT shear rate s_nu, or the
 * RLBM frequency.
 * ------------------------------------------------------------------------- */
/* lbm::launch_step_gpu<D2Q9, float, CollisionType::BGK> */
int lbm_launch_step_gpu_d2q9_float_bgk(const float* current_populations, float* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, float omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D2Q9, float, CollisionType::TRT> */
int lbm_launch_step_gpu_d2q9_float_trt(const float* current_populations, float* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, float omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D2Q9, float, CollisionType::MRT> */
int lbm_launch_step_gpu_d2q9_float_mrt(const float* current_populations, float* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, float omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D2Q9, float, CollisionType::RLBM> */
int lbm_launch_step_gpu_d2q9_float_rlbm(const float* current_populations, float* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, float omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D2Q9, double, CollisionType::BGK> */
int lbm_launch_step_gpu_d2q9_double_bgk(const double* current_populations, double* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, double omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D2Q9, double, CollisionType::TRT> */
int lbm_launch_step_gpu_d2q9_double_trt(const double* current_populations, double* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, double omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D2Q9, double, CollisionType::MRT> */
int lbm_launch_step_gpu_d2q9_double_mrt(const double* current_populations, double* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, double omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D2Q9, double, CollisionType::RLBM> */
int lbm_launch_step_gpu_d2q9_double_rlbm(const double* current_populations, double* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, double omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D3Q19, float, CollisionType::BGK> */
int lbm_launch_step_gpu_d3q19_float_bgk(const float* current_populations, float* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, float omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D3Q19, float, CollisionType::TRT> */
int lbm_launch_step_gpu_d3q19_float_trt(const float* current_populations, float* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, float omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D3Q19, float, CollisionType::MRT> */
int lbm_launch_step_gpu_d3q19_float_mrt(const float* current_populations, float* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, float omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D3Q19, float, CollisionType::RLBM> */
int lbm_launch_step_gpu_d3q19_float_rlbm(const float* current_populations, float* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, float omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D3Q19, double, CollisionType::BGK> */
int lbm_launch_step_gpu_d3q19_double_bgk(const double* current_populations, double* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, double omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D3Q19, double, CollisionType::TRT> */
int lbm_launch_step_gpu_d3q19_double_trt(const double* current_populations, double* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, double omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D3Q19, double, CollisionType::MRT> */
int lbm_launch_step_gpu_d3q19_double_mrt(const double* current_populations, double* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, double omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D3Q19, double, CollisionType::RLBM> */
int lbm_launch_step_gpu_d3q19_double_rlbm(const double* current_populations, double* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, double omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D3Q27, float, CollisionType::BGK> */
int lbm_launch_step_gpu_d3q27_float_bgk(const float* current_populations, float* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, float omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D3Q27, float, CollisionType::TRT> */
int lbm_launch_step_gpu_d3q27_float_trt(const float* current_populations, float* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, float omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D3Q27, float, CollisionType::MRT> */
int lbm_launch_step_gpu_d3q27_float_mrt(const float* current_populations, float* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, float omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D3Q27, float, CollisionType::RLBM> */
int lbm_launch_step_gpu_d3q27_float_rlbm(const float* current_populations, float* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, float omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D3Q27, double, CollisionType::BGK> */
int lbm_launch_step_gpu_d3q27_double_bgk(const double* current_populations, double* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, double omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D3Q27, double, CollisionType::TRT> */
int lbm_launch_step_gpu_d3q27_double_trt(const double* current_populations, double* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, double omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D3Q27, double, CollisionType::MRT> */
int lbm_launch_step_gpu_d3q27_double_mrt(const double* current_populations, double* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, double omega,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_step_gpu<D3Q27, double, CollisionType::RLBM> */
int lbm_launch_step_gpu_d3q27_double_rlbm(const double* current_populations, double* next_populations,
    size_t x_extent, size_t y_extent, size_t z_extent, double omega,
    unsigned block_x, unsigned block_y, unsigned block_z);

/* ---------------------------------------------------------------------------
 * Passive-scalar advection-diffusion step. Each replaces
 *   template <FL, SL, Real> cudaError_t lbm::launch_scalar_step_gpu(
 *       const Real* current_scalar, Real* next_scalar, const Real* current_fluid,
 *       size_t x, size_t y, size_t z, Real omega_c, Real source_term = 0,
 *       dim3 block = {16, 8, 1})
 * (include/lattice_cuda.cuh:209-222, src/lattice_cuda.cu:539-589, instantiated
 * at :925-991). The fluid velocity is read at the destination cell.
 * ------------------------------------------------------------------------- */
/* lbm::launch_scalar_step_gpu<D2Q9, D2Q5, float> */
int lbm_launch_scalar_step_gpu_d2q9_d2q5_float(const float* current_scalar, float* next_scalar,
    const float* current_fluid, size_t x_extent, size_t y_extent, size_t z_extent,
    float omega_c, float source_term, unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_scalar_step_gpu<D2Q9, D2Q5, double> */
int lbm_launch_scalar_step_gpu_d2q9_d2q5_double(const double* current_scalar, double* next_scalar,
    const double* current_fluid, size_t x_extent, size_t y_extent, size_t z_extent,
    double omega_c, double source_term, unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_scalar_step_gpu<D3Q19, D3Q7, float> */
int lbm_launch_scalar_step_gpu_d3q19_d3q7_float(const float* current_scalar, float* next_scalar,
    const float* current_fluid, size_t x_extent, size_t y_extent, size_t z_extent,
    float omega_c, float source_term, unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_scalar_step_gpu<D3Q19, D3Q7, double> */
int lbm_launch_scalar_step_gpu_d3q19_d3q7_double(const double* current_scalar, double* next_scalar,
    const double* current_fluid, size_t x_extent, size_t y_extent, size_t z_extent,
    double omega_c, double source_term, unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_scalar_step_gpu<D3Q27, D3Q7, float> */
int lbm_launch_scalar_step_gpu_d3q27_d3q7_float(const float* current_scalar, float* next_scalar,
    const float* current_fluid, size_t x_extent, size_t y_extent, size_t z_extent,
    float omega_c, float source_term, unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_scalar_step_gpu<D3Q27, D3Q7, double> */
int lbm_launch_scalar_step_gpu_d3q27_d3q7_double(const double* current_scalar, double* next_scalar,
    const double* current_fluid, size_t x_extent, size_t y_extent, size_t z_extent,
    double omega_c, double source_term, unsigned block_x, unsigned block_y, unsigned block_z);

/* ---------------------------------------------------------------------------
 * Fused A + B -> C advection-diffusion-reaction step. Each replaces
 *   template <FL, SL, Real> cudaError_t lbm::launch_reaction_AB_gpu(
 *       const Real* current_a, Real* next_a, const Real* current_b,
 *       Real* next_b, const Real* current_fluid, size_t x, size_t y, size_t z,
 *       Real omega_c, Real k_react, dim3 block = {16, 8, 1})
 * (include/lattice_cuda.cuh:276-291, src/lattice_cuda.cu:610-666,
 * instantiated at :1012-1029).
 * ------------------------------------------------------------------------- */
/* lbm::launch_reaction_AB_gpu<D2Q9, D2Q5, float> */
int lbm_launch_reaction_ab_gpu_d2q9_d2q5_float(const float* current_a, float* next_a,
    const float* current_b, float* next_b, const float* current_fluid,
    size_t x_extent, size_t y_extent, size_t z_extent, float omega_c, float k_react,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_reaction_AB_gpu<D2Q9, D2Q5, double> */
int lbm_launch_reaction_ab_gpu_d2q9_d2q5_double(const double* current_a, double* next_a,
    const double* current_b, double* next_b, const double* current_fluid,
    size_t x_extent, size_t y_extent, size_t z_extent, double omega_c, double k_react,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_reaction_AB_gpu<D3Q19, D3Q7, float> */
int lbm_launch_reaction_ab_gpu_d3q19_d3q7_float(const float* current_a, float* next_a,
    const float* current_b, float* next_b, const float* current_fluid,
    size_t x_extent, size_t y_extent, size_t z_extent, float omega_c, float k_react,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_reaction_AB_gpu<D3Q19, D3Q7, double> */
int lbm_launch_reaction_ab_gpu_d3q19_d3q7_double(const double* current_a, double* next_a,
    const double* current_b, double* next_b, const double* current_fluid,
    size_t x_extent, size_t y_extent, size_t z_extent, double omega_c, double k_react,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_reaction_AB_gpu<D3Q27, D3Q7, float> */
int lbm_launch_reaction_ab_gpu_d3q27_d3q7_float(const float* current_a, float* next_a,
    const float* current_b, float* next_b, const float* current_fluid,
    size_t x_extent, size_t y_extent, size_t z_extent, float omega_c, float k_react,
    unsigned block_x, unsigned block_y, unsigned block_z);
/* lbm::launch_reaction_AB_gpu<D3Q27, D3Q7, double> */
int lbm_launch_reaction_ab_gpu_d3q27_d3q7_double(const double* current_a, double* next_a,
    const double* current_b, double* next_b, const double* current_fluid,
    size_t x_extent, size_t y_extent, size_t z_extent, double omega_c, double k_react,
    unsigned block_x, unsigned block_y, unsigned block_z);

/* ---------------------------------------------------------------------------
 * Stream-ordered extensions (no reference counterpart unless stated).
 * `precision` selects float or double for every population pointer.
 * ------------------------------------------------------------------------- */

/* Any of the 24 step instantiations above, on `stream` (same validation). */
int lbm_step_async(int lattice, int precision, int collision, const void* current_populations,
    void* next_populations, size_t x_extent, size_t y_extent, size_t z_extent, double omega,
    void* stream);

/* Any of the 6 scalar-step instantiations above; `fluid_lattice` picks the pair. */
int lbm_scalar_step_async(int fluid_lattice, int precision, const void* current_scalar,
    void* next_scalar, const void* current_fluid, size_t x_extent, size_t y_extent,
    size_t z_extent, double omega_c, double source_term, void* stream);

/* Any of the 6 reaction instantiations above. */
int lbm_reaction_ab_async(int fluid_lattice, int precision, const void* current_a, void* next_a,
    const void* current_b, void* next_b, const void* current_fluid, size_t x_extent,
    size_t y_extent, size_t z_extent, double omega_c, double k_react, void* stream);

/* One launch doing what the reference's reaction driver does with two
 * (src/simulate_reaction.cpp:518-543): the fluid step, then the reaction step
 * advected by the post-step fluid. The velocity is recomputed from the
 * post-collision populations held in registers, which are the values the
 * separate reaction launch would read back, so the result is the same and the
 * fluid is not re-read. When `stats_partials` is non-null the launch also
 * accumulates the reactive statistics of the post-step scalar fields into it
 * (FP64 per-block partial sums; size from lbm_stats_partials_bytes);
 * lbm_reactive_stats_finalize_async then turns them into the 8 diagnostics. */
int lbm_fluid_reaction_ab_async(int fluid_lattice, int precision, int collision,
    const void* current_fluid, void* next_fluid, const void* current_a, void* next_a,
    const void* current_b, void* next_b, size_t x_extent, size_t y_extent, size_t z_extent,
    double omega, double omega_c, double k_react, double* stats_partials,
    size_t stats_partials_bytes, void* stream);

/* The same coupled step on shifted 16-bit populations (`format` LBM_F16S,
 * LBM_BF16S, LBM_E3M12S or LBM_Q15S; no reference counterpart): the fluid is
 * stored as codes of S (f_i / w_i - rho0) and collides on the deviations (BGK,
 * TRT, or MRT on D2Q9 / D3Q19), the scalars as codes of S (g_i / w_i - c0)
 * (c0 a reference concentration, e.g. 0.5 for fields in [0, 1]), reacted in
 * FP32 as the FP32 step reacts them; half the bytes of the FP32 step. Fields are
 * encoded and decoded with lbm_encode_shifted_async / lbm_decode_shifted_async
 * (rho0 for the fluid, c0 for the scalars). Statistics partials as above, of the
 * FP32 values the step encodes. */
int lbm_fluid_reaction_ab_shifted_async(int fluid_lattice, int format, int collision,
    const void* current_fluid, void* next_fluid, const void* current_a, void* next_a,
    const void* current_b, void* next_b, size_t x_extent, size_t y_extent, size_t z_extent,
    double omega, double omega_c, double k_react, float rho0, float c0, double* stats_partials,
    size_t stats_partials_bytes, void* stream);

/* Bytes of FP64 partial sums the statistics kernels write for this domain. */
size_t lbm_stats_partials_bytes(int fluid_lattice, size_t x_extent, size_t y_extent,
    size_t z_extent);

/* Reactive-mixing statistics of two scalar fields, replacing the host loop of
 * lbm::compute_reactive_stats (include/lattice_io.hpp:256-338). Sums of C_A,
 * C_B, C_A^2, C_B^2 and C_A C_B are accumulated in FP64 with a fixed-order
 * two-pass reduction (deterministic run to run). `partials` is caller-owned
 * scratch of lbm_stats_partials_bytes bytes. `diagnostics` (device, 8
 * doubles) receives mean_A, mean_B, var_A, var_B, covariance,
 * segregation_intensity, true_reaction_rate, mixed_reaction_rate
 * (ReactiveDiagnostics, include/lattice_io.hpp:148-166). As in the
 * reference, k_react is taken in the population precision. */
int lbm_reactive_stats_async(int scalar_lattice, int precision, const void* current_a,
    const void* current_b, size_t x_extent, size_t y_extent, size_t z_extent, double k_react,
    double* partials, size_t partials_bytes, double* diagnostics, void* stream);

/* ---------------------------------------------------------------------------
 * Shifted 16-bit population storage (no reference counterpart). A population
 * is stored as a 16-bit code of v_i = S (f_i / w_i - rho0), round to nearest,
 * and read back as f_i = w_i (rho0 + v_i / S):
 *   LBM_F16S   IEEE binary16, S = 4096
 *   LBM_BF16S  bfloat16, S = 1
 *   LBM_E3M12S sign | 3-bit exponent E | 12-bit mantissa m, S = 1, standing
 *              for |v| = 2^(E-6) (1 + m/4096) - 2^-6: uniform 2^-18 grid near
 *              zero, 13-bit relative precision above ~1/64, |v| < 3.98,
 *              saturating
 *   LBM_Q15S   16-bit fixed point, v rounded to an integer, S = 32768:
 *              uniform 2^-15 grid over |f/w - rho0| < 1; stored offset
 *              binary (code = round(v) + 32768), saturating (NaN to one
 *              of the bounds)
 * Half the bytes of FP32 storage; collision in FP32 registers (BGK, TRT and
 * D2Q9 / D3Q19 MRT on the deviations v, D3Q27 MRT and RLBM on the decoded f
 * with the FP32 operator code). Where the step collides on the deviations it
 * rounds FP16 and BF16 stochastically (unbiased; the random bits come from
 * the values themselves, so the step is deterministic); conversions and the
 * other paths round to nearest. Buffers are uint16 [Q, Z, Y, X]; x_extent
 * must be a multiple of 4 and buffers 8-byte aligned (else
 * cudaErrorInvalidValue). rho0 is the reference density of the shift. With
 * x_extent a multiple of 8 (at most 1024) and 16-byte aligned buffers, the
 * D2Q9 / D3Q19 BGK, TRT and MRT steps stage each row's source rows in shared
 * memory with bulk copies (see lbm_stage_timeouts).
 * ------------------------------------------------------------------------- */
int lbm_step_shifted_async(int lattice, int format, int collision,
    const void* current_populations, void* next_populations, size_t x_extent,
    size_t y_extent, size_t z_extent, float omega, float rho0, void* stream);

/* Blocks of the row-staged 16-bit step (no reference counterpart) that gave
 * up waiting for a shared-memory row copy, since the count was last reset, on
 * the current device; every wait in that kernel is bounded, so a copy that
 * never lands ends the launch with this count raised instead of hanging it.
 * `reset` non-zero clears the count. Synchronous; returns 0xFFFFFFFF if the
 * count cannot be read. */
unsigned int lbm_stage_timeouts(int reset);

/* FP32/FP64 populations (`precision`) -> shifted 16-bit form, any lattice
 * (fluid or scalar; scalars shift by w_i * rho0 with rho0 a reference
 * concentration). */
int lbm_encode_shifted_async(int lattice, int format, int precision, const void* populations,
    void* shifted, size_t x_extent, size_t y_extent, size_t z_extent, float rho0, void* stream);

/* Shifted 16-bit form -> FP32/FP64 populations. */
int lbm_decode_shifted_async(int lattice, int format, int precision, const void* shifted,
    void* populations, size_t x_extent, size_t y_extent, size_t z_extent, float rho0,
    void* stream);

/* ---------------------------------------------------------------------------
 * Discrete reverse-mode adjoint (no reference counterpart). Objective:
 * J = sum_x 0.5 rho |u|^2 of the state after `steps` collide-stream steps
 * (BGK or TRT; MRT on D2Q9 / D3Q19) started from f^0 = f_eq(rho0, u0). The gradient driver runs
 * the forward pass storing a checkpoint every `checkpoint_interval` steps,
 * then for each segment, last first, recomputes the segment's states from
 * its checkpoint and runs the adjoint steps back through it. Outputs (device):
 * objective_and_dtau[0] = J, [1] = dJ/dtau (FP64, deterministic), and
 * grad_u0 = dJ/du0 [D, Z, Y, X] in the population precision. The workspace
 * (checkpoints, one segment, two adjoint fields, FP64 slots) is caller-owned
 * device memory of lbm_ke_gradient_workspace_bytes bytes; rho0, u0 and
 * grad_u0 must not overlap it. Cost: about 2 forward runs + 1 adjoint run.
 * ------------------------------------------------------------------------- */
size_t lbm_ke_gradient_workspace_bytes(int lattice, int precision, size_t x_extent,
    size_t y_extent, size_t z_extent, int steps, int checkpoint_interval);

int lbm_ke_gradient_async(int lattice, int precision, int collision, const void* rho0,
    const void* u0, size_t x_extent, size_t y_extent, size_t z_extent, double tau, int steps,
    int checkpoint_interval, void* workspace, size_t workspace_bytes, double* objective_and_dtau,
    void* grad_u0, void* stream);

/* One adjoint step: lambda = J_step(f^n)^T lambda_next, where f^n is the state
 * the forward step started from (pull formulation; the adjoint scatters). If
 * dtau_slots is non-null, each block adds lambda_next . dC/dtau over its cells
 * to its own FP64 slot (lbm_stats_partials_bytes / 5 slots). */
int lbm_adjoint_step_async(int lattice, int precision, int collision, const void* populations,
    const void* lambda_next, void* lambda, size_t x_extent, size_t y_extent, size_t z_extent,
    double tau, double* dtau_slots, void* stream);

/* Reactive-mixing gradients (no reference counterpart): the checkpointed
 * discrete adjoint of the coupled step of lbm_fluid_reaction_ab_async (fluid
 * BGK or TRT, or MRT on D2Q9 / D3Q19, then the A + B -> C reaction step of launch_reaction_AB_gpu on
 * the post-step fluid, src/simulate_reaction.cpp:518-543). Initial state:
 * f^0 = f_eq(rho0, u0), A^0 = g_eq(a0, u0), B^0 = g_eq(b0, u0) (fields [Z,Y,X],
 * u0 [D,Z,Y,X], population precision). Objective of the state after `steps`:
 *   LBM_OBJECTIVE_MEAN_PRODUCT  <C> = <a0> - <C_A>   (mean product formed)
 *   LBM_OBJECTIVE_SEGREGATION   I_s = cov(C_A, C_B) / (<C_A> <C_B>), as
 *                               compute_reactive_stats (lattice_io.hpp:318-337)
 * result (device, 4 doubles): J, dJ/dk, dJ/dtau, dJ/dtau_c (omega = 1/tau,
 * omega_c = 1/tau_c rounded to the population precision, as the launchers
 * take them); grad_a0 = dJ/da0 and, if non-null, grad_b0 = dJ/db0 ([Z,Y,X]) and
 * grad_u0 = dJ/du0 ([D,Z,Y,X]: through f^0, A^0 and B^0).
 * Workspace of lbm_reactive_gradient_workspace_bytes bytes, not overlapping
 * the inputs or outputs. Cost: about 2 forward runs + 1 adjoint run. */
#define LBM_OBJECTIVE_MEAN_PRODUCT 0
#define LBM_OBJECTIVE_SEGREGATION 1
/* storage: LBM_NATIVE keeps the forward states in `precision`; a 16-bit format
 * (LBM_F16S, ..., precision LBM_FLOAT) runs the forward and its recomputation
 * with lbm_fluid_reaction_ab_shifted_async (fluid shifted by 1, scalars by c0)
 * and stores the states in 16 bits; the adjoint then runs in FP32 about the
 * decoded states (the rounding is not differentiated: the encoding counts as
 * the identity). */
size_t lbm_reactive_gradient_workspace_bytes(int fluid_lattice, int precision, int storage,
    size_t x_extent, size_t y_extent, size_t z_extent, int steps, int checkpoint_interval);
int lbm_reactive_gradient_async(int fluid_lattice, int precision, int storage, float c0,
    int collision, int objective, const void* rho0, const void* u0, const void* a0,
    const void* b0, size_t x_extent, size_t y_extent, size_t z_extent, double tau, double tau_c,
    double k_react, int steps, int checkpoint_interval, void* workspace, size_t workspace_bytes,
    double* result, void* grad_a0, void* grad_b0, void* grad_u0, void* stream);

/* The same second pass writing into row *row_counter of a device table of
 * table_rows x 8 doubles (rows at or past table_rows are not written), then
 * advancing *row_counter (device). No reference counterpart: the destination
 * row is read on the device, so a sequence of steps with this call at its end
 * can be captured once in a CUDA graph and replayed to fill successive rows
 * (the reference driver logs a row every output_frequency steps,
 * simulate_reaction.cpp:557-580). */
int lbm_reactive_stats_append_async(int fluid_lattice, int precision, size_t x_extent,
    size_t y_extent, size_t z_extent, double k_react, const double* partials,
    size_t partials_bytes, double* table, size_t table_rows, unsigned long long* row_counter,
    void* stream);

/* Statistics of a domain split across ranks (no reference counterpart): each
 * rank reduces its partials (from a statistics launch over its cells) to the
 * five FP64 sums of C_A, C_B, C_A^2, C_B^2, C_A C_B (device, 5 doubles); the
 * ranks add their sums (an all-reduce of five doubles); then
 * lbm_reactive_stats_from_sums_async forms the 8 diagnostics of the totals
 * over `cells` cells (k_react in `precision`, as compute_reactive_stats takes
 * it). On one rank the two calls give the bits of
 * lbm_reactive_stats_finalize_async. */
int lbm_reactive_stats_sums_async(int fluid_lattice, size_t x_extent, size_t y_extent,
    size_t z_extent, const double* partials, size_t partials_bytes, double* sums, void* stream);
int lbm_reactive_stats_from_sums_async(int precision, const double* sums, double cells,
    double k_react, double* diagnostics, void* stream);

/* Allocation-free form of lbm_reactive_stats_async. No counterpart in the
 * reference. For callers that cannot allocate device memory, e.g. a plugin or
 * FFI binding inside an application that owns every device allocation and
 * passes this library only the two scalar fields: the FP64 partial sums go to
 * a fixed array inside the library (5 MiB, reserved on every GPU that loads
 * the library until the process exits) instead of caller scratch. Limit:
 * ceil(x_extent / 128) * y_extent * z_extent <= LBM_STATS_NOALLOC_MAX_BLOCKS
 * (e.g. 256^3 or 1024^2); larger domains return cudaErrorInvalidValue. Each
 * call looks up the array's address in the calling thread's current CUDA
 * context (host-side; the address belongs to the context, so contexts the host
 * creates or switches itself, and device resets, are handled). The first call
 * in a context may load the library's device code into it: make it before any
 * stream capture. All calls in a context share the array: calls that overlap
 * on the GPU (other streams, other threads) race, so serialise them. */
#define LBM_STATS_NOALLOC_MAX_BLOCKS 131072
int lbm_reactive_stats_noalloc_async(int scalar_lattice, int precision, const void* current_a,
    const void* current_b, size_t x_extent, size_t y_extent, size_t z_extent, double k_react,
    double* diagnostics, void* stream);

/* Second pass of the statistics over partials written by a fused launch. */
int lbm_reactive_stats_finalize_async(int fluid_lattice, int precision, size_t x_extent,
    size_t y_extent, size_t z_extent, double k_react, const double* partials,
    size_t partials_bytes, double* diagnostics, void* stream);

/* Equilibrium initialisation from macroscopic fields (device, `precision`):
 * rho[N] (density, or concentration for D2Q5/D3Q7) and u[D*N] component-major.
 * Per cell it evaluates lbm::compute_equilibrium (lattice_physics.hpp:267-290)
 * or lbm::compute_scalar_equilibrium (:643-659), the initialisation every
 * reference driver and test performs on the host. */
int lbm_init_equilibrium_async(int lattice, int precision, const void* rho, const void* u,
    void* populations, size_t x_extent, size_t y_extent, size_t z_extent, void* stream);

/* ---- fluid diagnostics and blow-up guard ---------------------------------
 * Replace the host loops of lbm::log_diagnostics (lattice_io.hpp:182-234) and
 * of compute_max_velocity with its crash test (turbulent_tgv_3d.cpp:150-173,
 * :302-316), which need the whole field on the host (main.cpp:595-606).
 * diagnostics (device, 5 doubles):
 *   [0] total mass           sum of rho          (FP64 sum of Real terms)
 *   [1] total kinetic energy sum of 0.5 rho |u|^2 (FP64 sum of Real terms)
 *   [2] max |u| over the cells whose |u| is not NaN (log_diagnostics' max)
 *   [3] number of cells whose |u| is not finite
 *   [4] 1.0 if [3] > 0 or [2] > speed_limit (the driver's crash test), else 0.0
 * Per-cell rho, |u|^2, 0.5 rho |u|^2 and |u| are computed in the population
 * precision as the reference computes them; the reference's Real accumulators
 * become FP64 ones added in a fixed order (run-to-run identical).
 * partials: device scratch of lbm_diagnostics_partials_bytes() bytes. */
size_t lbm_diagnostics_partials_bytes(int lattice, size_t x_extent, size_t y_extent,
    size_t z_extent);
int lbm_fluid_diagnostics_async(int lattice, int precision, const void* populations,
    size_t x_extent, size_t y_extent, size_t z_extent, double speed_limit, double* partials,
    size_t partials_bytes, double* diagnostics, void* stream);
/* One collide-stream step (as lbm_step_async) that also reduces the
 * diagnostics of the state it writes, at no extra memory traffic: the
 * populations a thread writes in the pull scheme are the next buffer's
 * populations of its own cells. Same five values as lbm_fluid_diagnostics_async
 * on next_populations (the FP64 sums may differ in the last bits: the cells are
 * grouped into other blocks). */
int lbm_step_diagnostics_async(int lattice, int precision, int collision,
    const void* current_populations, void* next_populations, size_t x_extent, size_t y_extent,
    size_t z_extent, double omega, double speed_limit, double* partials, size_t partials_bytes,
    double* diagnostics, void* stream);

/* ---- z-slab decomposition (multi-GPU) ---------------------------------------
 * No reference counterpart. A periodic 3-D box (D3Q19 or D3Q27) cut into
 * z-slabs, one per rank; each slab is a [Q, z_extent, Y, X] field in the
 * reference layout. The populations that cross a slab face travel in face
 * buffers of lbm_slab_face_elems() elements ([k, Y, X], the k populations with
 * c_z = +1 (or -1) in ascending order):
 *   halo_lo  c_z = +1 populations of the lower neighbour's top plane
 *   halo_hi  c_z = -1 populations of the upper neighbour's bottom plane
 *   send_lo  this step's c_z = -1 populations of plane 0 (the lower neighbour's halo_hi)
 *   send_hi  this step's c_z = +1 populations of plane z_extent-1 (the upper one's halo_lo)
 * lbm_step_slab_async steps planes [z_begin, z_end): plane 0 reads halo_lo
 * and writes send_lo, the top plane reads halo_hi and writes send_hi; other
 * planes touch no face buffer (those pointers may be null when the range
 * does not include a face). A box stepped as slabs with the face buffers
 * exchanged between steps is bit-identical to the box stepped whole.
 * Requirements as the vectorised step: x_extent even and buffers aligned to
 * 2 elements for D3Q19 float; D3Q27 double MRT / RLBM are not available.
 * lbm_slab_pack_async fills send_lo / send_hi from a state (before the first
 * exchange). */
size_t lbm_slab_face_elems(int lattice, size_t x_extent, size_t y_extent);
int lbm_step_slab_async(int lattice, int precision, int collision,
    const void* current_populations, void* next_populations, size_t x_extent, size_t y_extent,
    size_t z_extent, double omega, const void* halo_lo, const void* halo_hi, void* send_lo,
    void* send_hi, size_t z_begin, size_t z_end, void* stream);
int lbm_slab_pack_async(int lattice, int precision, const void* populations, size_t x_extent,
    size_t y_extent, size_t z_extent, void* send_lo, void* send_hi, void* stream);
/* The z-slab step on shifted 16-bit storage (lbm_step_shifted_async's formats
 * and operators, D3Q19 or D3Q27): face buffers of lbm_slab_face_elems 16-bit
 * codes, otherwise as lbm_step_slab_async. A box stepped as slabs gives the
 * codes of the box stepped whole. lbm_slab_pack_shifted_async fills the send
 * buffers from a 16-bit state. */
int lbm_step_slab_shifted_async(int lattice, int format, int collision,
    const void* current_populations, void* next_populations, size_t x_extent, size_t y_extent,
    size_t z_extent, float omega, float rho0, const void* halo_lo, const void* halo_hi,
    void* send_lo, void* send_hi, size_t z_begin, size_t z_end, void* stream);
int lbm_slab_pack_shifted_async(int lattice, const void* populations, size_t x_extent,
    size_t y_extent, size_t z_extent, void* send_lo, void* send_hi, void* stream);
/* The face exchange of slabs that share one device (every rank of a box in one
 * process): copies src[i] to dst[i], `bytes` each, for i < count <= 64, in one
 * launch. src and dst are host arrays of device pointers; no destination may
 * overlap a source or another destination. */
int lbm_copy_buffers_async(int count, const void* const* src, void* const* dst, size_t bytes,
    void* stream);

/* The coupled fluid + A + B -> C step of lbm_fluid_reaction_ab_async on a
 * z-slab (D3Q19 or D3Q27 fluid with two D3Q7 species). One face buffer per
 * side of lbm_fluid_reaction_slab_face_elems() elements: the fluid's crossing
 * populations as for lbm_step_slab_async, then species A's and then B's (one
 * [Y, X] plane each: c_z = +1 in send_hi / halo_lo, c_z = -1 in send_lo /
 * halo_hi). All four face buffers are required for every plane range. With
 * stats_partials non-null the launch writes the statistics partials of its
 * planes' new scalar fields at their places in a buffer of
 * lbm_stats_partials_bytes(fluid_lattice, x, y, z_extent) bytes, so a step
 * split into several plane ranges fills it once; lbm_reactive_stats_sums_async
 * then gives the rank's five sums. A box stepped as slabs is bit-identical to
 * the box stepped whole. lbm_fluid_reaction_slab_pack_async fills the send
 * buffers from a state (before the first exchange). */
size_t lbm_fluid_reaction_slab_face_elems(int fluid_lattice, size_t x_extent, size_t y_extent);
int lbm_fluid_reaction_slab_async(int fluid_lattice, int precision, int collision,
    const void* current_fluid, void* next_fluid, const void* current_a, void* next_a,
    const void* current_b, void* next_b, size_t x_extent, size_t y_extent, size_t z_extent,
    double omega, double omega_c, double k_react, const void* halo_lo, const void* halo_hi,
    void* send_lo, void* send_hi, size_t z_begin, size_t z_end, double* stats_partials,
    size_t stats_partials_bytes, void* stream);
int lbm_fluid_reaction_slab_pack_async(int fluid_lattice, int precision, const void* fluid,
    const void* a, const void* b, size_t x_extent, size_t y_extent, size_t z_extent,
    void* send_lo, void* send_hi, void* stream);

/* The gradient of lbm_reactive_gradient_async on a z-slab (no reference
 * counterpart): D3Q19 (BGK, TRT, MRT) or D3Q27 (BGK, TRT) fluid with two D3Q7
 * species, states stored as lbm_reactive_gradient_async stores them (storage
 * LBM_NATIVE: in the precision; a 16-bit format: codes, scalars shifted by c0,
 * precision LBM_FLOAT). Every rank runs the whole-box sequence on its slab
 * (z_extent = its own planes, total_cells = cells of the whole box); the face
 * buffers have the layout above with elements of the stored states (state
 * faces: forward steps and packs) or of the precision (the adjoint's scatter
 * sends), and each exchange moves send_hi(r) into halo_lo(r + 1) and send_lo(r)
 * into halo_hi(r - 1):
 *   initial state  lbm_init_equilibrium_async (16-bit: in FP32, then
 *                 lbm_encode_shifted_async, fluid shifted by 1, scalars by c0);
 *   forward step  lbm_reactive_slab_forward_async (velocity, [3, Z, Y, X] in the
 *                 precision, may be null for states the backward sweep
 *                 recomputes), then an exchange;
 *   adjoint step  n (state n and u^{n+1} stored): state n's halos (those the
 *                 exchange after the step that produced it delivered, kept with
 *                 the state; or lbm_reactive_slab_pack_async of state n and an
 *                 exchange), then
 *                 lbm_reactive_slab_adjoint_step_async (lambda^{n+1} ->
 *                 lambda^n; velocity_adjoint is [3, Z, Y, X] scratch; adds to
 *                 the per-warp slots of lbm_reactive_slab_slots_bytes, zeroed
 *                 by the caller before the first step), an exchange of the
 *                 scatter sends it wrote, and
 *                 lbm_reactive_slab_adjoint_unpack_async(halo_lo, halo_hi) into
 *                 lambda^n;
 *   seed          lbm_reactive_slab_seed_async of the final state (segregation:
 *                 the whole box's eight diagnostics, e.g. from
 *                 lbm_reactive_stats_sums_async over ranks and
 *                 lbm_reactive_stats_from_sums_async); objective partials of
 *                 lbm_reactive_slab_objective_bytes;
 *   end           lbm_reactive_slab_init_gradients_async (grad_b0, grad_u0
 *                 may be null), lbm_reactive_slab_sums_async (the rank's four
 *                 FP64 sums), an all-reduce (sum) of those four doubles, and
 *                 lbm_reactive_slab_result_async -> result[4] = J, dJ/dk,
 *                 dJ/dtau, dJ/dtau_c.
 * A slab's adjoint fields and initial-state gradients are bit-identical to the
 * whole box's given the same seed; the four scalars differ from the whole
 * box's only in the order of the FP64 sums. */
size_t lbm_reactive_slab_slots_bytes(int fluid_lattice, size_t x_extent, size_t y_extent,
    size_t z_extent);
size_t lbm_reactive_slab_objective_bytes(int fluid_lattice, size_t x_extent, size_t y_extent,
    size_t z_extent);
int lbm_reactive_slab_pack_async(int fluid_lattice, int precision, int storage,
    const void* fluid, const void* a, const void* b, size_t x_extent, size_t y_extent,
    size_t z_extent, void* send_lo, void* send_hi, void* stream);
int lbm_reactive_slab_forward_async(int fluid_lattice, int precision, int storage, float c0,
    int collision, const void* current_fluid, void* next_fluid, const void* current_a,
    void* next_a, const void* current_b, void* next_b, void* velocity, size_t x_extent,
    size_t y_extent, size_t z_extent, double tau, double tau_c, double k_react,
    const void* halo_lo, const void* halo_hi, void* send_lo, void* send_hi, void* stream);
int lbm_reactive_slab_adjoint_step_async(int fluid_lattice, int precision, int storage,
    float c0, int collision, const void* fluid_n, const void* a_n, const void* b_n,
    const void* halo_lo,
    const void* halo_hi, const void* velocity_next, const void* lambda_fluid_next,
    const void* lambda_a_next, const void* lambda_b_next, void* lambda_fluid, void* lambda_a,
    void* lambda_b, void* velocity_adjoint, void* send_lo, void* send_hi, size_t x_extent,
    size_t y_extent, size_t z_extent, double tau, double tau_c, double k_react, double* slots,
    size_t slots_bytes, void* stream);
int lbm_reactive_slab_adjoint_unpack_async(int fluid_lattice, int precision,
    const void* recv_lo, const void* recv_hi, void* lambda_fluid, void* lambda_a,
    void* lambda_b, size_t x_extent, size_t y_extent, size_t z_extent, void* stream);
int lbm_reactive_slab_seed_async(int fluid_lattice, int precision, int storage, float c0,
    int objective, const void* a_final, const void* b_final, const void* a0, const double* diagnostics,
    void* lambda_fluid, void* lambda_a, void* lambda_b, size_t x_extent, size_t y_extent,
    size_t z_extent, double total_cells, double* objective_partials, size_t partials_bytes,
    void* stream);
int lbm_reactive_slab_init_gradients_async(int fluid_lattice, int precision, int objective,
    const void* rho0, const void* u0, const void* a0, const void* b0, const void* lambda_fluid,
    const void* lambda_a, const void* lambda_b, size_t x_extent, size_t y_extent,
    size_t z_extent, double total_cells, void* grad_a0, void* grad_b0, void* grad_u0,
    void* stream);
int lbm_reactive_slab_sums_async(int fluid_lattice, size_t x_extent, size_t y_extent,
    size_t z_extent, const double* slots, size_t slots_bytes, const double* objective_partials,
    size_t partials_bytes, double* sums, void* stream);
int lbm_reactive_slab_result_async(int precision, int objective, const double* sums,
    const double* diagnostics, double total_cells, double tau_c, double* result, void* stream);

/* ---- output ----------------------------------------------------------------
 * Macroscopic fields for output, computed on the device from the populations
 * as the reference's VTK writer computes them on the host (write_vtk,
 * lattice_io.hpp:386-451; compute_macro_state): density[N], velocity[D*N]
 * (component-major) and speed[N] = |u|, in the population precision. Any of
 * the three may be null (not all). For D2Q5 / D3Q7 `density` receives the
 * concentration and velocity / speed must be null. */
int lbm_macro_fields_async(int lattice, int precision, const void* populations,
    size_t x_extent, size_t y_extent, size_t z_extent, void* density, void* velocity,
    void* speed, void* stream);

/* Host functions (plain host pointers; no GPU work). Return 0 or one of: */
#define LBM_IO_BAD_ARGUMENT 1
#define LBM_IO_OPEN_FAILED 2
#define LBM_IO_WRITE_FAILED 3
#define LBM_IO_BAD_FILE 4
#define LBM_IO_MISMATCH 5
/* The legacy ASCII VTK file of lbm::write_vtk (lattice_io.hpp:386-451), byte
 * for byte, from host copies of lbm_macro_fields_async's three outputs
 * (dims 2 or 3; the reference names it lbm_<step, 6 digits>.vtk). */
int lbm_write_vtk_legacy(const char* path, int dims, size_t x_extent, size_t y_extent,
    size_t z_extent, size_t time_step, int precision, const void* density,
    const void* velocity, const void* speed);
/* Restart files (no reference counterpart): a 64-byte header (magic
 * "LBCUBEP1", lattice, precision, extents, time step) and the raw [Q,Z,Y,X]
 * populations. lbm_read_populations checks the header against the arguments
 * (LBM_IO_MISMATCH) and returns the stored time step. */
int lbm_write_populations(const char* path, int lattice, int precision, size_t x_extent,
    size_t y_extent, size_t z_extent, size_t time_step, const void* populations);
int lbm_read_populations(const char* path, int lattice, int precision, size_t x_extent,
    size_t y_extent, size_t z_extent, size_t* time_step, void* populations);

#ifdef __cplusplus
}  /* extern "C" */
#endif
#endif /* LBCUBE_B200_H */
