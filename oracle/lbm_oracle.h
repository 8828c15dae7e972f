/*
 * Test infrastructure: the CPU oracle for the B200 lattice Boltzmann engine.
 *
 * A plain-C restatement of LB-Cube's serial CPU path (include/lattice_core.hpp,
 * include/lattice_physics.hpp, include/lattice_mrt.hpp, include/lattice_io.hpp).
 * Only the tests, the smoke check and the benchmark's CPU-baseline leg use it:
 * it is the checker, never part of the engine. Every expression keeps the
 * reference's evaluation order, so with floating-point contraction disabled
 * (oracle/Makefile) it reproduces the reference's results bit for bit; the
 * tests pin that against the reference itself (oracle/_ref) and against the
 * reference tests' golden vectors.
 *
 * Populations are flat [Q, Z, Y, X] arrays, X fastest (lattice_memory.hpp:55-102).
 * Enum codes:
 *   lattice   0 D2Q9, 1 D3Q19, 2 D3Q27, 3 D2Q5, 4 D3Q7
 *   precision 0 float, 1 double
 *   collision 0 BGK, 1 TRT, 2 MRT, 3 RLBM
 * Every function returns 0 on success and -1 on an unsupported combination.
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* `steps` fused pull collide-stream steps (step_cpu, lattice_core.hpp:146-216). */
int oracle_step(int lattice, int precision, int collision, const void* in, void* out,
                size_t nx, size_t ny, size_t nz, double omega, int steps);

/* Passive scalar with a uniform source, fluid frozen (step_scalar_cpu, :238-337).
 * `fluid_lattice` selects the pair D2Q9/D2Q5, D3Q19/D3Q7 or D3Q27/D3Q7. */
int oracle_scalar_step(int fluid_lattice, int precision, const void* s_in, void* s_out,
                       const void* fluid, size_t nx, size_t ny, size_t nz, double omega_c,
                       double source, int steps);

/* Fused A+B->C step, fluid frozen (step_reaction_AB, :357-474). */
int oracle_reaction_ab(int fluid_lattice, int precision, const void* a_in, void* a_out,
                       const void* b_in, void* b_out, const void* fluid, size_t nx,
                       size_t ny, size_t nz, double omega_c, double k_react, int steps);

/* The reference driver's coupled loop (src/simulate_reaction.cpp:548-554): one
 * fluid step, then one reaction step that reads the post-step fluid. In place. */
int oracle_coupled_reaction(int fluid_lattice, int precision, int collision, void* fluid,
                            void* a, void* b, size_t nx, size_t ny, size_t nz, double omega,
                            double omega_c, double k_react, int steps);

/* compute_reactive_stats (lattice_io.hpp:256-338). out[8] = mean_A, mean_B,
 * var_A, var_B, covariance, segregation_intensity, true_rate, mixed_rate.
 * accumulate_f64 = 0 keeps the reference's Real accumulators; 1 sums in double. */
int oracle_reactive_stats(int scalar_lattice, int precision, const void* a, const void* b,
                          size_t nx, size_t ny, size_t nz, double k_react,
                          int accumulate_f64, double* out);

/* log_diagnostics sums (lattice_io.hpp:182-234): out[3] = total mass, total
 * kinetic energy 0.5*rho*|u|^2, max |u|, accumulated in Real. */
int oracle_fluid_diagnostics(int lattice, int precision, const void* f, size_t nx, size_t ny,
                             size_t nz, double* out);

/* The engine's device diagnostics restated: log_diagnostics' per-cell terms in
 * the population precision, summed in double; out[5] = total mass, total
 * kinetic energy, max |u| (NaN speeds skipped, as std::max skips them),
 * number of non-finite |u|, crash flag (non-finite |u| or max |u| >
 * speed_limit, turbulent_tgv_3d.cpp:302-316). */
int oracle_fluid_diagnostics64(int lattice, int precision, const void* f, size_t nx, size_t ny,
                               size_t nz, double speed_limit, double* out);

/* Per-cell density and velocity (compute_macro_state, lattice_physics.hpp:227-249)
 * widened to double: rho[N], u[D*N] (component-major). */
int oracle_macro_fields(int lattice, int precision, const void* f, size_t nx, size_t ny,
                        size_t nz, double* rho, double* u);

/* Equilibrium populations of one cell (compute_equilibrium, :267-290, or
 * compute_scalar_equilibrium, :643-659, for lattices 3 and 4 where `rho` is
 * the concentration). u has D entries. */
int oracle_equilibrium(int lattice, int precision, double rho, const double* u, void* out);

/* Equilibrium field from per-cell rho[N] and u[D*N] (component-major), the
 * initialisation every reference driver and test uses. */
int oracle_init_equilibrium(int lattice, int precision, const double* rho, const double* u,
                            void* out, size_t nx, size_t ny, size_t nz);

/* MRT moment transforms in double (lattice_mrt.hpp:439-534, :617-892, :1023-1225). */
int oracle_mrt_moments(int lattice, const double* f, double* m);
int oracle_mrt_populations(int lattice, const double* m, double* f);

/* Exact one-step A+B->C source (compute_reaction_ab_source, :712-743). */
double oracle_reaction_source_f64(double a, double b, double k_react);
float oracle_reaction_source_f32(float a, float b, float k_react);

#ifdef __cplusplus
}
#endif
#endif /* LBM_ORACLE_H */
