/*
 * Test infrastructure: CPU oracle (see lbm_oracle.h). This file holds the
 * lattice tables and the precision-independent entry points; the arithmetic
 * lives in lbm_oracle_impl.h, included once for float and once for double.
 *
 * Lattice tables restate include/lattice_traits.hpp:62-305 (velocity order,
 * weights, cs^2, opposite map). They have to be identical to the reference's
 * because the [Q, Z, Y, X] population order is part of the data format.
 */
#include "lbm_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int D, Q;
  double cs2;
  const double* w;
  const int* c; /* [Q * D], component d of velocity i at c[i * D + d] */
  const int* opp;
} lattice_t;

/* D2Q9, lattice_traits.hpp:62-97 */
static const double W_D2Q9[9] = {4.0 / 9.0,  1.0 / 9.0,  1.0 / 9.0,  1.0 / 9.0, 1.0 / 9.0,
                                 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
static const int C_D2Q9[18] = {0, 0, 1, 0, 0, 1, -1, 0, 0, -1, 1, 1, -1, 1, -1, -1, 1, -1};
static const int O_D2Q9[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};

/* D3Q19, lattice_traits.hpp:105-156 */
static const double W_D3Q19[19] = {
    1.0 / 3.0,  1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0,
    1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
    1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
static const int C_D3Q19[57] = {0,  0,  0,  1, 0, 0,  -1, 0,  0,  0,  1,  0,  0, -1, 0,
                                0,  0,  1,  0, 0, -1, 1,  1,  0,  -1, 1,  0,  1, -1, 0,
                                -1, -1, 0,  1, 0, 1,  -1, 0,  1,  1,  0,  -1, -1, 0, -1,
                                0,  1,  1,  0, -1, 1, 0,  1,  -1, 0,  -1, -1};
static const int O_D3Q19[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};

/* D3Q27, lattice_traits.hpp:165-227 */
static const double W_D3Q27[27] = {
    8.0 / 27.0,  2.0 / 27.0,  2.0 / 27.0,  2.0 / 27.0,  2.0 / 27.0,  2.0 / 27.0,  2.0 / 27.0,
    1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,
    1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 216.0, 1.0 / 216.0,
    1.0 / 216.0, 1.0 / 216.0, 1.0 / 216.0, 1.0 / 216.0, 1.0 / 216.0, 1.0 / 216.0};
static const int C_D3Q27[81] = {
    0,  0,  0,  1,  0,  0,  -1, 0,  0,  0, 1,  0,  0,  -1, 0,  0,  0,  1,  0,  0,  -1,
    1,  1,  0,  -1, 1,  0,  1,  -1, 0,  -1, -1, 0,  1,  0,  1,  -1, 0,  1,  1,  0,  -1,
    -1, 0,  -1, 0,  1,  1,  0,  -1, 1,  0,  1,  -1, 0,  -1, -1, 1,  1,  1,  -1, 1,  1,
    1,  -1, 1,  -1, -1, 1,  1,  1,  -1, -1, 1,  -1, 1,  -1, -1, -1, -1, -1};
static const int O_D3Q27[27] = {0,  2,  1,  4,  3,  6,  5,  10, 9,  8,  7,  14, 13, 12,
                                11, 18, 17, 16, 15, 26, 25, 24, 23, 22, 21, 20, 19};

/* D2Q5, lattice_traits.hpp:236-265 */
static const double W_D2Q5[5] = {1.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0};
static const int C_D2Q5[10] = {0, 0, 1, 0, 0, 1, -1, 0, 0, -1};
static const int O_D2Q5[5] = {0, 3, 4, 1, 2};

/* D3Q7, lattice_traits.hpp:273-305 (cs^2 = 1/4) */
static const double W_D3Q7[7] = {1.0 / 4.0, 1.0 / 8.0, 1.0 / 8.0, 1.0 / 8.0,
                                 1.0 / 8.0, 1.0 / 8.0, 1.0 / 8.0};
static const int C_D3Q7[21] = {0, 0, 0, 1, 0, 0, -1, 0, 0, 0, 1, 0, 0, -1, 0, 0, 0, 1, 0, 0, -1};
static const int O_D3Q7[7] = {0, 2, 1, 4, 3, 6, 5};

static const lattice_t LATTICES[5] = {
    {2, 9, 1.0 / 3.0, W_D2Q9, C_D2Q9, O_D2Q9},
    {3, 19, 1.0 / 3.0, W_D3Q19, C_D3Q19, O_D3Q19},
    {3, 27, 1.0 / 3.0, W_D3Q27, C_D3Q27, O_D3Q27},
    {2, 5, 1.0 / 3.0, W_D2Q5, C_D2Q5, O_D2Q5},
    {3, 7, 1.0 / 4.0, W_D3Q7, C_D3Q7, O_D3Q7},
};

/* Scalar lattice paired with each fluid lattice (lattice_cuda.cu:912-1010). */
static int scalar_of(int fluid_lattice) { return fluid_lattice == 0 ? 3 : 4; }

/* Flat [Q, Z, Y, X] offset (lattice_cuda.cu:69-78, lattice_memory.hpp:88-97). */
static size_t pidx(int i, size_t x, size_t y, size_t z, size_t nx, size_t ny, size_t nz) {
  return (((size_t)i * nz + z) * ny + y) * nx + x;
}

/* Periodic upstream coordinate x - c (lattice_core.hpp:70-78). */
static size_t pull(size_t coord, int c, size_t n) {
  const ptrdiff_t s = (ptrdiff_t)coord - (ptrdiff_t)c + (ptrdiff_t)n;
  return (size_t)(s % (ptrdiff_t)n);
}

/* ---- integer MRT matrices, derived once from the forward transforms ---- */
/* The inverse transforms of D2Q9 and D3Q19 are M^T D^-1 (lattice_mrt.hpp:
 * 459-534, :663-892): population i is the sum over moment rows r of
 * (M[r][i] / |M_r|^2) * m[r], taken in the row order the reference writes its
 * terms in (ascending for D2Q9; 0..9,14,10,15,11,12,13,16,17,18 for D3Q19),
 * skipping zero coefficients. M is read off the forward transform applied to
 * unit vectors, which is exact. */
static int g_M9[9][9], g_N9[9];
static int g_M19[19][19], g_N19[19];
static int g_mrt_ready = 0;
static const int ORDER9[9] = {0, 1, 2, 3, 4, 5, 6, 7, 8};
static const int ORDER19[19] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 14, 10, 15, 11, 12, 13, 16, 17, 18};

#define REAL float
#define SFX f32
#define EXPR expf
#define SQRTR sqrtf
#define FABSR fabsf
#define REAL_EPS 1.1920928955078125e-07f
#include "lbm_oracle_impl.h"
#undef REAL
#undef SFX
#undef EXPR
#undef SQRTR
#undef FABSR
#undef REAL_EPS

#define REAL double
#define SFX f64
#define EXPR exp
#define SQRTR sqrt
#define FABSR fabs
#define REAL_EPS 2.220446049250313080847e-16
#include "lbm_oracle_impl.h"
#undef REAL
#undef SFX
#undef EXPR
#undef SQRTR
#undef FABSR
#undef REAL_EPS

static void mrt_init(void) {
  if (g_mrt_ready) return;
  double e[27], m[27];
  for (int j = 0; j < 9; ++j) {
    memset(e, 0, sizeof e);
    e[j] = 1.0;
    moments_d2q9_f64(e, m);
    for (int r = 0; r < 9; ++r) g_M9[r][j] = (int)m[r];
  }
  for (int j = 0; j < 19; ++j) {
    memset(e, 0, sizeof e);
    e[j] = 1.0;
    moments_d3q19_f64(e, m);
    for (int r = 0; r < 19; ++r) g_M19[r][j] = (int)m[r];
  }
  for (int r = 0; r < 9; ++r) {
    g_N9[r] = 0;
    for (int j = 0; j < 9; ++j) g_N9[r] += g_M9[r][j] * g_M9[r][j];
  }
  for (int r = 0; r < 19; ++r) {
    g_N19[r] = 0;
    for (int j = 0; j < 19; ++j) g_N19[r] += g_M19[r][j] * g_M19[r][j];
  }
  g_mrt_ready = 1;
}

static int fluid_ok(int lattice) { return lattice >= 0 && lattice <= 2; }

int oracle_step(int lattice, int precision, int collision, const void* in, void* out,
                size_t nx, size_t ny, size_t nz, double omega, int steps) {
  if (!fluid_ok(lattice) || collision < 0 || collision > 3 || steps < 0) return -1;
  const lattice_t* L = &LATTICES[lattice];
  if (L->D == 2) nz = 1;
  mrt_init();
  if (precision == 0) return run_steps_f32(L, lattice, collision, in, out, nx, ny, nz, (float)omega, steps);
  if (precision == 1) return run_steps_f64(L, lattice, collision, in, out, nx, ny, nz, omega, steps);
  return -1;
}

int oracle_scalar_step(int fluid_lattice, int precision, const void* s_in, void* s_out,
                       const void* fluid, size_t nx, size_t ny, size_t nz, double omega_c,
                       double source, int steps) {
  if (!fluid_ok(fluid_lattice) || steps < 0) return -1;
  const lattice_t* FL = &LATTICES[fluid_lattice];
  const lattice_t* SL = &LATTICES[scalar_of(fluid_lattice)];
  if (FL->D == 2) nz = 1;
  if (precision == 0)
    return scalar_steps_f32(FL, SL, s_in, s_out, fluid, nx, ny, nz, (float)omega_c, (float)source, steps);
  if (precision == 1)
    return scalar_steps_f64(FL, SL, s_in, s_out, fluid, nx, ny, nz, omega_c, source, steps);
  return -1;
}

int oracle_reaction_ab(int fluid_lattice, int precision, const void* a_in, void* a_out,
                       const void* b_in, void* b_out, const void* fluid, size_t nx,
                       size_t ny, size_t nz, double omega_c, double k_react, int steps) {
  if (!fluid_ok(fluid_lattice) || steps < 0) return -1;
  const lattice_t* FL = &LATTICES[fluid_lattice];
  const lattice_t* SL = &LATTICES[scalar_of(fluid_lattice)];
  if (FL->D == 2) nz = 1;
  if (precision == 0)
    return reaction_steps_f32(FL, SL, a_in, a_out, b_in, b_out, fluid, nx, ny, nz,
                              (float)omega_c, (float)k_react, steps);
  if (precision == 1)
    return reaction_steps_f64(FL, SL, a_in, a_out, b_in, b_out, fluid, nx, ny, nz, omega_c,
                              k_react, steps);
  return -1;
}

int oracle_coupled_reaction(int fluid_lattice, int precision, int collision, void* fluid,
                            void* a, void* b, size_t nx, size_t ny, size_t nz, double omega,
                            double omega_c, double k_react, int steps) {
  if (!fluid_ok(fluid_lattice) || collision < 0 || collision > 3 || steps < 0) return -1;
  const lattice_t* FL = &LATTICES[fluid_lattice];
  const lattice_t* SL = &LATTICES[scalar_of(fluid_lattice)];
  if (FL->D == 2) nz = 1;
  mrt_init();
  if (precision == 0)
    return coupled_steps_f32(FL, SL, fluid_lattice, collision, fluid, a, b, nx, ny, nz,
                             (float)omega, (float)omega_c, (float)k_react, steps);
  if (precision == 1)
    return coupled_steps_f64(FL, SL, fluid_lattice, collision, fluid, a, b, nx, ny, nz, omega,
                             omega_c, k_react, steps);
  return -1;
}

int oracle_reactive_stats(int scalar_lattice, int precision, const void* a, const void* b,
                          size_t nx, size_t ny, size_t nz, double k_react,
                          int accumulate_f64, double* out) {
  if (scalar_lattice != 3 && scalar_lattice != 4) return -1;
  const lattice_t* SL = &LATTICES[scalar_lattice];
  if (SL->D == 2) nz = 1;
  if (precision == 0) return reactive_stats_f32(SL, a, b, nx, ny, nz, (float)k_react, accumulate_f64, out);
  if (precision == 1) return reactive_stats_f64(SL, a, b, nx, ny, nz, k_react, accumulate_f64, out);
  return -1;
}

int oracle_fluid_diagnostics(int lattice, int precision, const void* f, size_t nx, size_t ny,
                             size_t nz, double* out) {
  if (!fluid_ok(lattice)) return -1;
  const lattice_t* L = &LATTICES[lattice];
  if (L->D == 2) nz = 1;
  if (precision == 0) return fluid_diagnostics_f32(L, f, nx, ny, nz, out);
  if (precision == 1) return fluid_diagnostics_f64(L, f, nx, ny, nz, out);
  return -1;
}

int oracle_fluid_diagnostics64(int lattice, int precision, const void* f, size_t nx, size_t ny,
                               size_t nz, double speed_limit, double* out) {
  if (!fluid_ok(lattice)) return -1;
  const lattice_t* L = &LATTICES[lattice];
  if (L->D == 2) nz = 1;
  if (precision == 0) return fluid_diagnostics64_f32(L, f, nx, ny, nz, speed_limit, out);
  if (precision == 1) return fluid_diagnostics64_f64(L, f, nx, ny, nz, speed_limit, out);
  return -1;
}

int oracle_macro_fields(int lattice, int precision, const void* f, size_t nx, size_t ny,
                        size_t nz, double* rho, double* u) {
  if (lattice < 0 || lattice > 4) return -1;
  const lattice_t* L = &LATTICES[lattice];
  if (L->D == 2) nz = 1;
  if (precision == 0) return macro_fields_f32(L, f, nx, ny, nz, rho, u);
  if (precision == 1) return macro_fields_f64(L, f, nx, ny, nz, rho, u);
  return -1;
}

int oracle_equilibrium(int lattice, int precision, double rho, const double* u, void* out) {
  if (lattice < 0 || lattice > 4) return -1;
  const lattice_t* L = &LATTICES[lattice];
  if (precision == 0) {
    float uu[3] = {0, 0, 0};
    for (int d = 0; d < L->D; ++d) uu[d] = (float)u[d];
    cell_equilibrium_f32(L, lattice >= 3, (float)rho, uu, (float*)out);
    return 0;
  }
  if (precision == 1) {
    double uu[3] = {0, 0, 0};
    for (int d = 0; d < L->D; ++d) uu[d] = u[d];
    cell_equilibrium_f64(L, lattice >= 3, rho, uu, (double*)out);
    return 0;
  }
  return -1;
}

int oracle_init_equilibrium(int lattice, int precision, const double* rho, const double* u,
                            void* out, size_t nx, size_t ny, size_t nz) {
  if (lattice < 0 || lattice > 4) return -1;
  const lattice_t* L = &LATTICES[lattice];
  if (L->D == 2) nz = 1;
  if (precision == 0) return init_equilibrium_f32(L, lattice >= 3, rho, u, out, nx, ny, nz);
  if (precision == 1) return init_equilibrium_f64(L, lattice >= 3, rho, u, out, nx, ny, nz);
  return -1;
}

int oracle_mrt_moments(int lattice, const double* f, double* m) {
  mrt_init();
  if (lattice == 0) { moments_d2q9_f64(f, m); return 0; }
  if (lattice == 1) { moments_d3q19_f64(f, m); return 0; }
  if (lattice == 2) { moments_d3q27_f64(f, m); return 0; }
  return -1;
}

int oracle_mrt_populations(int lattice, const double* m, double* f) {
  mrt_init();
  if (lattice == 0) { populations_d2q9_f64(m, f); return 0; }
  if (lattice == 1) { populations_d3q19_f64(m, f); return 0; }
  if (lattice == 2) { populations_d3q27_f64(m, f); return 0; }
  return -1;
}

double oracle_reaction_source_f64(double a, double b, double k) { return reaction_source_f64(a, b, k); }
float oracle_reaction_source_f32(float a, float b, float k) { return reaction_source_f32(a, b, k); }
