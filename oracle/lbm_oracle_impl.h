/*
 * Test infrastructure: precision-generic body of the CPU oracle, included by
 * lbm_oracle.c with REAL = float and REAL = double. Each function restates one
 * reference function and keeps its evaluation order (the comment gives the
 * reference file:line); C's left-to-right grouping of + - * matches C++'s.
 */
#define OR_CAT2(a, b) a##_##b
#define OR_CAT(a, b) OR_CAT2(a, b)
#define F(name) OR_CAT(name, SFX)
#define R(x) ((REAL)(x))
#define KQ(a, b) ((REAL)(a) / (REAL)(b))

/* Shim-Eigen dot product: ascending, starting from the first product
 * (oracle/shim/Eigen/Dense). */
static REAL F(dot)(const REAL* a, const REAL* b, int D) {
  REAL s = a[0] * b[0];
  for (int d = 1; d < D; ++d) s += a[d] * b[d];
  return s;
}

/* compute_macro_state, lattice_physics.hpp:227-249 */
static void F(macro)(const lattice_t* L, const REAL* f, REAL* rho, REAL* u) {
  REAL density = R(0);
  REAL mom[3] = {R(0), R(0), R(0)};
  for (int i = 0; i < L->Q; ++i) {
    const REAL p = f[i];
    density += p;
    for (int d = 0; d < L->D; ++d) mom[d] += p * (REAL)L->c[i * L->D + d];
  }
  *rho = density;
  for (int d = 0; d < L->D; ++d) u[d] = mom[d] / density;
}

/* compute_equilibrium, lattice_physics.hpp:267-290 */
static REAL F(feq)(const lattice_t* L, int i, REAL rho, const REAL* u) {
  REAL dir[3] = {R(0), R(0), R(0)};
  for (int d = 0; d < L->D; ++d) dir[d] = (REAL)L->c[i * L->D + d];
  const REAL weight = (REAL)L->w[i];
  const REAL cs2 = (REAL)L->cs2;
  const REAL inv_cs2 = R(1.0) / cs2;
  const REAL c_dot_u = F(dot)(dir, u, L->D);
  const REAL u_dot_u = F(dot)(u, u, L->D);
  return weight * rho *
         (R(1.0) + inv_cs2 * c_dot_u + R(0.5) * inv_cs2 * inv_cs2 * c_dot_u * c_dot_u -
          R(0.5) * inv_cs2 * u_dot_u);
}

/* compute_scalar_equilibrium, lattice_physics.hpp:643-659 */
static REAL F(geq)(const lattice_t* S, int i, REAL conc, const REAL* u) {
  REAL c_dot_u = R(0);
  for (int d = 0; d < S->D; ++d) c_dot_u += (REAL)S->c[i * S->D + d] * u[d];
  const REAL weight = (REAL)S->w[i];
  const REAL cs2 = (REAL)S->cs2;
  return weight * conc * (R(1.0) + c_dot_u / cs2);
}

static void F(cell_equilibrium)(const lattice_t* L, int scalar, REAL rho, const REAL* u,
                                REAL* out) {
  for (int i = 0; i < L->Q; ++i) out[i] = scalar ? F(geq)(L, i, rho, u) : F(feq)(L, i, rho, u);
}

/* collide_bgk, lattice_physics.hpp:307-318 */
static void F(collide_bgk)(const lattice_t* L, REAL* f, REAL omega) {
  REAL rho, u[3];
  F(macro)(L, f, &rho, u);
  for (int i = 0; i < L->Q; ++i) {
    const REAL eq = F(feq)(L, i, rho, u);
    f[i] += omega * (eq - f[i]);
  }
}

/* compute_omega_minus, lattice_physics.hpp:336-344, magic parameter 1/4 */
static REAL F(omega_minus)(REAL omega_plus) {
  const REAL magic = R(1) / R(4);
  const REAL tau_plus = R(1) / omega_plus;
  const REAL tau_minus = magic / (tau_plus - R(1) / R(2)) + R(1) / R(2);
  return R(1) / tau_minus;
}

/* collide_cell TRT branch (lattice_core.hpp:96-100) + collide_trt (physics:366-398) */
static void F(collide_trt)(const lattice_t* L, REAL* f, REAL omega_plus) {
  REAL rho, u[3], eq[27], post[27];
  F(macro)(L, f, &rho, u);
  const REAL omega_m = F(omega_minus)(omega_plus);
  for (int i = 0; i < L->Q; ++i) eq[i] = F(feq)(L, i, rho, u);
  for (int i = 0; i < L->Q; ++i) {
    const int inv = L->opp[i];
    const REAL even = R(0.5) * (f[i] + f[inv]);
    const REAL eq_even = R(0.5) * (eq[i] + eq[inv]);
    const REAL odd = R(0.5) * (f[i] - f[inv]);
    const REAL eq_odd = R(0.5) * (eq[i] - eq[inv]);
    post[i] = f[i] - omega_plus * (even - eq_even) - omega_m * (odd - eq_odd);
  }
  for (int i = 0; i < L->Q; ++i) f[i] = post[i];
}

/* ---------------------------- MRT D2Q9 --------------------------------- */
/* compute_moments_d2q9, lattice_mrt.hpp:439-455 */
static void F(moments_d2q9)(const REAL* f, REAL* m) {
  m[0] = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
  m[1] = -R(4) * f[0] - f[1] - f[2] - f[3] - f[4] + R(2) * (f[5] + f[6] + f[7] + f[8]);
  m[2] = R(4) * f[0] - R(2) * (f[1] + f[2] + f[3] + f[4]) + f[5] + f[6] + f[7] + f[8];
  m[3] = f[1] - f[3] + f[5] - f[6] - f[7] + f[8];
  m[4] = -R(2) * f[1] + R(2) * f[3] + f[5] - f[6] - f[7] + f[8];
  m[5] = f[2] - f[4] + f[5] + f[6] - f[7] - f[8];
  m[6] = -R(2) * f[2] + R(2) * f[4] + f[5] + f[6] - f[7] - f[8];
  m[7] = f[1] - f[2] + f[3] - f[4];
  m[8] = f[5] - f[6] + f[7] - f[8];
}

/* Generic M^T D^-1 inverse (see lbm_oracle.c); restates compute_populations_d2q9
 * (lattice_mrt.hpp:470-534) and compute_populations_d3q19 (:674-892). */
static void F(inverse_orth)(int Q, const int* order, const int* Mflat, const int* N,
                            const REAL* m, REAL* f) {
  for (int i = 0; i < Q; ++i) {
    int first = 1;
    REAL acc = R(0);
    for (int k = 0; k < Q; ++k) {
      const int r = order[k];
      const int coef = Mflat[r * Q + i];
      if (coef == 0) continue;
      const REAL term = KQ(coef, N[r]) * m[r];
      if (first) {
        acc = term;
        first = 0;
      } else {
        acc = acc + term;
      }
    }
    f[i] = acc;
  }
}

static void F(populations_d2q9)(const REAL* m, REAL* f) {
  F(inverse_orth)(9, ORDER9, &g_M9[0][0], g_N9, m, f);
}

/* collide_mrt_d2q9 (lattice_mrt.hpp:586-603) with the rates of
 * MrtRelaxationRates_D2Q9 (:38-65) and s_nu = omega (lattice_core.hpp:104-107) */
static void F(collide_mrt_d2q9)(REAL* f, REAL omega) {
  REAL rho, u[3], m[9];
  F(macro)(&LATTICES[0], f, &rho, u);
  F(moments_d2q9)(f, m);
  const REAL ux = u[0], uy = u[1];
  const REAL jx = rho * ux, jy = rho * uy;
  const REAL usq = ux * ux + uy * uy;
  const REAL eq1 = -R(2) * rho + R(3) * rho * usq;
  const REAL eq2 = rho - R(3) * rho * usq;
  const REAL eq4 = -jx;
  const REAL eq6 = -jy;
  const REAL eq7 = rho * (ux * ux - uy * uy);
  const REAL eq8 = rho * ux * uy;
  (void)jx;
  (void)jy;
  const REAL s_e = R(1.63), s_eps = R(1.14), s_q = R(1.92), s_nu = omega;
  m[1] -= s_e * (m[1] - eq1);
  m[2] -= s_eps * (m[2] - eq2);
  m[4] -= s_q * (m[4] - eq4);
  m[6] -= s_q * (m[6] - eq6);
  m[7] -= s_nu * (m[7] - eq7);
  m[8] -= s_nu * (m[8] - eq8);
  F(populations_d2q9)(m, f);
}

/* ---------------------------- MRT D3Q19 -------------------------------- */
/* compute_moments_d3q19, lattice_mrt.hpp:617-661 */
static void F(moments_d3q19)(const REAL* f, REAL* m) {
  m[0] = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8] + f[9] + f[10] + f[11] +
         f[12] + f[13] + f[14] + f[15] + f[16] + f[17] + f[18];
  m[1] = -R(30) * f[0] - R(11) * (f[1] + f[2] + f[3] + f[4] + f[5] + f[6]) +
         R(8) * (f[7] + f[8] + f[9] + f[10] + f[11] + f[12] + f[13] + f[14] + f[15] + f[16] +
                 f[17] + f[18]);
  m[2] = R(12) * f[0] - R(4) * (f[1] + f[2] + f[3] + f[4] + f[5] + f[6]) + f[7] + f[8] + f[9] +
         f[10] + f[11] + f[12] + f[13] + f[14] + f[15] + f[16] + f[17] + f[18];
  m[3] = f[1] - f[2] + f[7] - f[8] + f[9] - f[10] + f[11] - f[12] + f[13] - f[14];
  m[4] = -R(4) * f[1] + R(4) * f[2] + f[7] - f[8] + f[9] - f[10] + f[11] - f[12] + f[13] - f[14];
  m[5] = f[3] - f[4] + f[7] + f[8] - f[9] - f[10] + f[15] - f[16] + f[17] - f[18];
  m[6] = -R(4) * f[3] + R(4) * f[4] + f[7] + f[8] - f[9] - f[10] + f[15] - f[16] + f[17] - f[18];
  m[7] = f[5] - f[6] + f[11] + f[12] - f[13] - f[14] + f[15] + f[16] - f[17] - f[18];
  m[8] = -R(4) * f[5] + R(4) * f[6] + f[11] + f[12] - f[13] - f[14] + f[15] + f[16] - f[17] -
         f[18];
  m[9] = R(2) * (f[1] + f[2]) - f[3] - f[4] - f[5] - f[6] + f[7] + f[8] + f[9] + f[10] + f[11] +
         f[12] + f[13] + f[14] - R(2) * (f[15] + f[16] + f[17] + f[18]);
  m[10] = f[3] + f[4] - f[5] - f[6] + f[7] + f[8] + f[9] + f[10] - f[11] - f[12] - f[13] - f[14];
  m[11] = f[7] - f[8] - f[9] + f[10];
  m[12] = f[15] - f[16] - f[17] + f[18];
  m[13] = f[11] - f[12] - f[13] + f[14];
  m[14] = -R(4) * (f[1] + f[2]) + R(2) * (f[3] + f[4] + f[5] + f[6]) + f[7] + f[8] + f[9] +
          f[10] + f[11] + f[12] + f[13] + f[14] - R(2) * (f[15] + f[16] + f[17] + f[18]);
  m[15] = -R(2) * (f[3] + f[4]) + R(2) * (f[5] + f[6]) + f[7] + f[8] + f[9] + f[10] - f[11] -
          f[12] - f[13] - f[14];
  m[16] = f[7] - f[8] + f[9] - f[10] - f[11] + f[12] - f[13] + f[14];
  m[17] = -f[7] - f[8] + f[9] + f[10] + f[15] - f[16] + f[17] - f[18];
  m[18] = f[11] + f[12] - f[13] - f[14] - f[15] - f[16] + f[17] + f[18];
}

static void F(populations_d3q19)(const REAL* m, REAL* f) {
  F(inverse_orth)(19, ORDER19, &g_M19[0][0], g_N19, m, f);
}

/* compute_equilibrium_moments_d3q19 (lattice_mrt.hpp:908-947) and
 * collide_mrt_d3q19 (:971-1009): shear modes 9-13 relax with omega, every
 * other non-conserved mode with the hard-wired rate 1. */
static void F(collide_mrt_d3q19)(REAL* f, REAL omega) {
  REAL rho, u[3], m[19], eq[19];
  F(macro)(&LATTICES[1], f, &rho, u);
  F(moments_d3q19)(f, m);
  const REAL ux = u[0], uy = u[1], uz = u[2];
  const REAL jx = rho * ux, jy = rho * uy, jz = rho * uz;
  const REAL ux2 = ux * ux, uy2 = uy * uy, uz2 = uz * uz;
  const REAL usq = ux2 + uy2 + uz2;
  eq[0] = rho;
  eq[1] = -R(11) * rho + R(19) * rho * usq;
  eq[2] = R(3) * rho - (R(11) / R(2)) * rho * usq;
  eq[3] = jx;
  eq[4] = -(R(2) / R(3)) * jx;
  eq[5] = jy;
  eq[6] = -(R(2) / R(3)) * jy;
  eq[7] = jz;
  eq[8] = -(R(2) / R(3)) * jz;
  eq[9] = R(3) * rho * (R(2) * ux2 - uy2 - uz2);
  eq[10] = rho * (uy2 - uz2);
  eq[11] = rho * ux * uy;
  eq[12] = rho * uy * uz;
  eq[13] = rho * ux * uz;
  eq[14] = R(0);
  eq[15] = R(0);
  eq[16] = R(0);
  eq[17] = R(0);
  eq[18] = R(0);
  const REAL s[19] = {R(0), R(1), R(1), R(0), R(1), R(0), R(1), R(0), R(1), omega,
                      omega, omega, omega, omega, R(1), R(1), R(1), R(1), R(1)};
  for (int i = 0; i < 19; ++i) m[i] -= s[i] * (m[i] - eq[i]);
  F(populations_d3q19)(m, f);
}

/* ---------------------------- MRT D3Q27 -------------------------------- */
/* d3q27_axis_basis (lattice_mrt.hpp:218-230): P0 = 1, P1 = c, P2 = 3c^2 - 2 */
static REAL F(axis_basis)(int order, int c) {
  const REAL v = (REAL)c;
  if (order == 0) return R(1);
  if (order == 1) return v;
  return R(3) * v * v - R(2);
}
/* d3q27_axis_norm (lattice_mrt.hpp:410-426) */
static REAL F(axis_norm)(int order) { return order == 0 ? R(3) : (order == 1 ? R(2) : R(6)); }
#define T3(a, b, c) (((a) * 3 + (b)) * 3 + (c))

/* transform_to_moments_d3q27, lattice_mrt.hpp:1023-1117 */
static void F(moments_d3q27)(const REAL* f, REAL* m) {
  const lattice_t* L = &LATTICES[2];
  REAL p[27], xt[27], xyt[27], raw[27];
  for (int i = 0; i < 27; ++i)
    p[T3(L->c[3 * i] + 1, L->c[3 * i + 1] + 1, L->c[3 * i + 2] + 1)] = f[i];
  for (int ax = 0; ax < 3; ++ax)
    for (int iy = 0; iy < 3; ++iy)
      for (int iz = 0; iz < 3; ++iz) {
        REAL v = R(0);
        for (int ix = 0; ix < 3; ++ix) v += F(axis_basis)(ax, ix - 1) * p[T3(ix, iy, iz)];
        xt[T3(ax, iy, iz)] = v;
      }
  for (int ax = 0; ax < 3; ++ax)
    for (int ay = 0; ay < 3; ++ay)
      for (int iz = 0; iz < 3; ++iz) {
        REAL v = R(0);
        for (int iy = 0; iy < 3; ++iy) v += F(axis_basis)(ay, iy - 1) * xt[T3(ax, iy, iz)];
        xyt[T3(ax, ay, iz)] = v;
      }
  for (int ax = 0; ax < 3; ++ax)
    for (int ay = 0; ay < 3; ++ay)
      for (int az = 0; az < 3; ++az) {
        REAL v = R(0);
        for (int iz = 0; iz < 3; ++iz) v += F(axis_basis)(az, iz - 1) * xyt[T3(ax, ay, iz)];
        raw[T3(ax, ay, az)] = v;
      }
  const REAL r200 = raw[T3(2, 0, 0)], r020 = raw[T3(0, 2, 0)], r002 = raw[T3(0, 0, 2)];
  m[0] = raw[T3(0, 0, 0)];
  m[1] = raw[T3(1, 0, 0)];
  m[2] = raw[T3(0, 1, 0)];
  m[3] = raw[T3(0, 0, 1)];
  m[4] = r200 + r020 + r002;
  m[5] = R(2) * r200 - r020 - r002;
  m[6] = r020 - r002;
  m[7] = raw[T3(1, 1, 0)];
  m[8] = raw[T3(0, 1, 1)];
  m[9] = raw[T3(1, 0, 1)];
  m[10] = raw[T3(2, 1, 0)];
  m[11] = raw[T3(2, 0, 1)];
  m[12] = raw[T3(1, 2, 0)];
  m[13] = raw[T3(0, 2, 1)];
  m[14] = raw[T3(1, 0, 2)];
  m[15] = raw[T3(0, 1, 2)];
  m[16] = raw[T3(1, 1, 1)];
  m[17] = raw[T3(2, 2, 0)];
  m[18] = raw[T3(2, 0, 2)];
  m[19] = raw[T3(0, 2, 2)];
  m[20] = raw[T3(2, 1, 1)];
  m[21] = raw[T3(1, 2, 1)];
  m[22] = raw[T3(1, 1, 2)];
  m[23] = raw[T3(2, 2, 1)];
  m[24] = raw[T3(2, 1, 2)];
  m[25] = raw[T3(1, 2, 2)];
  m[26] = raw[T3(2, 2, 2)];
}

/* transform_to_populations_d3q27, lattice_mrt.hpp:1130-1225 */
static void F(populations_d3q27)(const REAL* m, REAL* f) {
  const lattice_t* L = &LATTICES[2];
  REAL raw[27], zi[27], yzi[27], p[27];
  raw[T3(0, 0, 0)] = m[0];
  raw[T3(1, 0, 0)] = m[1];
  raw[T3(0, 1, 0)] = m[2];
  raw[T3(0, 0, 1)] = m[3];
  raw[T3(2, 0, 0)] = (m[4] + m[5]) / R(3);
  raw[T3(0, 2, 0)] = (R(2) * m[4] - m[5] + R(3) * m[6]) / R(6);
  raw[T3(0, 0, 2)] = (R(2) * m[4] - m[5] - R(3) * m[6]) / R(6);
  raw[T3(1, 1, 0)] = m[7];
  raw[T3(0, 1, 1)] = m[8];
  raw[T3(1, 0, 1)] = m[9];
  raw[T3(2, 1, 0)] = m[10];
  raw[T3(2, 0, 1)] = m[11];
  raw[T3(1, 2, 0)] = m[12];
  raw[T3(0, 2, 1)] = m[13];
  raw[T3(1, 0, 2)] = m[14];
  raw[T3(0, 1, 2)] = m[15];
  raw[T3(1, 1, 1)] = m[16];
  raw[T3(2, 2, 0)] = m[17];
  raw[T3(2, 0, 2)] = m[18];
  raw[T3(0, 2, 2)] = m[19];
  raw[T3(2, 1, 1)] = m[20];
  raw[T3(1, 2, 1)] = m[21];
  raw[T3(1, 1, 2)] = m[22];
  raw[T3(2, 2, 1)] = m[23];
  raw[T3(2, 1, 2)] = m[24];
  raw[T3(1, 2, 2)] = m[25];
  raw[T3(2, 2, 2)] = m[26];
  for (int ax = 0; ax < 3; ++ax)
    for (int ay = 0; ay < 3; ++ay)
      for (int iz = 0; iz < 3; ++iz) {
        REAL v = R(0);
        for (int az = 0; az < 3; ++az)
          v += raw[T3(ax, ay, az)] * F(axis_basis)(az, iz - 1) / F(axis_norm)(az);
        zi[T3(ax, ay, iz)] = v;
      }
  for (int ax = 0; ax < 3; ++ax)
    for (int iy = 0; iy < 3; ++iy)
      for (int iz = 0; iz < 3; ++iz) {
        REAL v = R(0);
        for (int ay = 0; ay < 3; ++ay)
          v += zi[T3(ax, ay, iz)] * F(axis_basis)(ay, iy - 1) / F(axis_norm)(ay);
        yzi[T3(ax, iy, iz)] = v;
      }
  for (int ix = 0; ix < 3; ++ix)
    for (int iy = 0; iy < 3; ++iy)
      for (int iz = 0; iz < 3; ++iz) {
        REAL v = R(0);
        for (int ax = 0; ax < 3; ++ax)
          v += yzi[T3(ax, iy, iz)] * F(axis_basis)(ax, ix - 1) / F(axis_norm)(ax);
        p[T3(ix, iy, iz)] = v;
      }
  for (int i = 0; i < 27; ++i)
    f[i] = p[T3(L->c[3 * i] + 1, L->c[3 * i + 1] + 1, L->c[3 * i + 2] + 1)];
}

/* compute_equilibrium_moments_d3q27 (lattice_mrt.hpp:1242-1268) and
 * collide_mrt_d3q27 (:1284-1305) with MrtRelaxationRates_D3Q27 (:161-204). */
static void F(collide_mrt_d3q27)(REAL* f, REAL omega) {
  const lattice_t* L = &LATTICES[2];
  REAL rho, u[3], m[27], feqp[27], eq[27];
  F(macro)(L, f, &rho, u);
  F(moments_d3q27)(f, m);
  const REAL ux = u[0], uy = u[1], uz = u[2];
  const REAL usq = ux * ux + uy * uy + uz * uz;
  for (int i = 0; i < 27; ++i) {
    const REAL cx = (REAL)L->c[3 * i], cy = (REAL)L->c[3 * i + 1], cz = (REAL)L->c[3 * i + 2];
    const REAL cu = cx * ux + cy * uy + cz * uz;
    feqp[i] = (REAL)L->w[i] * rho * (R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * usq);
  }
  F(moments_d3q27)(feqp, eq);
  const REAL s_b = R(1.19), s_e = R(1.1), s_eps = R(1.2), s_q = R(1.2), s_nu = omega;
  const REAL s[27] = {R(0), R(0), R(0), R(0), s_b,  s_nu, s_nu, s_nu, s_nu,
                      s_nu, s_e,  s_e,  s_e,  s_e,  s_e,  s_e,  s_eps, s_q,
                      s_q,  s_q,  s_q,  s_q,  s_q,  s_q,  s_q,  s_q,  s_q};
  for (int i = 0; i < 27; ++i) m[i] -= s[i] * (m[i] - eq[i]);
  F(populations_d3q27)(m, f);
}

/* ---------------------------- RLBM -------------------------------------- */
/* collide_regularized, lattice_physics.hpp:422-605, with compute_pi_neq_*
 * (:116-211) inlined. */
static void F(collide_rlbm)(int lattice, REAL* f, REAL omega) {
  const lattice_t* L = &LATTICES[lattice];
  REAL rho, u[3], feq[27];
  F(macro)(L, f, &rho, u);
  for (int i = 0; i < L->Q; ++i) feq[i] = F(feq)(L, i, rho, u);
  const REAL hp = R(9) / R(2);
  const REAL cs2 = (REAL)L->cs2;
  if (lattice == 0) {
    REAL pxx = R(0), pyy = R(0), pxy = R(0);
    for (int i = 0; i < 9; ++i) {
      const REAL fn = f[i] - feq[i];
      const REAL cx = (REAL)L->c[2 * i], cy = (REAL)L->c[2 * i + 1];
      pxx += fn * cx * cx;
      pyy += fn * cy * cy;
      pxy += fn * cx * cy;
    }
    const REAL ux = u[0], uy = u[1];
    const REAL a_xxx = R(3) * ux * pxx;
    const REAL a_yyy = R(3) * uy * pyy;
    const REAL a_xxy = R(2) * ux * pxy + uy * pxx;
    const REAL a_xyy = R(2) * uy * pxy + ux * pyy;
    for (int i = 0; i < 9; ++i) {
      const REAL cx = (REAL)L->c[2 * i], cy = (REAL)L->c[2 * i + 1];
      const REAL q_xx = cx * cx - cs2, q_yy = cy * cy - cs2, q_xy = cx * cy;
      const REAL second = q_xx * pxx + q_yy * pyy + R(2) * q_xy * pxy;
      const REAL h_xxx = cx * cx * cx - R(3) * cs2 * cx;
      const REAL h_yyy = cy * cy * cy - R(3) * cs2 * cy;
      const REAL h_xxy = cx * cx * cy - cs2 * cy;
      const REAL h_xyy = cx * cy * cy - cs2 * cx;
      const REAL third = a_xxx * h_xxx + a_yyy * h_yyy + R(3) * (a_xxy * h_xxy + a_xyy * h_xyy);
      const REAL rec = (REAL)L->w[i] * hp * (second + third);
      f[i] = feq[i] + (R(1) - omega) * rec;
    }
    return;
  }
  REAL pxx = R(0), pyy = R(0), pzz = R(0), pxy = R(0), pxz = R(0), pyz = R(0);
  for (int i = 0; i < L->Q; ++i) {
    const REAL fn = f[i] - feq[i];
    const REAL cx = (REAL)L->c[3 * i], cy = (REAL)L->c[3 * i + 1], cz = (REAL)L->c[3 * i + 2];
    pxx += fn * cx * cx;
    pyy += fn * cy * cy;
    pzz += fn * cz * cz;
    pxy += fn * cx * cy;
    pxz += fn * cx * cz;
    pyz += fn * cy * cz;
  }
  const REAL ux = u[0], uy = u[1], uz = u[2];
  const REAL a_xxx = R(3) * ux * pxx;
  const REAL a_yyy = R(3) * uy * pyy;
  const REAL a_zzz = R(3) * uz * pzz;
  const REAL a_xxy = R(2) * ux * pxy + uy * pxx;
  const REAL a_xxz = R(2) * ux * pxz + uz * pxx;
  REAL a_xyy, a_yyz, a_xzz, a_yzz, a_xyz;
  a_yyz = R(2) * uy * pyz + uz * pyy;
  if (lattice == 1) {
    a_xyy = R(2) * uy * pxy + ux * pyy;
    a_xzz = R(2) * uz * pxz + ux * pzz;
    a_yzz = R(2) * uz * pyz + uy * pzz;
    a_xyz = R(0);
  } else {
    a_xyy = ux * pyy + R(2) * uy * pxy;
    a_xzz = ux * pzz + R(2) * uz * pxz;
    a_yzz = uy * pzz + R(2) * uz * pyz;
    a_xyz = ux * pyz + uy * pxz + uz * pxy;
  }
  for (int i = 0; i < L->Q; ++i) {
    const REAL cx = (REAL)L->c[3 * i], cy = (REAL)L->c[3 * i + 1], cz = (REAL)L->c[3 * i + 2];
    const REAL q_xx = cx * cx - cs2, q_yy = cy * cy - cs2, q_zz = cz * cz - cs2;
    const REAL q_xy = cx * cy, q_xz = cx * cz, q_yz = cy * cz;
    const REAL second =
        q_xx * pxx + q_yy * pyy + q_zz * pzz + R(2) * (q_xy * pxy + q_xz * pxz + q_yz * pyz);
    const REAL h_xxx = cx * cx * cx - R(3) * cs2 * cx;
    const REAL h_yyy = cy * cy * cy - R(3) * cs2 * cy;
    const REAL h_zzz = cz * cz * cz - R(3) * cs2 * cz;
    const REAL h_xxy = cx * cx * cy - cs2 * cy;
    const REAL h_xxz = cx * cx * cz - cs2 * cz;
    const REAL h_xyy = cx * cy * cy - cs2 * cx;
    const REAL h_yyz = cy * cy * cz - cs2 * cz;
    const REAL h_xzz = cx * cz * cz - cs2 * cx;
    const REAL h_yzz = cy * cz * cz - cs2 * cy;
    const REAL h_xyz = cx * cy * cz;
    REAL third;
    if (lattice == 1) {
      third = R(3) * (h_xxy + h_yzz) * (a_xxy + a_yzz) + (h_xxy - h_yzz) * (a_xxy - a_yzz) +
              R(3) * (h_xzz + h_xyy) * (a_xzz + a_xyy) + (h_xzz - h_xyy) * (a_xzz - a_xyy) +
              R(3) * (h_yyz + h_xxz) * (a_yyz + a_xxz) + (h_yyz - h_xxz) * (a_yyz - a_xxz);
    } else {
      third = a_xxx * h_xxx + a_yyy * h_yyy + a_zzz * h_zzz +
              R(3) * (a_xxy * h_xxy + a_xxz * h_xxz + a_xyy * h_xyy + a_yyz * h_yyz +
                      a_xzz * h_xzz + a_yzz * h_yzz) +
              R(6) * a_xyz * h_xyz;
    }
    const REAL rec = (REAL)L->w[i] * hp * (second + third);
    f[i] = feq[i] + (R(1) - omega) * rec;
  }
}

/* collide_cell dispatch, lattice_core.hpp:90-126 */
static void F(collide)(const lattice_t* L, int lattice, int collision, REAL* f, REAL omega) {
  switch (collision) {
    case 0: F(collide_bgk)(L, f, omega); break;
    case 1: F(collide_trt)(L, f, omega); break;
    case 2:
      if (lattice == 0) F(collide_mrt_d2q9)(f, omega);
      else if (lattice == 1) F(collide_mrt_d3q19)(f, omega);
      else F(collide_mrt_d3q27)(f, omega);
      break;
    default: F(collide_rlbm)(lattice, f, omega); break;
  }
}

/* step_cpu, lattice_core.hpp:146-216 (one step, cur -> next) */
static void F(step_once)(const lattice_t* L, int lattice, int collision, const REAL* cur,
                         REAL* next, size_t nx, size_t ny, size_t nz, REAL omega) {
  REAL f[27];
  for (size_t z = 0; z < nz; ++z)
    for (size_t y = 0; y < ny; ++y)
      for (size_t x = 0; x < nx; ++x) {
        for (int i = 0; i < L->Q; ++i) {
          const int cx = L->c[i * L->D], cy = L->c[i * L->D + 1];
          const int cz = L->D == 3 ? L->c[i * L->D + 2] : 0;
          const size_t sx = pull(x, cx, nx), sy = pull(y, cy, ny), sz = pull(z, cz, nz);
          f[i] = cur[pidx(i, sx, sy, sz, nx, ny, nz)];
        }
        F(collide)(L, lattice, collision, f, omega);
        for (int i = 0; i < L->Q; ++i) next[pidx(i, x, y, z, nx, ny, nz)] = f[i];
      }
}

static int F(run_steps)(const lattice_t* L, int lattice, int collision, const void* in, void* out,
                        size_t nx, size_t ny, size_t nz, REAL omega, int steps) {
  const size_t count = (size_t)L->Q * nx * ny * nz;
  REAL* a = (REAL*)malloc(count * sizeof(REAL));
  REAL* b = (REAL*)malloc(count * sizeof(REAL));
  if (!a || !b) {
    free(a);
    free(b);
    return -1;
  }
  memcpy(a, in, count * sizeof(REAL));
  for (int s = 0; s < steps; ++s) {
    F(step_once)(L, lattice, collision, a, b, nx, ny, nz, omega);
    REAL* t = a;
    a = b;
    b = t;
  }
  memcpy(out, a, count * sizeof(REAL));
  free(a);
  free(b);
  return 0;
}

/* compute_concentration, lattice_physics.hpp:618-627 */
static REAL F(concentration)(const lattice_t* S, const REAL* g) {
  REAL c = R(0);
  for (int i = 0; i < S->Q; ++i) c += g[i];
  return c;
}

/* collide_scalar_bgk, lattice_physics.hpp:677-694 */
static void F(collide_scalar)(const lattice_t* S, REAL* g, const REAL* u, REAL omega_c,
                              REAL source) {
  const REAL conc = F(concentration)(S, g);
  for (int i = 0; i < S->Q; ++i) {
    const REAL weight = (REAL)S->w[i];
    const REAL eq = F(geq)(S, i, conc, u);
    g[i] += omega_c * (eq - g[i]) + weight * source;
  }
}

/* compute_reaction_ab_source, lattice_physics.hpp:712-743 */
static REAL F(reaction_source)(REAL a, REAL b, REAL k) {
  const REAL abs_a = a < R(0) ? -a : a;
  const REAL abs_b = b < R(0) ? -b : b;
  const REAL diff = b - a;
  const REAL abs_diff = diff < R(0) ? -diff : diff;
  const REAL tol = R(64.0) * REAL_EPS * (R(1.0) + abs_a + abs_b);
  REAL a_after;
  if (abs_diff <= tol) {
    a_after = a / (R(1.0) + k * a);
  } else {
    const REAL att = EXPR(-k * diff);
    a_after = a * diff * att / (b - a * att);
  }
  return a_after - a;
}

/* Fluid velocity at the destination cell, read in place (lattice_core.hpp:259-265). */
static void F(fluid_velocity_at)(const lattice_t* FL, const REAL* fluid, size_t x, size_t y,
                                 size_t z, size_t nx, size_t ny, size_t nz, REAL* u) {
  REAL f[27], rho;
  for (int i = 0; i < FL->Q; ++i) f[i] = fluid[pidx(i, x, y, z, nx, ny, nz)];
  F(macro)(FL, f, &rho, u);
}

static void F(gather_scalar)(const lattice_t* S, const REAL* cur, size_t x, size_t y, size_t z,
                             size_t nx, size_t ny, size_t nz, REAL* g) {
  for (int i = 0; i < S->Q; ++i) {
    const int cx = S->c[i * S->D], cy = S->c[i * S->D + 1];
    const int cz = S->D == 3 ? S->c[i * S->D + 2] : 0;
    g[i] = cur[pidx(i, pull(x, cx, nx), pull(y, cy, ny), pull(z, cz, nz), nx, ny, nz)];
  }
}

/* step_scalar_cpu, lattice_core.hpp:238-337 */
static void F(scalar_once)(const lattice_t* FL, const lattice_t* S, const REAL* cur, REAL* next,
                           const REAL* fluid, size_t nx, size_t ny, size_t nz, REAL omega_c,
                           REAL source) {
  REAL g[27], u[3];
  for (size_t z = 0; z < nz; ++z)
    for (size_t y = 0; y < ny; ++y)
      for (size_t x = 0; x < nx; ++x) {
        F(fluid_velocity_at)(FL, fluid, x, y, z, nx, ny, nz, u);
        F(gather_scalar)(S, cur, x, y, z, nx, ny, nz, g);
        F(collide_scalar)(S, g, u, omega_c, source);
        for (int i = 0; i < S->Q; ++i) next[pidx(i, x, y, z, nx, ny, nz)] = g[i];
      }
}

/* step_reaction_AB, lattice_core.hpp:357-474 */
static void F(reaction_once)(const lattice_t* FL, const lattice_t* S, const REAL* a_cur,
                             REAL* a_next, const REAL* b_cur, REAL* b_next, const REAL* fluid,
                             size_t nx, size_t ny, size_t nz, REAL omega_c, REAL k) {
  REAL ga[27], gb[27], u[3];
  for (size_t z = 0; z < nz; ++z)
    for (size_t y = 0; y < ny; ++y)
      for (size_t x = 0; x < nx; ++x) {
        F(fluid_velocity_at)(FL, fluid, x, y, z, nx, ny, nz, u);
        F(gather_scalar)(S, a_cur, x, y, z, nx, ny, nz, ga);
        F(gather_scalar)(S, b_cur, x, y, z, nx, ny, nz, gb);
        const REAL ca = F(concentration)(S, ga);
        const REAL cb = F(concentration)(S, gb);
        const REAL src = F(reaction_source)(ca, cb, k);
        F(collide_scalar)(S, ga, u, omega_c, src);
        F(collide_scalar)(S, gb, u, omega_c, src);
        for (int i = 0; i < S->Q; ++i) {
          a_next[pidx(i, x, y, z, nx, ny, nz)] = ga[i];
          b_next[pidx(i, x, y, z, nx, ny, nz)] = gb[i];
        }
      }
}

static int F(scalar_steps)(const lattice_t* FL, const lattice_t* S, const void* s_in,
                           void* s_out, const void* fluid, size_t nx, size_t ny, size_t nz,
                           REAL omega_c, REAL source, int steps) {
  const size_t count = (size_t)S->Q * nx * ny * nz;
  REAL* a = (REAL*)malloc(count * sizeof(REAL));
  REAL* b = (REAL*)malloc(count * sizeof(REAL));
  if (!a || !b) {
    free(a);
    free(b);
    return -1;
  }
  memcpy(a, s_in, count * sizeof(REAL));
  for (int s = 0; s < steps; ++s) {
    F(scalar_once)(FL, S, a, b, (const REAL*)fluid, nx, ny, nz, omega_c, source);
    REAL* t = a;
    a = b;
    b = t;
  }
  memcpy(s_out, a, count * sizeof(REAL));
  free(a);
  free(b);
  return 0;
}

static int F(reaction_steps)(const lattice_t* FL, const lattice_t* S, const void* a_in,
                             void* a_out, const void* b_in, void* b_out, const void* fluid,
                             size_t nx, size_t ny, size_t nz, REAL omega_c, REAL k, int steps) {
  const size_t count = (size_t)S->Q * nx * ny * nz;
  REAL* a0 = (REAL*)malloc(count * sizeof(REAL));
  REAL* a1 = (REAL*)malloc(count * sizeof(REAL));
  REAL* b0 = (REAL*)malloc(count * sizeof(REAL));
  REAL* b1 = (REAL*)malloc(count * sizeof(REAL));
  if (!a0 || !a1 || !b0 || !b1) {
    free(a0);
    free(a1);
    free(b0);
    free(b1);
    return -1;
  }
  memcpy(a0, a_in, count * sizeof(REAL));
  memcpy(b0, b_in, count * sizeof(REAL));
  for (int s = 0; s < steps; ++s) {
    F(reaction_once)(FL, S, a0, a1, b0, b1, (const REAL*)fluid, nx, ny, nz, omega_c, k);
    REAL* t = a0;
    a0 = a1;
    a1 = t;
    t = b0;
    b0 = b1;
    b1 = t;
  }
  memcpy(a_out, a0, count * sizeof(REAL));
  memcpy(b_out, b0, count * sizeof(REAL));
  free(a0);
  free(a1);
  free(b0);
  free(b1);
  return 0;
}

static int F(coupled_steps)(const lattice_t* FL, const lattice_t* S, int lattice, int collision,
                            void* fluid, void* a, void* b, size_t nx, size_t ny, size_t nz,
                            REAL omega, REAL omega_c, REAL k, int steps) {
  const size_t nf = (size_t)FL->Q * nx * ny * nz, ns = (size_t)S->Q * nx * ny * nz;
  REAL* f1 = (REAL*)malloc(nf * sizeof(REAL));
  REAL* a1 = (REAL*)malloc(ns * sizeof(REAL));
  REAL* b1 = (REAL*)malloc(ns * sizeof(REAL));
  REAL* f0 = (REAL*)fluid;
  REAL* a0 = (REAL*)a;
  REAL* b0 = (REAL*)b;
  if (!f1 || !a1 || !b1) {
    free(f1);
    free(a1);
    free(b1);
    return -1;
  }
  for (int s = 0; s < steps; ++s) {
    F(step_once)(FL, lattice, collision, f0, f1, nx, ny, nz, omega);
    memcpy(f0, f1, nf * sizeof(REAL));
    F(reaction_once)(FL, S, a0, a1, b0, b1, f0, nx, ny, nz, omega_c, k);
    memcpy(a0, a1, ns * sizeof(REAL));
    memcpy(b0, b1, ns * sizeof(REAL));
  }
  free(f1);
  free(a1);
  free(b1);
  return 0;
}

/* compute_reactive_stats, lattice_io.hpp:256-338. `acc64` selects double
 * accumulators (the engine's choice) instead of the reference's Real ones. */
static int F(reactive_stats)(const lattice_t* S, const void* va, const void* vb, size_t nx,
                             size_t ny, size_t nz, REAL k, int acc64, double* out) {
  const REAL* A = (const REAL*)va;
  const REAL* B = (const REAL*)vb;
  REAL g[27];
  const size_t cells = nx * ny * nz;
  if (acc64) {
    double sa = 0, sb = 0, sa2 = 0, sb2 = 0, sab = 0;
    for (size_t z = 0; z < nz; ++z)
      for (size_t y = 0; y < ny; ++y)
        for (size_t x = 0; x < nx; ++x) {
          for (int i = 0; i < S->Q; ++i) g[i] = A[pidx(i, x, y, z, nx, ny, nz)];
          const double ca = (double)F(concentration)(S, g);
          for (int i = 0; i < S->Q; ++i) g[i] = B[pidx(i, x, y, z, nx, ny, nz)];
          const double cb = (double)F(concentration)(S, g);
          sa += ca;
          sb += cb;
          sa2 += ca * ca;
          sb2 += cb * cb;
          sab += ca * cb;
        }
    const double inv = 1.0 / (double)cells;
    const double ma = sa * inv, mb = sb * inv, ma2 = sa2 * inv, mb2 = sb2 * inv, mab = sab * inv;
    const double kk = (double)k;
    const double mixed = kk * ma * mb;
    const double cov = mab - ma * mb;
    const double mp = ma * mb;
    const double seg = fabs(mp) > 2.220446049250313080847e-16 ? cov / mp : 0.0;
    out[0] = ma;
    out[1] = mb;
    out[2] = ma2 - ma * ma;
    out[3] = mb2 - mb * mb;
    out[4] = cov;
    out[5] = seg;
    out[6] = kk * mab;
    out[7] = mixed;
    return 0;
  }
  REAL sa = R(0), sb = R(0), sa2 = R(0), sb2 = R(0), sab = R(0);
  for (size_t z = 0; z < nz; ++z)
    for (size_t y = 0; y < ny; ++y)
      for (size_t x = 0; x < nx; ++x) {
        for (int i = 0; i < S->Q; ++i) g[i] = A[pidx(i, x, y, z, nx, ny, nz)];
        const REAL ca = F(concentration)(S, g);
        for (int i = 0; i < S->Q; ++i) g[i] = B[pidx(i, x, y, z, nx, ny, nz)];
        const REAL cb = F(concentration)(S, g);
        sa += ca;
        sb += cb;
        sa2 += ca * ca;
        sb2 += cb * cb;
        sab += ca * cb;
      }
  const REAL inv = R(1) / (REAL)cells;
  const REAL ma = sa * inv, mb = sb * inv, ma2 = sa2 * inv, mb2 = sb2 * inv, mab = sab * inv;
  const REAL mixed = k * ma * mb;
  const REAL cov = mab - ma * mb;
  const REAL mp = ma * mb;
  const REAL seg = FABSR(mp) > REAL_EPS ? cov / mp : R(0);
  out[0] = ma;
  out[1] = mb;
  out[2] = ma2 - ma * ma;
  out[3] = mb2 - mb * mb;
  out[4] = cov;
  out[5] = seg;
  out[6] = k * mab;
  out[7] = mixed;
  return 0;
}

/* log_diagnostics sums, lattice_io.hpp:182-234 */
static int F(fluid_diagnostics)(const lattice_t* L, const void* vf, size_t nx, size_t ny,
                                size_t nz, double* out) {
  const REAL* fl = (const REAL*)vf;
  REAL f[27], rho, u[3];
  REAL mass = R(0), ke = R(0), umax = R(0);
  for (size_t z = 0; z < nz; ++z)
    for (size_t y = 0; y < ny; ++y)
      for (size_t x = 0; x < nx; ++x) {
        for (int i = 0; i < L->Q; ++i) f[i] = fl[pidx(i, x, y, z, nx, ny, nz)];
        F(macro)(L, f, &rho, u);
        const REAL s2 = F(dot)(u, u, L->D);
        mass += rho;
        ke += R(0.5) * rho * s2;
        const REAL sp = SQRTR(s2);
        umax = umax < sp ? sp : umax;
      }
  out[0] = mass;
  out[1] = ke;
  out[2] = umax;
  return 0;
}

/* The engine's diagnostics: the per-cell terms of log_diagnostics in REAL,
 * accumulated in double, plus the non-finite count and the crash flag of
 * turbulent_tgv_3d.cpp:150-173, :302-316 (compute_max_velocity returns +inf
 * on a non-finite speed; the driver stops on !isfinite(max) || max > limit). */
static int F(fluid_diagnostics64)(const lattice_t* L, const void* vf, size_t nx, size_t ny,
                                  size_t nz, double speed_limit, double* out) {
  const REAL* fl = (const REAL*)vf;
  REAL f[27], rho, u[3];
  double mass = 0.0, ke = 0.0, umax = 0.0, nonfinite = 0.0;
  for (size_t z = 0; z < nz; ++z)
    for (size_t y = 0; y < ny; ++y)
      for (size_t x = 0; x < nx; ++x) {
        for (int i = 0; i < L->Q; ++i) f[i] = fl[pidx(i, x, y, z, nx, ny, nz)];
        F(macro)(L, f, &rho, u);
        const REAL s2 = F(dot)(u, u, L->D);
        const REAL k = R(0.5) * rho * s2;
        const REAL sp = SQRTR(s2);
        mass += (double)rho;
        ke += (double)k;
        if (!isfinite(sp)) nonfinite += 1.0;
        umax = umax < (double)sp ? (double)sp : umax;
      }
  out[0] = mass;
  out[1] = ke;
  out[2] = umax;
  out[3] = nonfinite;
  out[4] = (nonfinite > 0.0 || umax > speed_limit) ? 1.0 : 0.0;
  return 0;
}

static int F(macro_fields)(const lattice_t* L, const void* vf, size_t nx, size_t ny, size_t nz,
                           double* rho_out, double* u_out) {
  const REAL* fl = (const REAL*)vf;
  const size_t cells = nx * ny * nz;
  REAL f[27], rho, u[3];
  for (size_t c = 0; c < cells; ++c) {
    for (int i = 0; i < L->Q; ++i) f[i] = fl[(size_t)i * cells + c];
    if (L->Q <= 7) {
      rho = F(concentration)(L, f);
      rho_out[c] = rho;
      continue;
    }
    F(macro)(L, f, &rho, u);
    rho_out[c] = rho;
    for (int d = 0; d < L->D; ++d) u_out[(size_t)d * cells + c] = u[d];
  }
  return 0;
}

static int F(init_equilibrium)(const lattice_t* L, int scalar, const double* rho,
                               const double* u, void* vout, size_t nx, size_t ny, size_t nz) {
  REAL* out = (REAL*)vout;
  const size_t cells = nx * ny * nz;
  REAL e[27], uu[3];
  for (size_t c = 0; c < cells; ++c) {
    for (int d = 0; d < L->D; ++d) uu[d] = (REAL)u[(size_t)d * cells + c];
    F(cell_equilibrium)(L, scalar, (REAL)rho[c], uu, e);
    for (int i = 0; i < L->Q; ++i) out[(size_t)i * cells + c] = e[i];
  }
  return 0;
}

#undef F
#undef R
#undef KQ
#undef OR_CAT
#undef OR_CAT2
#undef T3
