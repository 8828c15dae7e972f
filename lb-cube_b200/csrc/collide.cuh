// Per-cell collision operators, kept in registers.
//
// Every operator evaluates the same expression tree as LB-Cube's host/device
// physics functions (file:line given per function), so that, compiled without
// FMA contraction (--fmad=false, the engine's build), a step produces the same
// bits as the reference CPU path. Terms whose lattice coefficient is 0 are
// dropped and coefficients of +-1 become additions/subtractions: in IEEE
// arithmetic `x + f*0 == x` and `x + f*(+-1) == x +- f` exactly, so the value
// of every partial sum is unchanged (only the sign of an exact zero can differ).
#pragma once

#include <type_traits>

#include "lattices.cuh"

#define LB_I(I) decltype(I)::value

namespace lbcube {

// exp for the reaction source. The float version is evaluated in double and
// rounded once, which is (almost always) the correctly rounded single-precision
// value that the host libm's expf returns, so the float reaction step tracks
// the CPU path more closely than a single-precision device exp would. The
// argument is -k (B - A): small for any rate that a time step resolves, and
// for |x| < 2^-8 the double value comes from the Taylor polynomial of degree 5
// (Horner, fused multiply-adds): its truncation error x^6 / 720 < 5e-18 is
// below half a unit in the last place of double, so it is as accurate as a
// full double exp for a fraction of the instructions.
template <class Real>
__device__ __forceinline__ Real rexp(Real x);
template <>
__device__ __forceinline__ float rexp<float>(float x) {
  const double d = (double)x;
  if (fabs(d) < 0.00390625) {
    double p = fma(d, 1.0 / 120.0, 1.0 / 24.0);
    p = fma(p, d, 1.0 / 6.0);
    p = fma(p, d, 0.5);
    p = fma(p, d, 1.0);
    return (float)fma(p, d, 1.0);
  }
  return (float)exp(d);
}
template <>
__device__ __forceinline__ double rexp<double>(double x) { return exp(x); }

// Signed sum of velocity components u[d] for the non-zero entries of c_i, in
// ascending d: the value of the dot product c_i . u
// (lattice_physics.hpp:282, :648-652).
template <class L, int i, class Real>
__device__ __forceinline__ Real c_dot(const Real* u) {
  Real s = Real(0);
  bool first = true;
  static_for<L::D>([&](auto D) {
    constexpr int c = L::c[i][LB_I(D)];
    if constexpr (c != 0) {
      const Real t = c > 0 ? u[LB_I(D)] : -u[LB_I(D)];
      s = first ? t : s + t;
      first = false;
    }
  });
  return s;
}

// compute_macro_state (lattice_physics.hpp:227-249): rho = sum f_i in ascending
// i, j_d = sum f_i c_id, u = j / rho.
template <class L, class Real>
__device__ __forceinline__ void macro_state(const Real (&f)[L::Q], Real& rho, Real (&u)[L::D]) {
  Real density = f[0];
  static_for<L::Q - 1>([&](auto I) { density += f[LB_I(I) + 1]; });
  static_for<L::D>([&](auto D) {
    constexpr int d = LB_I(D);
    Real m = Real(0);
    static_for<L::Q>([&](auto I) {
      constexpr int c = L::c[LB_I(I)][d];
      if constexpr (c > 0) m = m + f[LB_I(I)];
      if constexpr (c < 0) m = m - f[LB_I(I)];
    });
    u[d] = m / density;
  });
  // The reference adds f_i * c_id for every i, so a non-finite population
  // makes every velocity component NaN (0 * inf, inf / inf, or a NaN density),
  // while finite populations give exactly the sums above (their zero terms
  // change nothing). Skipping the zero terms loses that, so restore it; a
  // finite density means every population is finite, so the common path only
  // tests the density.
  if (!isfinite(density)) {
    bool bad = false;
    static_for<L::Q>([&](auto I) { bad = bad || !isfinite(f[LB_I(I)]); });
    if (bad) static_for<L::D>([&](auto D) { u[LB_I(D)] = Real(NAN); });
  }
  rho = density;
}

template <class L, class Real>
__device__ __forceinline__ Real u_dot_u(const Real (&u)[L::D]) {
  Real s = u[0] * u[0];
  static_for<L::D - 1>([&](auto D) { s += u[LB_I(D) + 1] * u[LB_I(D) + 1]; });
  return s;
}

// compute_equilibrium (lattice_physics.hpp:267-290):
// w rho (1 + cu/cs2 + cu^2/(2 cs2^2) - u.u/(2 cs2)), grouped as the reference.
template <class L, int i, class Real>
__device__ __forceinline__ Real feq(Real rho, const Real (&u)[L::D], Real usq) {
  constexpr double wd = L::w[i];
  const Real weight = Real(wd);
  const Real inv_cs2 = Real(1.0) / Real(L::cs2);
  const Real cu = c_dot<L, i>(u);
  return weight * rho *
         (Real(1.0) + inv_cs2 * cu + Real(0.5) * inv_cs2 * inv_cs2 * cu * cu -
          Real(0.5) * inv_cs2 * usq);
}

// All Q equilibria of a cell, bit-identical to feq<L, i> for every i but
// computed once per opposite pair: with c_o = -c_i, cu_o = -cu_i exactly, so
// 3 cu_o = -(3 cu_i), 1 + 3 cu_o == 1 - 3 cu_i, and (4.5 cu_o) cu_o ==
// (4.5 cu_i) cu_i, all without rounding differences.
template <class L, class Real>
__device__ __forceinline__ void equilibria(Real rho, const Real (&u)[L::D], Real usq,
                                           Real (&eq)[L::Q]) {
  const Real inv_cs2 = Real(1.0) / Real(L::cs2);
  const Real a = Real(0.5) * inv_cs2 * inv_cs2;  // 4.5, exact
  const Real b = Real(0.5) * inv_cs2;            // 1.5, exact
  const Real tail = b * usq;
  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr int o = L::opp[i];
    constexpr double wd = L::w[i];
    const Real wr = Real(wd) * rho;
    if constexpr (i == o) {
      eq[i] = wr * (Real(1.0) - tail);  // c_i = 0: 1 + 3*0 + (4.5*0)*0 == 1
    } else if constexpr (i < o) {
      const Real cu = c_dot<L, i>(u);
      const Real p = inv_cs2 * cu;
      const Real t2 = a * cu * cu;
      eq[i] = wr * (Real(1.0) + p + t2 - tail);
      eq[o] = wr * (Real(1.0) - p + t2 - tail);
    }
  });
}

// collide_bgk (lattice_physics.hpp:307-318).
template <class L, class Real>
__device__ __forceinline__ void collide_bgk(Real (&f)[L::Q], Real omega) {
  Real rho, u[L::D], eq[L::Q];
  macro_state<L>(f, rho, u);
  const Real usq = u_dot_u<L>(u);
  equilibria<L>(rho, u, usq, eq);
  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    f[i] = f[i] + omega * (eq[i] - f[i]);
  });
}

// compute_omega_minus (lattice_physics.hpp:336-344) with Lambda = 1/4.
template <class Real>
__host__ __device__ inline Real trt_omega_minus(Real omega_plus) {
  const Real magic = Real{1} / Real{4};
  const Real tau_plus = Real{1} / omega_plus;
  const Real tau_minus = magic / (tau_plus - Real{1} / Real{2}) + Real{1} / Real{2};
  return Real{1} / tau_minus;
}

// collide_trt (lattice_physics.hpp:366-398) after compute_macro_state
// (lattice_core.hpp:96-100). omega_minus is precomputed once per launch.
// Evaluated once per opposite pair (i, o): the reference's even parts for i
// and o are the same values, its odd parts exact negatives, so
//   post_i = (f_i - A) - B,  post_o = (f_o - A) + B
// with A = w+ (even - eq_even), B = w- (odd_i - eq_odd_i) reproduces both of
// its results bit for bit. The rest population has odd part +0.
template <class L, class Real>
__device__ __forceinline__ void collide_trt(Real (&f)[L::Q], Real omega_plus, Real omega_minus) {
  Real rho, u[L::D], eq[L::Q];
  macro_state<L>(f, rho, u);
  const Real usq = u_dot_u<L>(u);
  equilibria<L>(rho, u, usq, eq);
  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr int o = L::opp[i];
    if constexpr (i == o) {
      f[i] = f[i] - omega_plus * (f[i] - eq[i]);
    } else if constexpr (i < o) {
      const Real even = Real{0.5} * (f[i] + f[o]);
      const Real eq_even = Real{0.5} * (eq[i] + eq[o]);
      const Real odd = Real{0.5} * (f[i] - f[o]);
      const Real eq_odd = Real{0.5} * (eq[i] - eq[o]);
      const Real A = omega_plus * (even - eq_even);
      const Real B = omega_minus * (odd - eq_odd);
      const Real fi = f[i] - A - B;
      const Real fo = f[o] - A + B;
      f[i] = fi;
      f[o] = fo;
    }
  });
}

// ----------------------------------------------------------------------------
// MRT. The forward transforms are written once, generic in the element type,
// with the reference's grouping; instantiated with int at compile time they
// give the integer moment matrix M whose rows are orthogonal, from which the
// inverse M^T D^-1 is taken (coefficient M[r][i] / |M_r|^2).
// ----------------------------------------------------------------------------

// compute_moments_d2q9 (lattice_mrt.hpp:439-455).
template <class T>
__host__ __device__ constexpr void moments_d2q9(const T* f, T* m) {
  m[0] = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
  m[1] = -T(4) * f[0] - f[1] - f[2] - f[3] - f[4] + T(2) * (f[5] + f[6] + f[7] + f[8]);
  m[2] = T(4) * f[0] - T(2) * (f[1] + f[2] + f[3] + f[4]) + f[5] + f[6] + f[7] + f[8];
  m[3] = f[1] - f[3] + f[5] - f[6] - f[7] + f[8];
  m[4] = -T(2) * f[1] + T(2) * f[3] + f[5] - f[6] - f[7] + f[8];
  m[5] = f[2] - f[4] + f[5] + f[6] - f[7] - f[8];
  m[6] = -T(2) * f[2] + T(2) * f[4] + f[5] + f[6] - f[7] - f[8];
  m[7] = f[1] - f[2] + f[3] - f[4];
  m[8] = f[5] - f[6] + f[7] - f[8];
}

// compute_moments_d3q19 (lattice_mrt.hpp:617-661).
template <class T>
__host__ __device__ constexpr void moments_d3q19(const T* f, T* m) {
  m[0] = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8] + f[9] + f[10] + f[11] +
         f[12] + f[13] + f[14] + f[15] + f[16] + f[17] + f[18];
  m[1] = -T(30) * f[0] - T(11) * (f[1] + f[2] + f[3] + f[4] + f[5] + f[6]) +
         T(8) * (f[7] + f[8] + f[9] + f[10] + f[11] + f[12] + f[13] + f[14] + f[15] + f[16] +
                 f[17] + f[18]);
  m[2] = T(12) * f[0] - T(4) * (f[1] + f[2] + f[3] + f[4] + f[5] + f[6]) + f[7] + f[8] + f[9] +
         f[10] + f[11] + f[12] + f[13] + f[14] + f[15] + f[16] + f[17] + f[18];
  m[3] = f[1] - f[2] + f[7] - f[8] + f[9] - f[10] + f[11] - f[12] + f[13] - f[14];
  m[4] = -T(4) * f[1] + T(4) * f[2] + f[7] - f[8] + f[9] - f[10] + f[11] - f[12] + f[13] - f[14];
  m[5] = f[3] - f[4] + f[7] + f[8] - f[9] - f[10] + f[15] - f[16] + f[17] - f[18];
  m[6] = -T(4) * f[3] + T(4) * f[4] + f[7] + f[8] - f[9] - f[10] + f[15] - f[16] + f[17] - f[18];
  m[7] = f[5] - f[6] + f[11] + f[12] - f[13] - f[14] + f[15] + f[16] - f[17] - f[18];
  m[8] = -T(4) * f[5] + T(4) * f[6] + f[11] + f[12] - f[13] - f[14] + f[15] + f[16] - f[17] -
         f[18];
  m[9] = T(2) * (f[1] + f[2]) - f[3] - f[4] - f[5] - f[6] + f[7] + f[8] + f[9] + f[10] + f[11] +
         f[12] + f[13] + f[14] - T(2) * (f[15] + f[16] + f[17] + f[18]);
  m[10] = f[3] + f[4] - f[5] - f[6] + f[7] + f[8] + f[9] + f[10] - f[11] - f[12] - f[13] - f[14];
  m[11] = f[7] - f[8] - f[9] + f[10];
  m[12] = f[15] - f[16] - f[17] + f[18];
  m[13] = f[11] - f[12] - f[13] + f[14];
  m[14] = -T(4) * (f[1] + f[2]) + T(2) * (f[3] + f[4] + f[5] + f[6]) + f[7] + f[8] + f[9] +
          f[10] + f[11] + f[12] + f[13] + f[14] - T(2) * (f[15] + f[16] + f[17] + f[18]);
  m[15] = -T(2) * (f[3] + f[4]) + T(2) * (f[5] + f[6]) + f[7] + f[8] + f[9] + f[10] - f[11] -
          f[12] - f[13] - f[14];
  m[16] = f[7] - f[8] + f[9] - f[10] - f[11] + f[12] - f[13] + f[14];
  m[17] = -f[7] - f[8] + f[9] + f[10] + f[15] - f[16] + f[17] - f[18];
  m[18] = f[11] + f[12] - f[13] - f[14] - f[15] - f[16] + f[17] + f[18];
}

template <int Q>
struct MomentMatrix {
  int m[Q][Q];
  int norm[Q];
};

template <int Q, class Fwd>
constexpr MomentMatrix<Q> make_moment_matrix(Fwd fwd) {
  MomentMatrix<Q> r{};
  for (int j = 0; j < Q; ++j) {
    int e[Q] = {};
    int col[Q] = {};
    e[j] = 1;
    fwd(e, col);
    for (int i = 0; i < Q; ++i) r.m[i][j] = col[i];
  }
  for (int i = 0; i < Q; ++i) {
    r.norm[i] = 0;
    for (int j = 0; j < Q; ++j) r.norm[i] += r.m[i][j] * r.m[i][j];
  }
  return r;
}

struct Mrt9 {
  static constexpr MomentMatrix<9> M =
      make_moment_matrix<9>([](const int* f, int* m) { moments_d2q9<int>(f, m); });
  // Order in which compute_populations_d2q9 adds the moment terms (lattice_mrt.hpp:470-534).
  static constexpr int order[9] = {0, 1, 2, 3, 4, 5, 6, 7, 8};
};
struct Mrt19 {
  static constexpr MomentMatrix<19> M =
      make_moment_matrix<19>([](const int* f, int* m) { moments_d3q19<int>(f, m); });
  // Order in which compute_populations_d3q19 adds the moment terms (lattice_mrt.hpp:674-892).
  static constexpr int order[19] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 14, 10, 15, 11, 12, 13, 16, 17, 18};
};

// f_i = sum over r (in the reference's order, zero coefficients skipped) of
// (M[r][i] / |M_r|^2) m_r, evaluated left to right from the first term.
template <class Mx, int Q, class Real>
__device__ __forceinline__ void inverse_orthogonal(const Real (&m)[Q], Real (&f)[Q]) {
  static_for<Q>([&](auto I) {
    constexpr int i = LB_I(I);
    Real acc = Real(0);
    bool first = true;
    static_for<Q>([&](auto K) {
      constexpr int r = Mx::order[LB_I(K)];
      constexpr int coef = Mx::M.m[r][i];
      constexpr int nrm = Mx::M.norm[r];
      if constexpr (coef != 0) {
        const Real term = (Real(coef) / Real(nrm)) * m[r];
        acc = first ? term : acc + term;
        first = false;
      }
    });
    f[i] = acc;
  });
}

// collide_mrt_d2q9 (lattice_mrt.hpp:586-603), equilibrium moments (:548-569),
// rates MrtRelaxationRates_D2Q9 (:38-65) with s_nu = omega (lattice_core.hpp:104-107).
template <class Real>
__device__ __forceinline__ void collide_mrt_d2q9(Real (&f)[9], Real omega) {
  Real rho, u[2], m[9];
  macro_state<D2Q9>(f, rho, u);
  moments_d2q9<Real>(f, m);
  const Real ux = u[0], uy = u[1];
  const Real jx = rho * ux, jy = rho * uy;
  const Real usq = ux * ux + uy * uy;
  const Real eq1 = -Real{2} * rho + Real{3} * rho * usq;
  const Real eq2 = rho - Real{3} * rho * usq;
  const Real eq4 = -jx, eq6 = -jy;
  const Real eq7 = rho * (ux * ux - uy * uy);
  const Real eq8 = rho * ux * uy;
  const Real s_e = Real(1.63), s_eps = Real(1.14), s_q = Real(1.92), s_nu = omega;
  m[1] -= s_e * (m[1] - eq1);
  m[2] -= s_eps * (m[2] - eq2);
  m[4] -= s_q * (m[4] - eq4);
  m[6] -= s_q * (m[6] - eq6);
  m[7] -= s_nu * (m[7] - eq7);
  m[8] -= s_nu * (m[8] - eq8);
  inverse_orthogonal<Mrt9>(m, f);
}

// collide_mrt_d3q19 (lattice_mrt.hpp:971-1009) with the equilibrium moments of
// :908-947. Only the shear modes 9-13 use omega; the other non-conserved modes
// relax with the rate 1 the reference hard-wires (:981-1001).
template <class Real>
__device__ __forceinline__ void collide_mrt_d3q19(Real (&f)[19], Real omega) {
  Real rho, u[3], m[19];
  macro_state<D3Q19>(f, rho, u);
  moments_d3q19<Real>(f, m);
  const Real ux = u[0], uy = u[1], uz = u[2];
  const Real jx = rho * ux, jy = rho * uy, jz = rho * uz;
  const Real ux2 = ux * ux, uy2 = uy * uy, uz2 = uz * uz;
  const Real usq = ux2 + uy2 + uz2;
  Real eq[19];
  eq[0] = rho;
  eq[1] = -Real{11} * rho + Real{19} * rho * usq;
  eq[2] = Real{3} * rho - (Real{11} / Real{2}) * rho * usq;
  eq[3] = jx;
  eq[4] = -(Real{2} / Real{3}) * jx;
  eq[5] = jy;
  eq[6] = -(Real{2} / Real{3}) * jy;
  eq[7] = jz;
  eq[8] = -(Real{2} / Real{3}) * jz;
  eq[9] = Real{3} * rho * (Real{2} * ux2 - uy2 - uz2);
  eq[10] = rho * (uy2 - uz2);
  eq[11] = rho * ux * uy;
  eq[12] = rho * uy * uz;
  eq[13] = rho * ux * uz;
  static_for<19>([&](auto I) {
    constexpr int i = LB_I(I);
    if constexpr (i == 0 || i == 3 || i == 5 || i == 7) {
      // conserved: m - 0 * (m - eq) == m
    } else if constexpr (i >= 9 && i <= 13) {
      m[i] -= omega * (m[i] - eq[i]);
    } else if constexpr (i >= 14) {
      m[i] -= Real{1} * (m[i] - Real{0});
    } else {
      m[i] -= Real{1} * (m[i] - eq[i]);
    }
  });
  inverse_orthogonal<Mrt19>(m, f);
}

// D3Q27 orthogonal tensor-product basis (lattice_mrt.hpp:218-426,
// :1023-1305). P0 = 1, P1 = c, P2 = 3c^2 - 2 on c in {-1, 0, 1}, i.e. the
// integer factors below; the separable transforms keep the reference's loop
// order, including the initial `value = 0` of every accumulation.
__host__ __device__ constexpr int p27_basis(int order, int c) {
  return order == 0 ? 1 : (order == 1 ? c : 3 * c * c - 2);
}
__host__ __device__ constexpr int p27_norm(int order) { return order == 0 ? 3 : (order == 1 ? 2 : 6); }
__host__ __device__ constexpr int t27(int a, int b, int c) { return (a * 3 + b) * 3 + c; }

// Position of lattice velocity i in the 3x3x3 tensor layout.
template <int i>
__host__ __device__ constexpr int tensor_slot27() {
  return t27(D3Q27::c[i][0] + 1, D3Q27::c[i][1] + 1, D3Q27::c[i][2] + 1);
}

// transform_to_moments_d3q27 (lattice_mrt.hpp:1023-1117). DROP leaves out the
// terms whose basis factor is 0 (the c = 0 term of each first-order sum): for
// finite populations each is +-0, and adding +-0 to a sum that starts at +0
// changes nothing (a round-to-nearest sum is -0 only when both addends are -0,
// so such a sum is never -0). Callers pass DROP only for finite inputs.
template <class Real, bool DROP = false>
__device__ __forceinline__ void moments_d3q27(const Real (&f)[27], Real (&m)[27]) {
  Real p[27], xt[27], xyt[27], raw[27];
  static_for<27>([&](auto I) { p[tensor_slot27<LB_I(I)>()] = f[LB_I(I)]; });
  static_for<27>([&](auto J) {  // J = (ax, iy, iz)
    constexpr int a = LB_I(J) / 9, b = (LB_I(J) / 3) % 3, c = LB_I(J) % 3;
    Real v = Real(0);
    static_for<3>([&](auto K) {
      constexpr int k = LB_I(K);
      if constexpr (!DROP || p27_basis(a, k - 1) != 0) v += Real(p27_basis(a, k - 1)) * p[t27(k, b, c)];
    });
    xt[t27(a, b, c)] = v;
  });
  static_for<27>([&](auto J) {  // (ax, ay, iz)
    constexpr int a = LB_I(J) / 9, b = (LB_I(J) / 3) % 3, c = LB_I(J) % 3;
    Real v = Real(0);
    static_for<3>([&](auto K) {
      constexpr int k = LB_I(K);
      if constexpr (!DROP || p27_basis(b, k - 1) != 0) v += Real(p27_basis(b, k - 1)) * xt[t27(a, k, c)];
    });
    xyt[t27(a, b, c)] = v;
  });
  static_for<27>([&](auto J) {  // (ax, ay, az)
    constexpr int a = LB_I(J) / 9, b = (LB_I(J) / 3) % 3, c = LB_I(J) % 3;
    Real v = Real(0);
    static_for<3>([&](auto K) {
      constexpr int k = LB_I(K);
      if constexpr (!DROP || p27_basis(c, k - 1) != 0) v += Real(p27_basis(c, k - 1)) * xyt[t27(a, b, k)];
    });
    raw[t27(a, b, c)] = v;
  });
  const Real r200 = raw[t27(2, 0, 0)], r020 = raw[t27(0, 2, 0)], r002 = raw[t27(0, 0, 2)];
  m[0] = raw[t27(0, 0, 0)];
  m[1] = raw[t27(1, 0, 0)];
  m[2] = raw[t27(0, 1, 0)];
  m[3] = raw[t27(0, 0, 1)];
  m[4] = r200 + r020 + r002;
  m[5] = Real{2} * r200 - r020 - r002;
  m[6] = r020 - r002;
  m[7] = raw[t27(1, 1, 0)];
  m[8] = raw[t27(0, 1, 1)];
  m[9] = raw[t27(1, 0, 1)];
  m[10] = raw[t27(2, 1, 0)];
  m[11] = raw[t27(2, 0, 1)];
  m[12] = raw[t27(1, 2, 0)];
  m[13] = raw[t27(0, 2, 1)];
  m[14] = raw[t27(1, 0, 2)];
  m[15] = raw[t27(0, 1, 2)];
  m[16] = raw[t27(1, 1, 1)];
  m[17] = raw[t27(2, 2, 0)];
  m[18] = raw[t27(2, 0, 2)];
  m[19] = raw[t27(0, 2, 2)];
  m[20] = raw[t27(2, 1, 1)];
  m[21] = raw[t27(1, 2, 1)];
  m[22] = raw[t27(1, 1, 2)];
  m[23] = raw[t27(2, 2, 1)];
  m[24] = raw[t27(2, 1, 2)];
  m[25] = raw[t27(1, 2, 2)];
  m[26] = raw[t27(2, 2, 2)];
}

// Correctly rounded x / D for D = 3 and D = 6 without a division
// instruction: Markstein's correction step (P. Markstein, "Computation of
// elementary functions on the IBM RISC System/6000 processor", IBM J. Res.
// Dev. 34(1), 1990; for divisors known in advance, N. Brisebarre, J.-M.
// Muller, S. K. Raina, IEEE Trans. Computers 53(8), 2004):
//   z = RN(1/D),  q0 = RN(x z),  r = x - q0 D (exact with one FMA),  q = RN(q0 + r z).
// With z within half an ulp of 1/D and q0 within one ulp of x / D, q is the
// correctly rounded quotient unless an intermediate value underflows or
// overflows (Markstein's theorem). FP32, against IEEE x / D over every input:
// identical for D = 3 except x = -0 (gives +0) and x = +-inf (gives NaN); for
// D = 6 identical except x = -0, +-inf and 0 < |x| <= 2^-125. populations_d3q27
// below uses it only where none of those can occur (FP64: away from the
// underflow range by a wide margin).
template <int D, class Real>
__device__ __forceinline__ Real div_exact_const(Real x) {
  constexpr Real z = Real(1) / Real(D);
  if constexpr (std::is_same_v<Real, float>) {
    const float q0 = __fmul_rn(x, z);
    const float r = __fmaf_rn(-q0, (float)D, x);
    return __fmaf_rn(r, z, q0);
  } else {
    const double q0 = __dmul_rn(x, z);
    const double r = __fma_rn(-q0, (double)D, x);
    return __fma_rn(r, z, q0);
  }
}

// Division policies of the D3Q27 population transform: (x * P) / N with
// N in {2, 3, 6} as IEEE divisions, or through div_exact_const (N = 3, 6)
// and the exact x * 0.5 (N = 2). Const::checked<N> says which dividends the
// fast transform must see in the range Const::safe accepts: in FP32 those of
// the divisions by 6 (division by 3 is exact for every finite FP32 input), in
// FP64 all of them.
struct Div27Ieee {
  template <int N, class Real>
  __device__ __forceinline__ static Real div(Real x) { return x / Real(N); }
};
template <class Real>
struct Div27Const {
  template <int N>
  __device__ __forceinline__ static Real div(Real x) {
    if constexpr (N == 2) return x * Real(0.5);
    else return div_exact_const<N>(x);
  }
  template <int N>
  static constexpr bool checked = std::is_same_v<Real, float> ? N == 6 : N != 2;
  // zero, or |x| >= 2^-124 (FP32) / 2^-960 (FP64)
  __device__ __forceinline__ static bool safe(Real x) {
    if constexpr (std::is_same_v<Real, float>) return x == 0.0f || fabsf(x) >= 0x1p-124f;
    else return x == 0.0 || fabs(x) >= 0x1p-960;
  }
  // every moment finite and small enough that nothing in the transform overflows
  __device__ __forceinline__ static bool bounded(Real m) {
    if constexpr (std::is_same_v<Real, float>) return fabsf(m) <= 0x1p100f;
    else return fabs(m) <= 0x1p900;
  }
};

// transform_to_populations_d3q27 (lattice_mrt.hpp:1130-1225). With
// CHECK, `ok` is cleared when a dividend that Div::checked names is outside
// the range Div::safe accepts. Each dividend is +-x or +-2x for a value x
// checked here (|2x| >= |x|, and the sign does not matter).
//
// DROP (fast transform only, whose result is used only when `ok` holds, i.e.
// every intermediate is finite): leaves out the terms whose basis factor is 0
// (+-0 added to a sum that starts at +0, see moments_d3q27) and forms
// (x * -2) / 6 as -(x / 3). Both are the correctly rounded -x/3 (x * -2 is
// exact), and the x = +-0 cases differ only in the sign of a zero term, which
// the sum absorbs.
template <class Real, class Div, bool CHECK, bool DROP = false>
__device__ __forceinline__ void populations_d3q27_with(const Real (&m)[27], Real (&f)[27], bool& ok) {
  Real raw[27], zi[27], yzi[27], p[27];
  auto check = [&](auto n, Real x) {
    if constexpr (CHECK) {
      if constexpr (Div::template checked<decltype(n)::value>) ok = ok && Div::safe(x);
    }
  };
  using N3 = std::integral_constant<int, 3>;
  using N6 = std::integral_constant<int, 6>;
  raw[t27(0, 0, 0)] = m[0];
  raw[t27(1, 0, 0)] = m[1];
  raw[t27(0, 1, 0)] = m[2];
  raw[t27(0, 0, 1)] = m[3];
  const Real d200 = m[4] + m[5];
  const Real d020 = Real{2} * m[4] - m[5] + Real{3} * m[6];
  const Real d002 = Real{2} * m[4] - m[5] - Real{3} * m[6];
  check(N3{}, d200);
  check(N6{}, d020);
  check(N6{}, d002);
  raw[t27(2, 0, 0)] = Div::template div<3>(d200);
  raw[t27(0, 2, 0)] = Div::template div<6>(d020);
  raw[t27(0, 0, 2)] = Div::template div<6>(d002);
  raw[t27(1, 1, 0)] = m[7];
  raw[t27(0, 1, 1)] = m[8];
  raw[t27(1, 0, 1)] = m[9];
  raw[t27(2, 1, 0)] = m[10];
  raw[t27(2, 0, 1)] = m[11];
  raw[t27(1, 2, 0)] = m[12];
  raw[t27(0, 2, 1)] = m[13];
  raw[t27(1, 0, 2)] = m[14];
  raw[t27(0, 1, 2)] = m[15];
  raw[t27(1, 1, 1)] = m[16];
  raw[t27(2, 2, 0)] = m[17];
  raw[t27(2, 0, 2)] = m[18];
  raw[t27(0, 2, 2)] = m[19];
  raw[t27(2, 1, 1)] = m[20];
  raw[t27(1, 2, 1)] = m[21];
  raw[t27(1, 1, 2)] = m[22];
  raw[t27(2, 2, 1)] = m[23];
  raw[t27(2, 1, 2)] = m[24];
  raw[t27(1, 2, 2)] = m[25];
  raw[t27(2, 2, 2)] = m[26];
  static_for<9>([&](auto J) {  // dividends of pass 1: order 0 (/3) and order 2 (/6) rows
    check(N3{}, raw[t27(LB_I(J) / 3, LB_I(J) % 3, 0)]);
    check(N6{}, raw[t27(LB_I(J) / 3, LB_I(J) % 3, 2)]);
  });
  static_for<27>([&](auto J) {  // (ax, ay, iz)
    constexpr int a = LB_I(J) / 9, b = (LB_I(J) / 3) % 3, c = LB_I(J) % 3;
    Real v = Real(0);
    static_for<3>([&](auto K) {
      constexpr int k = LB_I(K);
      constexpr int basis = p27_basis(k, c - 1);
      if constexpr (DROP && basis == 0) {
      } else if constexpr (DROP && basis == -2) {
        v += -Div::template div<3>(raw[t27(a, b, k)]);
      } else {
        v += Div::template div<p27_norm(k)>(raw[t27(a, b, k)] * Real(basis));
      }
    });
    zi[t27(a, b, c)] = v;
  });
  static_for<9>([&](auto J) {  // dividends of pass 2
    check(N3{}, zi[t27(LB_I(J) / 3, 0, LB_I(J) % 3)]);
    check(N6{}, zi[t27(LB_I(J) / 3, 2, LB_I(J) % 3)]);
  });
  static_for<27>([&](auto J) {  // (ax, iy, iz)
    constexpr int a = LB_I(J) / 9, b = (LB_I(J) / 3) % 3, c = LB_I(J) % 3;
    Real v = Real(0);
    static_for<3>([&](auto K) {
      constexpr int k = LB_I(K);
      constexpr int basis = p27_basis(k, b - 1);
      if constexpr (DROP && basis == 0) {
      } else if constexpr (DROP && basis == -2) {
        v += -Div::template div<3>(zi[t27(a, k, c)]);
      } else {
        v += Div::template div<p27_norm(k)>(zi[t27(a, k, c)] * Real(basis));
      }
    });
    yzi[t27(a, b, c)] = v;
  });
  static_for<9>([&](auto J) {  // dividends of pass 3
    check(N3{}, yzi[t27(0, LB_I(J) / 3, LB_I(J) % 3)]);
    check(N6{}, yzi[t27(2, LB_I(J) / 3, LB_I(J) % 3)]);
  });
  static_for<27>([&](auto J) {  // (ix, iy, iz)
    constexpr int a = LB_I(J) / 9, b = (LB_I(J) / 3) % 3, c = LB_I(J) % 3;
    Real v = Real(0);
    static_for<3>([&](auto K) {
      constexpr int k = LB_I(K);
      constexpr int basis = p27_basis(k, a - 1);
      if constexpr (DROP && basis == 0) {
      } else if constexpr (DROP && basis == -2) {
        v += -Div::template div<3>(yzi[t27(k, b, c)]);
      } else {
        v += Div::template div<p27_norm(k)>(yzi[t27(k, b, c)] * Real(basis));
      }
    });
    p[t27(a, b, c)] = v;
  });
  static_for<27>([&](auto I) { f[LB_I(I)] = p[tensor_slot27<LB_I(I)>()]; });
}

// Out of line, so that the rare fallback below keeps its divisions out of the
// kernel's instruction stream.
template <class Real>
static __device__ __noinline__ void populations_d3q27_ieee(const Real (&m)[27], Real (&f)[27]) {
  bool ok = true;
  populations_d3q27_with<Real, Div27Ieee, false>(m, f, ok);
}

// The fast transform (Div27Const) gives the bits of the IEEE one when every
// moment is bounded (so nothing overflows and no dividend is infinite) and
// every checked dividend is in the safe range; a zero quotient's sign never
// matters, since each one is added to a sum that starts at +0. Any other cell
// is recomputed with IEEE divisions.
template <class Real>
__device__ __forceinline__ void populations_d3q27(const Real (&m)[27], Real (&f)[27]) {
  using Div = Div27Const<Real>;
  bool ok = true;
  static_for<27>([&](auto K) { ok = ok && Div::bounded(m[LB_I(K)]); });
  populations_d3q27_with<Real, Div, true, true>(m, f, ok);
  if (!ok) {
    // copies: passing m or f itself to the out-of-line call would make them
    // addressable and move them to local memory on the fast path as well
    Real mc[27], fc[27];
    static_for<27>([&](auto K) { mc[LB_I(K)] = m[LB_I(K)]; });
    populations_d3q27_ieee<Real>(mc, fc);
    static_for<27>([&](auto K) { f[LB_I(K)] = fc[LB_I(K)]; });
  }
}

// Projected equilibrium populations of collide_mrt_d3q27 (lattice_mrt.hpp:1242-1268).
template <class Real>
__device__ __forceinline__ void equilibrium_d3q27(Real rho, const Real (&u)[3], Real (&fe)[27]) {
  const Real ux = u[0], uy = u[1], uz = u[2];
  const Real usq = ux * ux + uy * uy + uz * uz;
  static_for<27>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr double wd = D3Q27::w[i];
    const Real cu = c_dot<D3Q27, i>(u);
    fe[i] = Real(wd) * rho * (Real{1} + Real{3} * cu + Real{4.5} * cu * cu - Real{1.5} * usq);
  });
}

// Moment relaxation with MrtRelaxationRates_D3Q27 (lattice_mrt.hpp:161-204).
template <class Real>
__device__ __forceinline__ void relax_d3q27(Real (&m)[27], const Real (&eq)[27], Real omega) {
  const Real s_b = Real(1.19), s_e = Real(1.1), s_eps = Real(1.2), s_q = Real(1.2);
  static_for<27>([&](auto I) {
    constexpr int i = LB_I(I);
    if constexpr (i >= 4) {
      const Real s = i == 4 ? s_b : (i <= 9 ? omega : (i <= 15 ? s_e : (i == 16 ? s_eps : s_q)));
      m[i] -= s * (m[i] - eq[i]);
    }
  });
}

// The reference's collision term for term, with IEEE divisions: the path of
// every cell that the guard of collide_mrt_d3q27 sends away. Out of line, so
// its code stays out of the kernel's instruction stream.
template <class Real>
static __device__ __noinline__ void collide_mrt_d3q27_full(Real (&f)[27], Real omega) {
  Real rho, u[3], m[27], fe[27], eq[27];
  macro_state<D3Q27>(f, rho, u);
  moments_d3q27<Real>(f, m);
  equilibrium_d3q27<Real>(rho, u, fe);
  moments_d3q27<Real>(fe, eq);
  relax_d3q27<Real>(m, eq, omega);
  bool ok = true;
  populations_d3q27_with<Real, Div27Ieee, false>(m, f, ok);
}

// collide_mrt_d3q27 (lattice_mrt.hpp:1284-1305) with the projected
// equilibrium of :1242-1268 and MrtRelaxationRates_D3Q27 (:161-204).
// Guard: |rho| <= 2^60 and every |u_d| <= 2^20 (false for NaN). A finite
// density means every population is finite (a non-finite addend makes the
// sum inf or NaN), and the bounds keep every equilibrium population below
// 2^106, so both forward transforms may drop their zero-factor terms
// (moments_d3q27). Other cells run the full expression out of line.
template <class Real>
__device__ __forceinline__ void collide_mrt_d3q27(Real (&f)[27], Real omega) {
  Real rho, u[3];
  macro_state<D3Q27>(f, rho, u);
  const bool fast = fabs(rho) <= Real(0x1p60) && fabs(u[0]) <= Real(0x1p20) &&
                    fabs(u[1]) <= Real(0x1p20) && fabs(u[2]) <= Real(0x1p20);
  if (!fast) {
    // a copy: passing f itself would make it addressable (local memory)
    Real fc[27];
    static_for<27>([&](auto K) { fc[LB_I(K)] = f[LB_I(K)]; });
    collide_mrt_d3q27_full<Real>(fc, omega);
    static_for<27>([&](auto K) { f[LB_I(K)] = fc[LB_I(K)]; });
    return;
  }
  Real m[27], fe[27], eq[27];
  moments_d3q27<Real, true>(f, m);
  equilibrium_d3q27<Real>(rho, u, fe);
  moments_d3q27<Real, true>(fe, eq);
  relax_d3q27<Real>(m, eq, omega);
  populations_d3q27<Real>(m, f);
}

// ----------------------------------------------------------------------------
// Regularized (RLBM) collision, collide_regularized (lattice_physics.hpp:422-605)
// with compute_pi_neq_* (:116-211).
// ----------------------------------------------------------------------------
template <class L, class Real>
__device__ __forceinline__ void collide_rlbm(Real (&f)[L::Q], Real omega) {
  Real rho, u[L::D], fe[L::Q];
  macro_state<L>(f, rho, u);
  const Real usq = u_dot_u<L>(u);
  equilibria<L>(rho, u, usq, fe);
  const Real hp = Real{9} / Real{2};
  const Real cs2 = Real(L::cs2);
  // Pi_neq = sum_i (f_i - feq_i) c_i c_i, accumulated from zero in ascending i.
  Real pxx = Real(0), pyy = Real(0), pzz = Real(0), pxy = Real(0), pxz = Real(0), pyz = Real(0);
  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    const Real fn = f[i] - fe[i];
    constexpr int ix = L::c[i][0], iy = L::c[i][1], iz = L::c[i][2];
    const Real cx = Real(ix), cy = Real(iy), cz = Real(iz);
    (void)cz;
    pxx += fn * cx * cx;
    pyy += fn * cy * cy;
    pxy += fn * cx * cy;
    if constexpr (L::D == 3) {
      pzz += fn * cz * cz;
      pxz += fn * cx * cz;
      pyz += fn * cy * cz;
    }
  });
  if constexpr (L::id == kD2Q9) {
    const Real ux = u[0], uy = u[1];
    const Real a_xxx = Real{3} * ux * pxx;
    const Real a_yyy = Real{3} * uy * pyy;
    const Real a_xxy = Real{2} * ux * pxy + uy * pxx;
    const Real a_xyy = Real{2} * uy * pxy + ux * pyy;
    static_for<9>([&](auto I) {
      constexpr int i = LB_I(I);
      constexpr double wd = L::w[i];
      constexpr int ix = L::c[i][0], iy = L::c[i][1];
      const Real cx = Real(ix), cy = Real(iy);
      const Real q_xx = cx * cx - cs2, q_yy = cy * cy - cs2, q_xy = cx * cy;
      const Real second = q_xx * pxx + q_yy * pyy + Real{2} * q_xy * pxy;
      const Real h_xxx = cx * cx * cx - Real{3} * cs2 * cx;
      const Real h_yyy = cy * cy * cy - Real{3} * cs2 * cy;
      const Real h_xxy = cx * cx * cy - cs2 * cy;
      const Real h_xyy = cx * cy * cy - cs2 * cx;
      const Real third = a_xxx * h_xxx + a_yyy * h_yyy + Real{3} * (a_xxy * h_xxy + a_xyy * h_xyy);
      const Real rec = Real(wd) * hp * (second + third);
      f[i] = fe[i] + (Real{1} - omega) * rec;
    });
  } else {
    const Real ux = u[0], uy = u[1], uz = u[2];
    const Real a_xxx = Real{3} * ux * pxx;
    const Real a_yyy = Real{3} * uy * pyy;
    const Real a_zzz = Real{3} * uz * pzz;
    const Real a_xxy = Real{2} * ux * pxy + uy * pxx;
    const Real a_xxz = Real{2} * ux * pxz + uz * pxx;
    const Real a_yyz = Real{2} * uy * pyz + uz * pyy;
    Real a_xyy, a_xzz, a_yzz, a_xyz;
    if constexpr (L::id == kD3Q19) {
      a_xyy = Real{2} * uy * pxy + ux * pyy;
      a_xzz = Real{2} * uz * pxz + ux * pzz;
      a_yzz = Real{2} * uz * pyz + uy * pzz;
      a_xyz = Real(0);
    } else {
      a_xyy = ux * pyy + Real{2} * uy * pxy;
      a_xzz = ux * pzz + Real{2} * uz * pxz;
      a_yzz = uy * pzz + Real{2} * uz * pyz;
      a_xyz = ux * pyz + uy * pxz + uz * pxy;
    }
    static_for<L::Q>([&](auto I) {
      constexpr int i = LB_I(I);
      constexpr double wd = L::w[i];
      constexpr int ix = L::c[i][0], iy = L::c[i][1], iz = L::c[i][2];
    const Real cx = Real(ix), cy = Real(iy), cz = Real(iz);
      const Real q_xx = cx * cx - cs2, q_yy = cy * cy - cs2, q_zz = cz * cz - cs2;
      const Real q_xy = cx * cy, q_xz = cx * cz, q_yz = cy * cz;
      const Real second = q_xx * pxx + q_yy * pyy + q_zz * pzz +
                          Real{2} * (q_xy * pxy + q_xz * pxz + q_yz * pyz);
      const Real h_xxx = cx * cx * cx - Real{3} * cs2 * cx;
      const Real h_yyy = cy * cy * cy - Real{3} * cs2 * cy;
      const Real h_zzz = cz * cz * cz - Real{3} * cs2 * cz;
      const Real h_xxy = cx * cx * cy - cs2 * cy;
      const Real h_xxz = cx * cx * cz - cs2 * cz;
      const Real h_xyy = cx * cy * cy - cs2 * cx;
      const Real h_yyz = cy * cy * cz - cs2 * cz;
      const Real h_xzz = cx * cz * cz - cs2 * cx;
      const Real h_yzz = cy * cz * cz - cs2 * cy;
      const Real h_xyz = cx * cy * cz;
      (void)h_xxx, (void)h_yyy, (void)h_zzz, (void)h_xyz;  // unused by the D3Q19 branch
      Real third;
      if constexpr (L::id == kD3Q19) {
        third = Real{3} * (h_xxy + h_yzz) * (a_xxy + a_yzz) + (h_xxy - h_yzz) * (a_xxy - a_yzz) +
                Real{3} * (h_xzz + h_xyy) * (a_xzz + a_xyy) + (h_xzz - h_xyy) * (a_xzz - a_xyy) +
                Real{3} * (h_yyz + h_xxz) * (a_yyz + a_xxz) + (h_yyz - h_xxz) * (a_yyz - a_xxz);
      } else {
        third = a_xxx * h_xxx + a_yyy * h_yyy + a_zzz * h_zzz +
                Real{3} * (a_xxy * h_xxy + a_xxz * h_xxz + a_xyy * h_xyy + a_yyz * h_yyz +
                           a_xzz * h_xzz + a_yzz * h_yzz) +
                Real{6} * a_xyz * h_xyz;
      }
      const Real rec = Real(wd) * hp * (second + third);
      f[i] = fe[i] + (Real{1} - omega) * rec;
    });
  }
}

// collide_cell dispatch (lattice_core.hpp:90-126, lattice_cuda.cu:90-126).
template <class L, class Real, int CT>
__device__ __forceinline__ void collide(Real (&f)[L::Q], Real omega, Real omega_minus) {
  if constexpr (CT == kBGK) {
    collide_bgk<L>(f, omega);
  } else if constexpr (CT == kTRT) {
    collide_trt<L>(f, omega, omega_minus);
  } else if constexpr (CT == kMRT) {
    if constexpr (L::id == kD2Q9) collide_mrt_d2q9<Real>(f, omega);
    else if constexpr (L::id == kD3Q19) collide_mrt_d3q19<Real>(f, omega);
    else collide_mrt_d3q27<Real>(f, omega);
  } else {
    collide_rlbm<L>(f, omega);
  }
}

// ----------------------------------------------------------------------------
// Advection-diffusion (lattice_physics.hpp:607-743).
// ----------------------------------------------------------------------------

// compute_concentration: C = sum g_i in ascending i.
template <class S, class Real>
__device__ __forceinline__ Real concentration(const Real (&g)[S::Q]) {
  Real c = g[0];
  static_for<S::Q - 1>([&](auto I) { c += g[LB_I(I) + 1]; });
  return c;
}

// compute_scalar_equilibrium: w C (1 + (c.u) / cs2), with a true division by cs2.
template <class S, int i, class Real>
__device__ __forceinline__ Real geq(Real conc, const Real (&u)[S::D]) {
  constexpr double wd = S::w[i];
  const Real cu = c_dot<S, i>(u);
  const Real cs2 = Real(S::cs2);
  return Real(wd) * conc * (Real(1.0) + cu / cs2);
}

// collide_scalar_bgk: g_i += omega_c (g_eq - g_i) + w_i S.
template <class S, class Real>
__device__ __forceinline__ void collide_scalar(Real (&g)[S::Q], const Real (&u)[S::D], Real omega_c,
                                               Real source) {
  const Real conc = concentration<S>(g);
  static_for<S::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr double wd = S::w[i];
    const Real eq = geq<S, i>(conc, u);
    g[i] += omega_c * (eq - g[i]) + Real(wd) * source;
  });
}

template <class Real> struct RealEps;
template <> struct RealEps<float> { static constexpr float value = 1.1920928955078125e-07f; };
template <> struct RealEps<double> { static constexpr double value = 2.220446049250313080847e-16; };

// compute_reaction_ab_source: exact one-step A + B -> C batch solution; the
// returned increment is applied to both species.
template <class Real>
__device__ __forceinline__ Real reaction_source(Real a, Real b, Real k) {
  const Real abs_a = a < Real{} ? -a : a;
  const Real abs_b = b < Real{} ? -b : b;
  const Real diff = b - a;
  const Real abs_diff = diff < Real{} ? -diff : diff;
  const Real tol = Real(64.0) * RealEps<Real>::value * (Real(1.0) + abs_a + abs_b);
  Real a_after;
  if (abs_diff <= tol) {
    a_after = a / (Real(1.0) + k * a);
  } else {
    const Real att = rexp<Real>(-k * diff);
    a_after = a * diff * att / (b - a * att);
  }
  return a_after - a;
}

// Two species pulled, one exact A+B->C source applied to both
// (lattice_core.hpp:403-411).
template <class SL, class Real>
__device__ __forceinline__ void react_pair(Real (&a)[SL::Q], Real (&b)[SL::Q],
                                           const Real (&u)[SL::D], Real omega_c, Real k) {
  const Real ca = concentration<SL>(a);
  const Real cb = concentration<SL>(b);
  const Real src = reaction_source<Real>(ca, cb, k);
  collide_scalar<SL>(a, u, omega_c, src);
  collide_scalar<SL>(b, u, omega_c, src);
}

}  // namespace lbcube
