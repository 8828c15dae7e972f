// Per-cell pieces of the discrete adjoint of the collide-stream step (BGK,
// TRT), shared by the fluid adjoint (adjoint.cu) and the coupled
// fluid + A + B -> C adjoint (adjoint_reactive.cu).
//
// Forward step (lattice_core.hpp:146-216): f^{n+1}(x, i) = C_i(g(x)), with the
// pulled state g_j(x) = f^n(x - c_j, j). For an objective J(f^N), the adjoint
// lambda^n = dJ/df^n obeys
//   lambda^n(x - c_j, j) = mu_j(x),   mu(x) = J_C(g(x))^T lambda^{n+1}(x, .),
// a scatter that is a bijection for every j (race-free with ping-pong buffers).
// For f_eq = w rho (1 + 3 c.u + 4.5 (c.u)^2 - 1.5 u.u) as a function of
// rho = sum g and j = sum g c:
//   d f_eq_i / d rho = w_i (1 - 4.5 (c_i.u)^2 + 1.5 u.u)
//   d f_eq_i / d j_a = w_i (3 c_ia + 9 (c_i.u) c_ia - 3 u_a)
// so with Lambda_i the weights of f_eq_i in C (BGK: omega lambda_i; TRT:
// omega+ (lambda_i + lambda_o)/2 + omega- (lambda_i - lambda_o)/2),
//   mu_j = a lambda_j + b lambda_opp(j) + A + B . c_j,
//   A = sum_i Lambda_i d f_eq_i / d rho,   B_a = sum_i Lambda_i d f_eq_i / d j_a,
// with a = 1 - omega, b = 0 (BGK) or a = 1 - (omega+ + omega-)/2,
// b = (omega- - omega+)/2 (TRT): O(Q) work per cell.
#pragma once

#include "cells.cuh"
#include "collide.cuh"
#include "common.cuh"

namespace lbcube {

// Resident blocks of kThreads per SM that the fluid adjoint kernels' register
// allocation must allow: FP32 five (96 registers instead of 115), FP64 two
// (FP64 values take two registers each; five blocks spilled up to 1 KB).
template <class Real>
constexpr int kAdjointBlocks = sizeof(Real) == 4 ? 5 : 2;

struct AdjointParams {
  double omega, omega_minus;
  double domega_dtau, domega_minus_dtau;  // derivatives of the rates w.r.t. tau
};

template <class Real>
inline AdjointParams make_params(int collision, double tau) {
  AdjointParams ap{};
  const Real omega = Real(1) / Real(tau);
  ap.omega = omega;
  ap.domega_dtau = -(double)omega * (double)omega;
  if (collision == kTRT) {
    const Real omm = trt_omega_minus<Real>(omega);
    ap.omega_minus = omm;
    // tau- = Lambda / (tau - 1/2) + 1/2  =>  d omega- / d tau = omega-^2 Lambda / (tau - 1/2)^2
    const double t = (double)tau - 0.5;
    ap.domega_minus_dtau = (double)omm * (double)omm * 0.25 / (t * t);
  }
  return ap;
}

// mu = J_C(g)^T lambda at one cell, from the pulled pre-collision populations
// gv (with their rho and u) and lambda^{n+1} at the cell (lv). Returns the
// cell's lambda . dC/dtau (the tau-derivative of the step, evaluated per cell
// in the population precision). One pass over the opposite pairs (i, o):
// f_eq_i = E + O, f_eq_o = E - O with E = w rho (1 + 4.5 (c.u)^2 - 1.5 u.u) and
// O = 3 w rho c.u, so every sum needs only the pair's own values.
template <class L, class Real>
__device__ __forceinline__ double fluid_adjoint_cell_mrt(const Real (&gv)[L::Q], const Real (&lv)[L::Q],
                                                         Real rho, const Real (&u)[L::D],
                                                         const AdjointParams& ap, Real (&mu)[L::Q]);

template <class L, class Real, int CT>
__device__ __forceinline__ double fluid_adjoint_cell(const Real (&gv)[L::Q], const Real (&lv)[L::Q],
                                                     Real rho, const Real (&u)[L::D],
                                                     const AdjointParams& ap, Real (&mu)[L::Q]) {
  if constexpr (CT == kMRT) return fluid_adjoint_cell_mrt<L, Real>(gv, lv, rho, u, ap, mu);
  const Real usq = u_dot_u<L>(u);
  const Real om = Real(ap.omega), omm = Real(ap.omega_minus);
  const Real base = Real(1) - Real(1.5) * usq;
  Real dt1 = Real(0), dt2 = Real(0), W = Real(0), Aq = Real(0), B[L::D];
  static_for<L::D>([&](auto D) { B[LB_I(D)] = Real(0); });
  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr int o = L::opp[i];
    constexpr double wd = L::w[i];
    const Real wr = Real(wd) * rho;
    if constexpr (i == o) {  // rest population: f_eq = w rho (1 - 1.5 u.u)
      if constexpr (CT == kBGK) dt1 += lv[i] * (wr * base - gv[i]);
      else dt1 += lv[i] * (gv[i] - wr * base);
      W += Real(wd) * (om * lv[i]);
    } else if constexpr (i < o) {
      const Real cu = c_dot<L, i>(u);
      const Real E = wr * (base + Real(4.5) * cu * cu), O = Real(3) * wr * cu;
      Real sum, dif;  // Lam_i + Lam_o, Lam_i - Lam_o
      if constexpr (CT == kBGK) {
        sum = om * (lv[i] + lv[o]);
        dif = om * (lv[i] - lv[o]);
        dt1 += lv[i] * ((E + O) - gv[i]) + lv[o] * ((E - O) - gv[o]);
      } else {
        const Real lp = lv[i] + lv[o], lm = lv[i] - lv[o];
        sum = om * lp;
        dif = omm * lm;
        dt1 += lp * (Real(0.5) * (gv[i] + gv[o]) - E);  // (lambda_i + lambda_o) (g+ - f_eq+)
        dt2 += lm * (Real(0.5) * (gv[i] - gv[o]) - O);  // (lambda_i - lambda_o) (g- - f_eq-)
      }
      W += Real(wd) * sum;
      Aq += Real(wd) * sum * cu * cu;
      // w (Lam_i (3 + 9 cu) - Lam_o (3 - 9 cu)) = w (3 (Lam_i - Lam_o) + 9 cu (Lam_i + Lam_o))
      const Real s = Real(wd) * (Real(3) * dif + Real(9) * cu * sum);
      static_for<L::D>([&](auto D) {
        constexpr int c = L::c[i][LB_I(D)];
        if constexpr (c > 0) B[LB_I(D)] += s;
        if constexpr (c < 0) B[LB_I(D)] -= s;
      });
    }
  });
  const double dtau = CT == kBGK ? (double)dt1 * ap.domega_dtau
                                 : -((double)dt1 * ap.domega_dtau + (double)dt2 * ap.domega_minus_dtau);
  // A = sum_i w_i Lam_i (1 + 1.5 u.u) - 4.5 sum_i w_i Lam_i (c_i.u)^2
  // B = sum_i w_i Lam_i (3 + 9 c_i.u) c_i - 3 u sum_i w_i Lam_i
  const Real A = W * (Real(1) + Real(1.5) * usq) - Real(4.5) * Aq;
  static_for<L::D>([&](auto D) { B[LB_I(D)] -= Real(3) * W * u[LB_I(D)]; });
  const Real a = CT == kBGK ? Real(1) - om : Real(1) - Real(0.5) * (om + omm);
  const Real b = CT == kBGK ? Real(0) : Real(0.5) * (omm - om);
  static_for<L::Q>([&](auto I) {
    constexpr int j = LB_I(I);
    [[maybe_unused]] constexpr int o = L::opp[j];
    Real m = a * lv[j] + A + c_dot<L, j>(B);
    if constexpr (CT != kBGK) m += b * lv[o];
    mu[j] = m;
  });
  return dtau;
}

// ---- MRT (D2Q9, D3Q19) ---------------------------------------------------------
// Forward (collide_mrt_d2q9 / collide_mrt_d3q19): m = M g, m_post_k = m_k -
// s_k (m_k - m_eq_k(rho, j)) (s_k = 0 for rho and j), f = M^T D^-1 m_post. With
// nu = D^-1 M lambda the transpose is
//   mu_j = sum_k M_kj (1 - s_k) nu_k + A + B . c_j,
//   A = sum_k s_k nu_k d m_eq_k / d rho,   B_a = sum_k s_k nu_k d m_eq_k / d j_a,
// and lambda . df/domega = -sum over the omega-relaxed k of nu_k (m_k - m_eq_k).
// m_eq written in (rho, j): D2Q9 e = -2 rho + 3 j.j / rho, eps = rho - 3 j.j / rho,
// q_a = -j_a, p_xx = (jx^2 - jy^2) / rho, p_xy = jx jy / rho (rates 1.63, 1.14,
// 1.92, omega); D3Q19 e = -11 rho + 19 j.j / rho, eps = 3 rho - 5.5 j.j / rho,
// q_a = -2/3 j_a, 3p_xx = 3 (2 jx^2 - jy^2 - jz^2) / rho, p_ww = (jy^2 - jz^2) / rho,
// p_xy, p_yz, p_xz = j_a j_b / rho (rate omega), ghosts 0 (rate 1).
template <class L>
struct MrtAdj;
template <>
struct MrtAdj<D2Q9> {
  using Mx = Mrt9;
  __host__ __device__ static constexpr bool omega_rate(int k) { return k == 7 || k == 8; }
  template <class Real>
  __device__ __forceinline__ static Real rate(int k, Real omega) {
    return k == 1 ? Real(1.63) : k == 2 ? Real(1.14) : (k == 4 || k == 6) ? Real(1.92)
         : (k == 7 || k == 8) ? omega : Real(0);
  }
  // d m_eq_k / d rho and d m_eq_k / d j (u = j / rho), and m_eq_k itself
  template <int k, class Real>
  __device__ __forceinline__ static void deq(Real rho, const Real (&u)[2], Real usq, Real& dr,
                                             Real (&dj)[2], Real& eq) {
    dj[0] = dj[1] = Real(0);
    if constexpr (k == 1) { dr = -Real(2) - Real(3) * usq; dj[0] = Real(6) * u[0]; dj[1] = Real(6) * u[1]; eq = -Real(2) * rho + Real(3) * rho * usq; }
    else if constexpr (k == 2) { dr = Real(1) + Real(3) * usq; dj[0] = -Real(6) * u[0]; dj[1] = -Real(6) * u[1]; eq = rho - Real(3) * rho * usq; }
    else if constexpr (k == 4) { dr = Real(0); dj[0] = -Real(1); eq = -rho * u[0]; }
    else if constexpr (k == 6) { dr = Real(0); dj[1] = -Real(1); eq = -rho * u[1]; }
    else if constexpr (k == 7) { dr = -(u[0] * u[0] - u[1] * u[1]); dj[0] = Real(2) * u[0]; dj[1] = -Real(2) * u[1]; eq = rho * (u[0] * u[0] - u[1] * u[1]); }
    else if constexpr (k == 8) { dr = -u[0] * u[1]; dj[0] = u[1]; dj[1] = u[0]; eq = rho * u[0] * u[1]; }
    else { dr = Real(0); eq = Real(0); }
  }
};
template <>
struct MrtAdj<D3Q19> {
  using Mx = Mrt19;
  __host__ __device__ static constexpr bool omega_rate(int k) { return k >= 9 && k <= 13; }
  template <class Real>
  __device__ __forceinline__ static Real rate(int k, Real omega) {
    return (k == 0 || k == 3 || k == 5 || k == 7) ? Real(0) : (k >= 9 && k <= 13) ? omega : Real(1);
  }
  template <int k, class Real>
  __device__ __forceinline__ static void deq(Real rho, const Real (&u)[3], Real usq, Real& dr,
                                             Real (&dj)[3], Real& eq) {
    dj[0] = dj[1] = dj[2] = Real(0);
    if constexpr (k == 1) { dr = -Real(11) - Real(19) * usq; dj[0] = Real(38) * u[0]; dj[1] = Real(38) * u[1]; dj[2] = Real(38) * u[2]; eq = -Real(11) * rho + Real(19) * rho * usq; }
    else if constexpr (k == 2) { dr = Real(3) + Real(5.5) * usq; dj[0] = -Real(11) * u[0]; dj[1] = -Real(11) * u[1]; dj[2] = -Real(11) * u[2]; eq = Real(3) * rho - Real(5.5) * rho * usq; }
    else if constexpr (k == 4) { dr = Real(0); dj[0] = -Real(2) / Real(3); eq = -(Real(2) / Real(3)) * rho * u[0]; }
    else if constexpr (k == 6) { dr = Real(0); dj[1] = -Real(2) / Real(3); eq = -(Real(2) / Real(3)) * rho * u[1]; }
    else if constexpr (k == 8) { dr = Real(0); dj[2] = -Real(2) / Real(3); eq = -(Real(2) / Real(3)) * rho * u[2]; }
    else if constexpr (k == 9) {
      const Real t = Real(2) * u[0] * u[0] - u[1] * u[1] - u[2] * u[2];
      dr = -Real(3) * t; dj[0] = Real(12) * u[0]; dj[1] = -Real(6) * u[1]; dj[2] = -Real(6) * u[2]; eq = Real(3) * rho * t;
    }
    else if constexpr (k == 10) { dr = -(u[1] * u[1] - u[2] * u[2]); dj[1] = Real(2) * u[1]; dj[2] = -Real(2) * u[2]; eq = rho * (u[1] * u[1] - u[2] * u[2]); }
    else if constexpr (k == 11) { dr = -u[0] * u[1]; dj[0] = u[1]; dj[1] = u[0]; eq = rho * u[0] * u[1]; }
    else if constexpr (k == 12) { dr = -u[1] * u[2]; dj[1] = u[2]; dj[2] = u[1]; eq = rho * u[1] * u[2]; }
    else if constexpr (k == 13) { dr = -u[0] * u[2]; dj[0] = u[2]; dj[2] = u[0]; eq = rho * u[0] * u[2]; }
    else { dr = Real(0); eq = Real(0); }
  }
};

template <class L, class Real>
__device__ __forceinline__ double fluid_adjoint_cell_mrt(const Real (&gv)[L::Q], const Real (&lv)[L::Q],
                                                         Real rho, const Real (&u)[L::D],
                                                         const AdjointParams& ap, Real (&mu)[L::Q]) {
  using MA = MrtAdj<L>;
  using Mx = typename MA::Mx;
  const Real om = Real(ap.omega);
  const Real usq = u_dot_u<L>(u);
  Real A = Real(0), B[L::D], keep[L::Q];
  static_for<L::D>([&](auto D) { B[LB_I(D)] = Real(0); });
  Real dom = Real(0);  // lambda . df/domega
  static_for<L::Q>([&](auto KK) {
    constexpr int k = LB_I(KK);
    constexpr int nrm = Mx::M.norm[k];
    Real nu = Real(0);
    static_for<L::Q>([&](auto I) {
      constexpr int i = LB_I(I);
      constexpr int c = Mx::M.m[k][i];
      if constexpr (c == 1) nu += lv[i];
      else if constexpr (c == -1) nu -= lv[i];
      else if constexpr (c != 0) nu += Real(c) * lv[i];
    });
    nu = nu / Real(nrm);
    const Real s = MA::template rate<Real>(k, om);
    keep[k] = (Real(1) - s) * nu;
    Real dr, dj[L::D], eq;
    MA::template deq<k, Real>(rho, u, usq, dr, dj, eq);
    A += s * nu * dr;
    static_for<L::D>([&](auto D) { B[LB_I(D)] += s * nu * dj[LB_I(D)]; });
    if constexpr (MA::omega_rate(k)) {
      Real m = Real(0);  // forward moment of the pulled state
      static_for<L::Q>([&](auto I) {
        constexpr int i = LB_I(I);
        constexpr int c = Mx::M.m[k][i];
        if constexpr (c != 0) m += Real(c) * gv[i];
      });
      dom -= nu * (m - eq);
    }
  });
  static_for<L::Q>([&](auto J) {
    constexpr int j = LB_I(J);
    Real m = A + c_dot<L, j>(B);
    static_for<L::Q>([&](auto KK) {
      constexpr int k = LB_I(KK);
      constexpr int c = Mx::M.m[k][j];
      if constexpr (c != 0) m += Real(c) * keep[k];
    });
    mu[j] = m;
  });
  return (double)dom * ap.domega_dtau;
}

// Adjoint of the pull: mu_j(x) goes to lambda^n(x - c_j, j).
template <class L, class Real>
__device__ __forceinline__ void scatter(Real* __restrict__ lam, const Grid& g, const Neighbours& n,
                                        int x, int y, int z, const Real (&mu)[L::Q]) {
  const size_t plane = (size_t)g.plane;
  static_for<L::Q>([&](auto I) {
    constexpr int j = LB_I(I);
    constexpr int cx = L::c[j][0], cy = L::c[j][1], cz = L::c[j][2];
    const int tx = cx == 0 ? x : (cx > 0 ? n.xm : n.xp);
    const int ty = cy == 0 ? y : (cy > 0 ? n.ym : n.yp);
    const int tz = cz == 0 ? z : (cz > 0 ? n.zm : n.zp);
    lam[plane * j + ((tz * g.ny + ty) * g.nx + tx)] = mu[j];
  });
}

// Fixed-order sum of n doubles, times `scale`, into out[0] (one block of 1024).
static __global__ void __launch_bounds__(1024)
    sum_slots_kernel(const double* __restrict__ s, long long n, long long stride, double scale,
                     double* __restrict__ out) {
  __shared__ double sh[1024];
  double acc = 0.0;
  for (long long k = threadIdx.x; k < n; k += 1024) acc += s[k * stride];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int st = 512; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = sh[0] * scale;
}

}  // namespace lbcube
