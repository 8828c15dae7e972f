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
template <class L, class Real, int CT>
__device__ __forceinline__ double fluid_adjoint_cell(const Real (&gv)[L::Q], const Real (&lv)[L::Q],
                                                     Real rho, const Real (&u)[L::D],
                                                     const AdjointParams& ap, Real (&mu)[L::Q]) {
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
    constexpr int o = L::opp[j];
    Real m = a * lv[j] + A + c_dot<L, j>(B);
    if constexpr (CT != kBGK) m += b * lv[o];
    mu[j] = m;
  });
  return dtau;
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
