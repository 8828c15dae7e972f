// Checkpointed discrete adjoint of the coupled fluid + A + B -> C step, and
// the gradients of a reactive-mixing objective with respect to the reaction
// rate k, the fluid relaxation time tau, the scalar relaxation time tau_c, the
// initial concentration fields A0, B0 and the initial velocity field u0. No
// reference counterpart.
//
// Forward step n (src/simulate_reaction.cpp:518-543, one fused launch here):
//   f^{n+1} = S(f^n)                            fluid collide-stream
//   A^{n+1}_i(x) = a_i + w_c (g_eq_i(C_A, u) - a_i) + w_i S(C_A, C_B, k)
//   B^{n+1}_i(x) = b_i + w_c (g_eq_i(C_B, u) - b_i) + w_i S(C_A, C_B, k)
// with a_j = A^n(x - c_j, j), C_A = sum a (likewise b, C_B), u the fluid
// velocity of f^{n+1}(x), g_eq_i(C, u) = w_i C (1 + c_i.u / cs2)
// (lattice_physics.hpp:643-694) and S the exact batch source (:712-743).
//
// Adjoint step n, per cell x, with (lf, la, lb) = lambda^{n+1} at x:
//   sigma = sum_i w_i (la_i + lb_i)
//   abar_j = (1 - w_c) la_j + w_c sum_i la_i w_i (1 + c_i.u / cs2) + sigma dS/dC_A
//   bbar_j = (1 - w_c) lb_j + w_c sum_i lb_i w_i (1 + c_i.u / cs2) + sigma dS/dC_B
//   ubar   = (w_c / cs2) sum_i w_i c_i (C_A la_i + C_B lb_i)
//   lf_k  += (c_k - u) . ubar / rho            (u = j / rho of f^{n+1}(x))
// then the fluid adjoint (adjoint.cuh) on the updated lf; abar, bbar and the
// fluid mu scatter to the pull sources. dJ/dk gathers sigma dS/dk, dJ/dw_c
// gathers sum_i la_i (g_eq_i(C_A) - a_i) + lb_i (g_eq_i(C_B) - b_i).
// Two kernels per adjoint step: the reaction part reads the advecting velocity
// u^{n+1} that the forward pass stored with each state (exactly the value the
// forward reaction used) and writes ubar; the fluid part adds the ubar term at
// the linearisation point of its own pre-collision (rho, u), equal to the
// post-collision ones up to rounding (BGK and TRT conserve mass and momentum).
// Splitting keeps each kernel's registers, and so its occupancy, close to the
// plain fluid adjoint's. The source derivatives are evaluated in FP64 at the
// step's inputs on the branch the forward step took.
//
// Objectives (final state N, means over the N_c cells):
//   LBM_OBJECTIVE_MEAN_PRODUCT  <C> = <A0> - <C_A^N>   (C = A0 - A; transport
//                               conserves A, so this is the product formed)
//   LBM_OBJECTIVE_SEGREGATION   I_s = cov(C_A, C_B) / (<C_A> <C_B>) of
//                               compute_reactive_stats (lattice_io.hpp:318-337)
#include <algorithm>
#include <type_traits>

#include "adjoint.cuh"
#include "adr.cuh"
#include "adr_shifted.cuh"
#include "cells.cuh"
#include "collide.cuh"
#include "common.cuh"
#include "reduce.cuh"
#include "slab_faces.cuh"
#include "stream_vec.cuh"
#include "../../include/lbcube_b200.h"

namespace lbcube {

// dS/da, dS/db, dS/dk of reaction_source (collide.cuh) on the branch the
// forward evaluation takes for these Real inputs, in FP64.
//   near-equal branch: a' = a / (1 + k a)
//   otherwise:         a' = N / D, N = a d e, D = b - a e, d = b - a, e = exp(-k d)
template <class Real>
__device__ __forceinline__ void reaction_source_grad(Real a, Real b, Real k, double& dsa,
                                                     double& dsb, double& dsk) {
  const Real abs_a = a < Real{} ? -a : a;
  const Real abs_b = b < Real{} ? -b : b;
  const Real diff = b - a;
  const Real abs_diff = diff < Real{} ? -diff : diff;
  const Real tol = Real(64.0) * RealEps<Real>::value * (Real(1.0) + abs_a + abs_b);
  const double A = a, B = b, K = k;
  if (abs_diff <= tol) {
    const double q = 1.0 + K * A;
    const double r = 1.0 / (q * q);
    dsa = r - 1.0;
    dsb = 0.0;
    dsk = -A * A * r;
  } else {
    const double d = B - A;
    const double e = exp(-K * d);
    const double inv = 1.0 / (B - A * e);  // 1 / D
    const double ap = A * d * e * inv;      // N / D
    const double dna = e * (d - A + A * d * K), dnb = A * e * (1.0 - d * K), dnk = -A * d * d * e;
    const double dda = -e * (1.0 + A * K), ddb = 1.0 + A * K * e, ddk = A * d * e;
    dsa = (dna - ap * dda) * inv - 1.0;
    dsb = (dnb - ap * ddb) * inv;
    dsk = (dnk - ap * ddk) * inv;
  }
}

struct ReactiveParams {
  AdjointParams fluid;
  double omega_c, k;
  float rho0, c0;  // shifts of 16-bit stored states (fluid, scalars)
};

// Access to the stored forward states: native Real fields, or shifted 16-bit
// codes decoded to FP32 populations (fluid shifted by rho0, scalars by c0).
template <class Real>
struct NativeState {
  using elem = Real;
  template <class L>
  __device__ __forceinline__ static void pulled(const elem* __restrict__ p, const Grid& g,
                                                const Neighbours& n, int x, int y, int z, float,
                                                Real (&out)[L::Q]) {
    gather<L>(p, g, n, x, y, z, out);
  }
  template <class L>
  __device__ __forceinline__ static void local(const elem* __restrict__ p, const Grid& g, int cell,
                                               float, Real (&out)[L::Q]) {
    load_cell<L>(p, g, cell, out);
  }
  // the pull on a z-slab, across its faces from halo buffers
  template <class L>
  __device__ __forceinline__ static void pulled_slab(const elem* __restrict__ p, const Grid& g,
                                                     const Neighbours& n, int x, int y, int z, float,
                                                     const elem* __restrict__ halo_lo,
                                                     const elem* __restrict__ halo_hi,
                                                     Real (&out)[L::Q]) {
    gather_slab<L>(p, g, n, x, y, z, halo_lo, halo_hi, out);
  }
};
template <int FMT>
struct ShiftedState {
  using elem = unsigned short;
  template <class L>
  __device__ __forceinline__ static void pulled(const elem* __restrict__ p, const Grid& g,
                                                const Neighbours& n, int x, int y, int z, float ref,
                                                float (&out)[L::Q]) {
    unsigned short h[L::Q];
    gather<L>(p, g, n, x, y, z, h);
    static_for<L::Q>([&](auto I) {
      out[LB_I(I)] = ShiftedStorage<FMT>::template decode<L, LB_I(I)>(h[LB_I(I)], {ref});
    });
  }
  template <class L>
  __device__ __forceinline__ static void local(const elem* __restrict__ p, const Grid& g, int cell,
                                               float ref, float (&out)[L::Q]) {
    unsigned short h[L::Q];
    load_cell<L>(p, g, cell, h);
    static_for<L::Q>([&](auto I) {
      out[LB_I(I)] = ShiftedStorage<FMT>::template decode<L, LB_I(I)>(h[LB_I(I)], {ref});
    });
  }
  template <class L>
  __device__ __forceinline__ static void pulled_slab(const elem* __restrict__ p, const Grid& g,
                                                     const Neighbours& n, int x, int y, int z,
                                                     float ref, const elem* __restrict__ halo_lo,
                                                     const elem* __restrict__ halo_hi,
                                                     float (&out)[L::Q]) {
    unsigned short h[L::Q];
    gather_slab<L>(p, g, n, x, y, z, halo_lo, halo_hi, h);
    static_for<L::Q>([&](auto I) {
      out[LB_I(I)] = ShiftedStorage<FMT>::template decode<L, LB_I(I)>(h[LB_I(I)], {ref});
    });
  }
};

// FP64 slots of the reactive adjoint, one set per warp (kThreads / 32 per
// block): dJ/dk, dJ/dtau, dJ/domega_c. Each warp adds its own sums to its own
// slots, so no kernel waits on a block barrier, and the fixed slot order keeps
// the totals identical from run to run.
constexpr int kReactiveSlots = 3;
constexpr int kWarpsPerBlock = kThreads / 32;

// The face buffers of a z-slab (slab_faces.cuh): halos of the stored state the
// step pulls from (its elements: Real or 16-bit codes), and sends of the
// adjoint scatter (Real). Unused on the whole box.
template <class E, class Real>
struct SlabFaces {
  const E* halo_lo;
  const E* halo_hi;
  Real* send_lo;
  Real* send_hi;
};

// Reaction part of adjoint step n at every cell x: from the pulled A^n, B^n,
// lambda_A^{n+1}, lambda_B^{n+1} at x and the advecting velocity u^{n+1}(x)
// (stored by the forward pass), scatter abar and bbar to lambda^n_A, lambda^n_B,
// write ubar(x) = dJ/du^{n+1}(x) for the fluid part, and add the block's
// dJ/dk and dJ/domega_c to its slots.
// SLAB: the pulls and scatters cross the z faces through `faces` (native
// states only).
template <class FL, class Real, class SP, bool SLAB = false>
__global__ void __launch_bounds__(kThreads)
    reaction_adjoint_kernel(const typename SP::elem* __restrict__ an,
                            const typename SP::elem* __restrict__ bn,
                            const Real* __restrict__ u_next, const Real* __restrict__ la_next,
                            const Real* __restrict__ lb_next, Real* __restrict__ la,
                            Real* __restrict__ lb, Real* __restrict__ ubar_out, Grid g,
                            ReactiveParams rp, double* __restrict__ slots,
                            SlabFaces<typename SP::elem, Real> faces = {}) {
  pdl_enter();
  using SL = typename ScalarOf<FL>::type;
  const size_t a_off = (size_t)face_planes<FL>() * g.ny * g.nx;
  const size_t b_off = a_off + (size_t)face_planes<SL>() * g.ny * g.nx;
  int x, y, z;
  const bool active = cell_of(g, x, y, z);
  double acc[2] = {0.0, 0.0};
  if (active) {
    const Neighbours n = neighbours(g, x, y, z);
    const int cell = (z * g.ny + y) * g.nx + x;
    const size_t plane = (size_t)g.plane;
    Real u[FL::D];
    static_for<FL::D>([&](auto D) { u[LB_I(D)] = __ldg(u_next + plane * LB_I(D) + cell); });
    Real ga[SL::Q], gb[SL::Q], lA[SL::Q], lB[SL::Q];
    if constexpr (SLAB) {
      SP::template pulled_slab<SL>(an, g, n, x, y, z, rp.c0, faces.halo_lo + a_off,
                                   faces.halo_hi + a_off, ga);
      SP::template pulled_slab<SL>(bn, g, n, x, y, z, rp.c0, faces.halo_lo + b_off,
                                   faces.halo_hi + b_off, gb);
    } else {
      SP::template pulled<SL>(an, g, n, x, y, z, rp.c0, ga);
      SP::template pulled<SL>(bn, g, n, x, y, z, rp.c0, gb);
    }
    load_cell<SL>(la_next, g, cell, lA);
    load_cell<SL>(lb_next, g, cell, lB);
    const Real ca = concentration<SL>(ga), cb = concentration<SL>(gb);
    double dsa, dsb, dsk;
    reaction_source_grad<Real>(ca, cb, Real(rp.k), dsa, dsb, dsk);
    const Real oc = Real(rp.omega_c);
    const Real inv_cs2 = Real(1.0 / SL::cs2);
    Real sigma = Real(0), ea = Real(0), eb = Real(0), doc = Real(0), ubar[FL::D];
    static_for<FL::D>([&](auto D) { ubar[LB_I(D)] = Real(0); });
    static_for<SL::Q>([&](auto I) {
      constexpr int i = LB_I(I);
      constexpr double wd = SL::w[i];
      const Real w = Real(wd);
      const Real e = w * (Real(1) + c_dot<SL, i>(u) * inv_cs2);
      sigma += w * (lA[i] + lB[i]);
      ea += lA[i] * e;
      eb += lB[i] * e;
      doc += lA[i] * (geq<SL, i>(ca, u) - ga[i]) + lB[i] * (geq<SL, i>(cb, u) - gb[i]);
      const Real s = w * (ca * lA[i] + cb * lB[i]);
      static_for<FL::D>([&](auto D) {
        constexpr int c = SL::c[i][LB_I(D)];
        if constexpr (c > 0) ubar[LB_I(D)] += s;
        if constexpr (c < 0) ubar[LB_I(D)] -= s;
      });
    });
    static_for<FL::D>([&](auto D) { ubar_out[plane * LB_I(D) + cell] = ubar[LB_I(D)] * (oc * inv_cs2); });
    acc[0] = (double)sigma * dsk;
    acc[1] = (double)doc;
    const Real sa = Real((double)sigma * dsa), sb = Real((double)sigma * dsb);
    Real ma[SL::Q], mb[SL::Q];
    static_for<SL::Q>([&](auto I) {
      constexpr int j = LB_I(I);
      ma[j] = (Real(1) - oc) * lA[j] + oc * ea + sa;
      mb[j] = (Real(1) - oc) * lB[j] + oc * eb + sb;
    });
    if constexpr (SLAB) {
      scatter_slab<SL>(la, g, n, x, y, z, ma, faces.send_lo + a_off, faces.send_hi + a_off);
      scatter_slab<SL>(lb, g, n, x, y, z, mb, faces.send_lo + b_off, faces.send_hi + b_off);
    } else {
      scatter<SL>(la, g, n, x, y, z, ma);
      scatter<SL>(lb, g, n, x, y, z, mb);
    }
  }
  warp_sum<2>(acc);
  if ((threadIdx.x & 31) == 0) {
    slots[warp_slot(g) * kReactiveSlots + 0] += acc[0];
    slots[warp_slot(g) * kReactiveSlots + 2] += acc[1];
  }
}

// Fluid part of adjoint step n: lambda_f^{n+1}(x, k) gains
// (c_k - u) . ubar(x) / rho (u = j / rho of the cell), then the fluid adjoint
// of adjoint.cuh; dJ/dtau to the block's slot.
// Register budget kAdjointBlocks (adjoint.cuh).
template <class FL, class Real, int CT, class SP, bool SLAB = false>
__global__ void __launch_bounds__(kThreads, kAdjointBlocks<Real>)
    coupled_fluid_adjoint_kernel(const typename SP::elem* __restrict__ fn,
                                 const Real* __restrict__ lf_next, const Real* __restrict__ ubar_in,
                                 Real* __restrict__ lf, Grid g, AdjointParams ap, float rho0,
                                 double* __restrict__ slots,
                                 SlabFaces<typename SP::elem, Real> faces = {}) {
  pdl_enter();
  int x, y, z;
  const bool active = cell_of(g, x, y, z);
  double dtau = 0.0;
  if (active) {
    const Neighbours n = neighbours(g, x, y, z);
    const int cell = (z * g.ny + y) * g.nx + x;
    const size_t plane = (size_t)g.plane;
    Real gv[FL::Q], lv[FL::Q], mu[FL::Q], rho, u[FL::D], ub[FL::D];
    if constexpr (SLAB) SP::template pulled_slab<FL>(fn, g, n, x, y, z, rho0, faces.halo_lo, faces.halo_hi, gv);
    else SP::template pulled<FL>(fn, g, n, x, y, z, rho0, gv);
    load_cell<FL>(lf_next, g, cell, lv);
    static_for<FL::D>([&](auto D) { ub[LB_I(D)] = __ldg(ubar_in + plane * LB_I(D) + cell); });
    macro_state<FL>(gv, rho, u);
    Real uub = Real(0);
    static_for<FL::D>([&](auto D) { uub += u[LB_I(D)] * ub[LB_I(D)]; });
    const Real inv_rho = Real(1) / rho;
    static_for<FL::Q>([&](auto I) {
      constexpr int k = LB_I(I);
      lv[k] += (c_dot<FL, k>(ub) - uub) * inv_rho;
    });
    dtau = fluid_adjoint_cell<FL, Real, CT>(gv, lv, rho, u, ap, mu);
    if constexpr (SLAB) scatter_slab<FL>(lf, g, n, x, y, z, mu, faces.send_lo, faces.send_hi);
    else scatter<FL>(lf, g, n, x, y, z, mu);
  }
  double v[1] = {dtau};
  warp_sum<1>(v);
  if ((threadIdx.x & 31) == 0) slots[warp_slot(g) * kReactiveSlots + 1] += v[0];
}

// Seeds lambda^N = dJ/d(f^N, A^N, B^N) and writes the block's FP64 share of J.
//   MEAN_PRODUCT: lf = 0, la = -1/N_c, lb = 0; J partial = sum (A0 - C_A^N)
//   SEGREGATION:  with ma, mb, <ab> = cov + ma mb of the final fields (stats),
//     la = (C_B / (ma mb) - <ab> / (ma^2 mb)) / N_c,
//     lb = (C_A / (ma mb) - <ab> / (ma mb^2)) / N_c   (zero when |ma mb| <= eps,
//     where compute_reactive_stats sets I_s = 0)
template <class FL, class Real, int OBJ, class SP>
__global__ void __launch_bounds__(kThreads)
    reactive_seed_kernel(const typename SP::elem* __restrict__ aN,
                         const typename SP::elem* __restrict__ bN, const Real* __restrict__ a0,
                         const double* __restrict__ stats, Real* __restrict__ lf,
                         Real* __restrict__ la, Real* __restrict__ lb, Grid g, float c0,
                         double inv_n, double* __restrict__ j_slots) {
  using SL = typename ScalarOf<FL>::type;
  int x, y, z;
  const bool active = cell_of(g, x, y, z);
  double jpart = 0.0;
  if (active) {
    const int cell = (z * g.ny + y) * g.nx + x;
    const size_t plane = (size_t)g.plane;
    Real va[SL::Q], vb[SL::Q];
    SP::template local<SL>(aN, g, cell, c0, va);
    SP::template local<SL>(bN, g, cell, c0, vb);
    const Real ca = concentration<SL>(va), cb = concentration<SL>(vb);
    Real sa, sb;
    if constexpr (OBJ == LBM_OBJECTIVE_MEAN_PRODUCT) {
      jpart = (double)a0[cell] - (double)ca;
      sa = Real(-inv_n);
      sb = Real(0);
    } else {
      const double ma = stats[0], mb = stats[1], cov = stats[4];
      const double mp = ma * mb, ab = cov + mp;
      if (fabs(mp) > 2.220446049250313080847e-16) {
        sa = Real(inv_n * ((double)cb / mp - ab / (ma * mp)));
        sb = Real(inv_n * ((double)ca / mp - ab / (mb * mp)));
      } else {
        sa = sb = Real(0);
      }
    }
    static_for<SL::Q>([&](auto I) {
      la[plane * LB_I(I) + cell] = sa;
      lb[plane * LB_I(I) + cell] = sb;
    });
    static_for<FL::Q>([&](auto I) { lf[plane * LB_I(I) + cell] = Real(0); });
  }
  double v[1] = {jpart};
  block_sum_to<1>(v, j_slots + block_linear());
}

// dJ/dC0(x) for a scalar initialised as g_eq(C0(x), u0(x)):
//   direct + sum_i lambda^0_i(x) w_i (1 + c_i.u0 / cs2)
template <class FL, class Real>
__global__ void __launch_bounds__(kThreads)
    scalar_init_gradient_kernel(const Real* __restrict__ u0, const Real* __restrict__ lam0,
                                Real direct, Real* __restrict__ grad, Grid g) {
  using SL = typename ScalarOf<FL>::type;
  int x, y, z;
  if (!cell_of(g, x, y, z)) return;
  const int cell = (z * g.ny + y) * g.nx + x;
  const size_t plane = (size_t)g.plane;
  Real u[FL::D], lv[SL::Q];
  static_for<FL::D>([&](auto D) { u[LB_I(D)] = u0[plane * LB_I(D) + cell]; });
  load_cell<SL>(lam0, g, cell, lv);
  const Real inv_cs2 = Real(1.0 / SL::cs2);
  Real s = direct;
  static_for<SL::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr double wd = SL::w[i];
    s += lv[i] * (Real(wd) * (Real(1) + c_dot<SL, i>(u) * inv_cs2));
  });
  grad[cell] = s;
}

// dJ/du0(x) for f^0 = f_eq(rho0, u0), A^0 = g_eq(a0, u0), B^0 = g_eq(b0, u0):
//   sum_i lf_i w_i rho0 (3 c_ia + 9 (c_i.u0) c_ia - 3 u0_a)
//   + sum_i (la_i a0 + lb_i b0) w_i c_ia / cs2      (scalar lattice)
template <class FL, class Real>
__global__ void __launch_bounds__(kThreads)
    reactive_velocity_gradient_kernel(const Real* __restrict__ rho0, const Real* __restrict__ u0,
                                      const Real* __restrict__ a0, const Real* __restrict__ b0,
                                      const Real* __restrict__ lf, const Real* __restrict__ la,
                                      const Real* __restrict__ lb, Real* __restrict__ grad, Grid g) {
  using SL = typename ScalarOf<FL>::type;
  int x, y, z;
  if (!cell_of(g, x, y, z)) return;
  const int cell = (z * g.ny + y) * g.nx + x;
  const size_t plane = (size_t)g.plane;
  Real u[FL::D], gr[FL::D];
  static_for<FL::D>([&](auto D) {
    u[LB_I(D)] = u0[plane * LB_I(D) + cell];
    gr[LB_I(D)] = Real(0);
  });
  const Real r = rho0[cell], ca = a0[cell], cb = b0[cell];
  static_for<FL::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr double wd = FL::w[i];
    const Real wl = Real(wd) * r * __ldg(lf + plane * i + cell);
    const Real s = wl * (Real(3) + Real(9) * c_dot<FL, i>(u));
    static_for<FL::D>([&](auto D) {
      constexpr int c = FL::c[i][LB_I(D)];
      if constexpr (c > 0) gr[LB_I(D)] += s;
      if constexpr (c < 0) gr[LB_I(D)] -= s;
      gr[LB_I(D)] -= Real(3) * wl * u[LB_I(D)];
    });
  });
  const Real inv_cs2 = Real(1.0 / SL::cs2);
  static_for<SL::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr double wd = SL::w[i];
    const Real s = Real(wd) * inv_cs2 *
                   (ca * __ldg(la + plane * i + cell) + cb * __ldg(lb + plane * i + cell));
    static_for<FL::D>([&](auto D) {
      constexpr int c = SL::c[i][LB_I(D)];
      if constexpr (c > 0) gr[LB_I(D)] += s;
      if constexpr (c < 0) gr[LB_I(D)] -= s;
    });
  });
  static_for<FL::D>([&](auto D) { grad[plane * LB_I(D) + cell] = gr[LB_I(D)]; });
}

template <class FL, class Real, class SP>
cudaError_t launch_reactive_adjoint(int collision, const typename SP::elem* fn,
                                    const typename SP::elem* an, const typename SP::elem* bn,
                                    const Real* u_next, const Real* lf_next, const Real* la_next,
                                    const Real* lb_next, Real* lf, Real* la, Real* lb, Real* ubar,
                                    const Grid& g, const ReactiveParams& rp, double* slots,
                                    cudaStream_t s) {
  // programmatic dependent launches (both kernels open with pdl_enter)
  using Faces = SlabFaces<typename SP::elem, Real>;
  const dim3 grid = grid_dims(g), block(block_dims(g));
  cudaError_t err = launch_pdl(reaction_adjoint_kernel<FL, Real, SP, false>, grid, block, 0, s, an, bn,
                               u_next, la_next, lb_next, la, lb, ubar, g, rp, slots, Faces{});
  if (err != cudaSuccess) return err;
  if (collision == kBGK)
    return launch_pdl(coupled_fluid_adjoint_kernel<FL, Real, kBGK, SP, false>, grid, block, 0, s, fn,
                      lf_next, ubar, lf, g, rp.fluid, rp.rho0, slots, Faces{});
  if (collision == kTRT)
    return launch_pdl(coupled_fluid_adjoint_kernel<FL, Real, kTRT, SP, false>, grid, block, 0, s, fn,
                      lf_next, ubar, lf, g, rp.fluid, rp.rho0, slots, Faces{});
  if constexpr (FL::Q != 27)
    return launch_pdl(coupled_fluid_adjoint_kernel<FL, Real, kMRT, SP, false>, grid, block, 0, s, fn,
                      lf_next, ubar, lf, g, rp.fluid, rp.rho0, slots, Faces{});
  else
    return cudaErrorInvalidValue;
}

struct ReactiveLayout {
  size_t ffield, sfield, ufield, state;  // bytes: fluid, one scalar, velocity; one stored state
  size_t lfield, lsfield, lstate;        // bytes of the adjoint fields and one adjoint state
  long long ckpts, blocks;
  size_t off_ckpt, off_seg, off_lam, off_ubar, off_slots, off_j, off_part, off_stats, total;
};

// A stored state n holds f^n, A^n, B^n and the velocity u^n that advected the
// reaction step producing it; an adjoint state holds lambda_f, lambda_A,
// lambda_B (its velocity slot unused).
// elem: bytes of a stored population (2 for 16-bit states); real: bytes of
// the adjoint fields and the stored velocity.
inline ReactiveLayout reactive_layout(int FQ, int SQ, int D, size_t elem, size_t real,
                                      const Grid& g, int steps, int interval) {
  ReactiveLayout l{};
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  l.ffield = up((size_t)FQ * g.plane * elem);
  l.sfield = up((size_t)SQ * g.plane * elem);
  l.ufield = up((size_t)D * g.plane * real);
  l.state = l.ffield + 2 * l.sfield + l.ufield;
  l.lfield = up((size_t)FQ * g.plane * real);
  l.lsfield = up((size_t)SQ * g.plane * real);
  l.lstate = l.lfield + 2 * l.lsfield;
  l.ckpts = (steps + interval - 1) / interval + 1;
  l.blocks = g.blocks();
  l.off_ckpt = 0;
  l.off_seg = l.off_ckpt + (size_t)l.ckpts * l.state;
  l.off_lam = l.off_seg + (size_t)interval * l.state;
  l.off_ubar = l.off_lam + 2 * l.lstate;
  l.off_slots = l.off_ubar + l.ufield;
  l.off_j = l.off_slots + up((size_t)l.blocks * kWarpsPerBlock * kReactiveSlots * sizeof(double));
  l.off_part = l.off_j + up((size_t)l.blocks * sizeof(double));
  l.off_stats = l.off_part + up((size_t)l.blocks * kStatSums * sizeof(double));
  l.total = l.off_stats + 256;
  return l;
}

// FMT < 0: states stored in Real; otherwise 16-bit codes of that format (Real
// is float), fluid shifted by rho0 = 1 and scalars by c0.
template <class FL, class Real, int FMT>
cudaError_t reactive_gradient(int collision, int objective, const Real* rho0, const Real* u0,
                              const Real* a0, const Real* b0, const Grid& g, double tau,
                              double tau_c, double k, float c0, int steps, int interval, char* ws,
                              const ReactiveLayout& lay, double* out, Real* grad_a0, Real* grad_b0,
                              Real* grad_u0, cudaStream_t s) {
  using SL = typename ScalarOf<FL>::type;
  constexpr bool NATIVE = FMT < 0;
  using SP = std::conditional_t<NATIVE, NativeState<Real>, ShiftedState<(FMT < 0 ? 0 : FMT)>>;
  using E = typename SP::elem;
  constexpr int prec = sizeof(Real) == 4 ? LBM_FLOAT : LBM_DOUBLE;
  constexpr int api_format = FMT == kF16S ? LBM_F16S : FMT == kBF16S ? LBM_BF16S
                           : FMT == kE3M12S ? LBM_E3M12S : LBM_Q15S;
  const double omega = (double)(Real(1) / Real(tau));
  const double omega_c = (double)(Real(1) / Real(tau_c));
  struct State {
    E* f;
    E* a;
    E* b;
    Real* u;
  };
  struct Adj {
    Real* f;
    Real* a;
    Real* b;
  };
  auto at = [&](size_t off) {
    char* p = ws + off;
    return State{reinterpret_cast<E*>(p), reinterpret_cast<E*>(p + lay.ffield),
                 reinterpret_cast<E*>(p + lay.ffield + lay.sfield),
                 reinterpret_cast<Real*>(p + lay.ffield + 2 * lay.sfield)};
  };
  auto adj = [&](size_t off) {
    char* p = ws + off;
    return Adj{reinterpret_cast<Real*>(p), reinterpret_cast<Real*>(p + lay.lfield),
               reinterpret_cast<Real*>(p + lay.lfield + lay.lsfield)};
  };
  auto ckpt = [&](long long i) { return at(lay.off_ckpt + (size_t)i * lay.state); };
  auto seg = [&](long long i) { return at(lay.off_seg + (size_t)i * lay.state); };
  const Adj lam[2] = {adj(lay.off_lam), adj(lay.off_lam + lay.lstate)};
  double* slots = reinterpret_cast<double*>(ws + lay.off_slots);
  double* j_slots = reinterpret_cast<double*>(ws + lay.off_j);
  double* partials = reinterpret_cast<double*>(ws + lay.off_part);
  double* stats = reinterpret_cast<double*>(ws + lay.off_stats);
  cudaError_t err;
  Real* ubar = reinterpret_cast<Real*>(ws + lay.off_ubar);
  // one coupled forward step; `keep_u`: store the advecting velocity with the
  // new state (states that only pass through the ping-pong slots of the
  // forward pass are recomputed later and need none)
  auto step = [&](const State& c, const State& n, bool keep_u) -> cudaError_t {
    if constexpr (NATIVE) {
      if (keep_u)
        return fluid_reaction_with_velocity<FL, Real>(collision, c.f, n.f, c.a, n.a, c.b, n.b, n.u,
                                                      g, Real(omega), Real(omega_c), Real(k), s);
      return (cudaError_t)lbm_fluid_reaction_ab_async(FL::id, prec, collision, c.f, n.f, c.a, n.a,
                                                      c.b, n.b, g.nx, g.ny, g.nz, omega, omega_c, k,
                                                      nullptr, 0, s);
    } else {
      return fluid_reaction_shifted<FL, FMT>(collision, c.f, n.f, c.a, n.a, c.b, n.b,
                                             keep_u ? n.u : nullptr, nullptr, g, (float)omega,
                                             (float)omega_c, (float)k, 1.0f, c0, s);
    }
  };

  // forward: equilibrium initial state (16-bit: built in FP32 in the adjoint
  // buffers, then encoded), checkpoints every `interval` steps, the last
  // segment's states kept for the backward sweep
  const State s0 = ckpt(0);
  {
    Real* fi = NATIVE ? reinterpret_cast<Real*>(s0.f) : lam[0].f;
    Real* ai = NATIVE ? reinterpret_cast<Real*>(s0.a) : lam[0].a;
    Real* bi = NATIVE ? reinterpret_cast<Real*>(s0.b) : lam[0].b;
    if ((err = (cudaError_t)lbm_init_equilibrium_async(FL::id, prec, rho0, u0, fi, g.nx, g.ny, g.nz,
                                                       s)) != cudaSuccess)
      return err;
    if ((err = (cudaError_t)lbm_init_equilibrium_async(SL::id, prec, a0, u0, ai, g.nx, g.ny, g.nz,
                                                       s)) != cudaSuccess)
      return err;
    if ((err = (cudaError_t)lbm_init_equilibrium_async(SL::id, prec, b0, u0, bi, g.nx, g.ny, g.nz,
                                                       s)) != cudaSuccess)
      return err;
    if constexpr (!NATIVE) {
      const int r1 = lbm_encode_shifted_async(FL::id, api_format, LBM_FLOAT, fi, s0.f, g.nx, g.ny,
                                              g.nz, 1.0f, s);
      const int r2 = lbm_encode_shifted_async(SL::id, api_format, LBM_FLOAT, ai, s0.a, g.nx, g.ny,
                                              g.nz, c0, s);
      const int r3 = lbm_encode_shifted_async(SL::id, api_format, LBM_FLOAT, bi, s0.b, g.nx, g.ny,
                                              g.nz, c0, s);
      if (r1 != 0 || r2 != 0 || r3 != 0) return (cudaError_t)(r1 ? r1 : r2 ? r2 : r3);
    }
  }
  const long long nseg = (steps + interval - 1) / interval;
  const int last0 = (int)((nseg - 1) * interval);
  State cur = s0;
  for (int n = 0; n < steps; ++n) {
    State nxt;
    bool kept = true;
    if (n + 1 == steps || (n + 1) % interval == 0) {
      nxt = ckpt((n + 1 + interval - 1) / interval);
    } else if (n + 1 > last0) {
      nxt = seg(n + 1 - last0);
    } else {
      nxt = seg(n % 2);
      kept = false;
    }
    if ((err = step(cur, nxt, kept)) != cudaSuccess) return err;
    cur = nxt;
  }

  // seed lambda^N and J
  const Adj& lN = lam[steps % 2];
  if (objective == LBM_OBJECTIVE_SEGREGATION) {
    const Real* fa = reinterpret_cast<const Real*>(cur.a);
    const Real* fb = reinterpret_cast<const Real*>(cur.b);
    if constexpr (!NATIVE) {  // statistics of the decoded final fields (other adjoint buffer)
      const Adj& tmp = lam[(steps + 1) % 2];
      const int r1 = lbm_decode_shifted_async(SL::id, api_format, LBM_FLOAT, cur.a, tmp.a, g.nx,
                                              g.ny, g.nz, c0, s);
      const int r2 = lbm_decode_shifted_async(SL::id, api_format, LBM_FLOAT, cur.b, tmp.b, g.nx,
                                              g.ny, g.nz, c0, s);
      if (r1 != 0 || r2 != 0) return (cudaError_t)(r1 ? r1 : r2);
      fa = tmp.a;
      fb = tmp.b;
    }
    err = (cudaError_t)lbm_reactive_stats_async(SL::id, prec, fa, fb, g.nx, g.ny, g.nz, k, partials,
                                                (size_t)lay.blocks * kStatSums * sizeof(double),
                                                stats, s);
    if (err != cudaSuccess) return err;
    reactive_seed_kernel<FL, Real, LBM_OBJECTIVE_SEGREGATION, SP>
        <<<grid_dims(g), block_dims(g), 0, s>>>(cur.a, cur.b, a0, stats, lN.f, lN.a, lN.b, g, c0,
                                                1.0 / (double)g.plane, j_slots);
  } else {
    reactive_seed_kernel<FL, Real, LBM_OBJECTIVE_MEAN_PRODUCT, SP>
        <<<grid_dims(g), block_dims(g), 0, s>>>(cur.a, cur.b, a0, stats, lN.f, lN.a, lN.b, g, c0,
                                                1.0 / (double)g.plane, j_slots);
  }
  if ((err = cudaGetLastError()) != cudaSuccess) return err;
  if ((err = cudaMemsetAsync(slots, 0,
                             (size_t)lay.blocks * kWarpsPerBlock * kReactiveSlots * sizeof(double),
                             s)) != cudaSuccess)
    return err;

  ReactiveParams rp{};
  rp.fluid = make_params<Real>(collision, tau);
  rp.omega_c = omega_c;
  rp.k = (double)Real(k);
  rp.rho0 = 1.0f;
  rp.c0 = c0;
  for (long long kk = nseg - 1; kk >= 0; --kk) {
    const int n0 = (int)(kk * interval);
    const int n1 = (int)std::min<long long>((long long)steps, (kk + 1) * interval);
    State src = ckpt(kk);
    for (int n = n0 + 1; n < n1 && kk < nseg - 1; ++n) {
      if ((err = step(src, seg(n - n0), true)) != cudaSuccess) return err;
      src = seg(n - n0);
    }
    for (int n = n1 - 1; n >= n0; --n) {
      const State sn = n == n0 ? ckpt(kk) : seg(n - n0);
      const State sn1 = n + 1 == n1 ? ckpt(kk + 1) : seg(n + 1 - n0);  // holds u^{n+1}
      const Adj& ln = lam[(n + 1) % 2];
      const Adj& l = lam[n % 2];
      err = launch_reactive_adjoint<FL, Real, SP>(collision, sn.f, sn.a, sn.b, sn1.u, ln.f, ln.a,
                                                  ln.b, l.f, l.a, l.b, ubar, g, rp, slots, s);
      if (err != cudaSuccess) return err;
    }
  }

  // results: J, dJ/dk, dJ/dtau, dJ/dtau_c; dJ/dA0 (and dJ/dB0, dJ/du0). For
  // 16-bit states the encoding of the initial state counts as the identity.
  const Real direct_a = objective == LBM_OBJECTIVE_MEAN_PRODUCT ? Real(1.0 / (double)g.plane) : Real(0);
  scalar_init_gradient_kernel<FL, Real><<<grid_dims(g), block_dims(g), 0, s>>>(u0, lam[0].a, direct_a,
                                                                          grad_a0, g);
  if (grad_b0 != nullptr)
    scalar_init_gradient_kernel<FL, Real><<<grid_dims(g), block_dims(g), 0, s>>>(u0, lam[0].b, Real(0),
                                                                            grad_b0, g);
  if (grad_u0 != nullptr)
    reactive_velocity_gradient_kernel<FL, Real><<<grid_dims(g), block_dims(g), 0, s>>>(
        rho0, u0, a0, b0, lam[0].f, lam[0].a, lam[0].b, grad_u0, g);
  if (objective == LBM_OBJECTIVE_SEGREGATION) {
    if ((err = cudaMemcpyAsync(out, stats + 5, sizeof(double), cudaMemcpyDeviceToDevice, s)) !=
        cudaSuccess)
      return err;
  } else {
    sum_slots_kernel<<<1, 1024, 0, s>>>(j_slots, lay.blocks, 1, 1.0 / (double)g.plane, out);
  }
  const long long nslots = lay.blocks * kWarpsPerBlock;
  sum_slots_kernel<<<1, 1024, 0, s>>>(slots + 0, nslots, kReactiveSlots, 1.0, out + 1);
  sum_slots_kernel<<<1, 1024, 0, s>>>(slots + 1, nslots, kReactiveSlots, 1.0, out + 2);
  sum_slots_kernel<<<1, 1024, 0, s>>>(slots + 2, nslots, kReactiveSlots, -omega_c * omega_c,
                                      out + 3);
  return cudaGetLastError();
}

inline int scalar_q(int fluid_lattice) { return fluid_lattice == kD2Q9 ? 5 : 7; }
inline int fluid_q(int fluid_lattice) {
  return fluid_lattice == kD2Q9 ? 9 : (fluid_lattice == kD3Q19 ? 19 : 27);
}

// storage: LBM_NATIVE (states in Real) or a 16-bit format (Real float).
inline int storage_fmt(int storage) {
  return storage == LBM_F16S ? kF16S : storage == LBM_BF16S ? kBF16S
       : storage == LBM_E3M12S ? kE3M12S : storage == LBM_Q15S ? kQ15S : -1;
}

template <class Real>
cudaError_t reactive_dispatch(int lattice, int storage, float c0, int collision, int objective,
                              const void* rho0, const void* u0, const void* a0, const void* b0,
                              size_t nx, size_t ny, size_t nz, double tau, double tau_c, double k,
                              int steps, int interval, void* ws, size_t ws_bytes, double* out,
                              void* grad_a0, void* grad_b0, void* grad_u0, cudaStream_t s) {
  Grid g;
  const int dims = lattice == kD2Q9 ? 2 : 3;
  cudaError_t err = validate_domain(rho0 == nullptr || u0 == nullptr || a0 == nullptr ||
                                        b0 == nullptr || ws == nullptr || out == nullptr ||
                                        grad_a0 == nullptr,
                                    1, 1, 1, dims, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  if (lattice != kD2Q9 && lattice != kD3Q19 && lattice != kD3Q27) return cudaErrorInvalidValue;
  const bool mrt_ok = collision == kMRT && lattice != kD3Q27;
  if (steps < 1 || interval < 2 || (collision != kBGK && collision != kTRT && !mrt_ok) ||
      (objective != LBM_OBJECTIVE_MEAN_PRODUCT && objective != LBM_OBJECTIVE_SEGREGATION) ||
      !(tau > 0.5) || !(tau_c > 0.5))
    return cudaErrorInvalidValue;
  const int fmt = storage_fmt(storage);
  if (storage != LBM_NATIVE && (fmt < 0 || sizeof(Real) != 4)) return cudaErrorInvalidValue;
  const ReactiveLayout lay = reactive_layout(fluid_q(lattice), scalar_q(lattice), dims,
                                             fmt < 0 ? sizeof(Real) : 2, sizeof(Real), g, steps,
                                             interval);
  if (ws_bytes < lay.total) return cudaErrorInvalidValue;
  char* w = static_cast<char*>(ws);
#define LBCUBE_REACTIVE(FL, F)                                                                     \
  return reactive_gradient<FL, Real, F>(collision, objective, (const Real*)rho0, (const Real*)u0,  \
                                        (const Real*)a0, (const Real*)b0, g, tau, tau_c, k, c0,    \
                                        steps, interval, w, lay, out, (Real*)grad_a0,              \
                                        (Real*)grad_b0, (Real*)grad_u0, s)
#define LBCUBE_REACTIVE_FMT(FL)                                                                    \
  if (fmt < 0) LBCUBE_REACTIVE(FL, -1);                                                            \
  if constexpr (sizeof(Real) == 4) {                                                               \
    if (fmt == kF16S) LBCUBE_REACTIVE(FL, kF16S);                                                  \
    if (fmt == kBF16S) LBCUBE_REACTIVE(FL, kBF16S);                                                \
    if (fmt == kE3M12S) LBCUBE_REACTIVE(FL, kE3M12S);                                              \
    if (fmt == kQ15S) LBCUBE_REACTIVE(FL, kQ15S);                                                  \
  }                                                                                                \
  return cudaErrorInvalidValue;
  switch (lattice) {
    case kD2Q9: { LBCUBE_REACTIVE_FMT(D2Q9) }
    case kD3Q19: { LBCUBE_REACTIVE_FMT(D3Q19) }
    default: { LBCUBE_REACTIVE_FMT(D3Q27) }
  }
#undef LBCUBE_REACTIVE_FMT
#undef LBCUBE_REACTIVE
}

// ---- z-slab form -------------------------------------------------------------
// The same gradient over a box cut along z into slabs, one per rank
// (slab_faces.cuh for the face layout). The host sequence of reactive_gradient
// runs on every rank with its own slab; the per-step pieces are entries of
// their own because a face exchange or an all-reduce sits between them:
//   forward step   lbm_reactive_slab_forward_async (the coupled slab step,
//                  storing the advecting velocity), then a face exchange;
//   adjoint step   pack of the stored state's faces + exchange (the pulled
//                  halos), lbm_reactive_slab_adjoint_step_async (the two
//                  kernels above with slab pulls and scatters), exchange of the
//                  scatter sends, lbm_reactive_slab_adjoint_unpack_async;
//   seed / end     lbm_reactive_slab_seed_async, ..._init_gradients_async,
//                  the rank's FP64 sums (..._sums_async), an all-reduce of
//                  those four doubles, lbm_reactive_slab_result_async.
// Every cell does the whole box's arithmetic on the same inputs, so the
// adjoint fields and initial-state gradients of a slab are bit-identical to
// the whole box's (given the same seed); the four scalars differ only in the
// order of the FP64 sums.

// The neighbours' scatter sends into the slab's lambda^n (slab_faces.cuh).
template <class FL, class Real>
__global__ void __launch_bounds__(256)
    reactive_slab_unpack_kernel(const Real* __restrict__ recv_lo, const Real* __restrict__ recv_hi,
                                Real* __restrict__ lf, Real* __restrict__ la, Real* __restrict__ lb,
                                Grid g) {
  using SL = typename ScalarOf<FL>::type;
  const size_t n2 = (size_t)g.ny * g.nx;
  const size_t a_off = (size_t)face_planes<FL>() * n2;
  const size_t b_off = a_off + (size_t)face_planes<SL>() * n2;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < (long long)(2 * n2);
       e += (long long)gridDim.x * blockDim.x) {
    const int side = e < (long long)n2 ? 0 : 1;
    const size_t row = (size_t)(side == 0 ? e : e - (long long)n2);
    unscatter_slab<FL>(lf, g, side, row, recv_lo, recv_hi);
    unscatter_slab<SL>(la, g, side, row, recv_lo + a_off, recv_hi + a_off);
    unscatter_slab<SL>(lb, g, side, row, recv_lo + b_off, recv_hi + b_off);
  }
}

// J, dJ/dk, dJ/dtau, dJ/dtau_c from the all-reduced sums (objective partials,
// slots 0..2): the scaling of reactive_gradient's last four reductions.
static __global__ void reactive_slab_result_kernel(const double* __restrict__ sums,
                                                   const double* __restrict__ stats, int objective,
                                                   double inv_n, double omega_c,
                                                   double* __restrict__ out) {
  out[0] = objective == LBM_OBJECTIVE_SEGREGATION ? stats[5] : sums[0] * inv_n;
  out[1] = sums[1];
  out[2] = sums[2];
  out[3] = sums[3] * (-omega_c * omega_c);
}

// Checks shared by the slab entries; fills g (a 3-D slab of a D3Q19 / D3Q27
// fluid lattice).
inline cudaError_t slab_domain(int fluid_lattice, int precision, bool any_null, size_t nx,
                               size_t ny, size_t nz, Grid& g) {
  if (fluid_lattice != kD3Q19 && fluid_lattice != kD3Q27) return cudaErrorInvalidValue;
  if (precision != LBM_FLOAT && precision != LBM_DOUBLE) return cudaErrorInvalidValue;
  return validate_domain(any_null, 1, 1, 1, 3, nx, ny, nz, g);
}

inline bool slab_collision_ok(int fluid_lattice, int collision) {
  return collision == kBGK || collision == kTRT || (collision == kMRT && fluid_lattice != kD3Q27);
}

inline size_t slab_slots_bytes(const Grid& g) {
  return (size_t)g.blocks() * kWarpsPerBlock * kReactiveSlots * sizeof(double);
}

// One adjoint step on a slab; SP: the stored states' policy (NativeState<Real>
// or ShiftedState<FMT> with Real float).
template <class FL, class Real, class SP>
cudaError_t slab_adjoint_step(int collision, const typename SP::elem* fn,
                              const typename SP::elem* an, const typename SP::elem* bn,
                              const typename SP::elem* halo_lo, const typename SP::elem* halo_hi,
                              const Real* u_next, const Real* lf_next, const Real* la_next,
                              const Real* lb_next, Real* lf, Real* la, Real* lb, Real* ubar,
                              Real* send_lo, Real* send_hi, const Grid& g, double tau, double tau_c,
                              double k, float c0, double* slots, cudaStream_t s) {
  using SL = typename ScalarOf<FL>::type;
  using E = typename SP::elem;
  const size_t fe = (size_t)FL::Q * g.plane, se = (size_t)SL::Q * g.plane;
  const size_t ub = (size_t)FL::D * g.plane * sizeof(Real);
  const size_t he = (size_t)coupled_face_planes<FL>() * g.ny * g.nx;
  const Span reads[9] = {{fn, fe * sizeof(E)},      {an, se * sizeof(E)},
                         {bn, se * sizeof(E)},      {halo_lo, he * sizeof(E)},
                         {halo_hi, he * sizeof(E)}, {u_next, ub},
                         {lf_next, fe * sizeof(Real)}, {la_next, se * sizeof(Real)},
                         {lb_next, se * sizeof(Real)}};
  const Span writes[7] = {{lf, fe * sizeof(Real)},      {la, se * sizeof(Real)},
                          {lb, se * sizeof(Real)},      {ubar, ub},
                          {send_lo, he * sizeof(Real)}, {send_hi, he * sizeof(Real)},
                          {slots, slab_slots_bytes(g)}};
  if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  ReactiveParams rp{};
  rp.fluid = make_params<Real>(collision, tau);
  rp.omega_c = (double)(Real(1) / Real(tau_c));
  rp.k = (double)Real(k);
  rp.rho0 = 1.0f;
  rp.c0 = c0;
  if (collision != kBGK && collision != kTRT && (collision != kMRT || FL::Q == 27))
    return cudaErrorInvalidValue;
  const SlabFaces<E, Real> faces{halo_lo, halo_hi, send_lo, send_hi};
  // Planes 1 .. nz-2 pull and scatter only inside the slab: the whole-box
  // kernels (fewer registers than the SLAB forms); planes 0 and nz-1 the SLAB
  // forms. Every reaction launch precedes the fluid launches (they read its
  // ubar); slots are indexed by absolute plane.
  auto ranges = [&](auto each) {
    if (g.nz >= 3) each(1, g.nz - 2, 1, std::false_type{});
    each(0, g.nz >= 2 ? 2 : 1, g.nz - 1, std::true_type{});  // both face planes in one launch
  };
  ranges([&](int z0, int planes, int zs, auto slab) {
    constexpr bool SLAB = decltype(slab)::value;
    Grid gr = g;
    gr.z0 = z0;
    gr.zs = zs;
    dim3 grid = grid_dims(gr);
    grid.y = (unsigned)planes;
    launch_pdl(reaction_adjoint_kernel<FL, Real, SP, SLAB>, grid, dim3(block_dims(gr)), 0, s, an, bn,
               u_next, la_next, lb_next, la, lb, ubar, gr, rp, slots, faces);
  });
  ranges([&](int z0, int planes, int zs, auto slab) {
    constexpr bool SLAB = decltype(slab)::value;
    Grid gr = g;
    gr.z0 = z0;
    gr.zs = zs;
    dim3 grid = grid_dims(gr);
    grid.y = (unsigned)planes;
    const dim3 block(block_dims(gr));
    if (collision == kBGK)
      launch_pdl(coupled_fluid_adjoint_kernel<FL, Real, kBGK, SP, SLAB>, grid, block, 0, s, fn, lf_next,
                 ubar, lf, gr, rp.fluid, rp.rho0, slots, faces);
    else if (collision == kTRT)
      launch_pdl(coupled_fluid_adjoint_kernel<FL, Real, kTRT, SP, SLAB>, grid, block, 0, s, fn, lf_next,
                 ubar, lf, gr, rp.fluid, rp.rho0, slots, faces);
    else if constexpr (FL::Q != 27)
      launch_pdl(coupled_fluid_adjoint_kernel<FL, Real, kMRT, SP, SLAB>, grid, block, 0, s, fn, lf_next,
                 ubar, lf, gr, rp.fluid, rp.rho0, slots, faces);
  });
  return cudaGetLastError();
}

// Calls fn(FL{}, Real{}, std::integral_constant<int, FMT>{}) for a slab's
// fluid lattice, precision and storage (FMT -1: states in Real; a 16-bit
// format needs Real float).
template <class F>
int slab_dispatch(int fluid_lattice, int precision, int storage, F&& fn) {
  const int fmt = storage_fmt(storage);
  if (storage != LBM_NATIVE && (fmt < 0 || precision != LBM_FLOAT)) return (int)cudaErrorInvalidValue;
  auto by_format = [&](auto fl, auto r) -> int {
    if (fmt < 0) return fn(fl, r, std::integral_constant<int, -1>{});
    if constexpr (std::is_same_v<decltype(r), float>) {
      if (fmt == kF16S) return fn(fl, r, std::integral_constant<int, kF16S>{});
      if (fmt == kBF16S) return fn(fl, r, std::integral_constant<int, kBF16S>{});
      if (fmt == kE3M12S) return fn(fl, r, std::integral_constant<int, kE3M12S>{});
      if (fmt == kQ15S) return fn(fl, r, std::integral_constant<int, kQ15S>{});
    }
    return (int)cudaErrorInvalidValue;
  };
  if (fluid_lattice == kD3Q19 && precision == LBM_FLOAT) return by_format(D3Q19{}, 0.0f);
  if (fluid_lattice == kD3Q19 && precision == LBM_DOUBLE) return by_format(D3Q19{}, 0.0);
  if (fluid_lattice == kD3Q27 && precision == LBM_FLOAT) return by_format(D3Q27{}, 0.0f);
  if (fluid_lattice == kD3Q27 && precision == LBM_DOUBLE) return by_format(D3Q27{}, 0.0);
  return (int)cudaErrorInvalidValue;
}

template <class Real, int FMT>
using SlabState = std::conditional_t<(FMT < 0), NativeState<Real>, ShiftedState<(FMT < 0 ? 0 : FMT)>>;

}  // namespace lbcube

using namespace lbcube;

extern "C" size_t lbm_reactive_gradient_workspace_bytes(int fluid_lattice, int precision,
                                                        int storage, size_t x_extent,
                                                        size_t y_extent, size_t z_extent,
                                                        int steps, int checkpoint_interval) {
  Grid g;
  if (fluid_lattice != LBM_D2Q9 && fluid_lattice != LBM_D3Q19 && fluid_lattice != LBM_D3Q27)
    return 0;
  const int dims = fluid_lattice == LBM_D2Q9 ? 2 : 3;
  if (validate_domain(false, 1, 1, 1, dims, x_extent, y_extent, z_extent, g) != cudaSuccess)
    return 0;
  if (steps < 1 || checkpoint_interval < 2) return 0;
  if (precision != LBM_FLOAT && precision != LBM_DOUBLE) return 0;
  const int fmt = storage_fmt(storage);
  if (storage != LBM_NATIVE && (fmt < 0 || precision != LBM_FLOAT)) return 0;
  const size_t real = precision == LBM_DOUBLE ? 8 : 4;
  return reactive_layout(fluid_q(fluid_lattice), scalar_q(fluid_lattice), dims,
                         fmt < 0 ? real : 2, real, g, steps, checkpoint_interval)
      .total;
}

extern "C" int lbm_reactive_gradient_async(int fluid_lattice, int precision, int storage,
                                           float c0, int collision, int objective,
                                           const void* rho0, const void* u0, const void* a0,
                                           const void* b0, size_t x_extent, size_t y_extent,
                                           size_t z_extent, double tau, double tau_c,
                                           double k_react, int steps, int checkpoint_interval,
                                           void* workspace, size_t workspace_bytes,
                                           double* result, void* grad_a0, void* grad_b0,
                                           void* grad_u0, void* stream) {
  const cudaStream_t s = as_stream(stream);
  if (precision == LBM_FLOAT)
    return (int)reactive_dispatch<float>(fluid_lattice, storage, c0, collision, objective, rho0,
                                         u0, a0, b0, x_extent, y_extent, z_extent, tau, tau_c,
                                         k_react, steps, checkpoint_interval, workspace,
                                         workspace_bytes, result, grad_a0, grad_b0, grad_u0, s);
  if (precision == LBM_DOUBLE)
    return (int)reactive_dispatch<double>(fluid_lattice, storage, c0, collision, objective, rho0,
                                          u0, a0, b0, x_extent, y_extent, z_extent, tau, tau_c,
                                          k_react, steps, checkpoint_interval, workspace,
                                          workspace_bytes, result, grad_a0, grad_b0, grad_u0, s);
  return (int)cudaErrorInvalidValue;
}

// ---- z-slab entries -----------------------------------------------------------

extern "C" size_t lbm_reactive_slab_slots_bytes(int fluid_lattice, size_t x_extent,
                                                size_t y_extent, size_t z_extent) {
  Grid g;
  if (slab_domain(fluid_lattice, LBM_DOUBLE, false, x_extent, y_extent, z_extent, g) != cudaSuccess)
    return 0;
  return slab_slots_bytes(g);
}

extern "C" size_t lbm_reactive_slab_objective_bytes(int fluid_lattice, size_t x_extent,
                                                    size_t y_extent, size_t z_extent) {
  Grid g;
  if (slab_domain(fluid_lattice, LBM_DOUBLE, false, x_extent, y_extent, z_extent, g) != cudaSuccess)
    return 0;
  return (size_t)g.blocks() * sizeof(double);
}

extern "C" int lbm_reactive_slab_forward_async(
    int fluid_lattice, int precision, int storage, float c0, int collision,
    const void* current_fluid, void* next_fluid, const void* current_a, void* next_a,
    const void* current_b, void* next_b, void* velocity, size_t x_extent, size_t y_extent,
    size_t z_extent, double tau, double tau_c, double k_react, const void* halo_lo,
    const void* halo_hi, void* send_lo, void* send_hi, void* stream) {
  Grid g;
  cudaError_t err = slab_domain(fluid_lattice, precision,
                                current_fluid == nullptr || next_fluid == nullptr ||
                                    current_a == nullptr || next_a == nullptr ||
                                    current_b == nullptr || next_b == nullptr ||
                                    halo_lo == nullptr || halo_hi == nullptr ||
                                    send_lo == nullptr || send_hi == nullptr,
                                x_extent, y_extent, z_extent, g);
  if (err != cudaSuccess) return (int)err;
  if (!slab_collision_ok(fluid_lattice, collision) || !(tau > 0.5) || !(tau_c > 0.5))
    return (int)cudaErrorInvalidValue;
  const cudaStream_t s = as_stream(stream);
  return slab_dispatch(fluid_lattice, precision, storage, [&](auto fl, auto r, auto f) -> int {
    using FL = decltype(fl);
    using R = decltype(r);
    constexpr int FMT = decltype(f)::value;
    using E = typename SlabState<R, FMT>::elem;
    const size_t fe = FL::Q * (size_t)g.plane, se = 7 * (size_t)g.plane;
    const size_t ub = 3 * (size_t)g.plane * sizeof(R);
    const size_t hb = lbm_fluid_reaction_slab_face_elems(fluid_lattice, x_extent, y_extent) * sizeof(E);
    const Span reads[5] = {{current_fluid, fe * sizeof(E)}, {current_a, se * sizeof(E)},
                           {current_b, se * sizeof(E)},     {halo_lo, hb},
                           {halo_hi, hb}};
    const Span writes[6] = {{next_fluid, fe * sizeof(E)}, {next_a, se * sizeof(E)},
                            {next_b, se * sizeof(E)},     {send_lo, hb},
                            {send_hi, hb},                {velocity, velocity ? ub : 0}};
    if (any_overlap(reads, writes)) return (int)cudaErrorInvalidValue;
    // the relaxation rates as the whole-box gradient forms them
    if constexpr (FMT < 0) {
      return (int)fluid_reaction_slab_with_velocity<FL, R>(
          collision, (const R*)current_fluid, (R*)next_fluid, (const R*)current_a, (R*)next_a,
          (const R*)current_b, (R*)next_b, (R*)velocity, g, R(1) / R(tau), R(1) / R(tau_c),
          R(k_react), (const R*)halo_lo, (const R*)halo_hi, (R*)send_lo, (R*)send_hi, s);
    } else {
      return (int)fluid_reaction_shifted_slab<FL, FMT>(
          collision, (const E*)current_fluid, (E*)next_fluid, (const E*)current_a, (E*)next_a,
          (const E*)current_b, (E*)next_b, (float*)velocity, g, 1.0f / (float)tau,
          1.0f / (float)tau_c, (float)k_react, 1.0f, c0, (const E*)halo_lo, (const E*)halo_hi,
          (E*)send_lo, (E*)send_hi, s);
    }
  });
}

extern "C" int lbm_reactive_slab_adjoint_step_async(
    int fluid_lattice, int precision, int storage, float c0, int collision, const void* fluid_n,
    const void* a_n, const void* b_n, const void* halo_lo, const void* halo_hi,
    const void* velocity_next, const void* lambda_fluid_next, const void* lambda_a_next,
    const void* lambda_b_next, void* lambda_fluid, void* lambda_a, void* lambda_b,
    void* velocity_adjoint, void* send_lo, void* send_hi, size_t x_extent, size_t y_extent,
    size_t z_extent, double tau, double tau_c, double k_react, double* slots, size_t slots_bytes,
    void* stream) {
  Grid g;
  cudaError_t err = slab_domain(
      fluid_lattice, precision,
      fluid_n == nullptr || a_n == nullptr || b_n == nullptr || halo_lo == nullptr ||
          halo_hi == nullptr || velocity_next == nullptr || lambda_fluid_next == nullptr ||
          lambda_a_next == nullptr || lambda_b_next == nullptr || lambda_fluid == nullptr ||
          lambda_a == nullptr || lambda_b == nullptr || velocity_adjoint == nullptr ||
          send_lo == nullptr || send_hi == nullptr || slots == nullptr,
      x_extent, y_extent, z_extent, g);
  if (err != cudaSuccess) return (int)err;
  if (!slab_collision_ok(fluid_lattice, collision) || !(tau > 0.5) || !(tau_c > 0.5) ||
      slots_bytes < slab_slots_bytes(g))
    return (int)cudaErrorInvalidValue;
  const cudaStream_t s = as_stream(stream);
  return slab_dispatch(fluid_lattice, precision, storage, [&](auto fl, auto r, auto f) -> int {
    using FL = decltype(fl);
    using R = decltype(r);
    using SP = SlabState<R, decltype(f)::value>;
    using E = typename SP::elem;
    return (int)slab_adjoint_step<FL, R, SP>(
        collision, (const E*)fluid_n, (const E*)a_n, (const E*)b_n, (const E*)halo_lo,
        (const E*)halo_hi, (const R*)velocity_next, (const R*)lambda_fluid_next,
        (const R*)lambda_a_next, (const R*)lambda_b_next, (R*)lambda_fluid, (R*)lambda_a,
        (R*)lambda_b, (R*)velocity_adjoint, (R*)send_lo, (R*)send_hi, g, tau, tau_c, k_react, c0,
        slots, s);
  });
}

extern "C" int lbm_reactive_slab_adjoint_unpack_async(int fluid_lattice, int precision,
                                                      const void* recv_lo, const void* recv_hi,
                                                      void* lambda_fluid, void* lambda_a,
                                                      void* lambda_b, size_t x_extent,
                                                      size_t y_extent, size_t z_extent,
                                                      void* stream) {
  Grid g;
  cudaError_t err = slab_domain(fluid_lattice, precision,
                                recv_lo == nullptr || recv_hi == nullptr ||
                                    lambda_fluid == nullptr || lambda_a == nullptr ||
                                    lambda_b == nullptr,
                                x_extent, y_extent, z_extent, g);
  if (err != cudaSuccess) return (int)err;
  const size_t real = precision == LBM_DOUBLE ? 8 : 4;
  const size_t fq = fluid_lattice == kD3Q19 ? 19 : 27;
  const size_t hb = lbm_fluid_reaction_slab_face_elems(fluid_lattice, x_extent, y_extent) * real;
  const Span reads[2] = {{recv_lo, hb}, {recv_hi, hb}};
  const Span writes[3] = {{lambda_fluid, fq * g.plane * real},
                          {lambda_a, 7 * g.plane * real},
                          {lambda_b, 7 * g.plane * real}};
  if (any_overlap(reads, writes)) return (int)cudaErrorInvalidValue;
  const cudaStream_t s = as_stream(stream);
  const long long total = 2LL * g.ny * g.nx;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  return slab_dispatch(fluid_lattice, precision, LBM_NATIVE, [&](auto fl, auto r, auto) -> int {
    using FL = decltype(fl);
    using R = decltype(r);
    reactive_slab_unpack_kernel<FL, R><<<blocks, 256, 0, s>>>(
        (const R*)recv_lo, (const R*)recv_hi, (R*)lambda_fluid, (R*)lambda_a, (R*)lambda_b, g);
    return (int)cudaGetLastError();
  });
}

extern "C" int lbm_reactive_slab_seed_async(int fluid_lattice, int precision, int storage,
                                            float c0, int objective, const void* a_final,
                                            const void* b_final, const void* a0,
                                            const double* diagnostics, void* lambda_fluid,
                                            void* lambda_a, void* lambda_b, size_t x_extent,
                                            size_t y_extent, size_t z_extent, double total_cells,
                                            double* objective_partials, size_t partials_bytes,
                                            void* stream) {
  Grid g;
  cudaError_t err = slab_domain(
      fluid_lattice, precision,
      a_final == nullptr || b_final == nullptr || a0 == nullptr || lambda_fluid == nullptr ||
          lambda_a == nullptr || lambda_b == nullptr || objective_partials == nullptr ||
          (objective == LBM_OBJECTIVE_SEGREGATION && diagnostics == nullptr),
      x_extent, y_extent, z_extent, g);
  if (err != cudaSuccess) return (int)err;
  if ((objective != LBM_OBJECTIVE_MEAN_PRODUCT && objective != LBM_OBJECTIVE_SEGREGATION) ||
      !(total_cells >= (double)g.plane) || partials_bytes < (size_t)g.blocks() * sizeof(double))
    return (int)cudaErrorInvalidValue;
  const cudaStream_t s = as_stream(stream);
  const double inv_n = 1.0 / total_cells;
  return slab_dispatch(fluid_lattice, precision, storage, [&](auto fl, auto r, auto f) -> int {
    using FL = decltype(fl);
    using R = decltype(r);
    using SP = SlabState<R, decltype(f)::value>;
    using E = typename SP::elem;
    if (objective == LBM_OBJECTIVE_SEGREGATION)
      reactive_seed_kernel<FL, R, LBM_OBJECTIVE_SEGREGATION, SP><<<grid_dims(g), block_dims(g), 0, s>>>(
          (const E*)a_final, (const E*)b_final, (const R*)a0, diagnostics, (R*)lambda_fluid,
          (R*)lambda_a, (R*)lambda_b, g, c0, inv_n, objective_partials);
    else
      reactive_seed_kernel<FL, R, LBM_OBJECTIVE_MEAN_PRODUCT, SP><<<grid_dims(g), block_dims(g), 0, s>>>(
          (const E*)a_final, (const E*)b_final, (const R*)a0, diagnostics, (R*)lambda_fluid,
          (R*)lambda_a, (R*)lambda_b, g, c0, inv_n, objective_partials);
    return (int)cudaGetLastError();
  });
}

extern "C" int lbm_reactive_slab_init_gradients_async(
    int fluid_lattice, int precision, int objective, const void* rho0, const void* u0,
    const void* a0, const void* b0, const void* lambda_fluid, const void* lambda_a,
    const void* lambda_b, size_t x_extent, size_t y_extent, size_t z_extent, double total_cells,
    void* grad_a0, void* grad_b0, void* grad_u0, void* stream) {
  Grid g;
  cudaError_t err = slab_domain(fluid_lattice, precision,
                                u0 == nullptr || lambda_a == nullptr || grad_a0 == nullptr ||
                                    (grad_b0 != nullptr && lambda_b == nullptr) ||
                                    (grad_u0 != nullptr &&
                                     (rho0 == nullptr || a0 == nullptr || b0 == nullptr ||
                                      lambda_fluid == nullptr || lambda_b == nullptr)),
                                x_extent, y_extent, z_extent, g);
  if (err != cudaSuccess) return (int)err;
  if ((objective != LBM_OBJECTIVE_MEAN_PRODUCT && objective != LBM_OBJECTIVE_SEGREGATION) ||
      !(total_cells >= (double)g.plane))
    return (int)cudaErrorInvalidValue;
  const cudaStream_t s = as_stream(stream);
  return slab_dispatch(fluid_lattice, precision, LBM_NATIVE, [&](auto fl, auto r, auto) -> int {
    using FL = decltype(fl);
    using R = decltype(r);
    const R direct = objective == LBM_OBJECTIVE_MEAN_PRODUCT ? R(1.0 / total_cells) : R(0);
    scalar_init_gradient_kernel<FL, R><<<grid_dims(g), block_dims(g), 0, s>>>(
        (const R*)u0, (const R*)lambda_a, direct, (R*)grad_a0, g);
    if (grad_b0 != nullptr)
      scalar_init_gradient_kernel<FL, R><<<grid_dims(g), block_dims(g), 0, s>>>(
          (const R*)u0, (const R*)lambda_b, R(0), (R*)grad_b0, g);
    if (grad_u0 != nullptr)
      reactive_velocity_gradient_kernel<FL, R><<<grid_dims(g), block_dims(g), 0, s>>>(
          (const R*)rho0, (const R*)u0, (const R*)a0, (const R*)b0, (const R*)lambda_fluid,
          (const R*)lambda_a, (const R*)lambda_b, (R*)grad_u0, g);
    return (int)cudaGetLastError();
  });
}

extern "C" int lbm_reactive_slab_sums_async(int fluid_lattice, size_t x_extent, size_t y_extent,
                                            size_t z_extent, const double* slots,
                                            size_t slots_bytes, const double* objective_partials,
                                            size_t partials_bytes, double* sums, void* stream) {
  Grid g;
  cudaError_t err = slab_domain(fluid_lattice, LBM_DOUBLE,
                                slots == nullptr || objective_partials == nullptr || sums == nullptr,
                                x_extent, y_extent, z_extent, g);
  if (err != cudaSuccess) return (int)err;
  if (slots_bytes < slab_slots_bytes(g) || partials_bytes < (size_t)g.blocks() * sizeof(double))
    return (int)cudaErrorInvalidValue;
  const cudaStream_t s = as_stream(stream);
  const long long nslots = g.blocks() * kWarpsPerBlock;
  sum_slots_kernel<<<1, 1024, 0, s>>>(objective_partials, g.blocks(), 1, 1.0, sums);
  for (int k = 0; k < kReactiveSlots; ++k)
    sum_slots_kernel<<<1, 1024, 0, s>>>(slots + k, nslots, kReactiveSlots, 1.0, sums + 1 + k);
  return (int)cudaGetLastError();
}

extern "C" int lbm_reactive_slab_result_async(int precision, int objective, const double* sums,
                                              const double* diagnostics, double total_cells,
                                              double tau_c, double* result, void* stream) {
  if (sums == nullptr || result == nullptr ||
      (objective == LBM_OBJECTIVE_SEGREGATION && diagnostics == nullptr))
    return (int)cudaErrorInvalidDevicePointer;
  if ((precision != LBM_FLOAT && precision != LBM_DOUBLE) ||
      (objective != LBM_OBJECTIVE_MEAN_PRODUCT && objective != LBM_OBJECTIVE_SEGREGATION) ||
      !(total_cells >= 1.0) || !(tau_c > 0.5))
    return (int)cudaErrorInvalidValue;
  const double omega_c = precision == LBM_FLOAT ? (double)(1.0f / (float)tau_c) : 1.0 / tau_c;
  reactive_slab_result_kernel<<<1, 1, 0, as_stream(stream)>>>(sums, diagnostics, objective,
                                                              1.0 / total_cells, omega_c, result);
  return (int)cudaGetLastError();
}

