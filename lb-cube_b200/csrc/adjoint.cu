// Discrete reverse-mode adjoint of the collide-stream step (BGK, TRT; MRT on
// D2Q9 and D3Q19) and the checkpointed gradient of the final kinetic energy.
// No reference counterpart.
//
// adjoint_step_kernel applies the transposed step Jacobian of adjoint.cuh at
// every cell and scatters to the pull sources. The tau-derivative of the step,
// sum_x lambda^{n+1} . dC/dtau, is accumulated per block in FP64 into slots
// the block owns (deterministic over steps).
#include <algorithm>
#include <climits>

#include "adjoint.cuh"
#include "cells.cuh"
#include "collide.cuh"
#include "common.cuh"
#include "reduce.cuh"
#include "../../include/lbcube_b200.h"

namespace lbcube {

template <class L, class Real, int CT>
__global__ void __launch_bounds__(kThreads, kAdjointBlocks<Real>)
    adjoint_step_kernel(const Real* __restrict__ fn, const Real* __restrict__ lam_next,
                        Real* __restrict__ lam, Grid g, AdjointParams ap,
                        double* __restrict__ dtau_slots) {
  pdl_enter();
  int x, y, z;
  const bool active = cell_of(g, x, y, z);
  double dtau = 0.0;
  if (active) {
    const Neighbours n = neighbours(g, x, y, z);
    const int cell = (z * g.ny + y) * g.nx + x;
    Real gv[L::Q], lv[L::Q], mu[L::Q];
    gather<L>(fn, g, n, x, y, z, gv);  // pulled pre-collision state, as in the forward step
    load_cell<L>(lam_next, g, cell, lv);
    Real rho, u[L::D];
    macro_state<L>(gv, rho, u);
    dtau = fluid_adjoint_cell<L, Real, CT>(gv, lv, rho, u, ap, mu);
    scatter<L>(lam, g, n, x, y, z, mu);
  }
  if (dtau_slots != nullptr) {
    double v[1] = {dtau};
    __shared__ double tot;
    block_sum_to<1>(v, &tot);
    __syncthreads();
    if (threadIdx.x == 0) dtau_slots[block_linear()] += tot;
  }
}

// lambda^N = dJ/df^N for J = sum_x 0.5 rho |u|^2 (the total kinetic energy of
// log_diagnostics, lattice_io.hpp:182-234): lambda_i = c_i.u - 0.5 |u|^2.
// Per-block FP64 partial sums of J go to `ke_slots` (overwritten).
template <class L, class Real>
__global__ void __launch_bounds__(kThreads)
    ke_seed_kernel(const Real* __restrict__ f, Real* __restrict__ lam, Grid g,
                   double* __restrict__ ke_slots) {
  int x, y, z;
  const bool active = cell_of(g, x, y, z);
  double ke = 0.0;
  if (active) {
    const int cell = (z * g.ny + y) * g.nx + x;
    const size_t plane = (size_t)g.plane;
    Real fv[L::Q], rho, u[L::D];
    load_cell<L>(f, g, cell, fv);
    macro_state<L>(fv, rho, u);
    const Real usq = u_dot_u<L>(u);
    ke = 0.5 * (double)rho * (double)usq;
    static_for<L::Q>([&](auto I) {
      constexpr int i = LB_I(I);
      lam[plane * i + cell] = c_dot<L, i>(u) - Real(0.5) * usq;
    });
  }
  double v[1] = {ke};
  block_sum_to<1>(v, ke_slots + block_linear());
}

// dJ/du0(x) for f^0 = f_eq(rho0(x), u0(x)):
//   dJ/du0_a = sum_i lambda^0_i w_i rho0 (3 c_ia + 9 (c_i.u0) c_ia - 3 u0_a)
template <class L, class Real>
__global__ void __launch_bounds__(kThreads)
    velocity_gradient_kernel(const Real* __restrict__ rho0, const Real* __restrict__ u0,
                             const Real* __restrict__ lam0, Real* __restrict__ grad, Grid g) {
  int x, y, z;
  if (!cell_of(g, x, y, z)) return;
  const int cell = (z * g.ny + y) * g.nx + x;
  const size_t plane = (size_t)g.plane;
  Real u[L::D], lv[L::Q];
  static_for<L::D>([&](auto D) { u[LB_I(D)] = u0[plane * LB_I(D) + cell]; });
  load_cell<L>(lam0, g, cell, lv);
  const Real r = rho0[cell];
  Real gr[L::D];
  static_for<L::D>([&](auto D) { gr[LB_I(D)] = Real(0); });
  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr double wd = L::w[i];
    const Real wl = Real(wd) * r * lv[i];
    const Real s = wl * (Real(3) + Real(9) * c_dot<L, i>(u));
    static_for<L::D>([&](auto D) {
      constexpr int c = L::c[i][LB_I(D)];
      if constexpr (c > 0) gr[LB_I(D)] += s;
      if constexpr (c < 0) gr[LB_I(D)] -= s;
      gr[LB_I(D)] -= Real(3) * wl * u[LB_I(D)];
    });
  });
  static_for<L::D>([&](auto D) { grad[plane * LB_I(D) + cell] = gr[LB_I(D)]; });
}

template <class L, class Real>
cudaError_t launch_adjoint_step(int collision, const Real* fn, const Real* lam_next, Real* lam,
                                const Grid& g, const AdjointParams& ap, double* dtau_slots,
                                cudaStream_t s) {
  // programmatic dependent launches (the kernel opens with pdl_enter)
  const dim3 grid = grid_dims(g), block(block_dims(g));
  if (collision == kBGK)
    return launch_pdl(adjoint_step_kernel<L, Real, kBGK>, grid, block, 0, s, fn, lam_next, lam, g, ap,
                      dtau_slots);
  if (collision == kTRT)
    return launch_pdl(adjoint_step_kernel<L, Real, kTRT>, grid, block, 0, s, fn, lam_next, lam, g, ap,
                      dtau_slots);
  if constexpr (L::Q != 27) {
    if (collision != kMRT) return cudaErrorInvalidValue;
    return launch_pdl(adjoint_step_kernel<L, Real, kMRT>, grid, block, 0, s, fn, lam_next, lam, g, ap,
                      dtau_slots);
  } else {
    return cudaErrorInvalidValue;
  }
}

// Forward step used by the gradient driver (same engine launcher as the public API).
template <class Real>
cudaError_t forward_step(int lattice, int collision, const Real* cur, Real* nxt, const Grid& g,
                         double omega, cudaStream_t s) {
  return (cudaError_t)lbm_step_async(lattice, sizeof(Real) == 4 ? LBM_FLOAT : LBM_DOUBLE, collision,
                                     cur, nxt, g.nx, g.ny, g.nz, omega, s);
}

struct GradientLayout {
  size_t field;      // bytes of one population field
  long long ckpts;   // checkpoints stored (including the initial state)
  size_t off_ckpt, off_seg, off_lam, off_slots, total;
  long long slots;   // FP64 slots (blocks)
};

inline GradientLayout gradient_layout(int Q, size_t elem, const Grid& g, int steps, int interval) {
  GradientLayout l{};
  l.field = (size_t)Q * g.plane * elem;
  l.field = (l.field + 255) / 256 * 256;
  l.ckpts = (steps + interval - 1) / interval + 1;
  l.slots = g.blocks();
  l.off_ckpt = 0;
  l.off_seg = l.off_ckpt + (size_t)l.ckpts * l.field;
  l.off_lam = l.off_seg + (size_t)interval * l.field;
  l.off_slots = l.off_lam + 2 * l.field;
  l.total = l.off_slots + (size_t)(2 * l.slots) * sizeof(double);
  return l;
}

template <class L, class Real>
cudaError_t ke_gradient(int collision, const Real* rho0, const Real* u0, const Grid& g, double tau,
                        int steps, int interval, char* ws, const GradientLayout& lay, double* out,
                        Real* grad_u0, cudaStream_t s) {
  const double omega = (double)(Real(1) / Real(tau));
  auto ckpt = [&](long long k) { return reinterpret_cast<Real*>(ws + lay.off_ckpt + k * lay.field); };
  auto seg = [&](long long k) { return reinterpret_cast<Real*>(ws + lay.off_seg + k * lay.field); };
  Real* lam[2] = {reinterpret_cast<Real*>(ws + lay.off_lam),
                  reinterpret_cast<Real*>(ws + lay.off_lam + lay.field)};
  double* ke_slots = reinterpret_cast<double*>(ws + lay.off_slots);
  double* dtau_slots = ke_slots + lay.slots;
  cudaError_t err;

  // forward: f^0 = f_eq(rho0, u0) into checkpoint 0; checkpoints every `interval` steps
  err = (cudaError_t)lbm_init_equilibrium_async(L::id, sizeof(Real) == 4 ? LBM_FLOAT : LBM_DOUBLE,
                                                rho0, u0, ckpt(0), g.nx, g.ny, g.nz, s);
  if (err != cudaSuccess) return err;
  // Intermediate states ping-pong in two segment slots, except in the last
  // segment, whose states go straight to their segment slots so the backward
  // sweep need not recompute it.
  const long long nseg = (steps + interval - 1) / interval;
  const int last0 = (int)((nseg - 1) * interval);
  const Real* cur = ckpt(0);
  for (int n = 0; n < steps; ++n) {
    Real* nxt;
    if (n + 1 == steps || (n + 1) % interval == 0) {
      nxt = ckpt((n + 1 + interval - 1) / interval);
    } else if (n + 1 > last0) {
      nxt = seg(n + 1 - last0);
    } else {
      nxt = seg(n % 2);
    }
    err = forward_step<Real>(L::id, collision, cur, nxt, g, omega, s);
    if (err != cudaSuccess) return err;
    cur = nxt;
  }
  // seed: lambda^N and J from f^N (the last checkpoint written)
  ke_seed_kernel<L, Real><<<grid_dims(g), block_dims(g), 0, s>>>(cur, lam[steps % 2], g, ke_slots);
  if ((err = cudaGetLastError()) != cudaSuccess) return err;
  if ((err = cudaMemsetAsync(dtau_slots, 0, lay.slots * sizeof(double), s)) != cudaSuccess) return err;
  const AdjointParams ap = make_params<Real>(collision, tau);
  // backward over segments [k*interval, min((k+1)*interval, steps))
  for (long long k = nseg - 1; k >= 0; --k) {
    const int n0 = (int)(k * interval);
    const int n1 = (int)std::min<long long>((long long)steps, (k + 1) * interval);
    // recompute f^{n0+1} .. f^{n1-1} into the segment store from checkpoint k
    // (the last segment's states are already there)
    const Real* src = ckpt(k);
    for (int n = n0 + 1; n < n1 && k < nseg - 1; ++n) {
      err = forward_step<Real>(L::id, collision, src, seg(n - n0), g, omega, s);
      if (err != cudaSuccess) return err;
      src = seg(n - n0);
    }
    for (int n = n1 - 1; n >= n0; --n) {
      const Real* fn = n == n0 ? ckpt(k) : seg(n - n0);
      err = launch_adjoint_step<L, Real>(collision, fn, lam[(n + 1) % 2], lam[n % 2], g, ap,
                                         dtau_slots, s);
      if (err != cudaSuccess) return err;
    }
  }
  velocity_gradient_kernel<L, Real><<<grid_dims(g), block_dims(g), 0, s>>>(rho0, u0, lam[0], grad_u0, g);
  if ((err = cudaGetLastError()) != cudaSuccess) return err;
  sum_slots_kernel<<<1, 1024, 0, s>>>(ke_slots, lay.slots, 1, 1.0, out);
  sum_slots_kernel<<<1, 1024, 0, s>>>(dtau_slots, lay.slots, 1, 1.0, out + 1);
  return cudaGetLastError();
}

template <class Real>
cudaError_t gradient_dispatch(int lattice, int collision, const void* rho0, const void* u0,
                              size_t nx, size_t ny, size_t nz, double tau, int steps, int interval,
                              void* ws, size_t ws_bytes, double* out, void* grad, cudaStream_t s) {
  Grid g;
  const int dims = lattice == kD2Q9 ? 2 : 3;
  cudaError_t err = validate_domain(rho0 == nullptr || u0 == nullptr || ws == nullptr ||
                                        out == nullptr || grad == nullptr,
                                    1, 1, 1, dims, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  const bool mrt_ok = collision == kMRT && lattice != kD3Q27;
  if (steps < 1 || interval < 2 || (collision != kBGK && collision != kTRT && !mrt_ok) || !(tau > 0.5))
    return cudaErrorInvalidValue;
  const int Q = lattice == kD2Q9 ? 9 : (lattice == kD3Q19 ? 19 : 27);
  const GradientLayout lay = gradient_layout(Q, sizeof(Real), g, steps, interval);
  if (ws_bytes < lay.total) return cudaErrorInvalidValue;
  char* w = static_cast<char*>(ws);
  switch (lattice) {
    case kD2Q9:
      return ke_gradient<D2Q9, Real>(collision, (const Real*)rho0, (const Real*)u0, g, tau, steps,
                                     interval, w, lay, out, (Real*)grad, s);
    case kD3Q19:
      return ke_gradient<D3Q19, Real>(collision, (const Real*)rho0, (const Real*)u0, g, tau, steps,
                                      interval, w, lay, out, (Real*)grad, s);
    case kD3Q27:
      return ke_gradient<D3Q27, Real>(collision, (const Real*)rho0, (const Real*)u0, g, tau, steps,
                                      interval, w, lay, out, (Real*)grad, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace lbcube

using namespace lbcube;

extern "C" size_t lbm_ke_gradient_workspace_bytes(int lattice, int precision, size_t x_extent,
                                                  size_t y_extent, size_t z_extent, int steps,
                                                  int checkpoint_interval) {
  Grid g;
  const int dims = lattice == LBM_D2Q9 ? 2 : 3;
  if (validate_domain(false, 1, 1, 1, dims, x_extent, y_extent, z_extent, g) != cudaSuccess)
    return 0;
  if (steps < 1 || checkpoint_interval < 2) return 0;
  const int Q = lattice == LBM_D2Q9 ? 9 : (lattice == LBM_D3Q19 ? 19 : 27);
  return gradient_layout(Q, precision == LBM_DOUBLE ? 8 : 4, g, steps, checkpoint_interval).total;
}

extern "C" int lbm_ke_gradient_async(int lattice, int precision, int collision, const void* rho0,
                                     const void* u0, size_t x_extent, size_t y_extent,
                                     size_t z_extent, double tau, int steps,
                                     int checkpoint_interval, void* workspace,
                                     size_t workspace_bytes, double* objective_and_dtau,
                                     void* grad_u0, void* stream) {
  const cudaStream_t s = as_stream(stream);
  if (lattice < LBM_D2Q9 || lattice > LBM_D3Q27) return (int)cudaErrorInvalidValue;
  if (precision == LBM_FLOAT)
    return (int)gradient_dispatch<float>(lattice, collision, rho0, u0, x_extent, y_extent, z_extent,
                                         tau, steps, checkpoint_interval, workspace,
                                         workspace_bytes, objective_and_dtau, grad_u0, s);
  if (precision == LBM_DOUBLE)
    return (int)gradient_dispatch<double>(lattice, collision, rho0, u0, x_extent, y_extent,
                                          z_extent, tau, steps, checkpoint_interval, workspace,
                                          workspace_bytes, objective_and_dtau, grad_u0, s);
  return (int)cudaErrorInvalidValue;
}

extern "C" int lbm_adjoint_step_async(int lattice, int precision, int collision,
                                      const void* populations, const void* lambda_next,
                                      void* lambda, size_t x_extent, size_t y_extent,
                                      size_t z_extent, double tau, double* dtau_slots,
                                      void* stream) {
  Grid g;
  const int dims = lattice == LBM_D2Q9 ? 2 : 3;
  cudaError_t err = validate_domain(populations == nullptr || lambda_next == nullptr ||
                                        lambda == nullptr,
                                    1, 1, 1, dims, x_extent, y_extent, z_extent, g);
  if (err != cudaSuccess) return (int)err;
  if (!(tau > 0.5)) return (int)cudaErrorInvalidValue;
  const cudaStream_t s = as_stream(stream);
  const int Q = lattice == LBM_D2Q9 ? 9 : (lattice == LBM_D3Q19 ? 19 : 27);
  const size_t bytes = (size_t)Q * g.plane * (precision == LBM_DOUBLE ? 8 : 4);
  const Span reads[2] = {{populations, bytes}, {lambda_next, bytes}};
  const Span writes[1] = {{lambda, bytes}};
  if (any_overlap(reads, writes)) return (int)cudaErrorInvalidValue;
#define LBCUBE_ADJ(L, R)                                                                      \
  return (int)launch_adjoint_step<L, R>(collision, (const R*)populations, (const R*)lambda_next, \
                                        (R*)lambda, g, make_params<R>(collision, tau),          \
                                        dtau_slots, s)
  if (precision == LBM_FLOAT) {
    if (lattice == LBM_D2Q9) LBCUBE_ADJ(D2Q9, float);
    if (lattice == LBM_D3Q19) LBCUBE_ADJ(D3Q19, float);
    if (lattice == LBM_D3Q27) LBCUBE_ADJ(D3Q27, float);
  } else if (precision == LBM_DOUBLE) {
    if (lattice == LBM_D2Q9) LBCUBE_ADJ(D2Q9, double);
    if (lattice == LBM_D3Q19) LBCUBE_ADJ(D3Q19, double);
    if (lattice == LBM_D3Q27) LBCUBE_ADJ(D3Q27, double);
  }
#undef LBCUBE_ADJ
  return (int)cudaErrorInvalidValue;
}
