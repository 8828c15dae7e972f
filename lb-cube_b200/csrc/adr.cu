// Advection-diffusion(-reaction) kernels for D2Q5 / D3Q7 scalars.
//
// scalar_step_kernel    replaces kernel_scalar_step  (src/lattice_cuda.cu:234-327)
// reaction_ab_kernel    replaces kernel_reaction_AB  (src/lattice_cuda.cu:349-457)
// fluid_reaction_kernel fuses launch_step_gpu + launch_reaction_AB_gpu the way
//                       the reaction driver sequences them
//                       (src/simulate_reaction.cpp:518-543), optionally with
//                       the reactive-statistics partial sums of the new fields.
#include <algorithm>

#include "adr.cuh"
#include "slab_faces.cuh"
#include "cells.cuh"
#include "collide.cuh"
#include "common.cuh"
#include "reduce.cuh"
#include "../../include/lbcube_b200.h"

namespace lbcube {

template <class FL, class Real>
__global__ void __launch_bounds__(kThreads)
    scalar_step_kernel(const Real* __restrict__ cur_s, Real* __restrict__ nxt_s,
                       const Real* __restrict__ cur_f, Grid g, Real omega_c, Real source) {
  using SL = typename ScalarOf<FL>::type;
  pdl_enter();
  int x, y, z;
  if (!cell_of(g, x, y, z)) return;
  const int cell = (z * g.ny + y) * g.nx + x;
  Real f[FL::Q], u[FL::D], s[SL::Q];
  load_cell<FL>(cur_f, g, cell, f);
  fluid_velocity<FL>(f, u);
  gather<SL>(cur_s, g, neighbours(g, x, y, z), x, y, z, s);
  collide_scalar<SL>(s, u, omega_c, source);
  store_cell<SL>(nxt_s, g, cell, s);
}

template <class FL, class Real>
__global__ void __launch_bounds__(kThreads)
    reaction_ab_kernel(const Real* __restrict__ cur_a, Real* __restrict__ nxt_a,
                       const Real* __restrict__ cur_b, Real* __restrict__ nxt_b,
                       const Real* __restrict__ cur_f, Grid g, Real omega_c, Real k) {
  using SL = typename ScalarOf<FL>::type;
  pdl_enter();
  int x, y, z;
  if (!cell_of(g, x, y, z)) return;
  const int cell = (z * g.ny + y) * g.nx + x;
  Real f[FL::Q], u[FL::D], a[SL::Q], b[SL::Q];
  load_cell<FL>(cur_f, g, cell, f);
  fluid_velocity<FL>(f, u);
  const Neighbours n = neighbours(g, x, y, z);
  gather<SL>(cur_a, g, n, x, y, z, a);
  gather<SL>(cur_b, g, n, x, y, z, b);
  react_pair<SL>(a, b, u, omega_c, k);
  store_cell<SL>(nxt_a, g, cell, a);
  store_cell<SL>(nxt_b, g, cell, b);
}

// Fluid step + reaction step in one pass. The advecting velocity is
// recomputed from the post-collision fluid populations: they are bit for bit
// the values the reference's separate reaction launch reads back from the new
// fluid buffer at this cell, so the result equals the two-launch sequence.
// UOUT: also store that velocity, u_out[d * N + cell] (the reactive adjoint
// keeps it with each stored state).
template <class FL, class Real, int CT, bool STATS, bool UOUT>
__device__ __forceinline__ void fluid_reaction_body(const Real* __restrict__ cur_f, Real* __restrict__ nxt_f,
                                                    const Real* __restrict__ cur_a, Real* __restrict__ nxt_a,
                                                    const Real* __restrict__ cur_b, Real* __restrict__ nxt_b,
                                                    const Grid& g, Real omega, Real omega_minus,
                                                    Real omega_c, Real k, double* __restrict__ partials,
                                                    Real* __restrict__ u_out) {
  using SL = typename ScalarOf<FL>::type;
  pdl_enter();
  int x, y, z;
  const bool active = cell_of(g, x, y, z);
  double sums[kStatSums] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (active) {
    const int cell = (z * g.ny + y) * g.nx + x;
    const Neighbours n = neighbours(g, x, y, z);
    Real f[FL::Q], u[FL::D];
    gather<FL>(cur_f, g, n, x, y, z, f);
    collide<FL, Real, CT>(f, omega, omega_minus);
    store_cell<FL>(nxt_f, g, cell, f);
    fluid_velocity<FL>(f, u);
    if constexpr (UOUT) {
      static_for<FL::D>([&](auto D) { u_out[(size_t)g.plane * LB_I(D) + cell] = u[LB_I(D)]; });
    }
    Real a[SL::Q], b[SL::Q];
    gather<SL>(cur_a, g, n, x, y, z, a);
    gather<SL>(cur_b, g, n, x, y, z, b);
    react_pair<SL>(a, b, u, omega_c, k);
    store_cell<SL>(nxt_a, g, cell, a);
    store_cell<SL>(nxt_b, g, cell, b);
    if constexpr (STATS) {
      // concentration_at of the stored fields (lattice_io.hpp:125-133)
      const double ca = (double)concentration<SL>(a);
      const double cb = (double)concentration<SL>(b);
      sums[0] = ca;
      sums[1] = cb;
      sums[2] = ca * ca;
      sums[3] = cb * cb;
      sums[4] = ca * cb;
    }
  }
  // partials by absolute plane (plane_of): a launch over some planes writes
  // the partials of those planes' blocks
  if constexpr (STATS)
    block_sum_to<kStatSums>(sums, partials + ((long long)plane_of(g) * gridDim.x + blockIdx.x) *
                                                 kStatSums);
}

template <class FL, class Real, int CT, bool STATS, bool UOUT = false>
__global__ void __launch_bounds__(kThreads)
    fluid_reaction_kernel(const Real* __restrict__ cur_f, Real* __restrict__ nxt_f,
                          const Real* __restrict__ cur_a, Real* __restrict__ nxt_a,
                          const Real* __restrict__ cur_b, Real* __restrict__ nxt_b, Grid g,
                          Real omega, Real omega_minus, Real omega_c, Real k,
                          double* __restrict__ partials, Real* __restrict__ u_out = nullptr) {
  fluid_reaction_body<FL, Real, CT, STATS, UOUT>(cur_f, nxt_f, cur_a, nxt_a, cur_b, nxt_b, g, omega,
                                                 omega_minus, omega_c, k, partials, u_out);
}

// The statistics form of the FP32 D2Q9 step with the plain step's register
// budget (LBCUBE_STATS_MIN_BLOCKS resident blocks per SM): its FP64 sums and
// block reduction otherwise take 46 registers instead of 40, two resident
// blocks fewer (1024^2: 33.6 instead of 35.0 us per launch).
#ifndef LBCUBE_STATS_MIN_BLOCKS
#define LBCUBE_STATS_MIN_BLOCKS 12
#endif
template <class FL, class Real, int CT>
__global__ void __launch_bounds__(kThreads, LBCUBE_STATS_MIN_BLOCKS)
    fluid_reaction_stats_kernel(const Real* __restrict__ cur_f, Real* __restrict__ nxt_f,
                                const Real* __restrict__ cur_a, Real* __restrict__ nxt_a,
                                const Real* __restrict__ cur_b, Real* __restrict__ nxt_b, Grid g,
                                Real omega, Real omega_minus, Real omega_c, Real k,
                                double* __restrict__ partials) {
  fluid_reaction_body<FL, Real, CT, true, false>(cur_f, nxt_f, cur_a, nxt_a, cur_b, nxt_b, g, omega,
                                                 omega_minus, omega_c, k, partials, nullptr);
}

// ---- z-slab form of the coupled step ----------------------------------------
// Face layout and the halo gather / face sends: slab_faces.cuh. Every cell
// does the arithmetic of fluid_reaction_kernel, so a box stepped as slabs is
// bit-identical to the box stepped whole.

// Launch over planes g.z0 + k * g.zs (k < gridDim.y); statistics partials
// indexed by the absolute plane, so a step split into several launches writes
// every block's partial once.
// UOUT: also store the advecting velocity (the reactive adjoint keeps it with
// each stored state).
template <class FL, class Real, int CT, bool STATS, bool UOUT = false>
__global__ void __launch_bounds__(kThreads)
    fluid_reaction_slab_kernel(const Real* __restrict__ cur_f, Real* __restrict__ nxt_f,
                               const Real* __restrict__ cur_a, Real* __restrict__ nxt_a,
                               const Real* __restrict__ cur_b, Real* __restrict__ nxt_b, Grid g,
                               Real omega, Real omega_minus, Real omega_c, Real k,
                               const Real* __restrict__ halo_lo, const Real* __restrict__ halo_hi,
                               Real* __restrict__ send_lo, Real* __restrict__ send_hi,
                               double* __restrict__ partials, Real* __restrict__ u_out = nullptr) {
  using SL = typename ScalarOf<FL>::type;
  const size_t n2 = (size_t)g.ny * g.nx;
  const size_t a_off = (size_t)face_planes<FL>() * n2;
  const size_t b_off = a_off + (size_t)face_planes<SL>() * n2;
  pdl_enter();
  int x, y, z;
  const bool active = cell_of(g, x, y, z);
  double sums[kStatSums] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (active) {
    const int cell = (z * g.ny + y) * g.nx + x;
    const Neighbours n = neighbours(g, x, y, z);
    Real f[FL::Q], u[FL::D];
    gather_slab<FL>(cur_f, g, n, x, y, z, halo_lo, halo_hi, f);
    collide<FL, Real, CT>(f, omega, omega_minus);
    store_cell<FL>(nxt_f, g, cell, f);
    send_slab<FL>(g, x, y, z, f, send_lo, send_hi);
    fluid_velocity<FL>(f, u);
    if constexpr (UOUT) {
      static_for<FL::D>([&](auto D) { u_out[(size_t)g.plane * LB_I(D) + cell] = u[LB_I(D)]; });
    }
    Real a[SL::Q], b[SL::Q];
    gather_slab<SL>(cur_a, g, n, x, y, z, halo_lo + a_off, halo_hi + a_off, a);
    gather_slab<SL>(cur_b, g, n, x, y, z, halo_lo + b_off, halo_hi + b_off, b);
    react_pair<SL>(a, b, u, omega_c, k);
    store_cell<SL>(nxt_a, g, cell, a);
    store_cell<SL>(nxt_b, g, cell, b);
    send_slab<SL>(g, x, y, z, a, send_lo + a_off, send_hi + a_off);
    send_slab<SL>(g, x, y, z, b, send_lo + b_off, send_hi + b_off);
    if constexpr (STATS) {
      const double ca = (double)concentration<SL>(a);
      const double cb = (double)concentration<SL>(b);
      sums[0] = ca;
      sums[1] = cb;
      sums[2] = ca * ca;
      sums[3] = cb * cb;
      sums[4] = ca * cb;
    }
  }
  if constexpr (STATS) {
    const long long blk = (long long)plane_of(g) * gridDim.x + blockIdx.x;
    block_sum_to<kStatSums>(sums, partials + blk * kStatSums);
  }
}

// The face populations of a coupled state (fluid, A, B) into the send
// buffers: the exchange that precedes the first slab step.
template <class FL, class Real>
__global__ void __launch_bounds__(256)
    fluid_reaction_slab_pack_kernel(const Real* __restrict__ f, const Real* __restrict__ a,
                                    const Real* __restrict__ b, Real* __restrict__ send_lo,
                                    Real* __restrict__ send_hi, Grid g) {
  using SL = typename ScalarOf<FL>::type;
  const size_t n2 = (size_t)g.ny * g.nx;
  const size_t a_off = (size_t)face_planes<FL>() * n2;
  const size_t b_off = a_off + (size_t)face_planes<SL>() * n2;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < (long long)(2 * n2);
       e += (long long)gridDim.x * blockDim.x) {
    const int z = e < (long long)n2 ? 0 : g.nz - 1;
    const size_t row = (size_t)(e < (long long)n2 ? e : e - (long long)n2);
    const int y = (int)(row / g.nx), x = (int)(row - (size_t)y * g.nx);
    const int cell = (z * g.ny + y) * g.nx + x;
    Real ff[FL::Q], fa[SL::Q], fb[SL::Q];
    load_cell<FL>(f, g, cell, ff);
    load_cell<SL>(a, g, cell, fa);
    load_cell<SL>(b, g, cell, fb);
    auto send = [&](auto& vals, auto lat, size_t off) {
      using LL = decltype(lat);
      static_for<LL::Q>([&](auto I) {
        constexpr int i = LB_I(I);
        constexpr int cz = LL::c[i][2];
        if constexpr (cz > 0) {
          if (z == g.nz - 1) send_hi[off + zslot_of<LL>(i) * n2 + row] = vals[i];
        } else if constexpr (cz < 0) {
          if (z == 0) send_lo[off + zslot_of<LL>(i) * n2 + row] = vals[i];
        }
      });
    };
    send(ff, FL{}, 0);
    send(fa, SL{}, a_off);
    send(fb, SL{}, b_off);
  }
}

template <class FL, class Real, int CT>
cudaError_t launch_fluid_reaction_slab(const Real* cur_f, Real* nxt_f, const Real* cur_a,
                                       Real* nxt_a, const Real* cur_b, Real* nxt_b, size_t nx,
                                       size_t ny, size_t nz, Real omega, Real omega_c, Real k,
                                       const Real* halo_lo, const Real* halo_hi, Real* send_lo,
                                       Real* send_hi, size_t z_begin, size_t z_end,
                                       double* partials, size_t partials_bytes,
                                       cudaStream_t stream) {
  using SL = typename ScalarOf<FL>::type;
  Grid g;
  cudaError_t err = validate_domain(cur_f == nullptr || nxt_f == nullptr || cur_a == nullptr ||
                                        nxt_a == nullptr || cur_b == nullptr || nxt_b == nullptr ||
                                        halo_lo == nullptr || halo_hi == nullptr ||
                                        send_lo == nullptr || send_hi == nullptr,
                                    1, 1, 1, 3, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  if (z_begin >= z_end || z_end > (size_t)g.nz) return cudaErrorInvalidValue;
  const size_t sb = (size_t)SL::Q * g.plane * sizeof(Real);
  const size_t fb = (size_t)FL::Q * g.plane * sizeof(Real);
  const size_t hb = (size_t)coupled_face_planes<FL>() * g.ny * g.nx * sizeof(Real);
  const size_t need = (size_t)g.blocks() * kStatSums * sizeof(double);
  if (partials != nullptr && partials_bytes < need) return cudaErrorInvalidValue;
  const Span reads[5] = {{cur_f, fb}, {cur_a, sb}, {cur_b, sb}, {halo_lo, hb}, {halo_hi, hb}};
  const Span writes[6] = {{nxt_f, fb}, {nxt_a, sb}, {nxt_b, sb}, {send_lo, hb}, {send_hi, hb},
                          {partials, partials != nullptr ? need : 0}};
  if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  const Real omega_minus = CT == kTRT ? trt_omega_minus<Real>(omega) : Real(0);
  // planes 0 and nz-1 of the range: the SLAB form; planes in between pull and
  // send nothing across a face: the whole-box kernel (fewer registers)
  // `planes` planes from z0, `zs` apart
  auto launch = [&](int z0, int planes, int zs, bool face) {
    if (planes <= 0) return;
    Grid gr = g;
    gr.z0 = z0;
    gr.zs = zs;
    dim3 grid = grid_dims(gr);
    grid.y = (unsigned)planes;
    const dim3 block(block_dims(gr));
    Real* const none = nullptr;
    if (face && partials != nullptr)
      launch_pdl(fluid_reaction_slab_kernel<FL, Real, CT, true, false>, grid, block, 0, stream, cur_f, nxt_f,
                 cur_a, nxt_a, cur_b, nxt_b, gr, omega, omega_minus, omega_c, k, halo_lo, halo_hi, send_lo,
                 send_hi, partials, none);
    else if (face)
      launch_pdl(fluid_reaction_slab_kernel<FL, Real, CT, false, false>, grid, block, 0, stream, cur_f,
                 nxt_f, cur_a, nxt_a, cur_b, nxt_b, gr, omega, omega_minus, omega_c, k, halo_lo, halo_hi,
                 send_lo, send_hi, (double*)nullptr, none);
    else if (partials != nullptr)
      launch_pdl(fluid_reaction_kernel<FL, Real, CT, true, false>, grid, block, 0, stream, cur_f, nxt_f,
                 cur_a, nxt_a, cur_b, nxt_b, gr, omega, omega_minus, omega_c, k, partials, none);
    else
      launch_pdl(fluid_reaction_kernel<FL, Real, CT, false, false>, grid, block, 0, stream, cur_f, nxt_f,
                 cur_a, nxt_a, cur_b, nxt_b, gr, omega, omega_minus, omega_c, k, (double*)nullptr, none);
  };
  const int zb = (int)z_begin, ze = (int)z_end, last = g.nz - 1;
  const bool lo = zb == 0, hi = ze - 1 == last && last > 0 && zb <= last;
  launch(std::max(zb, 1), std::min(ze, last) - std::max(zb, 1), 1, false);
  if (lo && hi) {
    launch(0, 2, last, true);  // both face planes in one launch
  } else {
    if (lo) launch(0, 1, 1, true);
    if (hi) launch(last, 1, 1, true);
  }
  return cudaGetLastError();
}

template <class FL, class Real>
cudaError_t launch_fluid_reaction_slab_pack(const Real* f, const Real* a, const Real* b, size_t nx,
                                            size_t ny, size_t nz, Real* send_lo, Real* send_hi,
                                            cudaStream_t stream) {
  using SL = typename ScalarOf<FL>::type;
  Grid g;
  cudaError_t err = validate_domain(f == nullptr || a == nullptr || b == nullptr ||
                                        send_lo == nullptr || send_hi == nullptr,
                                    1, 1, 1, 3, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  const size_t hb = (size_t)coupled_face_planes<FL>() * g.ny * g.nx * sizeof(Real);
  const Span reads[3] = {{f, (size_t)FL::Q * g.plane * sizeof(Real)},
                         {a, (size_t)SL::Q * g.plane * sizeof(Real)},
                         {b, (size_t)SL::Q * g.plane * sizeof(Real)}};
  const Span writes[2] = {{send_lo, hb}, {send_hi, hb}};
  if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  const long long total = 2LL * g.ny * g.nx;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  fluid_reaction_slab_pack_kernel<FL, Real><<<blocks, 256, 0, stream>>>(f, a, b, send_lo, send_hi, g);
  return cudaGetLastError();
}

template <class FL, class Real>
cudaError_t launch_scalar(const Real* cur_s, Real* nxt_s, const Real* cur_f, size_t nx, size_t ny,
                          size_t nz, Real omega_c, Real source, unsigned bx, unsigned by,
                          unsigned bz, cudaStream_t stream) {
  using SL = typename ScalarOf<FL>::type;
  Grid g;
  cudaError_t err = validate_domain(cur_s == nullptr || nxt_s == nullptr || cur_f == nullptr, bx,
                                    by, bz, FL::D, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  const size_t sb = (size_t)SL::Q * g.plane * sizeof(Real);
  const size_t fb = (size_t)FL::Q * g.plane * sizeof(Real);
  const Span reads[2] = {{cur_s, sb}, {cur_f, fb}};
  const Span writes[1] = {{nxt_s, sb}};
  if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  return launch_pdl(scalar_step_kernel<FL, Real>, grid_dims(g), dim3(block_dims(g)), 0, stream, cur_s,
                    nxt_s, cur_f, g, omega_c, source);
}

template <class FL, class Real>
cudaError_t launch_reaction(const Real* cur_a, Real* nxt_a, const Real* cur_b, Real* nxt_b,
                            const Real* cur_f, size_t nx, size_t ny, size_t nz, Real omega_c,
                            Real k, unsigned bx, unsigned by, unsigned bz, cudaStream_t stream) {
  using SL = typename ScalarOf<FL>::type;
  Grid g;
  cudaError_t err =
      validate_domain(cur_a == nullptr || nxt_a == nullptr || cur_b == nullptr ||
                          nxt_b == nullptr || cur_f == nullptr,
                      bx, by, bz, FL::D, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  const size_t sb = (size_t)SL::Q * g.plane * sizeof(Real);
  const size_t fb = (size_t)FL::Q * g.plane * sizeof(Real);
  const Span reads[3] = {{cur_a, sb}, {cur_b, sb}, {cur_f, fb}};
  const Span writes[2] = {{nxt_a, sb}, {nxt_b, sb}};
  if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  return launch_pdl(reaction_ab_kernel<FL, Real>, grid_dims(g), dim3(block_dims(g)), 0, stream, cur_a,
                    nxt_a, cur_b, nxt_b, cur_f, g, omega_c, k);
}

template <class FL, class Real, int CT>
cudaError_t launch_fluid_reaction(const Real* cur_f, Real* nxt_f, const Real* cur_a, Real* nxt_a,
                                  const Real* cur_b, Real* nxt_b, size_t nx, size_t ny,
                                  size_t nz, Real omega, Real omega_c, Real k, double* partials,
                                  size_t partials_bytes, cudaStream_t stream) {
  using SL = typename ScalarOf<FL>::type;
  Grid g;
  cudaError_t err = validate_domain(cur_f == nullptr || nxt_f == nullptr || cur_a == nullptr ||
                                        nxt_a == nullptr || cur_b == nullptr || nxt_b == nullptr,
                                    1, 1, 1, FL::D, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  const size_t sb = (size_t)SL::Q * g.plane * sizeof(Real);
  const size_t fb = (size_t)FL::Q * g.plane * sizeof(Real);
  const Span reads[3] = {{cur_f, fb}, {cur_a, sb}, {cur_b, sb}};
  if (partials != nullptr) {
    const size_t need = (size_t)g.blocks() * kStatSums * sizeof(double);
    if (partials_bytes < need) return cudaErrorInvalidValue;
    const Span writes[4] = {{nxt_f, fb}, {nxt_a, sb}, {nxt_b, sb}, {partials, need}};
    if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  } else {
    const Span writes[3] = {{nxt_f, fb}, {nxt_a, sb}, {nxt_b, sb}};
    if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  }
  const Real omega_minus = CT == kTRT ? trt_omega_minus<Real>(omega) : Real(0);
  // launched as programmatic dependents of the previous launch (pdl_enter)
  if (partials != nullptr) {
    if constexpr (FL::Q == 9 && sizeof(Real) == 4 && LBCUBE_STATS_MIN_BLOCKS > 0)
      return launch_pdl(fluid_reaction_stats_kernel<FL, Real, CT>, grid_dims(g), dim3(block_dims(g)), 0,
                        stream, cur_f, nxt_f, cur_a, nxt_a, cur_b, nxt_b, g, omega, omega_minus,
                        omega_c, k, partials);
    else
      return launch_pdl(fluid_reaction_kernel<FL, Real, CT, true, false>, grid_dims(g),
                        dim3(block_dims(g)), 0, stream, cur_f, nxt_f, cur_a, nxt_a, cur_b, nxt_b, g,
                        omega, omega_minus, omega_c, k, partials, (Real*)nullptr);
  }
  return launch_pdl(fluid_reaction_kernel<FL, Real, CT, false, false>, grid_dims(g), dim3(block_dims(g)),
                    0, stream, cur_f, nxt_f, cur_a, nxt_a, cur_b, nxt_b, g, omega, omega_minus, omega_c,
                    k, (double*)nullptr, (Real*)nullptr);
}

// The fused step with the advecting velocity stored (no statistics), for the
// reactive adjoint's forward and recomputation passes. Buffers are checked by
// the caller (they are slices of its workspace).
template <class FL, class Real>
cudaError_t fluid_reaction_with_velocity(int collision, const Real* cur_f, Real* nxt_f,
                                         const Real* cur_a, Real* nxt_a, const Real* cur_b,
                                         Real* nxt_b, Real* u_out, const Grid& g, Real omega,
                                         Real omega_c, Real k, cudaStream_t s) {
  // programmatic dependent launches (the kernel opens with pdl_enter)
  const dim3 grid = grid_dims(g), block(block_dims(g));
  double* const none = nullptr;
  if (collision == kBGK)
    return launch_pdl(fluid_reaction_kernel<FL, Real, kBGK, false, true>, grid, block, 0, s, cur_f, nxt_f,
                      cur_a, nxt_a, cur_b, nxt_b, g, omega, Real(0), omega_c, k, none, u_out);
  if (collision == kTRT)
    return launch_pdl(fluid_reaction_kernel<FL, Real, kTRT, false, true>, grid, block, 0, s, cur_f, nxt_f,
                      cur_a, nxt_a, cur_b, nxt_b, g, omega, trt_omega_minus<Real>(omega), omega_c, k,
                      none, u_out);
  if (collision == kMRT)
    return launch_pdl(fluid_reaction_kernel<FL, Real, kMRT, false, true>, grid, block, 0, s, cur_f, nxt_f,
                      cur_a, nxt_a, cur_b, nxt_b, g, omega, Real(0), omega_c, k, none, u_out);
  return cudaErrorInvalidValue;
}

// The slab form of fluid_reaction_with_velocity (all planes of the slab, no
// statistics; u_out may be null): for the decomposed reactive adjoint. Planes
// 1 .. nz-2 pull and send nothing across a face, so they run the whole-box
// kernel (fewer registers than the SLAB form); planes 0 and nz-1 run the SLAB
// form. Buffers are checked by the caller.
template <class FL, class Real>
cudaError_t fluid_reaction_slab_with_velocity(int collision, const Real* cur_f, Real* nxt_f,
                                              const Real* cur_a, Real* nxt_a, const Real* cur_b,
                                              Real* nxt_b, Real* u_out, const Grid& g, Real omega,
                                              Real omega_c, Real k, const Real* halo_lo,
                                              const Real* halo_hi, Real* send_lo, Real* send_hi,
                                              cudaStream_t s) {
  auto run = [&](auto ct) -> cudaError_t {
    constexpr int CT = decltype(ct)::value;
    const Real om = CT == kTRT ? trt_omega_minus<Real>(omega) : Real(0);
    auto launch = [&](int z0, int planes, int zs, bool face) {
      Grid gr = g;
      gr.z0 = z0;
      gr.zs = zs;
      dim3 grid = grid_dims(gr);
      grid.y = (unsigned)planes;
      const dim3 block(block_dims(gr));
      double* const none = nullptr;
      if (face && u_out != nullptr)
        launch_pdl(fluid_reaction_slab_kernel<FL, Real, CT, false, true>, grid, block, 0, s, cur_f, nxt_f,
                   cur_a, nxt_a, cur_b, nxt_b, gr, omega, om, omega_c, k, halo_lo, halo_hi, send_lo,
                   send_hi, none, u_out);
      else if (face)
        launch_pdl(fluid_reaction_slab_kernel<FL, Real, CT, false, false>, grid, block, 0, s, cur_f,
                   nxt_f, cur_a, nxt_a, cur_b, nxt_b, gr, omega, om, omega_c, k, halo_lo, halo_hi,
                   send_lo, send_hi, none, (Real*)nullptr);
      else if (u_out != nullptr)
        launch_pdl(fluid_reaction_kernel<FL, Real, CT, false, true>, grid, block, 0, s, cur_f, nxt_f,
                   cur_a, nxt_a, cur_b, nxt_b, gr, omega, om, omega_c, k, none, u_out);
      else
        launch_pdl(fluid_reaction_kernel<FL, Real, CT, false, false>, grid, block, 0, s, cur_f, nxt_f,
                   cur_a, nxt_a, cur_b, nxt_b, gr, omega, om, omega_c, k, none, (Real*)nullptr);
    };
    if (g.nz >= 3) launch(1, g.nz - 2, 1, false);
    launch(0, g.nz >= 2 ? 2 : 1, g.nz - 1, true);  // both face planes in one launch
    return cudaGetLastError();
  };
  if (collision == kBGK) return run(std::integral_constant<int, kBGK>{});
  if (collision == kTRT) return run(std::integral_constant<int, kTRT>{});
  if (collision == kMRT) return run(std::integral_constant<int, kMRT>{});
  return cudaErrorInvalidValue;
}

#define LBCUBE_FRSV_INST(FL, R)                                                                     \
  template cudaError_t fluid_reaction_slab_with_velocity<FL, R>(                                   \
      int, const R*, R*, const R*, R*, const R*, R*, R*, const Grid&, R, R, R, const R*, const R*, \
      R*, R*, cudaStream_t);
LBCUBE_FRSV_INST(D3Q19, float)
LBCUBE_FRSV_INST(D3Q19, double)
LBCUBE_FRSV_INST(D3Q27, float)
LBCUBE_FRSV_INST(D3Q27, double)
#undef LBCUBE_FRSV_INST

#define LBCUBE_FRV(FL, R)                                                                     \
  template cudaError_t fluid_reaction_with_velocity<FL, R>(                                   \
      int, const R*, R*, const R*, R*, const R*, R*, R*, const Grid&, R, R, R, cudaStream_t);
LBCUBE_FRV(D2Q9, float)
LBCUBE_FRV(D2Q9, double)
LBCUBE_FRV(D3Q19, float)
LBCUBE_FRV(D3Q19, double)
LBCUBE_FRV(D3Q27, float)
LBCUBE_FRV(D3Q27, double)
#undef LBCUBE_FRV

template <class FL, class Real>
cudaError_t fused_by_collision(int collision, const void* cf, void* nf, const void* ca, void* na,
                               const void* cb, void* nb, size_t nx, size_t ny, size_t nz,
                               double omega, double omega_c, double k, double* partials,
                               size_t pbytes, cudaStream_t s) {
  const Real* f0 = static_cast<const Real*>(cf);
  Real* f1 = static_cast<Real*>(nf);
  const Real* a0 = static_cast<const Real*>(ca);
  Real* a1 = static_cast<Real*>(na);
  const Real* b0 = static_cast<const Real*>(cb);
  Real* b1 = static_cast<Real*>(nb);
  switch (collision) {
    case kBGK:
      return launch_fluid_reaction<FL, Real, kBGK>(f0, f1, a0, a1, b0, b1, nx, ny, nz, Real(omega),
                                                   Real(omega_c), Real(k), partials, pbytes, s);
    case kTRT:
      return launch_fluid_reaction<FL, Real, kTRT>(f0, f1, a0, a1, b0, b1, nx, ny, nz, Real(omega),
                                                   Real(omega_c), Real(k), partials, pbytes, s);
    case kMRT:
      return launch_fluid_reaction<FL, Real, kMRT>(f0, f1, a0, a1, b0, b1, nx, ny, nz, Real(omega),
                                                   Real(omega_c), Real(k), partials, pbytes, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace lbcube

using namespace lbcube;

#define LBCUBE_SCALAR_SYMBOL(fl, sl, FL, real)                                                   \
  extern "C" int lbm_launch_scalar_step_gpu_##fl##_##sl##_##real(                              \
      const real* current_scalar, real* next_scalar, const real* current_fluid,                \
      size_t x_extent, size_t y_extent, size_t z_extent, real omega_c, real source_term,       \
      unsigned block_x, unsigned block_y, unsigned block_z) {                                  \
    return (int)launch_scalar<FL, real>(current_scalar, next_scalar, current_fluid, x_extent,  \
                                        y_extent, z_extent, omega_c, source_term, block_x,     \
                                        block_y, block_z, (cudaStream_t)0);                    \
  }

#define LBCUBE_REACTION_SYMBOL(fl, sl, FL, real)                                                 \
  extern "C" int lbm_launch_reaction_ab_gpu_##fl##_##sl##_##real(                              \
      const real* current_a, real* next_a, const real* current_b, real* next_b,                \
      const real* current_fluid, size_t x_extent, size_t y_extent, size_t z_extent,            \
      real omega_c, real k_react, unsigned block_x, unsigned block_y, unsigned block_z) {      \
    return (int)launch_reaction<FL, real>(current_a, next_a, current_b, next_b, current_fluid, \
                                          x_extent, y_extent, z_extent, omega_c, k_react,      \
                                          block_x, block_y, block_z, (cudaStream_t)0);         \
  }

LBCUBE_SCALAR_SYMBOL(d2q9, d2q5, D2Q9, float)
LBCUBE_SCALAR_SYMBOL(d2q9, d2q5, D2Q9, double)
LBCUBE_SCALAR_SYMBOL(d3q19, d3q7, D3Q19, float)
LBCUBE_SCALAR_SYMBOL(d3q19, d3q7, D3Q19, double)
LBCUBE_SCALAR_SYMBOL(d3q27, d3q7, D3Q27, float)
LBCUBE_SCALAR_SYMBOL(d3q27, d3q7, D3Q27, double)

LBCUBE_REACTION_SYMBOL(d2q9, d2q5, D2Q9, float)
LBCUBE_REACTION_SYMBOL(d2q9, d2q5, D2Q9, double)
LBCUBE_REACTION_SYMBOL(d3q19, d3q7, D3Q19, float)
LBCUBE_REACTION_SYMBOL(d3q19, d3q7, D3Q19, double)
LBCUBE_REACTION_SYMBOL(d3q27, d3q7, D3Q27, float)
LBCUBE_REACTION_SYMBOL(d3q27, d3q7, D3Q27, double)

extern "C" int lbm_scalar_step_async(int fluid_lattice, int precision, const void* current_scalar,
                                     void* next_scalar, const void* current_fluid,
                                     size_t x_extent, size_t y_extent, size_t z_extent,
                                     double omega_c, double source_term, void* stream) {
  const cudaStream_t s = as_stream(stream);
#define LBCUBE_CASE(FL, real)                                                                     \
  return (int)launch_scalar<FL, real>(static_cast<const real*>(current_scalar),                  \
                                      static_cast<real*>(next_scalar),                           \
                                      static_cast<const real*>(current_fluid), x_extent,         \
                                      y_extent, z_extent, real(omega_c), real(source_term), 1, 1, \
                                      1, s)
  if (precision == LBM_FLOAT) {
    if (fluid_lattice == LBM_D2Q9) LBCUBE_CASE(D2Q9, float);
    if (fluid_lattice == LBM_D3Q19) LBCUBE_CASE(D3Q19, float);
    if (fluid_lattice == LBM_D3Q27) LBCUBE_CASE(D3Q27, float);
  } else if (precision == LBM_DOUBLE) {
    if (fluid_lattice == LBM_D2Q9) LBCUBE_CASE(D2Q9, double);
    if (fluid_lattice == LBM_D3Q19) LBCUBE_CASE(D3Q19, double);
    if (fluid_lattice == LBM_D3Q27) LBCUBE_CASE(D3Q27, double);
  }
#undef LBCUBE_CASE
  return (int)cudaErrorInvalidValue;
}

extern "C" int lbm_reaction_ab_async(int fluid_lattice, int precision, const void* current_a,
                                     void* next_a, const void* current_b, void* next_b,
                                     const void* current_fluid, size_t x_extent, size_t y_extent,
                                     size_t z_extent, double omega_c, double k_react,
                                     void* stream) {
  const cudaStream_t s = as_stream(stream);
#define LBCUBE_CASE(FL, real)                                                                 \
  return (int)launch_reaction<FL, real>(                                                     \
      static_cast<const real*>(current_a), static_cast<real*>(next_a),                       \
      static_cast<const real*>(current_b), static_cast<real*>(next_b),                       \
      static_cast<const real*>(current_fluid), x_extent, y_extent, z_extent, real(omega_c),  \
      real(k_react), 1, 1, 1, s)
  if (precision == LBM_FLOAT) {
    if (fluid_lattice == LBM_D2Q9) LBCUBE_CASE(D2Q9, float);
    if (fluid_lattice == LBM_D3Q19) LBCUBE_CASE(D3Q19, float);
    if (fluid_lattice == LBM_D3Q27) LBCUBE_CASE(D3Q27, float);
  } else if (precision == LBM_DOUBLE) {
    if (fluid_lattice == LBM_D2Q9) LBCUBE_CASE(D2Q9, double);
    if (fluid_lattice == LBM_D3Q19) LBCUBE_CASE(D3Q19, double);
    if (fluid_lattice == LBM_D3Q27) LBCUBE_CASE(D3Q27, double);
  }
#undef LBCUBE_CASE
  return (int)cudaErrorInvalidValue;
}

extern "C" int lbm_fluid_reaction_ab_async(int fluid_lattice, int precision, int collision,
                                           const void* current_fluid, void* next_fluid,
                                           const void* current_a, void* next_a,
                                           const void* current_b, void* next_b, size_t x_extent,
                                           size_t y_extent, size_t z_extent, double omega,
                                           double omega_c, double k_react,
                                           double* stats_partials, size_t stats_partials_bytes,
                                           void* stream) {
  const cudaStream_t s = as_stream(stream);
#define LBCUBE_CASE(FL, real)                                                                  \
  return (int)fused_by_collision<FL, real>(collision, current_fluid, next_fluid, current_a,   \
                                           next_a, current_b, next_b, x_extent, y_extent,     \
                                           z_extent, omega, omega_c, k_react, stats_partials, \
                                           stats_partials_bytes, s)
  if (precision == LBM_FLOAT) {
    if (fluid_lattice == LBM_D2Q9) LBCUBE_CASE(D2Q9, float);
    if (fluid_lattice == LBM_D3Q19) LBCUBE_CASE(D3Q19, float);
    if (fluid_lattice == LBM_D3Q27) LBCUBE_CASE(D3Q27, float);
  } else if (precision == LBM_DOUBLE) {
    if (fluid_lattice == LBM_D2Q9) LBCUBE_CASE(D2Q9, double);
    if (fluid_lattice == LBM_D3Q19) LBCUBE_CASE(D3Q19, double);
    if (fluid_lattice == LBM_D3Q27) LBCUBE_CASE(D3Q27, double);
  }
#undef LBCUBE_CASE
  return (int)cudaErrorInvalidValue;
}

extern "C" size_t lbm_fluid_reaction_slab_face_elems(int fluid_lattice, size_t x_extent,
                                                    size_t y_extent) {
  if (fluid_lattice == LBM_D3Q19) return (size_t)coupled_face_planes<D3Q19>() * x_extent * y_extent;
  if (fluid_lattice == LBM_D3Q27) return (size_t)coupled_face_planes<D3Q27>() * x_extent * y_extent;
  return 0;
}

extern "C" int lbm_fluid_reaction_slab_async(
    int fluid_lattice, int precision, int collision, const void* current_fluid, void* next_fluid,
    const void* current_a, void* next_a, const void* current_b, void* next_b, size_t x_extent,
    size_t y_extent, size_t z_extent, double omega, double omega_c, double k_react,
    const void* halo_lo, const void* halo_hi, void* send_lo, void* send_hi, size_t z_begin,
    size_t z_end, double* stats_partials, size_t stats_partials_bytes, void* stream) {
  const cudaStream_t s = as_stream(stream);
#define LBCUBE_SLAB(FL, R, CT)                                                                    \
  return (int)launch_fluid_reaction_slab<FL, R, CT>(                                             \
      static_cast<const R*>(current_fluid), static_cast<R*>(next_fluid),                         \
      static_cast<const R*>(current_a), static_cast<R*>(next_a), static_cast<const R*>(current_b), \
      static_cast<R*>(next_b), x_extent, y_extent, z_extent, R(omega), R(omega_c), R(k_react),   \
      static_cast<const R*>(halo_lo), static_cast<const R*>(halo_hi), static_cast<R*>(send_lo),  \
      static_cast<R*>(send_hi), z_begin, z_end, stats_partials, stats_partials_bytes, s)
#define LBCUBE_SLAB_OP(FL, R)                       \
  switch (collision) {                              \
    case kBGK: LBCUBE_SLAB(FL, R, kBGK);            \
    case kTRT: LBCUBE_SLAB(FL, R, kTRT);            \
    case kMRT: LBCUBE_SLAB(FL, R, kMRT);            \
    default: return (int)cudaErrorInvalidValue;     \
  }
  if (precision == LBM_FLOAT) {
    if (fluid_lattice == LBM_D3Q19) LBCUBE_SLAB_OP(D3Q19, float)
    if (fluid_lattice == LBM_D3Q27) LBCUBE_SLAB_OP(D3Q27, float)
  } else if (precision == LBM_DOUBLE) {
    if (fluid_lattice == LBM_D3Q19) LBCUBE_SLAB_OP(D3Q19, double)
    if (fluid_lattice == LBM_D3Q27) LBCUBE_SLAB_OP(D3Q27, double)
  }
#undef LBCUBE_SLAB_OP
#undef LBCUBE_SLAB
  return (int)cudaErrorInvalidValue;
}

// The pack for any stored form of the reactive gradient's states: elements of
// the precision (LBM_NATIVE) or 16-bit codes (a shifted format, LBM_FLOAT).
extern "C" int lbm_reactive_slab_pack_async(int fluid_lattice, int precision, int storage,
                                            const void* fluid, const void* a, const void* b,
                                            size_t x_extent, size_t y_extent, size_t z_extent,
                                            void* send_lo, void* send_hi, void* stream) {
  if (storage != LBM_NATIVE)
    return precision != LBM_FLOAT || (storage != LBM_F16S && storage != LBM_BF16S &&
                                      storage != LBM_E3M12S && storage != LBM_Q15S)
               ? (int)cudaErrorInvalidValue
           : fluid_lattice == LBM_D3Q19
               ? (int)launch_fluid_reaction_slab_pack<D3Q19, unsigned short>(
                     (const unsigned short*)fluid, (const unsigned short*)a,
                     (const unsigned short*)b, x_extent, y_extent, z_extent,
                     (unsigned short*)send_lo, (unsigned short*)send_hi, as_stream(stream))
           : fluid_lattice == LBM_D3Q27
               ? (int)launch_fluid_reaction_slab_pack<D3Q27, unsigned short>(
                     (const unsigned short*)fluid, (const unsigned short*)a,
                     (const unsigned short*)b, x_extent, y_extent, z_extent,
                     (unsigned short*)send_lo, (unsigned short*)send_hi, as_stream(stream))
               : (int)cudaErrorInvalidValue;
  return lbm_fluid_reaction_slab_pack_async(fluid_lattice, precision, fluid, a, b, x_extent,
                                            y_extent, z_extent, send_lo, send_hi, stream);
}

extern "C" int lbm_fluid_reaction_slab_pack_async(int fluid_lattice, int precision,
                                                  const void* fluid, const void* a, const void* b,
                                                  size_t x_extent, size_t y_extent, size_t z_extent,
                                                  void* send_lo, void* send_hi, void* stream) {
  const cudaStream_t s = as_stream(stream);
#define LBCUBE_PACK(FL, R)                                                                       \
  return (int)launch_fluid_reaction_slab_pack<FL, R>(                                           \
      static_cast<const R*>(fluid), static_cast<const R*>(a), static_cast<const R*>(b), x_extent, \
      y_extent, z_extent, static_cast<R*>(send_lo), static_cast<R*>(send_hi), s)
  if (precision == LBM_FLOAT) {
    if (fluid_lattice == LBM_D3Q19) LBCUBE_PACK(D3Q19, float);
    if (fluid_lattice == LBM_D3Q27) LBCUBE_PACK(D3Q27, float);
  } else if (precision == LBM_DOUBLE) {
    if (fluid_lattice == LBM_D3Q19) LBCUBE_PACK(D3Q19, double);
    if (fluid_lattice == LBM_D3Q27) LBCUBE_PACK(D3Q27, double);
  }
#undef LBCUBE_PACK
  return (int)cudaErrorInvalidValue;
}
