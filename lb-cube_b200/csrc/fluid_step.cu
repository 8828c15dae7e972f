// Fused pull-scheme collide-stream step for D2Q9 / D3Q19 / D3Q27 fluids.
//
// Replaces kernel_step and launch_step_gpu (src/lattice_cuda.cu:149-213,
// :476-520). One thread owns one destination cell: it gathers the Q incoming
// populations f_i(x - c_i) from the current buffer (periodic wrap by
// compare-and-select on 32-bit coordinates instead of the reference's 64-bit
// modulo), collides in registers and writes the Q results to the next buffer
// at its own cell. A warp covers 32 consecutive x cells, so each of the Q
// gathers and Q stores is one coalesced 128-byte row segment (shifted by at
// most one element for c_x != 0, which the L1/L2 sector reuse absorbs).
#include "collide.cuh"
#include "common.cuh"
#include "diag.cuh"
#include "stream_vec.cuh"
#include "../../include/lbcube_b200.h"

namespace lbcube {

template <class L, class Real, int CT>
__device__ __forceinline__ void step_cell(const Real* __restrict__ cur, Real* __restrict__ nxt,
                                          const Grid& g, int x, int y, int z, Real omega,
                                          Real omega_minus, Real (&f)[L::Q]) {
  const int xm = x == 0 ? g.nx - 1 : x - 1, xp = x == g.nx - 1 ? 0 : x + 1;
  const int ym = y == 0 ? g.ny - 1 : y - 1, yp = y == g.ny - 1 ? 0 : y + 1;
  const int zm = z == 0 ? g.nz - 1 : z - 1, zp = z == g.nz - 1 ? 0 : z + 1;
  const size_t plane = (size_t)g.plane;

  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
    // pull: source = destination - c_i (lattice_core.hpp:70-78)
    const int sx = cx == 0 ? x : (cx > 0 ? xm : xp);
    const int sy = cy == 0 ? y : (cy > 0 ? ym : yp);
    const int sz = cz == 0 ? z : (cz > 0 ? zm : zp);
    f[i] = __ldg(cur + plane * i + ((sz * g.ny + sy) * g.nx + sx));
  });

  collide<L, Real, CT>(f, omega, omega_minus);

  const int cell = (z * g.ny + y) * g.nx + x;
  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    nxt[plane * i + cell] = f[i];
  });
}

// DIAG: also reduce the diagnostics of the written state over the block
// (diag.cuh), as in fluid_step_vec_kernel.
template <class L, class Real, int CT, bool DIAG = false>
__global__ void __launch_bounds__(kThreads)
    fluid_step_kernel(const Real* __restrict__ cur, Real* __restrict__ nxt, Grid g, Real omega,
                      Real omega_minus, double* __restrict__ partials = nullptr) {
  int x, y, z;
  const bool active = cell_of(g, x, y, z);
  Real f[L::Q];
  if constexpr (DIAG) {
    DiagAcc acc;
    if (active) {
      step_cell<L, Real, CT>(cur, nxt, g, x, y, z, omega, omega_minus, f);
      diag_cell<L>(f, acc);
    }
    diag_block_to(acc, partials + block_linear() * kDiagPartials);
  } else {
    if (!active) return;
    step_cell<L, Real, CT>(cur, nxt, g, x, y, z, omega, omega_minus, f);
  }
}

// Cells per thread of the vectorised kernel, measured fastest on B200 at 256^3:
// 2 FP32 D2Q9 / D3Q19 cells (8-byte words; D3Q19 TRT 0.99 of the copy
// bandwidth against 0.80 at V = 4 and 0.76 at V = 1), 1 D3Q27 FP32 cell (BGK
// 0.86 against 0.75 at V = 2, TRT 0.80 against 0.58) and 1 FP64 cell.
// The plain step of native storage runs the vectorised kernel only for FP32
// D3Q19 BGK and TRT, where it is level with the one-cell kernel; every other
// lattice, operator and precision measured faster with the one-cell kernel
// (A/B at 256^3 / 4096^2, bitwise-identical outputs, fraction of the copy
// bandwidth): D3Q27 FP32 BGK 0.76 -> 0.97, TRT 0.74 -> 0.95, MRT 0.48 -> 0.56,
// RLBM 0.59 -> 0.68; D3Q27 FP64 BGK 0.91 -> 1.03, TRT 0.88 -> 1.03; D3Q19 FP32
// MRT 0.80 -> 0.87; D3Q19 FP64 MRT 0.86 -> 0.97, RLBM 0.74 -> 0.84; D2Q9 FP32
// 2-5 % and FP64 4-18 %. The one-cell kernel keeps fewer values live across
// the gather, so its warps hide the load latency without register pressure.
// The 16-bit storage and the slab step keep the vectorised kernel.
template <class L, class Real>
constexpr int kVecCells = (sizeof(Real) == 4 && L::Q != 27) ? 2 : 1;
template <class L, class Real, int CT>
constexpr bool kUseVec = sizeof(Real) == 4 && L::Q == 19 && (CT == kBGK || CT == kTRT);

template <class L, class Real, int CT>
cudaError_t launch_fluid_step(const Real* cur, Real* nxt, size_t nx, size_t ny, size_t nz,
                              Real omega, unsigned bx, unsigned by, unsigned bz,
                              cudaStream_t stream) {
  Grid g;
  cudaError_t err =
      validate_domain(cur == nullptr || nxt == nullptr, bx, by, bz, L::D, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  const size_t bytes = (size_t)L::Q * (size_t)g.plane * sizeof(Real);
  const Span reads[1] = {{cur, bytes}};
  const Span writes[1] = {{nxt, bytes}};
  if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  const Real omega_minus = CT == kTRT ? trt_omega_minus<Real>(omega) : Real(0);
  using S = NativeStorage<Real, kVecCells<L, Real>>;
  if (kUseVec<L, Real, CT> && vec_eligible<S>(g, cur, nxt)) {
    const VecGrid vg = make_vec_grid(g, S::V);
    launch_vec_step<L, S, CT>(vg, vec_grid_dims(vg), vec_block_threads(vg), stream, cur, nxt, omega,
                              omega_minus, typename S::Params{});
  } else {
    fluid_step_kernel<L, Real, CT><<<grid_dims(g), block_dims(g), 0, stream>>>(cur, nxt, g, omega,
                                                                           omega_minus);
  }
  return cudaGetLastError();
}

// One step plus the diagnostics of the state it writes (diag.cuh): the
// kernel writes one partial per block, the finalize pass reduces them.
template <class L, class Real, int CT>
cudaError_t launch_fluid_step_diag(const Real* cur, Real* nxt, size_t nx, size_t ny, size_t nz,
                                   Real omega, double speed_limit, double* partials,
                                   size_t pbytes, double* out, cudaStream_t stream) {
  Grid g;
  cudaError_t err = validate_domain(cur == nullptr || nxt == nullptr || partials == nullptr ||
                                        out == nullptr,
                                    1, 1, 1, L::D, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  const size_t need = (size_t)g.blocks() * kDiagPartials * sizeof(double);
  if (pbytes < need) return cudaErrorInvalidValue;
  const size_t bytes = (size_t)L::Q * (size_t)g.plane * sizeof(Real);
  const Span reads[1] = {{cur, bytes}};
  const Span writes[3] = {{nxt, bytes}, {partials, need}, {out, kDiagOut * sizeof(double)}};
  if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  const Real omega_minus = CT == kTRT ? trt_omega_minus<Real>(omega) : Real(0);
  using S = NativeStorage<Real, kVecCells<L, Real>>;
  long long count;
  if (kUseVec<L, Real, CT> && vec_eligible<S>(g, cur, nxt)) {
    const VecGrid vg = make_vec_grid(g, S::V);
    const dim3 grid = vec_grid_dims(vg);
    count = (long long)grid.x * grid.y;  // <= g.blocks(): a vector block spans >= one row block
    fluid_step_vec_kernel<L, S, CT, true><<<grid, vec_block_threads(vg), 0, stream>>>(
        cur, nxt, vg, omega, omega_minus, typename S::Params{}, partials);
  } else {
    count = g.blocks();
    fluid_step_kernel<L, Real, CT, true><<<grid_dims(g), block_dims(g), 0, stream>>>(
        cur, nxt, g, omega, omega_minus, partials);
  }
  err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  return launch_diag_finalize(partials, count, speed_limit, out, stream);
}

template <class Real, int CT>
cudaError_t diag_dispatch_lattice(int lattice, const void* cur, void* nxt, size_t nx, size_t ny,
                                  size_t nz, double omega, double speed_limit, double* partials,
                                  size_t pbytes, double* out, cudaStream_t s) {
  const Real* c = static_cast<const Real*>(cur);
  Real* n = static_cast<Real*>(nxt);
  const Real w = Real(omega);
  switch (lattice) {
    case kD2Q9: return launch_fluid_step_diag<D2Q9, Real, CT>(c, n, nx, ny, nz, w, speed_limit, partials, pbytes, out, s);
    case kD3Q19: return launch_fluid_step_diag<D3Q19, Real, CT>(c, n, nx, ny, nz, w, speed_limit, partials, pbytes, out, s);
    case kD3Q27: return launch_fluid_step_diag<D3Q27, Real, CT>(c, n, nx, ny, nz, w, speed_limit, partials, pbytes, out, s);
    default: return cudaErrorInvalidValue;
  }
}

template <class Real>
cudaError_t diag_dispatch_collision(int lattice, int collision, const void* cur, void* nxt,
                                    size_t nx, size_t ny, size_t nz, double omega,
                                    double speed_limit, double* partials, size_t pbytes,
                                    double* out, cudaStream_t s) {
  switch (collision) {
    case kBGK: return diag_dispatch_lattice<Real, kBGK>(lattice, cur, nxt, nx, ny, nz, omega, speed_limit, partials, pbytes, out, s);
    case kTRT: return diag_dispatch_lattice<Real, kTRT>(lattice, cur, nxt, nx, ny, nz, omega, speed_limit, partials, pbytes, out, s);
    case kMRT: return diag_dispatch_lattice<Real, kMRT>(lattice, cur, nxt, nx, ny, nz, omega, speed_limit, partials, pbytes, out, s);
    case kRLBM: return diag_dispatch_lattice<Real, kRLBM>(lattice, cur, nxt, nx, ny, nz, omega, speed_limit, partials, pbytes, out, s);
    default: return cudaErrorInvalidValue;
  }
}

template <class Real, int CT>
cudaError_t dispatch_lattice(int lattice, const void* cur, void* nxt, size_t nx, size_t ny,
                             size_t nz, double omega, cudaStream_t s) {
  const Real* c = static_cast<const Real*>(cur);
  Real* n = static_cast<Real*>(nxt);
  switch (lattice) {
    case kD2Q9: return launch_fluid_step<D2Q9, Real, CT>(c, n, nx, ny, nz, Real(omega), 1, 1, 1, s);
    case kD3Q19: return launch_fluid_step<D3Q19, Real, CT>(c, n, nx, ny, nz, Real(omega), 1, 1, 1, s);
    case kD3Q27: return launch_fluid_step<D3Q27, Real, CT>(c, n, nx, ny, nz, Real(omega), 1, 1, 1, s);
    default: return cudaErrorInvalidValue;
  }
}

template <class Real>
cudaError_t dispatch_collision(int lattice, int collision, const void* cur, void* nxt, size_t nx,
                               size_t ny, size_t nz, double omega, cudaStream_t s) {
  switch (collision) {
    case kBGK: return dispatch_lattice<Real, kBGK>(lattice, cur, nxt, nx, ny, nz, omega, s);
    case kTRT: return dispatch_lattice<Real, kTRT>(lattice, cur, nxt, nx, ny, nz, omega, s);
    case kMRT: return dispatch_lattice<Real, kMRT>(lattice, cur, nxt, nx, ny, nz, omega, s);
    case kRLBM: return dispatch_lattice<Real, kRLBM>(lattice, cur, nxt, nx, ny, nz, omega, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace lbcube

using namespace lbcube;

#define LBCUBE_STEP_SYMBOL(lat, LAT, real, op, OP)                                                \
  extern "C" int lbm_launch_step_gpu_##lat##_##real##_##op(                                     \
      const real* current_populations, real* next_populations, size_t x_extent,                 \
      size_t y_extent, size_t z_extent, real omega, unsigned block_x, unsigned block_y,         \
      unsigned block_z) {                                                                       \
    return (int)launch_fluid_step<LAT, real, OP>(current_populations, next_populations,        \
                                                 x_extent, y_extent, z_extent, omega, block_x, \
                                                 block_y, block_z, (cudaStream_t)0);            \
  }

#define LBCUBE_STEP_OPS(lat, LAT, real)              \
  LBCUBE_STEP_SYMBOL(lat, LAT, real, bgk, kBGK)      \
  LBCUBE_STEP_SYMBOL(lat, LAT, real, trt, kTRT)      \
  LBCUBE_STEP_SYMBOL(lat, LAT, real, mrt, kMRT)      \
  LBCUBE_STEP_SYMBOL(lat, LAT, real, rlbm, kRLBM)

LBCUBE_STEP_OPS(d2q9, D2Q9, float)
LBCUBE_STEP_OPS(d2q9, D2Q9, double)
LBCUBE_STEP_OPS(d3q19, D3Q19, float)
LBCUBE_STEP_OPS(d3q19, D3Q19, double)
LBCUBE_STEP_OPS(d3q27, D3Q27, float)
LBCUBE_STEP_OPS(d3q27, D3Q27, double)

extern "C" int lbm_step_async(int lattice, int precision, int collision,
                              const void* current_populations, void* next_populations,
                              size_t x_extent, size_t y_extent, size_t z_extent, double omega,
                              void* stream) {
  const cudaStream_t s = as_stream(stream);
  if (precision == LBM_FLOAT)
    return (int)dispatch_collision<float>(lattice, collision, current_populations,
                                          next_populations, x_extent, y_extent, z_extent, omega, s);
  if (precision == LBM_DOUBLE)
    return (int)dispatch_collision<double>(lattice, collision, current_populations,
                                           next_populations, x_extent, y_extent, z_extent, omega,
                                           s);
  return (int)cudaErrorInvalidValue;
}

extern "C" int lbm_step_diagnostics_async(int lattice, int precision, int collision,
                                          const void* current_populations,
                                          void* next_populations, size_t x_extent,
                                          size_t y_extent, size_t z_extent, double omega,
                                          double speed_limit, double* partials,
                                          size_t partials_bytes, double* diagnostics,
                                          void* stream) {
  const cudaStream_t s = as_stream(stream);
  if (precision == LBM_FLOAT)
    return (int)diag_dispatch_collision<float>(lattice, collision, current_populations,
                                               next_populations, x_extent, y_extent, z_extent,
                                               omega, speed_limit, partials, partials_bytes,
                                               diagnostics, s);
  if (precision == LBM_DOUBLE)
    return (int)diag_dispatch_collision<double>(lattice, collision, current_populations,
                                                next_populations, x_extent, y_extent, z_extent,
                                                omega, speed_limit, partials, partials_bytes,
                                                diagnostics, s);
  return (int)cudaErrorInvalidValue;
}
