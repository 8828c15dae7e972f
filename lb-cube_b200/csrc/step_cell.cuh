// One-cell-per-thread fused pull-scheme collide-stream step for D2Q9 / D3Q19 /
// D3Q27 fluids, and the rule that picks it over the vectorised kernel
// (stream_vec.cuh); shared by the periodic step (fluid_step.cu) and the
// interior planes of the slab step (slab.cu).
//
// Replaces kernel_step (src/lattice_cuda.cu:149-213). One thread owns one
// destination cell: it gathers the Q incoming populations f_i(x - c_i) from
// the current buffer (periodic wrap by compare-and-select on 32-bit
// coordinates instead of the reference's 64-bit modulo), collides in registers
// and writes the Q results to the next buffer at its own cell. A warp covers 32
// consecutive x cells, so each of the Q gathers and Q stores is one coalesced
// 128-byte row segment (shifted by at most one element for c_x != 0, which the
// L1/L2 sector reuse absorbs). Planes g.z0 + k * g.zs (k < gridDim.y) are stepped.
#pragma once
#include "collide.cuh"
#include "common.cuh"
#include "diag.cuh"

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
  pdl_enter();
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

// The Q population planes of a buffer as separate base pointers, passed as
// kernel parameters (read from the constant bank): every gather and store is
// then one wide multiply-add of a 32-bit in-plane offset, where base + plane * i
// otherwise costs 64-bit arithmetic per population. Used for MRT on D3Q19 and
// D3Q27, where it measured faster (A/B, same box, bit-identical outputs:
// D3Q19 FP64 MRT 0.94 -> 0.98 of the copy bandwidth at 256^3, D3Q27 FP32 MRT
// 0.56 -> 0.585 at 224^3; D3Q19 FP32 MRT and D3Q27 BGK level; RLBM 1.5-7 % and
// D2Q9 MRT 2.5 % slower, so those keep fluid_step_kernel). LBCUBE_PLANE_PTRS = 0
// turns it off.
#ifndef LBCUBE_PLANE_PTRS
#define LBCUBE_PLANE_PTRS 1
#endif
template <class L, class Real, int CT>
constexpr bool kUsePlanes = LBCUBE_PLANE_PTRS != 0 && CT == kMRT && L::Q >= 19;
template <class Real, int Q>
struct Planes {
  Real* p[Q];
};
template <class Real, int Q>
inline Planes<Real, Q> planes_of(Real* base, const Grid& g) {
  Planes<Real, Q> r;
  for (int i = 0; i < Q; ++i) r.p[i] = base + (size_t)g.plane * i;
  return r;
}

// fluid_step_kernel (no diagnostics) on plane pointers: the same gather,
// collision and stores, so the same bits.
template <class L, class Real, int CT>
__global__ void __launch_bounds__(kThreads)
    fluid_step_planes_kernel(const Planes<const Real, L::Q> cur, const Planes<Real, L::Q> nxt,
                             Grid g, Real omega, Real omega_minus) {
  pdl_enter();
  int x, y, z;
  if (!cell_of(g, x, y, z)) return;
  const int xm = x == 0 ? g.nx - 1 : x - 1, xp = x == g.nx - 1 ? 0 : x + 1;
  const int ym = y == 0 ? g.ny - 1 : y - 1, yp = y == g.ny - 1 ? 0 : y + 1;
  const int zm = z == 0 ? g.nz - 1 : z - 1, zp = z == g.nz - 1 ? 0 : z + 1;
  Real f[L::Q];
  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
    const int sx = cx == 0 ? x : (cx > 0 ? xm : xp);
    const int sy = cy == 0 ? y : (cy > 0 ? ym : yp);
    const int sz = cz == 0 ? z : (cz > 0 ? zm : zp);
    f[i] = __ldg(cur.p[i] + ((sz * g.ny + sy) * g.nx + sx));
  });
  collide<L, Real, CT>(f, omega, omega_minus);
  const int cell = (z * g.ny + y) * g.nx + x;
  static_for<L::Q>([&](auto I) { nxt.p[LB_I(I)][cell] = f[LB_I(I)]; });
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
// 2-5 % and FP64 4-18 %. Two cells per thread double the live populations
// (D3Q19 FP32 MRT: 80 registers against 40); at one cell per thread (D3Q27
// FP32, FP64) both kernels hold the same values, and they differ in the
// gather: the vectorised kernel exchanges x-neighbours by warp shuffles with
// extra loads at the warp edges, the one-cell kernel loads every neighbour
// directly (overlapping row segments, served by L1).
// The slab step follows the same rule on its interior planes; its face planes
// and the 16-bit storage keep the vectorised kernel.
template <class L, class Real>
constexpr int kVecCells = (sizeof(Real) == 4 && L::Q != 27) ? 2 : 1;
template <class L, class Real, int CT>
constexpr bool kUseVec = sizeof(Real) == 4 && L::Q == 19 && (CT == kBGK || CT == kTRT);

}  // namespace lbcube
