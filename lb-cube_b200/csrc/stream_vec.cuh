// Vectorised pull collide-stream: V consecutive cells per thread, every
// population row moved as aligned words of V elements (2 to 16 bytes).
//
// Thread t of a row segment owns cells x0 .. x0+V-1 (x0 = V * t). For a
// population with c_x = 0 its V inputs are one aligned word of the source
// row. For c_x = +1 (source x - 1) they are the previous lane's last element
// followed by the first V-1 elements of the thread's own word; for c_x = -1
// (source x + 1) the last V-1 elements followed by the next lane's first
// element. Words are decoded first and the neighbour's decoded value comes
// from a warp shuffle; the lanes at a warp edge or at the periodic x boundary
// load and decode that one element instead. Stores are aligned words. Requires nx % V == 0 and word-aligned
// buffers (the launcher checks and otherwise uses the one-cell kernel). A
// warp never spans two rows (threads along x are a multiple of 32), so the
// lane before an active lane always holds the cells just before it.
//
// The storage format is a policy:
//   NativeStorage<Real, V>  FP32/FP64 populations (bit-identical to the one-cell
//                           kernel: same collision code, only the memory access differs)
//   ShiftedStorage<fmt, V>  16-bit shifted populations decoded to FP32 f
//   DevStorage<fmt, V>      16-bit shifted populations collided as deviations
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstring>
#include <type_traits>

#include "collide.cuh"
#include "collide_dev.cuh"
#include "common.cuh"
#include "diag.cuh"

namespace lbcube {

// A row segment of V elements, moved as one word.
template <class E, int V>
struct RowWord {
  E v[V];
};

// ---- storage policies -------------------------------------------------------
// Each policy decodes a loaded word into V compute values (decode_word), one
// element of a neighbour (decode), encodes V results into a word
// (encode_word) and runs the collision of one cell (collide_cell).
template <class Real, int VEC = 16 / sizeof(Real)>
struct NativeStorage {
  using elem = Real;
  using compute = Real;
  static constexpr int V = VEC;
  static constexpr bool kBudgeted = false;
  struct Params {};
  template <class L, int i>
  __device__ __forceinline__ static compute decode(elem v, const Params&) { return v; }
  template <class L, int i>
  __device__ __forceinline__ static elem encode(compute f, const Params&) { return f; }
  template <class L, int i>
  __device__ __forceinline__ static void decode_word(const RowWord<elem, V>& w, compute (&out)[V],
                                                     const Params&) {
#pragma unroll
    for (int j = 0; j < V; ++j) out[j] = w.v[j];
  }
  template <class L, int i>
  __device__ __forceinline__ static RowWord<elem, V> encode_word(const compute (&in)[V],
                                                                const Params&) {
    RowWord<elem, V> w;
#pragma unroll
    for (int j = 0; j < V; ++j) w.v[j] = in[j];
    return w;
  }
  template <class L, int CT>
  __device__ __forceinline__ static void collide_cell(compute (&f)[L::Q], compute omega,
                                                      compute omega_minus, const Params&) {
    collide<L, compute, CT>(f, omega, omega_minus);
  }
};

// Shifted 16-bit storage of LB populations: the stored code h_i stands for
//   v_i = S (f_i / w_i - rho0)      (the codec of each format, collide_dev.cuh)
// so f_i = w_i (rho0 + v_i / S). Subtracting the rest state w_i rho0 keeps
// only the small deviation (a few 1e-2 of w_i at Mach 0.1), dividing by w_i
// puts every direction on the same scale, and S places that range where the
// format resolves it best. This policy decodes to f and runs the reference
// collision (MRT, RLBM, conversions); DevStorage below collides on v directly.
template <int FMT, int VEC = 4>
struct ShiftedStorage {
  using elem = unsigned short;
  using compute = float;
  static constexpr int V = VEC;  // cells per thread, decoded to FP32 in registers
  static constexpr bool kBudgeted = false;
  struct Params {
    float rho0;
  };
  template <class L, int i>
  __device__ __forceinline__ static compute decode(elem h, const Params& p) {
    constexpr double wd = L::w[i];
    return float(wd) * fmaf(Codec<FMT>::decode(h), 1.0f / Codec<FMT>::S, p.rho0);
  }
  template <class L, int i>
  __device__ __forceinline__ static elem encode(compute f, const Params& p) {
    constexpr double wd = L::w[i];
    return Codec<FMT>::encode((f * float(1.0 / wd) - p.rho0) * Codec<FMT>::S);
  }
  template <class L, int i>
  __device__ __forceinline__ static void decode_word(const RowWord<elem, V>& w, compute (&out)[V],
                                                     const Params& p) {
#pragma unroll
    for (int j = 0; j < V; ++j) out[j] = decode<L, i>(w.v[j], p);
  }
  template <class L, int i>
  __device__ __forceinline__ static RowWord<elem, V> encode_word(const compute (&in)[V],
                                                                const Params& p) {
    RowWord<elem, V> w;
#pragma unroll
    for (int j = 0; j < V; ++j) w.v[j] = encode<L, i>(in[j], p);
    return w;
  }
  template <class L, int CT>
  __device__ __forceinline__ static void collide_cell(compute (&f)[L::Q], compute omega,
                                                      compute omega_minus, const Params&) {
    collide<L, compute, CT>(f, omega, omega_minus);
  }
};

// 16-bit storage whose collision runs on the stored deviations (BGK, TRT).
template <int FMT, int VEC = 4>
struct DevStorage {
  static_assert(VEC % 2 == 0, "codes are converted in pairs");
  using elem = unsigned short;
  using compute = float;
  static constexpr int V = VEC;
  static constexpr bool kBudgeted = true;
  struct Params {
    float rho0;
  };
  template <class L, int i>
  __device__ __forceinline__ static compute decode(elem h, const Params&) {
    return Codec<FMT>::decode(h);
  }
  template <class L, int i>
  __device__ __forceinline__ static elem encode(compute v, const Params&) {
    return Codec<FMT>::encode(v);
  }
  // V is even: the word holds V/2 32-bit pairs, converted pairwise.
  template <class L, int i>
  __device__ __forceinline__ static void decode_word(const RowWord<elem, V>& w, compute (&out)[V],
                                                     const Params&) {
    unsigned int u[V / 2];
    memcpy(u, &w, sizeof(u));
#pragma unroll
    for (int k = 0; k < V / 2; ++k) {
      const float2 d = Codec<FMT>::decode2(u[k]);
      out[2 * k] = d.x;
      out[2 * k + 1] = d.y;
    }
  }
  template <class L, int i>
  __device__ __forceinline__ static RowWord<elem, V> encode_word(const compute (&in)[V],
                                                                const Params&) {
    unsigned int u[V / 2];
#pragma unroll
    for (int k = 0; k < V / 2; ++k) u[k] = Codec<FMT>::encode2(in[2 * k], in[2 * k + 1]);
    RowWord<elem, V> w;
    memcpy(&w, u, sizeof(u));
    return w;
  }
  __device__ __forceinline__ static float2 decode_pair(unsigned int w) { return Codec<FMT>::decode2(w); }
  __device__ __forceinline__ static unsigned int encode_pair(float a, float b) {
    return Codec<FMT>::encode2(a, b);
  }
  template <class L, int CT>
  __device__ __forceinline__ static void collide_cell(compute (&v)[L::Q], compute omega,
                                                      compute omega_minus, const Params& p) {
    static_assert(CT == kBGK || CT == kTRT || (CT == kMRT && L::Q != 27),
                  "deviation-space collision is BGK, TRT, or D2Q9 / D3Q19 MRT");
    if constexpr (CT == kMRT) collide_dev_mrt<L, FMT>(v, omega, p.rho0);
    else collide_dev<L, CT, FMT>(v, omega, omega_minus, p.rho0);
  }
};

// ---- word access ------------------------------------------------------------
template <int B> struct WordOf;
template <> struct WordOf<2> { using type = unsigned short; };
template <> struct WordOf<4> { using type = unsigned int; };
template <> struct WordOf<8> { using type = uint2; };
template <> struct WordOf<16> { using type = uint4; };

template <class E, int V>
__device__ __forceinline__ RowWord<E, V> load_word(const E* __restrict__ p) {
  using W = typename WordOf<sizeof(E) * V>::type;
  const W w = __ldg(reinterpret_cast<const W*>(p));
  RowWord<E, V> r;
  memcpy(&r, &w, sizeof(W));
  return r;
}

template <class E, int V>
__device__ __forceinline__ void store_word(E* __restrict__ p, const RowWord<E, V>& r) {
  using W = typename WordOf<sizeof(E) * V>::type;
  W w;
  memcpy(&w, &r, sizeof(W));
  *reinterpret_cast<W*>(p) = w;
}

// Launch shape of the vectorised kernel: TX threads along x (a multiple of 32,
// at most kThreads) cover TX * V cells of a row; TY = kThreads / TX rows per
// block. grid.x = xblocks * ceil(ny / TY), grid.y = nz.
struct VecGrid {
  Grid g;
  int tx, ty, xblocks, yblocks;
  int z0;  // first plane of the launch (grid.y planes from here); 0 for a whole box
};

inline VecGrid make_vec_grid(const Grid& g, int V) {
  VecGrid v;
  v.g = g;
  const int lanes_needed = (g.nx / V + 31) / 32 * 32;
  v.tx = lanes_needed < kThreads ? lanes_needed : kThreads;
  v.ty = kThreads / v.tx;
  v.xblocks = (g.nx / V + v.tx - 1) / v.tx;
  v.yblocks = (g.ny + v.ty - 1) / v.ty;
  v.z0 = 0;
  return v;
}

// ---- z-slab decomposition ---------------------------------------------------
// A rank owns planes [0, nz) of its slab; the populations that cross a slab
// face arrive in halo planes instead of the periodic wrap. Population i with
// c_z = +1 is pulled from z - 1: at z = 0 it is read from halo_lo; c_z = -1 at
// z = nz - 1 from halo_hi. A halo (or send) buffer holds the crossing
// populations of one face in ascending i: [zslot, ny, nx].
template <class L>
__host__ __device__ constexpr int zslot(int i) {
  int k = 0;
  for (int j = 0; j < i; ++j) k += L::c[j][2] == L::c[i][2] ? 1 : 0;
  return k;
}
template <class L>
__host__ __device__ constexpr int zcount() {
  int k = 0;
  for (int j = 0; j < L::Q; ++j) k += L::c[j][2] > 0 ? 1 : 0;
  return k;
}

template <class E>
struct SlabArgs {
  const E* halo_lo;  // c_z = +1 populations of the lower neighbour's top plane
  const E* halo_hi;  // c_z = -1 populations of the upper neighbour's bottom plane
  E* send_lo;        // this step's c_z = -1 populations of plane 0 (for the lower neighbour)
  E* send_hi;        // this step's c_z = +1 populations of plane nz - 1 (for the upper one)
  int z_begin;       // first plane of this launch
  int z_step = 1;    // planes between consecutive blockIdx.y (both faces in one launch: nz - 1)
};

// Gathers the Q populations of V cells (x0 .. x0+V-1, row y, slice z) and
// decodes them. All 32 lanes of every warp must call it (shuffles); inactive
// lanes (x0 >= nx or y >= ny) load nothing and contribute nothing.
template <class L, class S, bool SLAB = false>
__device__ __forceinline__ void gather_vec(const typename S::elem* __restrict__ cur, const Grid& g,
                                           int x0, int y, int z, bool active,
                                           const typename S::Params& p,
                                           typename S::compute (&f)[S::V][L::Q],
                                           const SlabArgs<typename S::elem>& slab = {}) {
  using E = typename S::elem;
  constexpr int V = S::V;
  const int lane = threadIdx.x & 31;
  const int ym = y == 0 ? g.ny - 1 : y - 1, yp = y == g.ny - 1 ? 0 : y + 1;
  const int zm = z == 0 ? g.nz - 1 : z - 1, zp = z == g.nz - 1 ? 0 : z + 1;
  const size_t plane = (size_t)g.plane;
  const bool left_edge = lane == 0 || x0 == 0;
  const bool right_edge = lane == 31 || x0 + V == g.nx;
  const int xl = x0 == 0 ? g.nx - 1 : x0 - 1;
  const int xr = x0 + V == g.nx ? 0 : x0 + V;
  // In-plane row offsets fit in 32 bits (a plane has at most 2^31 - 1 cells,
  // checked at launch): 64-bit arithmetic only for the plane base cur + plane i,
  // which is the same for every thread.
  const int zoff[3] = {zm * g.ny, z * g.ny, zp * g.ny};
  const int ysel[3] = {ym, y, yp};
  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
    const int sy = cy == 0 ? y : (cy > 0 ? ym : yp);
    const E* row;
    if constexpr (SLAB && cz > 0) {
      row = z == 0 ? slab.halo_lo + (size_t)(zslot<L>(i) * g.ny + sy) * g.nx
                   : cur + plane * i + (size_t)((z - 1) * g.ny + sy) * g.nx;
    } else if constexpr (SLAB && cz < 0) {
      row = z == g.nz - 1 ? slab.halo_hi + (size_t)(zslot<L>(i) * g.ny + sy) * g.nx
                          : cur + plane * i + (size_t)((z + 1) * g.ny + sy) * g.nx;
    } else {
      const int off = (zoff[cz > 0 ? 0 : (cz < 0 ? 2 : 1)] + ysel[cy > 0 ? 0 : (cy < 0 ? 2 : 1)]) * g.nx;
      row = (cur + plane * i) + off;
    }
    using R = typename S::compute;
    R val[V];
    if (active) {
      S::template decode_word<L, i>(load_word<E, V>(row + x0), val, p);
    } else {
#pragma unroll
      for (int j = 0; j < V; ++j) val[j] = R(0);
    }
    if constexpr (cx == 0) {
#pragma unroll
      for (int j = 0; j < V; ++j) f[j][i] = val[j];
    } else if constexpr (cx > 0) {  // source x - 1
      R left = __shfl_up_sync(0xffffffffu, val[V - 1], 1);
      if (active && left_edge) left = S::template decode<L, i>(__ldg(row + xl), p);
      f[0][i] = left;
#pragma unroll
      for (int j = 1; j < V; ++j) f[j][i] = val[j - 1];
    } else {  // source x + 1
      R right = __shfl_down_sync(0xffffffffu, val[0], 1);
      if (active && right_edge) right = S::template decode<L, i>(__ldg(row + xr), p);
#pragma unroll
      for (int j = 0; j < V - 1; ++j) f[j][i] = val[j + 1];
      f[V - 1][i] = right;
    }
  });
}

template <class L, class S, bool SLAB = false>
__device__ __forceinline__ void store_vec(typename S::elem* __restrict__ nxt, const Grid& g, int x0,
                                          int y, int z, const typename S::Params& p,
                                          const typename S::compute (&f)[S::V][L::Q],
                                          const SlabArgs<typename S::elem>& slab = {}) {
  using E = typename S::elem;
  constexpr int V = S::V;
  const size_t plane = (size_t)g.plane;
  const int cell = (z * g.ny + y) * g.nx + x0;  // < plane <= 2^31 - 1
  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr int cz = L::c[i][2];
    typename S::compute col[V];
#pragma unroll
    for (int j = 0; j < V; ++j) col[j] = f[j][i];
    const RowWord<E, V> w = S::template encode_word<L, i>(col, p);
    store_word<E, V>((nxt + plane * i) + cell, w);
    if constexpr (SLAB && cz > 0) {  // leaves through the top face
      if (z == g.nz - 1) store_word<E, V>(slab.send_hi + (size_t)(zslot<L>(i) * g.ny + y) * g.nx + x0, w);
    } else if constexpr (SLAB && cz < 0) {  // leaves through the bottom face
      if (z == 0) store_word<E, V>(slab.send_lo + (size_t)(zslot<L>(i) * g.ny + y) * g.nx + x0, w);
    }
  });
}

// DIAG: also reduce the diagnostics of the new state (diag.cuh) over the
// block into partials[block_linear() * kDiagPartials ..]. In the pull scheme
// the populations a thread writes are exactly the next buffer's populations of
// its own cells, so this costs no memory traffic. Native storage only.
// SLAB: one launch over planes slab.z_begin + k * slab.z_step (k < gridDim.y)
// of a z-slab, with halo planes at the slab faces (see SlabArgs).
template <class L, class S, int CT, bool DIAG, bool SLAB>
__device__ __forceinline__ void fluid_step_vec_body(const typename S::elem* __restrict__ cur,
                                                    typename S::elem* __restrict__ nxt,
                                                    const VecGrid& vg, typename S::compute omega,
                                                    typename S::compute omega_minus,
                                                    const typename S::Params& p,
                                                    double* __restrict__ partials,
                                                    const SlabArgs<typename S::elem>& slab) {
  pdl_enter();
  using R = typename S::compute;
  constexpr int V = S::V;
  const Grid& g = vg.g;
  const int yb = blockIdx.x / vg.xblocks;
  const int xb = blockIdx.x - yb * vg.xblocks;
  const int x0 = (xb * vg.tx + (int)(threadIdx.x % vg.tx)) * V;
  const int y = yb * vg.ty + (int)(threadIdx.x / vg.tx);
  const int z = SLAB ? slab.z_begin + (int)blockIdx.y * slab.z_step : vg.z0 + (int)blockIdx.y;
  const bool active = x0 < g.nx && y < g.ny;
  R f[V][L::Q];
  gather_vec<L, S, SLAB>(cur, g, x0, y < g.ny ? y : 0, z, active, p, f, slab);
  if constexpr (DIAG) {
    static_assert(std::is_same_v<typename S::elem, R>, "diagnostics need native storage");
    DiagAcc acc;
    if (active) {
#pragma unroll
      for (int j = 0; j < V; ++j) S::template collide_cell<L, CT>(f[j], omega, omega_minus, p);
      store_vec<L, S>(nxt, g, x0, y, z, p, f);
#pragma unroll
      for (int j = 0; j < V; ++j) diag_cell<L>(f[j], acc);
    }
    diag_block_to(acc, partials + block_linear() * kDiagPartials);
  } else {
    if (!active) return;
#pragma unroll
    for (int j = 0; j < V; ++j) S::template collide_cell<L, CT>(f[j], omega, omega_minus, p);
    store_vec<L, S, SLAB>(nxt, g, x0, y, z, p, f, slab);
  }
}

template <class L, class S, int CT, bool DIAG = false, bool SLAB = false>
__global__ void __launch_bounds__(kThreads)
    fluid_step_vec_kernel(const typename S::elem* __restrict__ cur,
                          typename S::elem* __restrict__ nxt, VecGrid vg,
                          typename S::compute omega, typename S::compute omega_minus,
                          typename S::Params p, double* __restrict__ partials = nullptr,
                          SlabArgs<typename S::elem> slab = {}) {
  fluid_step_vec_body<L, S, CT, DIAG, SLAB>(cur, nxt, vg, omega, omega_minus, p, partials, slab);
}

// The plain step on 16-bit storage with a register budget: at least
// kShiftedMinBlocks blocks of kThreads per SM. Four cells of 19 populations per
// thread leave the compiler free to interleave the cells' collisions up to
// 128 registers (4 blocks per SM), which an issue-bound kernel pays for in
// latency it cannot hide.
#ifndef LBCUBE_SHIFTED_MIN_BLOCKS
#define LBCUBE_SHIFTED_MIN_BLOCKS 5
#endif
constexpr int kShiftedMinBlocks = LBCUBE_SHIFTED_MIN_BLOCKS;

template <class L, class S, int CT>
__global__ void __launch_bounds__(kThreads, kShiftedMinBlocks)
    fluid_step_vec16_kernel(const typename S::elem* __restrict__ cur,
                            typename S::elem* __restrict__ nxt, VecGrid vg,
                            typename S::compute omega, typename S::compute omega_minus,
                            typename S::Params p) {
  fluid_step_vec_body<L, S, CT, false, false>(cur, nxt, vg, omega, omega_minus, p, nullptr, {});
}

// Launches the plain vectorised step. (Register budgets, i.e. launch bounds
// with a minimum block count, were timed at 4..8 blocks per SM for every
// lattice, precision and operator of the native storage; where they won, for
// FP32 D3Q19 MRT and RLBM, the one-cell kernel (step_cell.cuh) won by more and
// now runs those. An explicit count of 1 is not the compiler's default: it
// lets the allocation grow, e.g. 64 -> 94 registers for the FP32 D3Q19 TRT
// step.) 16-bit storage colliding on the deviations runs the budgeted kernel
// above for D2Q9 and D3Q19 (D3Q27 and the decoded RLBM spill under it).
template <class L, class S, int CT>
inline void launch_vec_step(const VecGrid& vg, dim3 grid, unsigned threads, cudaStream_t stream,
                            const typename S::elem* cur, typename S::elem* nxt,
                            typename S::compute omega, typename S::compute omega_minus,
                            const typename S::Params& p) {
  // programmatic dependent launches (pdl_enter opens the body)
  if constexpr (S::kBudgeted && L::Q <= 19)
    launch_pdl(fluid_step_vec16_kernel<L, S, CT>, grid, dim3(threads), 0, stream, cur, nxt, vg, omega,
               omega_minus, p);
  else
    launch_pdl(fluid_step_vec_kernel<L, S, CT, false, false>, grid, dim3(threads), 0, stream, cur, nxt,
               vg, omega, omega_minus, p, (double*)nullptr, SlabArgs<typename S::elem>{});
}

template <class S>
inline bool vec_eligible(const Grid& g, const void* a, const void* b) {
  constexpr uintptr_t align = sizeof(typename S::elem) * S::V;
  return g.nx % S::V == 0 && ((uintptr_t)a % align) == 0 && ((uintptr_t)b % align) == 0;
}

inline dim3 vec_grid_dims(const VecGrid& v) {
  return dim3((unsigned)(v.xblocks * v.yblocks), (unsigned)v.g.nz, 1);
}

// Threads per block of the vectorised kernel: exactly tx * ty (<= kThreads).
inline unsigned vec_block_threads(const VecGrid& v) { return (unsigned)(v.tx * v.ty); }

}  // namespace lbcube
