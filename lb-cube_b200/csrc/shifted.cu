// Shifted 16-bit population storage (FP16, BF16, E3M12 or Q15) with FP32
// collision.
//
// An extension with no reference counterpart. Populations are stored as codes
// of v_i = S (f_i / w_i - rho0) in 16 bits (collide_dev.cuh), halving the bytes
// per lattice update (D3Q19: 76 B instead of 152 B). BGK and TRT collide on
// the deviations v directly (DevStorage); MRT and RLBM decode to f, run the
// reference operator and re-encode (ShiftedStorage). Rounding to 16 bits is to
// nearest. Encode/decode kernels convert between FP32/FP64 populations and the
// 16-bit form.
#include <algorithm>
#include <type_traits>

#include "collide.cuh"
#include "common.cuh"
#include "stream_staged.cuh"
#include "stream_vec.cuh"
#include "../../include/lbcube_b200.h"

namespace lbcube {

// Cells per thread of the 16-bit kernels: four (8-byte words of codes).
#ifndef LBCUBE_SHIFTED_CELLS
#define LBCUBE_SHIFTED_CELLS 4
#endif
template <int FMT>
constexpr int kShiftedCells = LBCUBE_SHIFTED_CELLS;

// The plain step on the deviation-collision formats goes through the
// row-staged kernel (stream_staged.cuh) wherever its requirements hold.
#ifndef LBCUBE_SHIFTED_STAGED
#define LBCUBE_SHIFTED_STAGED 1
#endif
constexpr bool kShiftedStaged = LBCUBE_SHIFTED_STAGED != 0;

// BGK, TRT and the D2Q9 / D3Q19 MRT collide on the stored deviations; D3Q27
// MRT and RLBM decode to f and run the reference operator.
template <class L, int FMT, int CT>
using ShiftedPolicy =
    std::conditional_t<CT == kBGK || CT == kTRT || (CT == kMRT && L::Q != 27),
                       DevStorage<FMT, kShiftedCells<FMT>>,
                       ShiftedStorage<FMT, kShiftedCells<FMT>>>;

template <class L, int FMT, int CT>
cudaError_t launch_shifted_step(const void* cur, void* nxt, size_t nx, size_t ny, size_t nz,
                                float omega, float rho0, cudaStream_t stream) {
  using S = ShiftedPolicy<L, FMT, CT>;
  Grid g;
  cudaError_t err = validate_domain(cur == nullptr || nxt == nullptr, 1, 1, 1, L::D, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  const size_t bytes = (size_t)L::Q * g.plane * sizeof(typename S::elem);
  const Span reads[1] = {{cur, bytes}};
  const Span writes[1] = {{nxt, bytes}};
  if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  // the public contract for every format: x_extent a multiple of 4, buffers
  // 8-byte aligned (covers the word shape of both cell counts)
  if (g.nx % 4 != 0 || (uintptr_t)cur % 8 != 0 || (uintptr_t)nxt % 8 != 0)
    return cudaErrorInvalidValue;
  if (!vec_eligible<S>(g, cur, nxt)) return cudaErrorInvalidValue;  // nx % V, word alignment
  const float omega_minus = CT == kTRT ? trt_omega_minus<float>(omega) : 0.0f;
  if constexpr (kShiftedStaged && S::kBudgeted && S::V == 4 && L::Q <= 19) {
    if (staged_eligible<L>(g, cur, nxt))
      return launch_staged_step<L, S, CT>(g, stream, static_cast<const unsigned short*>(cur),
                                          static_cast<unsigned short*>(nxt), omega, omega_minus,
                                          typename S::Params{rho0});
  }
  const VecGrid vg = make_vec_grid(g, S::V);
  launch_vec_step<L, S, CT>(vg, vec_grid_dims(vg), vec_block_threads(vg), stream,
                            static_cast<const unsigned short*>(cur),
                            static_cast<unsigned short*>(nxt), omega,
                            omega_minus, typename S::Params{rho0});
  return cudaGetLastError();
}

template <class L, int FMT>
cudaError_t shifted_by_collision(int collision, const void* cur, void* nxt, size_t nx, size_t ny,
                                 size_t nz, float omega, float rho0, cudaStream_t s) {
  switch (collision) {
    case kBGK: return launch_shifted_step<L, FMT, kBGK>(cur, nxt, nx, ny, nz, omega, rho0, s);
    case kTRT: return launch_shifted_step<L, FMT, kTRT>(cur, nxt, nx, ny, nz, omega, rho0, s);
    case kMRT: return launch_shifted_step<L, FMT, kMRT>(cur, nxt, nx, ny, nz, omega, rho0, s);
    case kRLBM: return launch_shifted_step<L, FMT, kRLBM>(cur, nxt, nx, ny, nz, omega, rho0, s);
    default: return cudaErrorInvalidValue;
  }
}

template <int FMT>
cudaError_t shifted_by_lattice(int lattice, int collision, const void* cur, void* nxt, size_t nx,
                               size_t ny, size_t nz, float omega, float rho0, cudaStream_t s) {
  switch (lattice) {
    case kD2Q9: return shifted_by_collision<D2Q9, FMT>(collision, cur, nxt, nx, ny, nz, omega, rho0, s);
    case kD3Q19: return shifted_by_collision<D3Q19, FMT>(collision, cur, nxt, nx, ny, nz, omega, rho0, s);
    case kD3Q27: return shifted_by_collision<D3Q27, FMT>(collision, cur, nxt, nx, ny, nz, omega, rho0, s);
    default: return cudaErrorInvalidValue;
  }
}

// ---- z-slab form -----------------------------------------------------------------
// One step of planes [z_begin, z_end) of a z-slab of a box on 16-bit storage:
// populations crossing a face are pulled from halo buffers of codes and the
// leaving codes stored into send buffers (layout of lbm_slab_face_elems). Where
// the row-staged kernel applies it steps every plane of the range, its bulk
// copies reading the halo rows at the faces, so a box stepped as slabs gives
// the bits of the box stepped whole; otherwise the vectorised kernel steps the
// interior planes and its SLAB form the face planes.
template <class L, int FMT, int CT>
cudaError_t launch_shifted_slab_step(const void* cur_v, void* nxt_v, size_t nx, size_t ny,
                                     size_t nz, float omega, float rho0, const void* hl_v,
                                     const void* hh_v, void* sl_v, void* sh_v, size_t z_begin,
                                     size_t z_end, cudaStream_t stream) {
  using S = ShiftedPolicy<L, FMT, CT>;
  using E = unsigned short;
  const E* cur = static_cast<const E*>(cur_v);
  E* nxt = static_cast<E*>(nxt_v);
  const E *hl = static_cast<const E*>(hl_v), *hh = static_cast<const E*>(hh_v);
  E *sl = static_cast<E*>(sl_v), *sh = static_cast<E*>(sh_v);
  Grid g;
  cudaError_t err = validate_domain(cur == nullptr || nxt == nullptr, 1, 1, 1, 3, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  if (L::D != 3 || z_begin >= z_end || z_end > nz) return cudaErrorInvalidValue;
  const bool lo_face = z_begin == 0, hi_face = z_end == nz;
  if ((lo_face && (hl == nullptr || sl == nullptr)) || (hi_face && (hh == nullptr || sh == nullptr)))
    return cudaErrorInvalidDevicePointer;
  if (nz == 1 && (hl == nullptr || hh == nullptr || sl == nullptr || sh == nullptr))
    return cudaErrorInvalidDevicePointer;
  const size_t bytes = (size_t)L::Q * g.plane * sizeof(E);
  const size_t hbytes = (size_t)zcount<L>() * g.ny * g.nx * sizeof(E);
  const Span reads[3] = {{cur, bytes}, {hl, hl ? hbytes : 0}, {hh, hh ? hbytes : 0}};
  const Span writes[3] = {{nxt, bytes}, {sl, sl ? hbytes : 0}, {sh, sh ? hbytes : 0}};
  if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  // the public contract of the 16-bit step (x_extent a multiple of 4, 8-byte
  // aligned buffers), face buffers included
  if (g.nx % 4 != 0 || !vec_eligible<S>(g, cur, nxt)) return cudaErrorInvalidValue;
  for (const void* q : {hl_v, hh_v, (const void*)sl, (const void*)sh})
    if ((uintptr_t)q % 8 != 0) return cudaErrorInvalidValue;
  const float omega_minus = CT == kTRT ? trt_omega_minus<float>(omega) : 0.0f;
  const typename S::Params p{rho0};
  const SlabArgs<E> faces{hl, hh, sl, sh, 0};
  if constexpr (kShiftedStaged && S::kBudgeted && S::V == 4 && L::Q <= 19) {
    bool faces16 = true;
    for (const void* q : {hl_v, hh_v, (const void*)sl, (const void*)sh})
      faces16 = faces16 && (uintptr_t)q % 16 == 0;
    if (faces16 && staged_eligible<L>(g, cur, nxt))
      return launch_staged_step<L, S, CT, true>(g, stream, cur, nxt, omega, omega_minus, p,
                                                (int)z_begin, (int)z_end, faces);
  }
  VecGrid vg = make_vec_grid(g, S::V);
  const size_t ib = std::max<size_t>(z_begin, 1), ie = std::min<size_t>(z_end, nz - 1);
  if (ib < ie) {
    vg.z0 = (int)ib;
    dim3 grid = vec_grid_dims(vg);
    grid.y = (unsigned)(ie - ib);
    launch_vec_step<L, S, CT>(vg, grid, vec_block_threads(vg), stream, cur, nxt, omega, omega_minus, p);
    vg.z0 = 0;
  }
  // `count` face planes from z, `step` apart (both faces in one launch where
  // the range has both)
  auto face = [&](size_t z, unsigned count, int step) {
    dim3 grid = vec_grid_dims(vg);
    grid.y = count;
    SlabArgs<E> f = faces;
    f.z_begin = (int)z;
    f.z_step = step;
    launch_pdl(fluid_step_vec_kernel<L, S, CT, false, true>, grid, dim3(vec_block_threads(vg)), 0, stream,
               cur, nxt, vg, omega, omega_minus, p, (double*)nullptr, f);
  };
  if (lo_face && hi_face && nz > 1) {
    face(0, 2, (int)nz - 1);
  } else {
    if (lo_face) face(0, 1, 1);
    if (hi_face && nz > 1) face(nz - 1, 1, 1);
  }
  return cudaGetLastError();
}

template <class L, int FMT>
cudaError_t shifted_slab_by_collision(int collision, const void* cur, void* nxt, size_t nx,
                                      size_t ny, size_t nz, float omega, float rho0, const void* hl,
                                      const void* hh, void* sl, void* sh, size_t z0, size_t z1,
                                      cudaStream_t s) {
  switch (collision) {
    case kBGK: return launch_shifted_slab_step<L, FMT, kBGK>(cur, nxt, nx, ny, nz, omega, rho0, hl, hh, sl, sh, z0, z1, s);
    case kTRT: return launch_shifted_slab_step<L, FMT, kTRT>(cur, nxt, nx, ny, nz, omega, rho0, hl, hh, sl, sh, z0, z1, s);
    case kMRT: return launch_shifted_slab_step<L, FMT, kMRT>(cur, nxt, nx, ny, nz, omega, rho0, hl, hh, sl, sh, z0, z1, s);
    case kRLBM: return launch_shifted_slab_step<L, FMT, kRLBM>(cur, nxt, nx, ny, nz, omega, rho0, hl, hh, sl, sh, z0, z1, s);
    default: return cudaErrorInvalidValue;
  }
}

template <int FMT>
cudaError_t shifted_slab_by_lattice(int lattice, int collision, const void* cur, void* nxt,
                                    size_t nx, size_t ny, size_t nz, float omega, float rho0,
                                    const void* hl, const void* hh, void* sl, void* sh, size_t z0,
                                    size_t z1, cudaStream_t s) {
  switch (lattice) {
    case kD3Q19: return shifted_slab_by_collision<D3Q19, FMT>(collision, cur, nxt, nx, ny, nz, omega, rho0, hl, hh, sl, sh, z0, z1, s);
    case kD3Q27: return shifted_slab_by_collision<D3Q27, FMT>(collision, cur, nxt, nx, ny, nz, omega, rho0, hl, hh, sl, sh, z0, z1, s);
    default: return cudaErrorInvalidValue;
  }
}

// ---- conversions --------------------------------------------------------------
// grid.y = population i (its weight w_i is a compile-time constant of the
// block's branch), grid-stride over the cells of that plane.
template <class L, int FMT, class Real, bool ENCODE>
__global__ void __launch_bounds__(256)
    convert_kernel(const void* __restrict__ in, void* __restrict__ out, long long plane,
                   float rho0) {
  using S = ShiftedStorage<FMT>;
  const typename S::Params p{rho0};
  const int i = (int)blockIdx.y;
  static_for<L::Q>([&](auto I) {
    constexpr int q = LB_I(I);
    if (q != i) return;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < plane;
         c += (long long)gridDim.x * blockDim.x) {
      const long long e = (long long)q * plane + c;
      if constexpr (ENCODE) {
        const float f = (float)static_cast<const Real*>(in)[e];
        static_cast<unsigned short*>(out)[e] = S::template encode<L, q>(f, p);
      } else {
        const float f = S::template decode<L, q>(static_cast<const unsigned short*>(in)[e], p);
        static_cast<Real*>(out)[e] = (Real)f;
      }
    }
  });
}

// FP32 fields whose planes are a multiple of 4 cells, both buffers 16-byte
// aligned: four cells per thread and iteration (one 16-byte load or store of
// FP32 values, one 8-byte store or load of codes). Same per-element codec.
template <class L, int FMT, bool ENCODE>
__global__ void __launch_bounds__(256)
    convert4_kernel(const void* __restrict__ in, void* __restrict__ out, long long plane,
                    float rho0) {
  using S = ShiftedStorage<FMT>;
  const typename S::Params p{rho0};
  const int i = (int)blockIdx.y;
  const long long quads = plane / 4;
  static_for<L::Q>([&](auto I) {
    constexpr int q = LB_I(I);
    if (q != i) return;
    const long long base = (long long)q * quads;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < quads;
         c += (long long)gridDim.x * blockDim.x) {
      if constexpr (ENCODE) {
        const float4 f = __ldg(static_cast<const float4*>(in) + base + c);
        ushort4 h;
        h.x = S::template encode<L, q>(f.x, p);
        h.y = S::template encode<L, q>(f.y, p);
        h.z = S::template encode<L, q>(f.z, p);
        h.w = S::template encode<L, q>(f.w, p);
        static_cast<ushort4*>(out)[base + c] = h;
      } else {
        const ushort4 h = __ldg(static_cast<const ushort4*>(in) + base + c);
        float4 f;
        f.x = S::template decode<L, q>(h.x, p);
        f.y = S::template decode<L, q>(h.y, p);
        f.z = S::template decode<L, q>(h.z, p);
        f.w = S::template decode<L, q>(h.w, p);
        static_cast<float4*>(out)[base + c] = f;
      }
    }
  });
}

template <class L, int FMT, bool ENCODE>
cudaError_t launch_convert(int precision, const void* in, void* out, size_t nx, size_t ny,
                           size_t nz, float rho0, cudaStream_t s) {
  Grid g;
  cudaError_t err = validate_domain(in == nullptr || out == nullptr, 1, 1, 1, L::D, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  if (precision != LBM_FLOAT && precision != LBM_DOUBLE) return cudaErrorInvalidValue;
  const size_t wide = (size_t)L::Q * g.plane * (precision == LBM_FLOAT ? 4 : 8);
  const size_t narrow = (size_t)L::Q * g.plane * 2;
  const Span reads[1] = {{in, ENCODE ? wide : narrow}};
  const Span writes[1] = {{out, ENCODE ? narrow : wide}};
  if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  if (precision == LBM_FLOAT && g.plane % 4 == 0 && (uintptr_t)in % 16 == 0 &&
      (uintptr_t)out % 16 == 0) {
    const dim3 grid4((unsigned)std::min<long long>((g.plane / 4 + 255) / 256, 148LL * 8),
                     (unsigned)L::Q, 1);
    convert4_kernel<L, FMT, ENCODE><<<grid4, 256, 0, s>>>(in, out, g.plane, rho0);
    return cudaGetLastError();
  }
  const dim3 grid((unsigned)std::min<long long>((g.plane + 255) / 256, 148LL * 8), (unsigned)L::Q, 1);
  if (precision == LBM_FLOAT)
    convert_kernel<L, FMT, float, ENCODE><<<grid, 256, 0, s>>>(in, out, g.plane, rho0);
  else
    convert_kernel<L, FMT, double, ENCODE><<<grid, 256, 0, s>>>(in, out, g.plane, rho0);
  return cudaGetLastError();
}

template <int FMT, bool ENCODE>
cudaError_t convert_by_lattice(int lattice, int precision, const void* in, void* out, size_t nx,
                               size_t ny, size_t nz, float rho0, cudaStream_t s) {
  switch (lattice) {
    case kD2Q9: return launch_convert<D2Q9, FMT, ENCODE>(precision, in, out, nx, ny, nz, rho0, s);
    case kD3Q19: return launch_convert<D3Q19, FMT, ENCODE>(precision, in, out, nx, ny, nz, rho0, s);
    case kD3Q27: return launch_convert<D3Q27, FMT, ENCODE>(precision, in, out, nx, ny, nz, rho0, s);
    case kD2Q5: return launch_convert<D2Q5, FMT, ENCODE>(precision, in, out, nx, ny, nz, rho0, s);
    case kD3Q7: return launch_convert<D3Q7, FMT, ENCODE>(precision, in, out, nx, ny, nz, rho0, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace lbcube

using namespace lbcube;

extern "C" int lbm_step_shifted_async(int lattice, int format, int collision,
                                      const void* current_populations, void* next_populations,
                                      size_t x_extent, size_t y_extent, size_t z_extent,
                                      float omega, float rho0, void* stream) {
  const cudaStream_t s = as_stream(stream);
  if (format == LBM_F16S)
    return (int)shifted_by_lattice<kF16S>(lattice, collision, current_populations,
                                          next_populations, x_extent, y_extent, z_extent, omega,
                                          rho0, s);
  if (format == LBM_BF16S)
    return (int)shifted_by_lattice<kBF16S>(lattice, collision, current_populations,
                                           next_populations, x_extent, y_extent, z_extent, omega,
                                           rho0, s);
  if (format == LBM_E3M12S)
    return (int)shifted_by_lattice<kE3M12S>(lattice, collision, current_populations,
                                            next_populations, x_extent, y_extent, z_extent, omega,
                                            rho0, s);
  if (format == LBM_Q15S)
    return (int)shifted_by_lattice<kQ15S>(lattice, collision, current_populations,
                                          next_populations, x_extent, y_extent, z_extent, omega,
                                          rho0, s);
  return (int)cudaErrorInvalidValue;
}

extern "C" int lbm_step_slab_shifted_async(int lattice, int format, int collision,
                                           const void* current_populations, void* next_populations,
                                           size_t x_extent, size_t y_extent, size_t z_extent,
                                           float omega, float rho0, const void* halo_lo,
                                           const void* halo_hi, void* send_lo, void* send_hi,
                                           size_t z_begin, size_t z_end, void* stream) {
  const cudaStream_t s = as_stream(stream);
#define LBCUBE_SLAB16(F)                                                                           \
  return (int)shifted_slab_by_lattice<F>(lattice, collision, current_populations, next_populations, \
                                         x_extent, y_extent, z_extent, omega, rho0, halo_lo,       \
                                         halo_hi, send_lo, send_hi, z_begin, z_end, s)
  if (format == LBM_F16S) LBCUBE_SLAB16(kF16S);
  if (format == LBM_BF16S) LBCUBE_SLAB16(kBF16S);
  if (format == LBM_E3M12S) LBCUBE_SLAB16(kE3M12S);
  if (format == LBM_Q15S) LBCUBE_SLAB16(kQ15S);
#undef LBCUBE_SLAB16
  return (int)cudaErrorInvalidValue;
}

extern "C" unsigned int lbm_stage_timeouts(int reset) {
  unsigned int n = 0;
  if (cudaMemcpyFromSymbol(&n, g_stage_timeouts, sizeof(n)) != cudaSuccess) return ~0u;
  if (reset) {
    const unsigned int zero = 0;
    if (cudaMemcpyToSymbol(g_stage_timeouts, &zero, sizeof(zero)) != cudaSuccess) return ~0u;
  }
  return n;
}

extern "C" int lbm_encode_shifted_async(int lattice, int format, int precision,
                                        const void* populations, void* shifted, size_t x_extent,
                                        size_t y_extent, size_t z_extent, float rho0,
                                        void* stream) {
  const cudaStream_t s = as_stream(stream);
  if (format == LBM_F16S)
    return (int)convert_by_lattice<kF16S, true>(lattice, precision, populations, shifted,
                                                x_extent, y_extent, z_extent, rho0, s);
  if (format == LBM_BF16S)
    return (int)convert_by_lattice<kBF16S, true>(lattice, precision, populations, shifted,
                                                 x_extent, y_extent, z_extent, rho0, s);
  if (format == LBM_E3M12S)
    return (int)convert_by_lattice<kE3M12S, true>(lattice, precision, populations, shifted,
                                                  x_extent, y_extent, z_extent, rho0, s);
  if (format == LBM_Q15S)
    return (int)convert_by_lattice<kQ15S, true>(lattice, precision, populations, shifted,
                                                x_extent, y_extent, z_extent, rho0, s);
  return (int)cudaErrorInvalidValue;
}

extern "C" int lbm_decode_shifted_async(int lattice, int format, int precision,
                                        const void* shifted, void* populations, size_t x_extent,
                                        size_t y_extent, size_t z_extent, float rho0,
                                        void* stream) {
  const cudaStream_t s = as_stream(stream);
  if (format == LBM_F16S)
    return (int)convert_by_lattice<kF16S, false>(lattice, precision, shifted, populations,
                                                 x_extent, y_extent, z_extent, rho0, s);
  if (format == LBM_BF16S)
    return (int)convert_by_lattice<kBF16S, false>(lattice, precision, shifted, populations,
                                                  x_extent, y_extent, z_extent, rho0, s);
  if (format == LBM_E3M12S)
    return (int)convert_by_lattice<kE3M12S, false>(lattice, precision, shifted, populations,
                                                   x_extent, y_extent, z_extent, rho0, s);
  if (format == LBM_Q15S)
    return (int)convert_by_lattice<kQ15S, false>(lattice, precision, shifted, populations,
                                                 x_extent, y_extent, z_extent, rho0, s);
  return (int)cudaErrorInvalidValue;
}
