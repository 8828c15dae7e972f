// Collide-stream step of one z-slab of a periodic box split across ranks.
//
// No reference counterpart (the reference runs one domain on one device). The
// box is cut into slabs along z; each rank owns nz_local planes in the
// reference's [Q, Z, Y, X] layout and steps them with the same kernels as the
// periodic box (kUseVec, step_cell.cuh), except that the populations crossing
// a slab face are pulled from halo planes (SlabArgs, stream_vec.cuh) and the
// ones leaving through a face are also stored, in the same pass, into send
// planes for the neighbour. One exchange per step moves the send planes into
// the neighbours' halo planes (zcount<L>() of Q populations per face: 5 of 19
// for D3Q19, 9 of 27 for D3Q27); the host side runs it on NCCL point-to-point
// (lb-cube_b200/slab.py). Every cell does the arithmetic of the periodic step,
// so a box stepped as slabs is bit-identical to the box stepped whole.
//
// Launch ranges: interior planes [1, nz-1) read no halo and may run while the
// exchange of the previous step is in flight; the boundary planes 0 and nz-1
// run after it. Within one call, interior planes run the periodic-box kernel
// and only the boundary planes the SLAB form.
#include <algorithm>

#include "collide.cuh"
#include "common.cuh"
#include "step_cell.cuh"
#include "stream_vec.cuh"
#include "../../include/lbcube_b200.h"

namespace lbcube {

template <class L, class Real, int CT>
cudaError_t launch_slab_step(const Real* cur, Real* nxt, size_t nx, size_t ny, size_t nz,
                             Real omega, const Real* halo_lo, const Real* halo_hi, Real* send_lo,
                             Real* send_hi, size_t z_begin, size_t z_end, cudaStream_t s) {
  Grid g;
  cudaError_t err = validate_domain(cur == nullptr || nxt == nullptr, 1, 1, 1, 3, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  if (z_begin >= z_end || z_end > nz) return cudaErrorInvalidValue;
  const bool lo_face = z_begin == 0, hi_face = z_end == nz;
  if ((lo_face && (halo_lo == nullptr || send_lo == nullptr)) ||
      (hi_face && (halo_hi == nullptr || send_hi == nullptr)))
    return cudaErrorInvalidDevicePointer;
  // a face plane reads both halos when nz == 1
  if (nz == 1 && (halo_lo == nullptr || halo_hi == nullptr || send_lo == nullptr || send_hi == nullptr))
    return cudaErrorInvalidDevicePointer;
  using S = NativeStorage<Real, kVecCells<L, Real>>;  // as the periodic step
  if (!vec_eligible<S>(g, cur, nxt)) return cudaErrorInvalidValue;
  const size_t bytes = (size_t)L::Q * g.plane * sizeof(Real);
  const size_t hbytes = (size_t)zcount<L>() * g.ny * g.nx * sizeof(Real);
  const Span reads[3] = {{cur, bytes}, {halo_lo, halo_lo ? hbytes : 0}, {halo_hi, halo_hi ? hbytes : 0}};
  const Span writes[3] = {{nxt, bytes}, {send_lo, send_lo ? hbytes : 0}, {send_hi, send_hi ? hbytes : 0}};
  if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  constexpr uintptr_t align = sizeof(Real) * S::V;
  for (const void* p : {(const void*)halo_lo, (const void*)halo_hi, (const void*)send_lo, (const void*)send_hi})
    if ((uintptr_t)p % align != 0) return cudaErrorInvalidValue;
  const Real omega_minus = CT == kTRT ? trt_omega_minus<Real>(omega) : Real(0);
  VecGrid vg = make_vec_grid(g, S::V);
  // Interior planes [1, nz - 1) of the range pull only within the slab (no
  // wrap) and send nothing: the periodic-box kernel that the plain step uses
  // for this lattice, operator and precision (kUseVec) steps them, from plane
  // z0 on. Only the face planes run the SLAB form (halo rows, face sends),
  // whose extra addressing and stores cost about 30 % per plane.
  const size_t ib = std::max<size_t>(z_begin, 1), ie = std::min<size_t>(z_end, nz - 1);
  if (ib < ie) {
    if constexpr (kUseVec<L, Real, CT>) {
      vg.z0 = (int)ib;
      dim3 grid = vec_grid_dims(vg);
      grid.y = (unsigned)(ie - ib);
      launch_vec_step<L, S, CT>(vg, grid, vec_block_threads(vg), s, cur, nxt, omega, omega_minus,
                                typename S::Params{});
      vg.z0 = 0;
    } else {
      Grid gi = g;
      gi.z0 = (int)ib;
      dim3 grid = grid_dims(gi);
      grid.y = (unsigned)(ie - ib);
      launch_pdl(fluid_step_kernel<L, Real, CT, false>, grid, dim3(block_dims(gi)), 0, s, cur, nxt, gi,
                 omega, omega_minus, (double*)nullptr);
    }
  }
  // the face planes: `count` planes from z, `step` apart (both faces of the
  // slab in one launch where the range has both)
  auto faces = [&](size_t z, unsigned count, int step) {
    dim3 grid = vec_grid_dims(vg);
    grid.y = count;
    SlabArgs<Real> slab{halo_lo, halo_hi, send_lo, send_hi, (int)z};
    slab.z_step = step;
    launch_pdl(fluid_step_vec_kernel<L, S, CT, false, true>, grid, dim3(vec_block_threads(vg)), 0, s, cur,
               nxt, vg, omega, omega_minus, typename S::Params{}, (double*)nullptr, slab);
  };
  if (lo_face && hi_face && nz > 1) {
    faces(0, 2, (int)nz - 1);
  } else {
    if (lo_face) faces(0, 1, 1);
    if (hi_face && nz > 1) faces(nz - 1, 1, 1);
  }
  return cudaGetLastError();
}

// Copies the face populations of a slab state into the send planes (the
// exchange that precedes the first step).
template <class L, class Real>
__global__ void __launch_bounds__(256)
    slab_pack_kernel(const Real* __restrict__ f, Real* __restrict__ send_lo,
                     Real* __restrict__ send_hi, int nx, int ny, int nz) {
  const long long n2 = (long long)nx * ny;
  const long long total = (long long)zcount<L>() * n2;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(e / n2);
    const long long r = e - k * n2;
    static_for<L::Q>([&](auto I) {
      constexpr int i = LB_I(I);
      constexpr int cz = L::c[i][2];
      if constexpr (cz > 0) {
        if (zslot<L>(i) == k) send_hi[e] = f[(size_t)i * n2 * nz + (size_t)(nz - 1) * n2 + r];
      } else if constexpr (cz < 0) {
        if (zslot<L>(i) == k) send_lo[e] = f[(size_t)i * n2 * nz + r];
      }
    });
  }
}

template <class L, class Real>
cudaError_t launch_slab_pack(const Real* f, size_t nx, size_t ny, size_t nz, Real* send_lo,
                             Real* send_hi, cudaStream_t s) {
  Grid g;
  cudaError_t err = validate_domain(f == nullptr || send_lo == nullptr || send_hi == nullptr, 1, 1,
                                    1, 3, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  const size_t hbytes = (size_t)zcount<L>() * g.ny * g.nx * sizeof(Real);
  const Span reads[1] = {{f, (size_t)L::Q * g.plane * sizeof(Real)}};
  const Span writes[2] = {{send_lo, hbytes}, {send_hi, hbytes}};
  if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  const long long total = (long long)zcount<L>() * g.nx * g.ny;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  slab_pack_kernel<L, Real><<<blocks, 256, 0, s>>>(f, send_lo, send_hi, g.nx, g.ny, g.nz);
  return cudaGetLastError();
}

template <class Real, int CT>
cudaError_t slab_by_lattice(int lattice, const void* cur, void* nxt, size_t nx, size_t ny, size_t nz,
                            double omega, const void* hl, const void* hh, void* sl, void* sh,
                            size_t z0, size_t z1, cudaStream_t s) {
  const Real* c = static_cast<const Real*>(cur);
  Real* n = static_cast<Real*>(nxt);
  const Real *l = static_cast<const Real*>(hl), *h = static_cast<const Real*>(hh);
  Real *a = static_cast<Real*>(sl), *b = static_cast<Real*>(sh);
  switch (lattice) {
    case kD3Q19:
      return launch_slab_step<D3Q19, Real, CT>(c, n, nx, ny, nz, Real(omega), l, h, a, b, z0, z1, s);
    case kD3Q27:
      if constexpr (sizeof(Real) == 8 && (CT == kMRT || CT == kRLBM)) return cudaErrorInvalidValue;
      else return launch_slab_step<D3Q27, Real, CT>(c, n, nx, ny, nz, Real(omega), l, h, a, b, z0, z1, s);
    default: return cudaErrorInvalidValue;
  }
}

template <class Real>
cudaError_t slab_by_collision(int lattice, int collision, const void* cur, void* nxt, size_t nx,
                              size_t ny, size_t nz, double omega, const void* hl, const void* hh,
                              void* sl, void* sh, size_t z0, size_t z1, cudaStream_t s) {
  switch (collision) {
    case kBGK: return slab_by_lattice<Real, kBGK>(lattice, cur, nxt, nx, ny, nz, omega, hl, hh, sl, sh, z0, z1, s);
    case kTRT: return slab_by_lattice<Real, kTRT>(lattice, cur, nxt, nx, ny, nz, omega, hl, hh, sl, sh, z0, z1, s);
    case kMRT: return slab_by_lattice<Real, kMRT>(lattice, cur, nxt, nx, ny, nz, omega, hl, hh, sl, sh, z0, z1, s);
    case kRLBM: return slab_by_lattice<Real, kRLBM>(lattice, cur, nxt, nx, ny, nz, omega, hl, hh, sl, sh, z0, z1, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace lbcube

using namespace lbcube;

extern "C" size_t lbm_slab_face_elems(int lattice, size_t x_extent, size_t y_extent) {
  if (lattice == LBM_D3Q19) return (size_t)zcount<D3Q19>() * x_extent * y_extent;
  if (lattice == LBM_D3Q27) return (size_t)zcount<D3Q27>() * x_extent * y_extent;
  return 0;
}

extern "C" int lbm_step_slab_async(int lattice, int precision, int collision,
                                   const void* current_populations, void* next_populations,
                                   size_t x_extent, size_t y_extent, size_t z_extent, double omega,
                                   const void* halo_lo, const void* halo_hi, void* send_lo,
                                   void* send_hi, size_t z_begin, size_t z_end, void* stream) {
  const cudaStream_t s = as_stream(stream);
  if (precision == LBM_FLOAT)
    return (int)slab_by_collision<float>(lattice, collision, current_populations, next_populations,
                                         x_extent, y_extent, z_extent, omega, halo_lo, halo_hi,
                                         send_lo, send_hi, z_begin, z_end, s);
  if (precision == LBM_DOUBLE)
    return (int)slab_by_collision<double>(lattice, collision, current_populations, next_populations,
                                          x_extent, y_extent, z_extent, omega, halo_lo, halo_hi,
                                          send_lo, send_hi, z_begin, z_end, s);
  return (int)cudaErrorInvalidValue;
}

extern "C" int lbm_slab_pack_async(int lattice, int precision, const void* populations,
                                   size_t x_extent, size_t y_extent, size_t z_extent, void* send_lo,
                                   void* send_hi, void* stream) {
  const cudaStream_t s = as_stream(stream);
#define LBCUBE_PACK(L, R)                                                                          \
  return (int)launch_slab_pack<L, R>(static_cast<const R*>(populations), x_extent, y_extent,      \
                                     z_extent, static_cast<R*>(send_lo), static_cast<R*>(send_hi), s)
  if (precision == LBM_FLOAT) {
    if (lattice == LBM_D3Q19) LBCUBE_PACK(D3Q19, float);
    if (lattice == LBM_D3Q27) LBCUBE_PACK(D3Q27, float);
  } else if (precision == LBM_DOUBLE) {
    if (lattice == LBM_D3Q19) LBCUBE_PACK(D3Q19, double);
    if (lattice == LBM_D3Q27) LBCUBE_PACK(D3Q27, double);
  }
#undef LBCUBE_PACK
  return (int)cudaErrorInvalidValue;
}

// The pack of a slab state on 16-bit storage (codes of any format).
extern "C" int lbm_slab_pack_shifted_async(int lattice, const void* populations, size_t x_extent,
                                           size_t y_extent, size_t z_extent, void* send_lo,
                                           void* send_hi, void* stream) {
  using E = unsigned short;
  const E* f = static_cast<const E*>(populations);
  if (lattice == LBM_D3Q19)
    return (int)launch_slab_pack<D3Q19, E>(f, x_extent, y_extent, z_extent, static_cast<E*>(send_lo),
                                           static_cast<E*>(send_hi), as_stream(stream));
  if (lattice == LBM_D3Q27)
    return (int)launch_slab_pack<D3Q27, E>(f, x_extent, y_extent, z_extent, static_cast<E*>(send_lo),
                                           static_cast<E*>(send_hi), as_stream(stream));
  return (int)cudaErrorInvalidValue;
}

// ---- face copies between slabs held by one process ----------------------------
// The exchange of ranks that share one device (every rank of a box stepped in
// one process): `count` buffers of `bytes` bytes each copied in one launch, one
// block column per buffer, 16-byte words where both addresses allow it. The
// pointer lists travel as a kernel parameter.
namespace lbcube {

constexpr int kMaxCopies = 64;

struct CopyList {
  const unsigned char* src[kMaxCopies];
  unsigned char* dst[kMaxCopies];
};

static __global__ void __launch_bounds__(256)
    copy_buffers_kernel(const CopyList list, size_t bytes) {
  pdl_enter();
  const unsigned char* __restrict__ src = list.src[blockIdx.y];
  unsigned char* __restrict__ dst = list.dst[blockIdx.y];
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if ((((uintptr_t)src | (uintptr_t)dst) & 15u) == 0) {
    const size_t words = bytes / 16;
    for (size_t i = t; i < words; i += stride)
      reinterpret_cast<uint4*>(dst)[i] = reinterpret_cast<const uint4*>(src)[i];
    for (size_t i = words * 16 + t; i < bytes; i += stride) dst[i] = src[i];
  } else {
    for (size_t i = t; i < bytes; i += stride) dst[i] = src[i];
  }
}

}  // namespace lbcube

extern "C" int lbm_copy_buffers_async(int count, const void* const* src, void* const* dst,
                                      size_t bytes, void* stream) {
  if (src == nullptr || dst == nullptr) return (int)cudaErrorInvalidDevicePointer;
  if (count < 0 || count > kMaxCopies) return (int)cudaErrorInvalidValue;
  if (count == 0 || bytes == 0) return (int)cudaSuccess;
  CopyList list{};
  for (int i = 0; i < count; ++i) {
    if (src[i] == nullptr || dst[i] == nullptr) return (int)cudaErrorInvalidDevicePointer;
    list.src[i] = static_cast<const unsigned char*>(src[i]);
    list.dst[i] = static_cast<unsigned char*>(dst[i]);
  }
  // no copy may write into a buffer that another copy of the list reads or writes
  for (int i = 0; i < count; ++i)
    for (int j = 0; j < count; ++j) {
      const Span a[1] = {{src[j], bytes}};
      const Span b[1] = {{dst[i], bytes}};
      if (any_overlap(a, b)) return (int)cudaErrorInvalidValue;
      if (j > i) {
        const Span c[1] = {{dst[j], bytes}};
        if (any_overlap(c, b)) return (int)cudaErrorInvalidValue;
      }
    }
  const size_t words = (bytes + 15) / 16;
  const unsigned blocks_x = (unsigned)std::min<size_t>((words + 255) / 256, 64);
  // a programmatic dependent launch, like the slab steps around it
  return (int)launch_pdl(copy_buffers_kernel, dim3(blocks_x, (unsigned)count), dim3(256), 0, as_stream(stream),
                         list, bytes);
}
