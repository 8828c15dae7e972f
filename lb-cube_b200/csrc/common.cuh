// Launch geometry and argument validation shared by every kernel family.
#pragma once

#include <cuda_runtime.h>

#include <climits>
#include <cstddef>
#include <cstdint>
#include <utility>

#include "lattices.cuh"

namespace lbcube {

// Most threads per block. In the one-cell-per-thread kernels each thread owns
// one cell of an x-row and a block covers bx <= kThreads consecutive cells of
// one (y, z) row.
constexpr int kThreads = 128;

// Domain extents and the block decomposition: grid.x = xblocks * ny
// (row-major over y, then x-block), grid.y = nz; xblocks = ceil(nx / kThreads)
// blocks of bx threads, bx = ceil(nx / xblocks) rounded up to a warp, so that a
// row of, e.g., 192 cells runs as two full blocks of 96 rather than 128 + 64.
struct Grid {
  int nx, ny, nz;
  int xblocks;
  int bx;           // threads per block
  long long plane;  // cells per population plane, nx * ny * nz (< 2^31)
  int z0 = 0;       // first z plane of the launch
  int zs = 1;       // planes between consecutive blockIdx.y: z = z0 + blockIdx.y * zs (both face
                    // planes of a slab in one launch: z0 = 0, zs = nz - 1)

  __host__ __device__ long long blocks() const { return (long long)xblocks * ny * nz; }
};

// The z plane of this block.
__device__ __forceinline__ int plane_of(const Grid& g) { return g.z0 + (int)blockIdx.y * g.zs; }

__device__ __forceinline__ bool cell_of(const Grid& g, int& x, int& y, int& z) {
  const int row = blockIdx.x / g.xblocks;
  const int xb = blockIdx.x - row * g.xblocks;
  x = xb * g.bx + threadIdx.x;
  y = row;
  z = plane_of(g);
  return x < g.nx;
}

// Linear block index used to address per-block partial sums.
__device__ __forceinline__ long long block_linear() {
  return (long long)blockIdx.y * gridDim.x + blockIdx.x;
}

// Programmatic dependent launch. pdl_enter() at the top of a kernel waits
// until the grid it depends on has completed and its writes are visible (a
// no-op unless the kernel was launched with the programmatic-serialization
// attribute), then lets the next launch in the stream be scheduled, so that
// launch's blocks take the SMs that this grid's last blocks free instead of
// waiting for the whole grid to drain. launch_pdl launches with that attribute.
#ifndef LBCUBE_PDL
#define LBCUBE_PDL 1
#endif
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <class... KArgs, class... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t s, Args&&... args) {
  if (!LBCUBE_PDL) {
    kernel<<<grid, block, smem, s>>>(std::forward<Args>(args)...);
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

inline dim3 grid_dims(const Grid& g) { return dim3((unsigned)(g.xblocks * g.ny), (unsigned)g.nz, 1); }
inline unsigned block_dims(const Grid& g) { return (unsigned)g.bx; }

// Validation in the reference's order (src/lattice_cuda.cu:488-503), then the
// engine's own limits. On success fills `g`.
inline cudaError_t validate_domain(bool any_null, unsigned bx, unsigned by, unsigned bz, int dims,
                                   size_t nx, size_t ny, size_t nz, Grid& g) {
  if (any_null) return cudaErrorInvalidDevicePointer;
  if (bx == 0 || by == 0 || bz == 0) return cudaErrorInvalidConfiguration;
  if (dims == 2) nz = 1;
  if (nx == 0 || ny == 0 || nz == 0) return cudaErrorInvalidValue;
  if (nx > (size_t)INT_MAX || ny > (size_t)INT_MAX || nz > 65535) return cudaErrorInvalidValue;
  const unsigned long long cells = (unsigned long long)nx * ny;
  if (cells > (unsigned long long)INT_MAX || cells * nz > (unsigned long long)INT_MAX)
    return cudaErrorInvalidValue;
  g.nx = (int)nx;
  g.ny = (int)ny;
  g.nz = (int)nz;
  g.xblocks = (int)((nx + kThreads - 1) / kThreads);
  g.bx = (int)(((nx + g.xblocks - 1) / g.xblocks + 31) / 32 * 32);
  g.plane = (long long)(cells * nz);
  if ((long long)g.xblocks * g.ny > (long long)INT_MAX) return cudaErrorInvalidValue;
  return cudaSuccess;
}

struct Span {
  const void* p;
  size_t bytes;
};

inline bool overlaps(Span a, Span b) {
  const uintptr_t a0 = (uintptr_t)a.p, a1 = a0 + a.bytes;
  const uintptr_t b0 = (uintptr_t)b.p, b1 = b0 + b.bytes;
  return a0 < b1 && b0 < a1;
}

// Every written buffer must be disjoint from every other buffer of the call.
template <int NR, int NW>
inline bool any_overlap(const Span (&reads)[NR], const Span (&writes)[NW]) {
  for (int w = 0; w < NW; ++w) {
    for (int r = 0; r < NR; ++r)
      if (overlaps(writes[w], reads[r])) return true;
    for (int v = w + 1; v < NW; ++v)
      if (overlaps(writes[w], writes[v])) return true;
  }
  return false;
}

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace lbcube
