// Reactive-mixing statistics on the device, replacing the host loop of
// compute_reactive_stats (include/lattice_io.hpp:256-338).
//
// Pass 1 (stats_partials_kernel, or the epilogue of fluid_reaction_kernel)
// writes per-block FP64 sums of C_A, C_B, C_A^2, C_B^2, C_A C_B. Pass 2
// (stats_finalize_kernel, one cluster of blocks) adds the partials in a fixed order and
// forms the eight ReactiveDiagnostics fields (lattice_io.hpp:148-166) with the
// reference's formulas (:318-337), in FP64.
#include <cooperative_groups.h>

#include "collide.cuh"
#include "common.cuh"
#include "reduce.cuh"
#include "../../include/lbcube_b200.h"

namespace lbcube {

template <class SL, class Real>
__global__ void __launch_bounds__(kThreads)
    stats_partials_kernel(const Real* __restrict__ a, const Real* __restrict__ b, Grid g,
                          double* __restrict__ partials) {
  pdl_enter();
  int x, y, z;
  const bool active = cell_of(g, x, y, z);
  double sums[kStatSums] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (active) {
    const size_t plane = (size_t)g.plane;
    const int cell = (z * g.ny + y) * g.nx + x;
    Real ga[SL::Q], gb[SL::Q];
    static_for<SL::Q>([&](auto I) {
      ga[LB_I(I)] = __ldg(a + plane * LB_I(I) + cell);
      gb[LB_I(I)] = __ldg(b + plane * LB_I(I) + cell);
    });
    const double ca = (double)concentration<SL>(ga);
    const double cb = (double)concentration<SL>(gb);
    sums[0] = ca;
    sums[1] = cb;
    sums[2] = ca * ca;
    sums[3] = cb * cb;
    sums[4] = ca * cb;
  }
  block_sum_to<kStatSums>(sums, partials + block_linear() * kStatSums);
}

constexpr int kFinalThreads = 1024;
// Blocks of the second pass: one thread-block cluster (distributed shared
// memory), each block taking every kFinalBlocks-th run of kFinalThreads
// partials, so a pass over the 8 192 partials of a 1024^2 launch is one load
// per thread instead of eight dependent ones. LBCUBE_FINAL_BLOCKS = 1: one block.
#ifndef LBCUBE_FINAL_BLOCKS
#define LBCUBE_FINAL_BLOCKS 8
#endif
constexpr int kFinalBlocks = LBCUBE_FINAL_BLOCKS;

// Adds the partials in a fixed order (per thread the partials
// blockIdx.x * kFinalThreads + threadIdx.x + j * kFinalBlocks * kFinalThreads
// in ascending j, then a fixed tree within each block, then the blocks' totals
// in rank order); returns true in the one thread that holds the five sums in s.
// Every thread of the cluster must call it.
__device__ __forceinline__ bool sum_partials(const double* __restrict__ partials, long long blocks,
                                             double (&s)[kStatSums]) {
  __shared__ double sh[kFinalThreads][kStatSums];
#pragma unroll
  for (int q = 0; q < kStatSums; ++q) s[q] = 0.0;
  for (long long blk = (long long)blockIdx.x * kFinalThreads + threadIdx.x; blk < blocks;
       blk += (long long)kFinalBlocks * kFinalThreads) {
#pragma unroll
    for (int q = 0; q < kStatSums; ++q) s[q] += partials[blk * kStatSums + q];
  }
#pragma unroll
  for (int q = 0; q < kStatSums; ++q) sh[threadIdx.x][q] = s[q];
  __syncthreads();
  for (int stride = kFinalThreads / 2; stride > 0; stride >>= 1) {
    if ((int)threadIdx.x < stride) {
#pragma unroll
      for (int q = 0; q < kStatSums; ++q) sh[threadIdx.x][q] += sh[threadIdx.x + stride][q];
    }
    __syncthreads();
  }
  if constexpr (kFinalBlocks == 1) {
#pragma unroll
    for (int q = 0; q < kStatSums; ++q) s[q] = sh[0][q];
    return threadIdx.x == 0;
  } else {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    cluster.sync();  // every block's total is in its shared memory
    const bool holder = cluster.block_rank() == 0 && threadIdx.x == 0;
    if (holder) {
#pragma unroll
      for (int q = 0; q < kStatSums; ++q) s[q] = sh[0][q];
      for (unsigned int r = 1; r < (unsigned int)kFinalBlocks; ++r) {
        const double* remote = cluster.map_shared_rank(&sh[0][0], r);
#pragma unroll
        for (int q = 0; q < kStatSums; ++q) s[q] += remote[q];
      }
    }
    cluster.sync();  // the other blocks keep their shared memory until it has been read
    return holder;
  }
}

// The eight ReactiveDiagnostics fields from the five sums over `cells` cells
// (the reference's formulas, lattice_io.hpp:318-337, in FP64).
__device__ __forceinline__ void diagnostics_from_sums(const double (&s)[kStatSums], double cells,
                                                      double k, double* __restrict__ out) {
  const double inv = 1.0 / cells;
  const double ma = s[0] * inv, mb = s[1] * inv;
  const double ma2 = s[2] * inv, mb2 = s[3] * inv, mab = s[4] * inv;
  const double cov = mab - ma * mb;
  const double mp = ma * mb;
  const double eps = 2.220446049250313080847e-16;
  out[0] = ma;
  out[1] = mb;
  out[2] = ma2 - ma * ma;
  out[3] = mb2 - mb * mb;
  out[4] = cov;
  out[5] = fabs(mp) > eps ? cov / mp : 0.0;
  out[6] = k * mab;
  out[7] = k * ma * mb;
}

__global__ void __cluster_dims__(kFinalBlocks, 1, 1) __launch_bounds__(kFinalThreads)
    stats_finalize_kernel(const double* __restrict__ partials, long long blocks, long long cells,
                          double k, double* __restrict__ out) {
  pdl_enter();
  double s[kStatSums];
  if (sum_partials(partials, blocks, s)) diagnostics_from_sums(s, (double)cells, k, out);
}

// Finalize into the next row of a device table: row *row_counter (if below
// rows), then the counter advances. The destination is read on the device, so
// a captured sequence of steps plus this launch can be replayed to fill
// successive rows.
__global__ void __cluster_dims__(kFinalBlocks, 1, 1) __launch_bounds__(kFinalThreads)
    stats_append_kernel(const double* __restrict__ partials, long long blocks, long long cells,
                        double k, double* __restrict__ table, unsigned long long rows,
                        unsigned long long* __restrict__ row_counter) {
  pdl_enter();
  double s[kStatSums];
  if (sum_partials(partials, blocks, s)) {
    const unsigned long long row = *row_counter;
    if (row < rows) diagnostics_from_sums(s, (double)cells, k, table + row * 8);
    *row_counter = row + 1;
  }
}

// The five sums alone: a rank's share of the statistics of a decomposed domain.
__global__ void __cluster_dims__(kFinalBlocks, 1, 1) __launch_bounds__(kFinalThreads)
    stats_sums_kernel(const double* __restrict__ partials, long long blocks, double* __restrict__ out) {
  pdl_enter();
  double s[kStatSums];
  if (sum_partials(partials, blocks, s)) {
#pragma unroll
    for (int q = 0; q < kStatSums; ++q) out[q] = s[q];
  }
}

__global__ void stats_from_sums_kernel(const double* __restrict__ sums, double cells, double k,
                                       double* __restrict__ out) {
  double s[kStatSums];
#pragma unroll
  for (int q = 0; q < kStatSums; ++q) s[q] = sums[q];
  diagnostics_from_sums(s, cells, k, out);
}

cudaError_t launch_finalize(const Grid& g, double k, const double* partials, double* out,
                            cudaStream_t s) {
  // programmatic dependent launches (the statistics kernels open with pdl_enter)
  return launch_pdl(stats_finalize_kernel, dim3(kFinalBlocks), dim3(kFinalThreads), 0, s, partials,
                    (long long)g.blocks(), (long long)g.plane, k, out);
}

template <class SL, class Real>
cudaError_t launch_stats(const void* va, const void* vb, size_t nx, size_t ny, size_t nz, double k,
                         double* partials, size_t pbytes, double* out, cudaStream_t s) {
  const Real* a = static_cast<const Real*>(va);
  const Real* b = static_cast<const Real*>(vb);
  Grid g;
  cudaError_t err = validate_domain(a == nullptr || b == nullptr || partials == nullptr ||
                                        out == nullptr,
                                    1, 1, 1, SL::D, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  const size_t need = (size_t)g.blocks() * kStatSums * sizeof(double);
  if (pbytes < need) return cudaErrorInvalidValue;
  const size_t sb = (size_t)SL::Q * g.plane * sizeof(Real);
  const Span reads[2] = {{a, sb}, {b, sb}};
  const Span writes[2] = {{partials, need}, {out, 8 * sizeof(double)}};
  if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  err = launch_pdl(stats_partials_kernel<SL, Real>, grid_dims(g), dim3(block_dims(g)), 0, s, a, b, g,
                   partials);
  if (err != cudaSuccess) return err;
  // k_react has the population precision, as in compute_reactive_stats<SL, Real>.
  return launch_finalize(g, (double)(Real)k, partials, out, s);
}

}  // namespace lbcube

using namespace lbcube;

extern "C" size_t lbm_stats_partials_bytes(int fluid_lattice, size_t x_extent, size_t y_extent,
                                           size_t z_extent) {
  Grid g;
  const int dims = fluid_lattice == LBM_D2Q9 || fluid_lattice == LBM_D2Q5 ? 2 : 3;
  if (validate_domain(false, 1, 1, 1, dims, x_extent, y_extent, z_extent, g) != cudaSuccess)
    return 0;
  return (size_t)g.blocks() * kStatSums * sizeof(double);
}

extern "C" int lbm_reactive_stats_async(int scalar_lattice, int precision, const void* current_a,
                                        const void* current_b, size_t x_extent, size_t y_extent,
                                        size_t z_extent, double k_react, double* partials,
                                        size_t partials_bytes, double* diagnostics,
                                        void* stream) {
  const cudaStream_t s = as_stream(stream);
  if (scalar_lattice == LBM_D2Q5) {
    if (precision == LBM_FLOAT)
      return (int)launch_stats<D2Q5, float>(current_a, current_b, x_extent, y_extent, z_extent,
                                            k_react, partials, partials_bytes, diagnostics, s);
    if (precision == LBM_DOUBLE)
      return (int)launch_stats<D2Q5, double>(current_a, current_b, x_extent, y_extent, z_extent,
                                             k_react, partials, partials_bytes, diagnostics, s);
  } else if (scalar_lattice == LBM_D3Q7) {
    if (precision == LBM_FLOAT)
      return (int)launch_stats<D3Q7, float>(current_a, current_b, x_extent, y_extent, z_extent,
                                            k_react, partials, partials_bytes, diagnostics, s);
    if (precision == LBM_DOUBLE)
      return (int)launch_stats<D3Q7, double>(current_a, current_b, x_extent, y_extent, z_extent,
                                             k_react, partials, partials_bytes, diagnostics, s);
  }
  return (int)cudaErrorInvalidValue;
}

extern "C" int lbm_reactive_stats_finalize_async(int fluid_lattice, int precision,
                                                 size_t x_extent, size_t y_extent,
                                                 size_t z_extent, double k_react,
                                                 const double* partials,
                                                 size_t partials_bytes, double* diagnostics,
                                                 void* stream) {
  Grid g;
  const int dims = fluid_lattice == LBM_D2Q9 || fluid_lattice == LBM_D2Q5 ? 2 : 3;
  cudaError_t err = validate_domain(partials == nullptr || diagnostics == nullptr, 1, 1, 1, dims,
                                    x_extent, y_extent, z_extent, g);
  if (err != cudaSuccess) return (int)err;
  if (partials_bytes < (size_t)g.blocks() * kStatSums * sizeof(double))
    return (int)cudaErrorInvalidValue;
  if (precision != LBM_FLOAT && precision != LBM_DOUBLE) return (int)cudaErrorInvalidValue;
  const double k = precision == LBM_FLOAT ? (double)(float)k_react : k_react;
  return (int)launch_finalize(g, k, partials, diagnostics, as_stream(stream));
}

extern "C" int lbm_reactive_stats_append_async(int fluid_lattice, int precision, size_t x_extent,
                                               size_t y_extent, size_t z_extent, double k_react,
                                               const double* partials, size_t partials_bytes,
                                               double* table, size_t table_rows,
                                               unsigned long long* row_counter, void* stream) {
  Grid g;
  const int dims = fluid_lattice == LBM_D2Q9 || fluid_lattice == LBM_D2Q5 ? 2 : 3;
  cudaError_t err = validate_domain(partials == nullptr || table == nullptr || row_counter == nullptr,
                                    1, 1, 1, dims, x_extent, y_extent, z_extent, g);
  if (err != cudaSuccess) return (int)err;
  const size_t need = (size_t)g.blocks() * kStatSums * sizeof(double);
  if (partials_bytes < need || table_rows == 0) return (int)cudaErrorInvalidValue;
  if (precision != LBM_FLOAT && precision != LBM_DOUBLE) return (int)cudaErrorInvalidValue;
  const Span reads[1] = {{partials, need}};
  const Span writes[2] = {{table, table_rows * 8 * sizeof(double)}, {row_counter, sizeof(unsigned long long)}};
  if (any_overlap(reads, writes)) return (int)cudaErrorInvalidValue;
  const double k = precision == LBM_FLOAT ? (double)(float)k_react : k_react;
  return (int)launch_pdl(stats_append_kernel, dim3(kFinalBlocks), dim3(kFinalThreads), 0, as_stream(stream),
                         (const double*)partials, (long long)g.blocks(), (long long)g.plane, k, table,
                         (unsigned long long)table_rows, row_counter);
}

// Statistics of a domain split across ranks: each rank reduces its partials
// to the five sums (lbm_reactive_stats_sums_async), the ranks add the sums
// (an all-reduce of five doubles), and lbm_reactive_stats_from_sums_async
// forms the diagnostics from the totals. On one rank the two calls give the
// bits of lbm_reactive_stats_finalize_async.
extern "C" int lbm_reactive_stats_sums_async(int fluid_lattice, size_t x_extent, size_t y_extent,
                                             size_t z_extent, const double* partials,
                                             size_t partials_bytes, double* sums, void* stream) {
  Grid g;
  const int dims = fluid_lattice == LBM_D2Q9 || fluid_lattice == LBM_D2Q5 ? 2 : 3;
  cudaError_t err = validate_domain(partials == nullptr || sums == nullptr, 1, 1, 1, dims,
                                    x_extent, y_extent, z_extent, g);
  if (err != cudaSuccess) return (int)err;
  if (partials_bytes < (size_t)g.blocks() * kStatSums * sizeof(double)) return (int)cudaErrorInvalidValue;
  return (int)launch_pdl(stats_sums_kernel, dim3(kFinalBlocks), dim3(kFinalThreads), 0, as_stream(stream),
                         partials, (long long)g.blocks(), sums);
}

extern "C" int lbm_reactive_stats_from_sums_async(int precision, const double* sums, double cells,
                                                  double k_react, double* diagnostics,
                                                  void* stream) {
  if (sums == nullptr || diagnostics == nullptr) return (int)cudaErrorInvalidDevicePointer;
  if (precision != LBM_FLOAT && precision != LBM_DOUBLE) return (int)cudaErrorInvalidValue;
  if (!(cells >= 1.0)) return (int)cudaErrorInvalidValue;
  const double k = precision == LBM_FLOAT ? (double)(float)k_react : k_react;
  stats_from_sums_kernel<<<1, 1, 0, as_stream(stream)>>>(sums, cells, k, diagnostics);
  return (int)cudaGetLastError();
}

// ----------------------------------------------------------------------------
// Allocation-free statistics.
//
// For callers that cannot allocate device memory: for example a solver plugin
// or an FFI binding inside a host application that owns every device
// allocation through its own pool and hands this library only the scalar
// fields, so it has no way to obtain the partial-sum scratch that
// lbm_reactive_stats_async needs. Here the scratch is a file-scope device
// array of fixed size, reserved on every GPU that loads the library until the
// process exits; nothing is allocated per call.
// ----------------------------------------------------------------------------
namespace lbcube {

// Partial sums for up to this many 128-cell row segments (blocks):
// ceil(nx / 128) * ny * nz <= 131072, e.g. 256^3 or 1024^2. 5 MiB per GPU.
constexpr long long kNoAllocMaxBlocks = 131072;
static_assert(kNoAllocMaxBlocks == LBM_STATS_NOALLOC_MAX_BLOCKS,
              "the array size and the limit the header publishes must agree");
static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxBlocks * kStatSums];

// Device address of g_noalloc_partials in the calling thread's current
// context. In host code the array's name only stands in for the symbol. The
// address belongs to the context the library's device code is loaded in, not
// to the device ordinal: a host that creates or switches contexts itself
// (cuCtxCreate, cuCtxSetCurrent), or resets the device, gets the array at
// another address. So it is looked up on every call (a host-side query, no
// device work); the first lookup in a context may load the library's device
// code into it.
static cudaError_t noalloc_scratch(double** out) {
  void* p = nullptr;
  const cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_partials);
  if (err != cudaSuccess) return err;
  *out = static_cast<double*>(p);
  return cudaSuccess;
}

}  // namespace lbcube

extern "C" int lbm_reactive_stats_noalloc_async(int scalar_lattice, int precision,
                                                const void* current_a, const void* current_b,
                                                size_t x_extent, size_t y_extent,
                                                size_t z_extent, double k_react,
                                                double* diagnostics, void* stream) {
  double* scratch = nullptr;
  const cudaError_t err = noalloc_scratch(&scratch);
  if (err != cudaSuccess) return (int)err;
  // Every block overwrites its own partial slots and the second pass reads
  // only those, so nothing left in the array by an earlier call is used and
  // nothing needs clearing. A domain with more blocks than the array holds is
  // rejected with cudaErrorInvalidValue by the capacity check.
  const size_t capacity = (size_t)kNoAllocMaxBlocks * kStatSums * sizeof(double);
  return lbm_reactive_stats_async(scalar_lattice, precision, current_a, current_b, x_extent,
                                  y_extent, z_extent, k_react, scratch, capacity, diagnostics,
                                  stream);
}
