// Row-staged pull collide-stream on shifted 16-bit populations.
//
// The step on 16-bit storage moves half the bytes of the FP32 step, so its
// per-cell instruction budget at the HBM roofline is half as large, and a
// thread that waits for its own loads before colliding leaves the SM idle.
// This kernel takes the loads off the threads: one block owns a run of
// output rows of one plane (a row is the nx cells of one (y, z)); for every
// output row the Q source rows it pulls from (row (y - c_y, z - c_z) of
// population plane i, periodic) are copied whole into shared memory by the
// bulk-copy engine (cp.async.bulk, completion on an mbarrier), kStages rows
// ahead of the row being collided. Threads read their four cells' words of each
// population from shared memory (the x-shifted ones with one more 16-bit read
// at the row's periodic neighbour and two byte permutes), collide two cells
// at a time in registers and store aligned 8-byte words.
//
// Shared memory: kStages x Q rows x nx codes (D3Q19, nx = 256: 9.5 KiB per
// stage). Requirements (checked by the launcher, which otherwise uses the
// register-gather kernel of stream_vec.cuh): nx a multiple of 8 and at most
// 4 * kMaxRowThreads, buffers 16-byte aligned (every row copy then starts on
// a 16-byte boundary and moves a multiple of 16 bytes).
//
// Every wait on an mbarrier is bounded: after kWaitLimit polls a block records
// the timeout in g_stage_timeouts, waits (bounded again) for the copies it has
// in flight and returns, so a fault in the copy path ends the launch instead
// of hanging the GPU; lbm_stage_timeouts reports the count.
#pragma once

#include <cstdint>

#include "collide_dev.cuh"
#include "common.cuh"
#include "stream_vec.cuh"

namespace lbcube {

#ifndef LBCUBE_STAGES
#define LBCUBE_STAGES 3
#endif
#ifndef LBCUBE_STAGED_ROWS
#define LBCUBE_STAGED_ROWS 8
#endif
#ifndef LBCUBE_STAGED_MIN_BLOCKS
#define LBCUBE_STAGED_MIN_BLOCKS 2
#endif
constexpr int kStages = LBCUBE_STAGES;          // rows in flight per block
constexpr int kStagedRows = LBCUBE_STAGED_ROWS;  // output rows per block
constexpr int kMaxRowThreads = 256;  // threads per block: nx / 4, rounded up to a warp
constexpr long long kWaitLimit = 1LL << 22;

// Blocks that gave up waiting for a row copy (or found their shared memory
// misaligned) since the count was last read; one per translation unit that
// launches the kernel.
static __device__ unsigned int g_stage_timeouts;

__device__ __forceinline__ unsigned int smem_addr(const void* p) {
  return (unsigned int)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned int bar, unsigned int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned int bar, unsigned int bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

// Polls the barrier's phase `parity` at most kWaitLimit times.
__device__ __forceinline__ bool mbar_wait(unsigned int bar, unsigned int parity) {
  for (long long it = 0; it < kWaitLimit; ++it) {
    unsigned int done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Global -> shared bulk copy of `bytes` (a multiple of 16, both addresses
// 16-byte aligned), completing on barrier `bar`. No multicast.
__device__ __forceinline__ void bulk_copy_g2s(unsigned int dst, const void* src, unsigned int bytes,
                                              unsigned int bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

struct StagedGrid {
  int nx, ny, nz;
  long long plane;
  int rows;       // end of the launch's rows (exclusive); ny * nz for every row
  int row_bytes;  // nx * 2
  int row0;       // first row of the launch
};

// Issues the Q source rows of output row `r` into stage buffer `buf`. SLAB: a
// z-slab of a box (slab_faces.cuh layout of the halo buffers): at plane 0 the
// c_z = +1 rows come from halo_lo, at plane nz - 1 the c_z = -1 rows from
// halo_hi, instead of the periodic wrap.
template <class L, bool SLAB = false>
__device__ __forceinline__ void issue_row(const unsigned short* __restrict__ cur, const StagedGrid& g,
                                          int r, unsigned int buf, unsigned int bar,
                                          const SlabArgs<unsigned short>& slab = {}) {
  const int z = r / g.ny, y = r - z * g.ny;
  const int ym = y == 0 ? g.ny - 1 : y - 1, yp = y == g.ny - 1 ? 0 : y + 1;
  const int zm = z == 0 ? g.nz - 1 : z - 1, zp = z == g.nz - 1 ? 0 : z + 1;
  mbar_expect_tx(bar, (unsigned int)(L::Q * g.row_bytes));
  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr int cy = L::c[i][1], cz = L::c[i][2];
    const int sy = cy == 0 ? y : (cy > 0 ? ym : yp);
    const int sz = cz == 0 ? z : (cz > 0 ? zm : zp);
    const unsigned short* src = cur + g.plane * i + ((long long)sz * g.ny + sy) * g.nx;
    if constexpr (SLAB && cz > 0) {
      if (z == 0) src = slab.halo_lo + ((long long)zslot<L>(i) * g.ny + sy) * g.nx;
    } else if constexpr (SLAB && cz < 0) {
      if (z == g.nz - 1) src = slab.halo_hi + ((long long)zslot<L>(i) * g.ny + sy) * g.nx;
    }
    bulk_copy_g2s(buf + (unsigned int)(i * g.row_bytes), src, (unsigned int)g.row_bytes, bar);
  });
}

template <class L, class S, int CT, bool SLAB = false>
__global__ void __launch_bounds__(kMaxRowThreads, LBCUBE_STAGED_MIN_BLOCKS)
    fluid_step_staged_kernel(const unsigned short* __restrict__ cur,
                             unsigned short* __restrict__ nxt, StagedGrid g, float omega,
                             float omega_minus, typename S::Params p,
                             SlabArgs<unsigned short> slab = {}) {
  static_assert(S::V == 4, "four cells per thread");
  pdl_enter();
  // kStages row buffers, then the kStages mbarriers (8-byte aligned: a stage
  // is a multiple of 16 bytes)
  extern __shared__ __align__(128) unsigned char smem[];
  const int stage_bytes = L::Q * g.row_bytes;
  const unsigned int base = smem_addr(smem);
  const unsigned int bars = base + kStages * stage_bytes;
  const int t = threadIdx.x;
  if ((base & 15u) != 0u) {  // bulk copies need 16-byte aligned destinations
    if (t == 0) atomicAdd(&g_stage_timeouts, 1u);
    return;
  }
  const int r0 = g.row0 + blockIdx.x * kStagedRows;
  const int nrows = min(kStagedRows, g.rows - r0);
  const int x0 = 4 * t;
  const bool active = x0 < g.nx;
  const int xl = x0 == 0 ? g.nx - 1 : x0 - 1;  // periodic left neighbour of the first cell
  const int xr = x0 + 4 == g.nx ? 0 : x0 + 4;  // and right neighbour of the last
  if (t == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(bars + 8 * s, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  int issued = 0;  // rows whose copies have been issued (thread 0's count)
  if (t == 0)
    for (; issued < kStages && issued < nrows; ++issued)
      issue_row<L, SLAB>(cur, g, r0 + issued, base + issued * stage_bytes, bars + 8 * issued, slab);
  bool failed = false;
  for (int k = 0; k < nrows; ++k) {
    const int s = k % kStages;
    const bool ok = mbar_wait(bars + 8 * s, (unsigned int)((k / kStages) & 1));
    // this thread's four cells of every population, x-shifted rows assembled
    unsigned int raw[L::Q][2];
    if (ok && active) {
      static_for<L::Q>([&](auto I) {
        constexpr int i = LB_I(I);
        constexpr int cx = L::c[i][0];
        const unsigned char* row = smem + s * stage_bytes + i * g.row_bytes;
        const uint2 own = *reinterpret_cast<const uint2*>(row + 2 * x0);
        if constexpr (cx == 0) {
          raw[i][0] = own.x;
          raw[i][1] = own.y;
        } else if constexpr (cx > 0) {  // cells x0-1 .. x0+2
          const unsigned int left = *reinterpret_cast<const unsigned short*>(row + 2 * xl);
          raw[i][0] = __byte_perm(left, own.x, 0x5410);
          raw[i][1] = __byte_perm(own.x, own.y, 0x5432);
        } else {  // cells x0+1 .. x0+4
          const unsigned int right = *reinterpret_cast<const unsigned short*>(row + 2 * xr);
          raw[i][0] = __byte_perm(own.x, own.y, 0x5432);
          raw[i][1] = __byte_perm(own.y, right, 0x5432);
        }
      });
    }
    // every thread has read stage s (or one of them gave up waiting: then all leave)
    if (!__syncthreads_and(ok)) {
      failed = true;
      break;
    }
    if (t == 0 && issued < nrows) {
      issue_row<L, SLAB>(cur, g, r0 + issued, base + s * stage_bytes, bars + 8 * s, slab);
      ++issued;
    }
    if (active) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        float va[L::Q], vb[L::Q];
        static_for<L::Q>([&](auto I) {
          const float2 d = S::decode_pair(raw[LB_I(I)][h]);
          va[LB_I(I)] = d.x;
          vb[LB_I(I)] = d.y;
        });
        S::template collide_cell<L, CT>(va, omega, omega_minus, p);
        S::template collide_cell<L, CT>(vb, omega, omega_minus, p);
        static_for<L::Q>([&](auto I) { raw[LB_I(I)][h] = S::encode_pair(va[LB_I(I)], vb[LB_I(I)]); });
      }
      const long long cell = (long long)(r0 + k) * g.nx + x0;
      static_for<L::Q>([&](auto I) {
        constexpr int i = LB_I(I);
        *reinterpret_cast<uint2*>(nxt + g.plane * i + cell) = make_uint2(raw[i][0], raw[i][1]);
      });
      if constexpr (SLAB) {  // the populations leaving through a face, at the cells' own (x, y)
        const int z = (r0 + k) / g.ny, y = (r0 + k) - z * g.ny;
        static_for<L::Q>([&](auto I) {
          constexpr int i = LB_I(I);
          constexpr int cz = L::c[i][2];
          const long long at = ((long long)zslot<L>(i) * g.ny + y) * g.nx + x0;
          if constexpr (cz > 0) {
            if (z == g.nz - 1) *reinterpret_cast<uint2*>(slab.send_hi + at) = make_uint2(raw[i][0], raw[i][1]);
          } else if constexpr (cz < 0) {
            if (z == 0) *reinterpret_cast<uint2*>(slab.send_lo + at) = make_uint2(raw[i][0], raw[i][1]);
          }
        });
      }
    }
  }
  if (failed && t == 0) {
    // a copy never completed: record it, then give every copy this block
    // issued (the last row issued into each stage) a bounded wait to land
    // before the block's shared memory is released
    atomicAdd(&g_stage_timeouts, 1u);
    for (int s = 0; s < kStages && s < issued; ++s) {
      const int last = s + ((issued - 1 - s) / kStages) * kStages;
      mbar_wait(bars + 8 * s, (unsigned int)((last / kStages) & 1));
    }
  }
}

// Threads per block of the staged kernel for rows of nx cells.
inline int staged_threads(int nx) { return (nx / 4 + 31) / 32 * 32; }

template <class L>
inline bool staged_eligible(const Grid& g, const void* a, const void* b) {
  return L::Q <= 19 && g.nx % 8 == 0 && staged_threads(g.nx) <= kMaxRowThreads &&
         (uintptr_t)a % 16 == 0 && (uintptr_t)b % 16 == 0;
}

// Planes [z_begin, z_end) (every plane by default); SLAB: the planes of a
// z-slab, with its halo and send buffers in `slab`.
template <class L, class S, int CT, bool SLAB = false>
inline cudaError_t launch_staged_step(const Grid& g, cudaStream_t stream, const unsigned short* cur,
                                      unsigned short* nxt, float omega, float omega_minus,
                                      const typename S::Params& p, int z_begin = 0, int z_end = -1,
                                      const SlabArgs<unsigned short>& slab = {}) {
  StagedGrid sg;
  sg.nx = g.nx;
  sg.ny = g.ny;
  sg.nz = g.nz;
  sg.plane = g.plane;
  sg.row0 = z_begin * g.ny;
  sg.rows = (z_end < 0 ? g.nz : z_end) * g.ny;
  sg.row_bytes = g.nx * 2;
  if (sg.rows <= sg.row0) return cudaSuccess;
  const size_t smem = (size_t)kStages * L::Q * sg.row_bytes + kStages * 8;
  auto kernel = fluid_step_staged_kernel<L, S, CT, SLAB>;
  if (smem > 48 * 1024) {
    const cudaError_t err =
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
  }
  const unsigned blocks = (unsigned)((sg.rows - sg.row0 + kStagedRows - 1) / kStagedRows);
  return launch_pdl(kernel, dim3(blocks), dim3((unsigned)staged_threads(g.nx)), smem, stream, cur, nxt, sg,
                    omega, omega_minus, p, slab);
}

}  // namespace lbcube
