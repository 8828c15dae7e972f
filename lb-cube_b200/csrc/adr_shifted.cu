// The coupled fluid + A + B -> C step (fluid_reaction_kernel of adr.cu) on
// shifted 16-bit populations. No reference counterpart.
//
// The fluid is stored as codes of v_i = S (f_i / w_i - rho0) and collides on
// the deviations (collide_dev / collide_dev_mrt); the two scalars are stored as
// codes of S (g_i / w_i - c0) with c0 a reference concentration, decoded to
// FP32, advected and reacted exactly as in the FP32 step (react_pair: the
// scalar BGK with the exact A + B -> C source, lattice_physics.hpp:677-743)
// with the fluid velocity of the post-collision deviations, and re-encoded.
// Halves the bytes of the coupled step (D3Q19 + 2 D3Q7: 132 B per cell
// instead of 264). Statistics, when requested, are those of the FP32 values
// the step encodes.
#include "adr_shifted.cuh"
#include "cells.cuh"
#include "collide.cuh"
#include "collide_dev.cuh"
#include "common.cuh"
#include "reduce.cuh"
#include "slab_faces.cuh"
#include "stream_vec.cuh"
#include "../../include/lbcube_b200.h"

namespace lbcube {

// Pull-gather of 16-bit codes, decoded to deviations (fluid) or to
// populations (scalars, shifted by c0).
template <class L, int FMT, bool DEVIATION>
__device__ __forceinline__ void gather_codes(const unsigned short* __restrict__ cur, const Grid& g,
                                             const Neighbours& n, int x, int y, int z, float c0,
                                             float (&out)[L::Q]) {
  const size_t plane = (size_t)g.plane;
  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
    const int sx = cx == 0 ? x : (cx > 0 ? n.xm : n.xp);
    const int sy = cy == 0 ? y : (cy > 0 ? n.ym : n.yp);
    const int sz = cz == 0 ? z : (cz > 0 ? n.zm : n.zp);
    const unsigned short h = __ldg(cur + plane * i + ((sz * g.ny + sy) * g.nx + sx));
    if constexpr (DEVIATION) out[i] = Codec<FMT>::decode(h);
    else out[i] = ShiftedStorage<FMT>::template decode<L, i>(h, {c0});
  });
}

// Pull-gather of 16-bit codes on a z-slab (halo planes of codes at the faces,
// slab_faces.cuh), decoded as gather_codes does.
template <class L, int FMT, bool DEVIATION>
__device__ __forceinline__ void gather_codes_slab(const unsigned short* __restrict__ cur, const Grid& g,
                                                  const Neighbours& n, int x, int y, int z, float c0,
                                                  const unsigned short* __restrict__ halo_lo,
                                                  const unsigned short* __restrict__ halo_hi,
                                                  float (&out)[L::Q]) {
  unsigned short h[L::Q];
  gather_slab<L>(cur, g, n, x, y, z, halo_lo, halo_hi, h);
  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    if constexpr (DEVIATION) out[i] = Codec<FMT>::decode(h[i]);
    else out[i] = ShiftedStorage<FMT>::template decode<L, i>(h[i], {c0});
  });
}

// The face buffers of a slab of 16-bit states (codes; layout of slab_faces.cuh).
struct CodeFaces {
  const unsigned short* halo_lo;
  const unsigned short* halo_hi;
  unsigned short* send_lo;
  unsigned short* send_hi;
};

// SLAB: a z-slab of a box, the pulls across its faces from `faces` and the
// leaving codes stored into its send buffers (every plane of the slab).
template <class FL, int FMT, int CT, bool STATS, bool UOUT, bool SLAB = false>
__global__ void __launch_bounds__(kThreads)
    fluid_reaction_shifted_kernel(const unsigned short* __restrict__ cur_f,
                                  unsigned short* __restrict__ nxt_f,
                                  const unsigned short* __restrict__ cur_a,
                                  unsigned short* __restrict__ nxt_a,
                                  const unsigned short* __restrict__ cur_b,
                                  unsigned short* __restrict__ nxt_b, Grid g, float omega,
                                  float omega_minus, float omega_c, float k, float rho0, float c0,
                                  double* __restrict__ partials, float* __restrict__ u_out,
                                  CodeFaces faces = {}) {
  using SL = typename ScalarOf<FL>::type;
  const size_t a_off = (size_t)face_planes<FL>() * g.ny * g.nx;
  const size_t b_off = a_off + (size_t)face_planes<SL>() * g.ny * g.nx;
  pdl_enter();
  int x, y, z;
  const bool active = cell_of(g, x, y, z);
  double sums[kStatSums] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (active) {
    const int cell = (z * g.ny + y) * g.nx + x;
    const size_t plane = (size_t)g.plane;
    const Neighbours n = neighbours(g, x, y, z);
    float v[FL::Q], u[FL::D];
    if constexpr (SLAB) gather_codes_slab<FL, FMT, true>(cur_f, g, n, x, y, z, 0.0f, faces.halo_lo, faces.halo_hi, v);
    else gather_codes<FL, FMT, true>(cur_f, g, n, x, y, z, 0.0f, v);
    if constexpr (CT == kMRT) collide_dev_mrt<FL, FMT>(v, omega, rho0);
    else collide_dev<FL, CT, FMT>(v, omega, omega_minus, rho0);
    unsigned short hf[FL::Q];
    static_for<FL::Q>([&](auto I) {
      hf[LB_I(I)] = Codec<FMT>::encode(v[LB_I(I)]);
      nxt_f[plane * LB_I(I) + cell] = hf[LB_I(I)];
    });
    if constexpr (SLAB) send_slab<FL>(g, x, y, z, hf, faces.send_lo, faces.send_hi);
    dev_velocity<FL, FMT>(v, rho0, u);
    if constexpr (UOUT) static_for<FL::D>([&](auto D) { u_out[plane * LB_I(D) + cell] = u[LB_I(D)]; });
    float a[SL::Q], b[SL::Q];
    if constexpr (SLAB) {
      gather_codes_slab<SL, FMT, false>(cur_a, g, n, x, y, z, c0, faces.halo_lo + a_off, faces.halo_hi + a_off, a);
      gather_codes_slab<SL, FMT, false>(cur_b, g, n, x, y, z, c0, faces.halo_lo + b_off, faces.halo_hi + b_off, b);
    } else {
      gather_codes<SL, FMT, false>(cur_a, g, n, x, y, z, c0, a);
      gather_codes<SL, FMT, false>(cur_b, g, n, x, y, z, c0, b);
    }
    react_pair<SL>(a, b, u, omega_c, k);
    const typename ShiftedStorage<FMT>::Params sp{c0};
    unsigned short ha[SL::Q], hb[SL::Q];
    static_for<SL::Q>([&](auto I) {
      constexpr int i = LB_I(I);
      ha[i] = ShiftedStorage<FMT>::template encode<SL, i>(a[i], sp);
      hb[i] = ShiftedStorage<FMT>::template encode<SL, i>(b[i], sp);
      nxt_a[plane * i + cell] = ha[i];
      nxt_b[plane * i + cell] = hb[i];
    });
    if constexpr (SLAB) {
      send_slab<SL>(g, x, y, z, ha, faces.send_lo + a_off, faces.send_hi + a_off);
      send_slab<SL>(g, x, y, z, hb, faces.send_lo + b_off, faces.send_hi + b_off);
    }
    if constexpr (STATS) {
      const double sa = (double)concentration<SL>(a), sb = (double)concentration<SL>(b);
      sums[0] = sa;
      sums[1] = sb;
      sums[2] = sa * sa;
      sums[3] = sb * sb;
      sums[4] = sa * sb;
    }
  }
  if constexpr (STATS) block_sum_to<kStatSums>(sums, partials + block_linear() * kStatSums);
}

template <class FL, int FMT, int CT>
cudaError_t launch_shifted_coupled(const unsigned short* cf, unsigned short* nf,
                                   const unsigned short* ca, unsigned short* na,
                                   const unsigned short* cb, unsigned short* nb, float* u_out,
                                   double* partials, const Grid& g, float omega, float omega_c,
                                   float k, float rho0, float c0, cudaStream_t s) {
  const float om = CT == kTRT ? trt_omega_minus<float>(omega) : 0.0f;
  // programmatic dependent launches (the kernel opens with pdl_enter)
#define LBCUBE_SC(ST, UO)                                                                          \
  return launch_pdl(fluid_reaction_shifted_kernel<FL, FMT, CT, ST, UO, false>, grid_dims(g),      \
                    dim3(block_dims(g)), 0, s, cf, nf, ca, na, cb, nb, g, omega, om, omega_c, k,  \
                    rho0, c0, partials, u_out, CodeFaces{})
  if (partials != nullptr && u_out != nullptr) LBCUBE_SC(true, true);
  if (partials != nullptr) LBCUBE_SC(true, false);
  if (u_out != nullptr) LBCUBE_SC(false, true);
  LBCUBE_SC(false, false);
#undef LBCUBE_SC
}

template <class FL, int FMT>
cudaError_t fluid_reaction_shifted(int collision, const unsigned short* cur_f,
                                   unsigned short* nxt_f, const unsigned short* cur_a,
                                   unsigned short* nxt_a, const unsigned short* cur_b,
                                   unsigned short* nxt_b, float* u_out, double* partials,
                                   const Grid& g, float omega, float omega_c, float k, float rho0,
                                   float c0, cudaStream_t s) {
  switch (collision) {
    case kBGK:
      return launch_shifted_coupled<FL, FMT, kBGK>(cur_f, nxt_f, cur_a, nxt_a, cur_b, nxt_b, u_out,
                                                   partials, g, omega, omega_c, k, rho0, c0, s);
    case kTRT:
      return launch_shifted_coupled<FL, FMT, kTRT>(cur_f, nxt_f, cur_a, nxt_a, cur_b, nxt_b, u_out,
                                                   partials, g, omega, omega_c, k, rho0, c0, s);
    case kMRT:
      if constexpr (FL::Q != 27)
        return launch_shifted_coupled<FL, FMT, kMRT>(cur_f, nxt_f, cur_a, nxt_a, cur_b, nxt_b,
                                                     u_out, partials, g, omega, omega_c, k, rho0,
                                                     c0, s);
      return cudaErrorInvalidValue;
    default: return cudaErrorInvalidValue;
  }
}

// The slab form of fluid_reaction_shifted (all planes, no statistics; u_out
// may be null). Buffers are checked by the caller.
template <class FL, int FMT>
cudaError_t fluid_reaction_shifted_slab(int collision, const unsigned short* cur_f,
                                        unsigned short* nxt_f, const unsigned short* cur_a,
                                        unsigned short* nxt_a, const unsigned short* cur_b,
                                        unsigned short* nxt_b, float* u_out, const Grid& g,
                                        float omega, float omega_c, float k, float rho0, float c0,
                                        const unsigned short* halo_lo, const unsigned short* halo_hi,
                                        unsigned short* send_lo, unsigned short* send_hi,
                                        cudaStream_t s) {
  // planes 1 .. nz-2 neither pull nor send across a face: the whole-box
  // kernel (fewer registers); planes 0 and nz-1: the SLAB form
  const CodeFaces faces{halo_lo, halo_hi, send_lo, send_hi};
  auto launch = [&](auto ct) -> cudaError_t {
    constexpr int CT = decltype(ct)::value;
    const float om = CT == kTRT ? trt_omega_minus<float>(omega) : 0.0f;
    auto range = [&](int z0, int planes, int zs, auto slab) {
      constexpr bool SLAB = decltype(slab)::value;
      Grid gr = g;
      gr.z0 = z0;
      gr.zs = zs;
      dim3 grid = grid_dims(gr);
      grid.y = (unsigned)planes;
      const dim3 block(block_dims(gr));
      double* const none = nullptr;
      if (u_out != nullptr)
        launch_pdl(fluid_reaction_shifted_kernel<FL, FMT, CT, false, true, SLAB>, grid, block, 0, s, cur_f,
                   nxt_f, cur_a, nxt_a, cur_b, nxt_b, gr, omega, om, omega_c, k, rho0, c0, none, u_out, faces);
      else
        launch_pdl(fluid_reaction_shifted_kernel<FL, FMT, CT, false, false, SLAB>, grid, block, 0, s, cur_f,
                   nxt_f, cur_a, nxt_a, cur_b, nxt_b, gr, omega, om, omega_c, k, rho0, c0, none,
                   (float*)nullptr, faces);
    };
    if (g.nz >= 3) range(1, g.nz - 2, 1, std::false_type{});
    range(0, g.nz >= 2 ? 2 : 1, g.nz - 1, std::true_type{});  // both face planes in one launch
    return cudaGetLastError();
  };
  switch (collision) {
    case kBGK: return launch(std::integral_constant<int, kBGK>{});
    case kTRT: return launch(std::integral_constant<int, kTRT>{});
    case kMRT:
      if constexpr (FL::Q != 27) return launch(std::integral_constant<int, kMRT>{});
      return cudaErrorInvalidValue;
    default: return cudaErrorInvalidValue;
  }
}

#define LBCUBE_FRSS(FL, F)                                                                        \
  template cudaError_t fluid_reaction_shifted_slab<FL, F>(                                        \
      int, const unsigned short*, unsigned short*, const unsigned short*, unsigned short*,        \
      const unsigned short*, unsigned short*, float*, const Grid&, float, float, float, float,    \
      float, const unsigned short*, const unsigned short*, unsigned short*, unsigned short*,      \
      cudaStream_t);
LBCUBE_FRSS(D3Q19, kF16S)
LBCUBE_FRSS(D3Q19, kBF16S)
LBCUBE_FRSS(D3Q19, kE3M12S)
LBCUBE_FRSS(D3Q19, kQ15S)
LBCUBE_FRSS(D3Q27, kF16S)
LBCUBE_FRSS(D3Q27, kBF16S)
LBCUBE_FRSS(D3Q27, kE3M12S)
LBCUBE_FRSS(D3Q27, kQ15S)
#undef LBCUBE_FRSS

#define LBCUBE_FRS(FL, F)                                                                         \
  template cudaError_t fluid_reaction_shifted<FL, F>(                                             \
      int, const unsigned short*, unsigned short*, const unsigned short*, unsigned short*,        \
      const unsigned short*, unsigned short*, float*, double*, const Grid&, float, float, float,  \
      float, float, cudaStream_t);
#define LBCUBE_FRS_ALL(FL) LBCUBE_FRS(FL, kF16S) LBCUBE_FRS(FL, kBF16S) LBCUBE_FRS(FL, kE3M12S) LBCUBE_FRS(FL, kQ15S)
LBCUBE_FRS_ALL(D2Q9)
LBCUBE_FRS_ALL(D3Q19)
LBCUBE_FRS_ALL(D3Q27)
#undef LBCUBE_FRS_ALL
#undef LBCUBE_FRS

template <int FMT>
cudaError_t coupled_by_lattice(int lattice, int collision, const void* cf, void* nf, const void* ca,
                               void* na, const void* cb, void* nb, size_t nx, size_t ny, size_t nz,
                               double omega, double omega_c, double k, float rho0, float c0,
                               double* partials, size_t pbytes, cudaStream_t s) {
  const int dims = lattice == kD2Q9 ? 2 : 3;
  Grid g;
  cudaError_t err = validate_domain(cf == nullptr || nf == nullptr || ca == nullptr ||
                                        na == nullptr || cb == nullptr || nb == nullptr,
                                    1, 1, 1, dims, nx, ny, nz, g);
  if (err != cudaSuccess) return err;
  const int FQ = lattice == kD2Q9 ? 9 : (lattice == kD3Q19 ? 19 : 27), SQ = dims == 2 ? 5 : 7;
  const size_t fb = (size_t)FQ * g.plane * 2, sb = (size_t)SQ * g.plane * 2;
  const size_t need = partials != nullptr ? (size_t)g.blocks() * kStatSums * sizeof(double) : 0;
  if (partials != nullptr && pbytes < need) return cudaErrorInvalidValue;
  const Span reads[3] = {{cf, fb}, {ca, sb}, {cb, sb}};
  const Span writes[4] = {{nf, fb}, {na, sb}, {nb, sb}, {partials, need}};
  if (any_overlap(reads, writes)) return cudaErrorInvalidValue;
  using U = unsigned short;
#define LBCUBE_CL(FL)                                                                             \
  return fluid_reaction_shifted<FL, FMT>(collision, (const U*)cf, (U*)nf, (const U*)ca, (U*)na, \
                                         (const U*)cb, (U*)nb, nullptr, partials, g, (float)omega, \
                                         (float)omega_c, (float)k, rho0, c0, s)
  switch (lattice) {
    case kD2Q9: LBCUBE_CL(D2Q9);
    case kD3Q19: LBCUBE_CL(D3Q19);
    case kD3Q27: LBCUBE_CL(D3Q27);
    default: return cudaErrorInvalidValue;
  }
#undef LBCUBE_CL
}

}  // namespace lbcube

using namespace lbcube;

extern "C" int lbm_fluid_reaction_ab_shifted_async(
    int fluid_lattice, int format, int collision, const void* current_fluid, void* next_fluid,
    const void* current_a, void* next_a, const void* current_b, void* next_b, size_t x_extent,
    size_t y_extent, size_t z_extent, double omega, double omega_c, double k_react, float rho0,
    float c0, double* stats_partials, size_t stats_partials_bytes, void* stream) {
  const cudaStream_t s = as_stream(stream);
#define LBCUBE_FMT(F)                                                                              \
  return (int)coupled_by_lattice<F>(fluid_lattice, collision, current_fluid, next_fluid,          \
                                    current_a, next_a, current_b, next_b, x_extent, y_extent,     \
                                    z_extent, omega, omega_c, k_react, rho0, c0, stats_partials,  \
                                    stats_partials_bytes, s)
  if (format == LBM_F16S) LBCUBE_FMT(kF16S);
  if (format == LBM_BF16S) LBCUBE_FMT(kBF16S);
  if (format == LBM_E3M12S) LBCUBE_FMT(kE3M12S);
  if (format == LBM_Q15S) LBCUBE_FMT(kQ15S);
#undef LBCUBE_FMT
  return (int)cudaErrorInvalidValue;
}
