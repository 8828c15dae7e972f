// Collision in the stored deviation variables of the 16-bit formats.
//
// A 16-bit shifted population stores v_i = S (f_i / w_i - rho0). BGK and TRT
// are linear in f apart from the macroscopic moments, so they can run on v
// directly: with dv = sum_i w_i v_i = S (rho - rho0), j_v = sum_i w_i c_i v_i
// = S j and R = S rho = S rho0 + dv (isotropy makes sum w_i c_i = 0),
//   u = j_v / R,   v_eq_i = dv + R (3 c_i.u + 4.5 (c_i.u)^2 - 1.5 u.u),
// and the post-collision values are the reference operators (BGK,
// lattice_physics.hpp:307-318; TRT, :366-398 with Lambda = 1/4) applied to v.
// Because w_i cancels inside every opposite pair, decoding and encoding are a
// single conversion each, and FP32 works on small deviations rather than on
// values near w_i. This is algebraically the reference collision; it is not
// bit-identical to it (the 16-bit rounding dominates by orders of magnitude).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstring>

#include "collide.cuh"

namespace lbcube {

enum ShiftedFormat : int { kF16S = 0, kBF16S = 1, kE3M12S = 2, kQ15S = 3 };

// E3M12: a 16-bit format of this engine's own layout for shifted populations,
// sign | 3-bit exponent E | 12-bit mantissa m, standing for the magnitude
//   |v| = 2^(E - 6) (1 + m / 4096) - 2^-6,     E = 0 .. 7
// i.e. |v| + 2^-6 is a 13-bit-significand float. The offset makes the grid
// uniform (spacing 2^-18 = 3.8e-6) near zero and relative (2^-13) from about
// 1/64 up; |v| < 4 - 2^-6 covers every stable LB state. Against IEEE FP16 it
// gives up range for two more significand bits: 4x finer rounding of the large
// deviations that dominate the velocity error. Conversions are a few integer
// and FP32 operations (no int/float conversion instructions); encoding rounds
// to nearest (ties to even) and saturates (NaN too).
__device__ __forceinline__ float e3m12_to_float(unsigned short h) {
  // |v| + 2^-6 has FP32 exponent E - 6 + 127 and mantissa m << 11
  const float y = __uint_as_float((((unsigned int)h & 0x7FFFu) << 11) + ((127u - 6u) << 23));
  return __uint_as_float(__float_as_uint(y - 0.015625f) | (((unsigned int)h & 0x8000u) << 16));
}

__device__ __forceinline__ unsigned short float_to_e3m12(float x) {
  const unsigned int sign = (__float_as_uint(x) >> 16) & 0x8000u;
  unsigned int t = __float_as_uint(fabsf(x) + 0.015625f) - ((127u - 6u) << 23);
  t += 0x3FFu + ((t >> 11) & 1u);  // round the 23-bit mantissa to 12 bits, ties to even
  return (unsigned short)(min(t >> 11, 0x7FFFu) | sign);  // saturate (Inf, NaN, |v| >= 4 - 2^-6)
}

// Codec of each 16-bit format: the code h stands for v = S (f/w - rho0).
//   F16S   IEEE binary16, S = 4096 (normal for |f/w - rho0| > 1.5e-8, finite < 16)
//   BF16S  bfloat16, S = 1
//   E3M12S the format above, S = 1 (|f/w - rho0| < 4 - 2^-6)
//   Q15S   16-bit two's-complement fixed point, code = round(v), S = 32768: a
//          uniform 2^-15 grid over |f/w - rho0| < 1, the range of every
//          subsonic state (|u| <~ 0.2); saturating, NaN gives 0 (v = 0).
// decode2 / encode2 convert the two codes of a 32-bit word (first element in
// the low half); F16/BF16 use paired packing conversions.
template <int FMT>
struct Codec;
template <>
struct Codec<kF16S> {
  static constexpr float S = 4096.0f;
  __device__ __forceinline__ static float decode(unsigned short h) { return __half2float(__ushort_as_half(h)); }
  __device__ __forceinline__ static unsigned short encode(float v) { return __half_as_ushort(__float2half_rn(v)); }
  __device__ __forceinline__ static float2 decode2(unsigned int w) {
    __half2 h;
    memcpy(&h, &w, 4);
    return __half22float2(h);
  }
  __device__ __forceinline__ static unsigned int encode2(float a, float b) {
    const __half2 h = __floats2half2_rn(a, b);
    unsigned int w;
    memcpy(&w, &h, 4);
    return w;
  }
};
template <>
struct Codec<kBF16S> {
  static constexpr float S = 1.0f;
  __device__ __forceinline__ static float decode(unsigned short h) { return __bfloat162float(__ushort_as_bfloat16(h)); }
  __device__ __forceinline__ static unsigned short encode(float v) { return __bfloat16_as_ushort(__float2bfloat16_rn(v)); }
  __device__ __forceinline__ static float2 decode2(unsigned int w) {
    return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xFFFF0000u));
  }
  __device__ __forceinline__ static unsigned int encode2(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    unsigned int w;
    memcpy(&w, &h, 4);
    return w;
  }
};
template <>
struct Codec<kE3M12S> {
  static constexpr float S = 1.0f;
  __device__ __forceinline__ static float decode(unsigned short h) { return e3m12_to_float(h); }
  __device__ __forceinline__ static unsigned short encode(float v) { return float_to_e3m12(v); }
  __device__ __forceinline__ static float2 decode2(unsigned int w) {
    return make_float2(e3m12_to_float((unsigned short)w), e3m12_to_float((unsigned short)(w >> 16)));
  }
  __device__ __forceinline__ static unsigned int encode2(float a, float b) {
    return (unsigned int)float_to_e3m12(a) | ((unsigned int)float_to_e3m12(b) << 16);
  }
};
template <>
struct Codec<kQ15S> {
  static constexpr float S = 32768.0f;
  __device__ __forceinline__ static float decode(unsigned short h) { return (float)(short)h; }
  __device__ __forceinline__ static unsigned short encode(float v) {
    unsigned short r;
    asm("cvt.rni.sat.s16.f32 %0, %1;" : "=h"(r) : "f"(v));  // saturating, NaN gives 0
    return r;
  }
  __device__ __forceinline__ static float2 decode2(unsigned int w) {
    return make_float2((float)(short)(w & 0xFFFFu), (float)(short)(w >> 16));
  }
  __device__ __forceinline__ static unsigned int encode2(float a, float b) {
    return (unsigned int)encode(a) | ((unsigned int)encode(b) << 16);
  }
};

// Distinct lattice weights: class k of population i, and a representative.
template <class L>
struct WeightClasses {
  __host__ __device__ static constexpr int of(int i) {
    int k = 0;
    for (int a = 0; a < i; ++a) {
      bool seen = false;
      for (int b = 0; b < a; ++b) seen = seen || L::w[b] == L::w[a];
      if (!seen) {
        if (L::w[a] == L::w[i]) return k;
        ++k;
      }
    }
    return k;
  }
  __host__ __device__ static constexpr int count_() {
    int n = 0;
    for (int i = 0; i < L::Q; ++i) n = of(i) + 1 > n ? of(i) + 1 : n;
    return n;
  }
  static constexpr int count = count_();
  __host__ __device__ static constexpr int first(int k) {
    for (int i = 0; i < L::Q; ++i)
      if (of(i) == k) return i;
    return 0;
  }
};

// BGK / TRT on deviation variables v (S-scaled), see the file comment.
template <class L, int CT, int FMT>
__device__ __forceinline__ void collide_dev(float (&v)[L::Q], float omega, float omega_minus,
                                            float rho0) {
  constexpr float S = Codec<FMT>::S;
  // moments with the weights factored out: per weight class, plain sums of v
  // and of c v, then one multiply-add per class
  constexpr int K = WeightClasses<L>::count;
  float sv[K], sj[K][L::D];
  static_for<K>([&](auto k) {
    sv[LB_I(k)] = 0.0f;
    static_for<L::D>([&](auto D) { sj[LB_I(k)][LB_I(D)] = 0.0f; });
  });
  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr int k = WeightClasses<L>::of(i);
    sv[k] += v[i];
    static_for<L::D>([&](auto D) {
      constexpr int c = L::c[i][LB_I(D)];
      if constexpr (c > 0) sj[k][LB_I(D)] += v[i];
      if constexpr (c < 0) sj[k][LB_I(D)] -= v[i];
    });
  });
  float dv = 0.0f, j[L::D];
  static_for<L::D>([&](auto D) { j[LB_I(D)] = 0.0f; });
  static_for<K>([&](auto kk) {
    constexpr int k = LB_I(kk);
    constexpr float w = (float)L::w[WeightClasses<L>::first(k)];
    dv = fmaf(w, sv[k], dv);
    static_for<L::D>([&](auto D) { j[LB_I(D)] = fmaf(w, sj[k][LB_I(D)], j[LB_I(D)]); });
  });
  const float R = fmaf(S, rho0, dv);  // S rho
  const float inv = __frcp_rn(R);
  float u[L::D];
  static_for<L::D>([&](auto D) { u[LB_I(D)] = j[LB_I(D)] * inv; });
  float usq = 0.0f;
  static_for<L::D>([&](auto D) { usq = fmaf(u[LB_I(D)], u[LB_I(D)], usq); });
  const float base = fmaf(-1.5f * R, usq, dv);  // v_eq of the rest population
  const float r3 = 3.0f * R, r45 = 4.5f * R;
  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr int o = L::opp[i];
    if constexpr (i == o) {
      v[i] = fmaf(omega, base - v[i], v[i]);
    } else if constexpr (i < o) {
      const float cu = c_dot<L, i>(u);
      const float eq_even = fmaf(r45 * cu, cu, base);  // dv + R (4.5 cu^2 - 1.5 u.u)
      const float eq_odd = r3 * cu;                     // R 3 cu
      if constexpr (CT == kBGK) {
        v[i] = fmaf(omega, (eq_even + eq_odd) - v[i], v[i]);
        v[o] = fmaf(omega, (eq_even - eq_odd) - v[o], v[o]);
      } else {
        const float A = omega * fmaf(0.5f, v[i] + v[o], -eq_even);
        const float B = omega_minus * fmaf(0.5f, v[i] - v[o], -eq_odd);
        const float vi = v[i] - A - B;
        const float vo = v[o] - A + B;
        v[i] = vi;
        v[o] = vo;
      }
    }
  });
}

}  // namespace lbcube
