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

// Velocity u = j / rho of deviation variables v (the moments of collide_dev).
template <class L, int FMT>
__device__ __forceinline__ void dev_velocity(const float (&v)[L::Q], float rho0, float (&u)[L::D]) {
  constexpr float S = Codec<FMT>::S;
  float dv = 0.0f, j[L::D];
  static_for<L::D>([&](auto D) { j[LB_I(D)] = 0.0f; });
  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    constexpr float w = (float)L::w[i];
    dv = fmaf(w, v[i], dv);
    static_for<L::D>([&](auto D) {
      constexpr int c = L::c[i][LB_I(D)];
      if constexpr (c > 0) j[LB_I(D)] = fmaf(w, v[i], j[LB_I(D)]);
      if constexpr (c < 0) j[LB_I(D)] = fmaf(-w, v[i], j[LB_I(D)]);
    });
  });
  const float inv = __frcp_rn(fmaf(S, rho0, dv));
  static_for<L::D>([&](auto D) { u[LB_I(D)] = j[LB_I(D)] * inv; });
}

// ---- MRT on deviation variables (D2Q9, D3Q19) -----------------------------------
// The reference MRT (collide_mrt_d2q9, lattice_mrt.hpp:586-603; collide_mrt_d3q19,
// :971-1009) relaxes the orthogonal moments m = M f towards m_eq and maps back
// with M^-1 = M^T D^-1 (D = diag |M_k|^2). In deviation form, with
// mu_k = S (m_k - rho0 m_k(rest)) = sum_j M_kj w_j v_j (m(rest) = M w, the moments
// of f = w), the post-collision deviations are
//   v_i = (1 / w_i) sum_k (M_ki / D_k) mu_post_k,
// mu_post = mu for conserved moments, mu_eq for moments relaxed with rate 1, and
// mu - s (mu - mu_eq) otherwise, where mu_eq is S (m_eq - rho0 m(rest)) of the
// reference's equilibrium moments written with R = S rho and j_v = S j = R u:
//   D2Q9  (:548-569)  e: -2 dv + 3 R u.u   eps: dv - 3 R u.u   q: -j_v
//                     p_xx: R (ux^2 - uy^2)  p_xy: R ux uy; rates 1.63, 1.14, 1.92, omega
//   D3Q19 (:908-947)  e: -11 dv + 19 R u.u  eps: 3 dv - 5.5 R u.u  q: -2/3 j_v
//                     3p_xx: 3 R (2ux^2 - uy^2 - uz^2)  p_ww: R (uy^2 - uz^2)
//                     p_xy, p_yz, p_xz: R u_a u_b; rates: omega on 9-13, 1 on the
//                     rest, ghost modes 14-18 with equilibrium 0 (:981-1001)
// Only the moments with a rate other than 1 are formed from v; algebraically
// this is the reference operator, evaluated in FP32 on the stored deviations.
template <class L>
struct DevMrt;

// kinds: 0 conserved, 1 relaxed with rate 1 (to mu_eq), 2 relaxed with rate s,
// 3 relaxed with rate 1 to an equilibrium of 0
template <>
struct DevMrt<D2Q9> {
  using Mx = Mrt9;
  static constexpr int kind[9] = {0, 2, 2, 0, 2, 0, 2, 2, 2};
  __device__ __forceinline__ static float rate(int k, float omega) {
    return k == 1 ? 1.63f : k == 2 ? 1.14f : (k == 4 || k == 6) ? 1.92f : omega;
  }
  template <int k>
  __device__ __forceinline__ static float eq(float dv, float R, const float (&u)[2], const float (&j)[2],
                                             float usq) {
    if constexpr (k == 1) return fmaf(3.0f * R, usq, -2.0f * dv);
    if constexpr (k == 2) return fmaf(-3.0f * R, usq, dv);
    if constexpr (k == 4) return -j[0];
    if constexpr (k == 6) return -j[1];
    if constexpr (k == 7) return R * (u[0] * u[0] - u[1] * u[1]);
    if constexpr (k == 8) return R * u[0] * u[1];
    return 0.0f;
  }
};

template <>
struct DevMrt<D3Q19> {
  using Mx = Mrt19;
  static constexpr int kind[19] = {0, 1, 1, 0, 1, 0, 1, 0, 1, 2, 2, 2, 2, 2, 3, 3, 3, 3, 3};
  __device__ __forceinline__ static float rate(int, float omega) { return omega; }
  template <int k>
  __device__ __forceinline__ static float eq(float dv, float R, const float (&u)[3], const float (&j)[3],
                                             float usq) {
    if constexpr (k == 1) return fmaf(19.0f * R, usq, -11.0f * dv);
    if constexpr (k == 2) return fmaf(-5.5f * R, usq, 3.0f * dv);
    if constexpr (k == 4) return (-2.0f / 3.0f) * j[0];
    if constexpr (k == 6) return (-2.0f / 3.0f) * j[1];
    if constexpr (k == 8) return (-2.0f / 3.0f) * j[2];
    if constexpr (k == 9) return 3.0f * R * (2.0f * u[0] * u[0] - u[1] * u[1] - u[2] * u[2]);
    if constexpr (k == 10) return R * (u[1] * u[1] - u[2] * u[2]);
    if constexpr (k == 11) return R * u[0] * u[1];
    if constexpr (k == 12) return R * u[1] * u[2];
    if constexpr (k == 13) return R * u[0] * u[2];
    return 0.0f;
  }
};

// Index of the momentum component a conserved moment k > 0 carries (3 -> x,
// 5 -> y, 7 -> z in both bases).
__host__ __device__ constexpr int conserved_axis(int k) { return (k - 3) / 2; }

template <class L, int FMT>
__device__ __forceinline__ void collide_dev_mrt(float (&v)[L::Q], float omega, float rho0) {
  using MR = DevMrt<L>;
  using Mx = typename MR::Mx;
  constexpr float S = Codec<FMT>::S;
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
  const float R = fmaf(S, rho0, dv);
  const float inv = __frcp_rn(R);
  float u[L::D];
  static_for<L::D>([&](auto D) { u[LB_I(D)] = j[LB_I(D)] * inv; });
  float usq = 0.0f;
  static_for<L::D>([&](auto D) { usq = fmaf(u[LB_I(D)], u[LB_I(D)], usq); });
  // post-collision deviation moments
  float mp[L::Q];
  static_for<L::Q>([&](auto KK) {
    constexpr int k = LB_I(KK);
    constexpr int kind = MR::kind[k];
    if constexpr (kind == 0) {
      if constexpr (k == 0) mp[k] = dv;
      else mp[k] = j[conserved_axis(k)];
    } else if constexpr (kind == 1) {
      mp[k] = MR::template eq<k>(dv, R, u, j, usq);
    } else if constexpr (kind == 2) {
      float m = 0.0f;
      static_for<L::Q>([&](auto JJ) {
        constexpr int jj = LB_I(JJ);
        constexpr int coef = Mx::M.m[k][jj];
        constexpr float cw = (float)(coef * L::w[jj]);
        if constexpr (coef != 0) m = fmaf(cw, v[jj], m);
      });
      const float e = MR::template eq<k>(dv, R, u, j, usq);
      mp[k] = fmaf(-MR::rate(k, omega), m - e, m);
    } else {
      mp[k] = 0.0f;
    }
  });
  static_for<L::Q>([&](auto I) {
    constexpr int i = LB_I(I);
    float acc = 0.0f;
    static_for<L::Q>([&](auto KK) {
      constexpr int k = LB_I(KK);
      constexpr int coef = Mx::M.m[k][i];
      constexpr int kind = MR::kind[k];
      constexpr float cb = (float)((double)coef / ((double)Mx::M.norm[k] * L::w[i]));
      if constexpr (coef != 0 && kind != 3) acc = fmaf(cb, mp[k], acc);
    });
    v[i] = acc;
  });
}

}  // namespace lbcube
