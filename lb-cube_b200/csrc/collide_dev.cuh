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
//   Q15S   16-bit fixed point, v = round(S (f/w - rho0)) with S = 32768: a
//          uniform 2^-15 grid over |f/w - rho0| < 1, the range of every
//          subsonic state (|u| <~ 0.2); stored offset-binary, saturating.
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
  // Stochastic rounding (sm_100a cvt.rs): each value rounds up with the
  // probability given by its discarded bits, so rounding errors carry no
  // bias. With round-to-nearest, the errors of a smooth flow are correlated
  // from step to step and cell to cell; TRT keeps its odd modes for ~1 /
  // omega_minus steps and drifts (D3Q19 256^3 Taylor-Green, 2000 steps:
  // velocity error 1.96e-3 with nearest rounding, 3.7e-4 stochastic). The
  // random bits mix both values' bit patterns by odd multipliers, so every
  // bit of them depends on the low bits of the other value of the pair: for a
  // given value they are uniform whenever the other one varies. (Two equal
  // values get bits that are a fixed scramble of the value itself, so a
  // steady uniform state rounds the same way every step, as nearest
  // rounding would.)
  __device__ __forceinline__ static unsigned int encode2(float a, float b) {
    const unsigned int rb = __float_as_uint(a) * 0x9E3779B1u + __float_as_uint(b) * 0x85EBCA77u;
    unsigned int w;
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(w) : "f"(b), "f"(a), "r"(rb));
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
  // stochastic rounding as for FP16
  __device__ __forceinline__ static unsigned int encode2(float a, float b) {
    const unsigned int rb = __float_as_uint(a) * 0x9E3779B1u + __float_as_uint(b) * 0x85EBCA77u;
    unsigned int w;
    asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(w) : "f"(b), "f"(a), "r"(rb));
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
  // float_to_e3m12 of a (low half) and b (high half), regrouped: the bias
  // subtraction joins the rounding add (the same sum mod 2^32; the bias has
  // no bits below 23, so bit 11 of the biased and unbiased words agree), and
  // the two signs go into the packed word at the end.
  __device__ __forceinline__ static unsigned int encode2(float a, float b) {
    constexpr unsigned int kRound = 0x3FFu - ((127u - 6u) << 23);
    const unsigned int ya = __float_as_uint(fabsf(a) + 0.015625f);
    const unsigned int yb = __float_as_uint(fabsf(b) + 0.015625f);
    const unsigned int ra = min((ya + kRound + ((ya >> 11) & 1u)) >> 11, 0x7FFFu);
    const unsigned int rb = min((yb + kRound + ((yb >> 11) & 1u)) >> 11, 0x7FFFu);
    return __byte_perm(ra, rb, 0x5410) | ((__float_as_uint(a) >> 16) & 0x8000u) |
           (__float_as_uint(b) & 0x80000000u);
  }
};
template <>
struct Codec<kQ15S> {
  static constexpr float S = 32768.0f;
  // code = round(v) + 32768 (offset binary). Decoding places the code in the
  // mantissa of 2^23 (0x4B00xxxx = 2^23 + code) and subtracts 2^23 + 2^15;
  // encoding adds 1.5 * 2^23 + 2^15, which rounds v to an integer (nearest,
  // ties to even) and leaves round(v) + 2^15 in the low 16 bits. Byte
  // permutes, adds, min/max and a saturating pack only: no int <-> float
  // conversion instruction. Saturating (NaN too, to one of the bounds).
  static constexpr unsigned int kDecodeHigh = 0x4B000000u;
  static constexpr float kDecodeBias = 8421376.0f;   // 2^23 + 2^15
  static constexpr float kEncodeBias = 12615680.0f;  // 1.5 * 2^23 + 2^15
  __device__ __forceinline__ static float clamp(float v) { return fminf(fmaxf(v, -32768.0f), 32767.0f); }
  __device__ __forceinline__ static float decode(unsigned short h) {
    return __uint_as_float(kDecodeHigh | h) - kDecodeBias;
  }
  __device__ __forceinline__ static unsigned short encode(float v) {
    return (unsigned short)__float_as_uint(clamp(v) + kEncodeBias);
  }
  __device__ __forceinline__ static float2 decode2(unsigned int w) {
    return make_float2(__uint_as_float(__byte_perm(w, kDecodeHigh, 0x7610)) - kDecodeBias,
                       __uint_as_float(__byte_perm(w, kDecodeHigh, 0x7632)) - kDecodeBias);
  }
  // round(v) + 2^15 as a 32-bit integer (exact for |v| < 2^22), then one
  // saturating pack of the two to 16 bits each (the first value low)
  __device__ __forceinline__ static unsigned int encode2(float a, float b) {
    const int ia = (int)(__float_as_uint(a + kEncodeBias) - 0x4B400000u);
    const int ib = (int)(__float_as_uint(b + kEncodeBias) - 0x4B400000u);
    unsigned int r;
    asm("cvt.pack.sat.u16.s32 %0, %1, %2;" : "=r"(r) : "r"(ib), "r"(ia));
    return r;
  }
};

// ---- opposite pairs and weight classes ---------------------------------------
// Every lattice here has one rest population (index 0) and (Q - 1) / 2 opposite
// pairs (i, opp[i]); pair p is the p-th i with i < opp[i], in ascending i. The
// deviation-space operators work on the pair sums s_p = v_i + v_o and
// differences d_p = v_i - v_o: dv is a weighted sum of s, j of d. Pairs with
// equal weights form a class, so each class costs one multiply.
template <class L>
struct PairsOf {
  static constexpr int count = (L::Q - 1) / 2;
  __host__ __device__ static constexpr int lo(int p) {
    int k = 0;
    for (int i = 0; i < L::Q; ++i)
      if (i < L::opp[i]) {
        if (k == p) return i;
        ++k;
      }
    return 0;
  }
  __host__ __device__ static constexpr int hi(int p) { return L::opp[lo(p)]; }
  __host__ __device__ static constexpr int klass(int p) {
    int k = 0;
    for (int a = 0; a < p; ++a) {
      bool seen = false;
      for (int b = 0; b < a; ++b) seen = seen || L::w[lo(b)] == L::w[lo(a)];
      if (!seen) {
        if (L::w[lo(a)] == L::w[lo(p)]) return k;
        ++k;
      }
    }
    return k;
  }
  __host__ __device__ static constexpr int classes() {
    int n = 0;
    for (int p = 0; p < count; ++p) n = klass(p) + 1 > n ? klass(p) + 1 : n;
    return n;
  }
  __host__ __device__ static constexpr double class_weight(int k) {
    for (int p = 0; p < count; ++p)
      if (klass(p) == k) return L::w[lo(p)];
    return 0.0;
  }
  __host__ __device__ static constexpr bool well_formed() {
    if (L::opp[0] != 0 || L::Q % 2 != 1) return false;
    for (int i = 1; i < L::Q; ++i)
      if (L::opp[i] == i || L::opp[L::opp[i]] != i || L::w[L::opp[i]] != L::w[i]) return false;
    return true;
  }
  static_assert(well_formed(), "one rest population and opposite pairs of equal weight");
};

// Adds `t` to `acc`, or starts it (no addition of a zero: x + 0 is not x for x = -0).
__device__ __forceinline__ void accumulate(float& acc, bool& first, float t) {
  acc = first ? t : acc + t;
  first = false;
}

// Pair sums and differences, dv = sum_i w_i v_i and j = sum_i w_i c_i v_i.
template <class L>
struct DevMoments {
  static constexpr int NP = PairsOf<L>::count;
  float s[NP], d[NP];
  float dv, j[L::D];
  __device__ __forceinline__ explicit DevMoments(const float (&v)[L::Q]) {
    using P = PairsOf<L>;
    constexpr int K = P::classes();
    static_for<NP>([&](auto PP) {
      constexpr int p = LB_I(PP);
      s[p] = v[P::lo(p)] + v[P::hi(p)];
      d[p] = v[P::lo(p)] - v[P::hi(p)];
    });
    dv = (float)L::w[0] * v[0];
    static_for<K>([&](auto KK) {
      constexpr int k = LB_I(KK);
      float cs = 0.0f;
      bool first = true;
      static_for<NP>([&](auto PP) {
        if constexpr (P::klass(LB_I(PP)) == k) accumulate(cs, first, s[LB_I(PP)]);
      });
      dv = fmaf((float)P::class_weight(k), cs, dv);
    });
    static_for<L::D>([&](auto DD) {
      constexpr int a = LB_I(DD);
      float ja = 0.0f;
      bool jfirst = true;
      static_for<K>([&](auto KK) {
        constexpr int k = LB_I(KK);
        float cd = 0.0f;
        bool first = true;
        static_for<NP>([&](auto PP) {
          constexpr int p = LB_I(PP);
          constexpr int c = L::c[P::lo(p)][a];
          if constexpr (P::klass(p) == k && c != 0) accumulate(cd, first, c > 0 ? d[p] : -d[p]);
        });
        if (!first) {
          const float t = (float)P::class_weight(k) * cd;
          ja = jfirst ? t : fmaf((float)P::class_weight(k), cd, ja);
          jfirst = false;
        }
      });
      j[a] = ja;
    });
  }
};

// 1 / x to within one ulp (the 16-bit paths round far more coarsely).
__device__ __forceinline__ float fast_rcp(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// BGK / TRT on deviation variables v (S-scaled), see the file comment. With
// v_eq_i = E_i + O_i split into the part even in c_i (E = dv + R (4.5 (c.u)^2 -
// 1.5 u.u)) and the odd part (O = 3 R c.u), BGK is v_i' = (1 - omega) v_i +
// omega v_eq_i. TRT relaxes the even part of a pair with omega and the odd part
// with omega_minus:
//   v_i' = (1 - (omega + omega_minus) / 2) v_i + ((omega_minus - omega) / 2) v_o
//          + omega E_i + omega_minus O_i,
// and the reference's magic parameter Lambda = 1/4 (compute_omega_minus,
// lattice_physics.hpp:336-344) makes omega + omega_minus = 2 exactly
// ((tau+ - 1/2)(tau- - 1/2) = 1/4 gives 1/tau+ + 1/tau- = 2), so the first
// term vanishes: each post-collision population is one multiply-add of its
// opposite plus the equilibrium. (omega_minus is the float of that value; the
// dropped term is below 1e-7 of v, far under the 16-bit rounding.)
template <class L, int CT, int FMT>
__device__ __forceinline__ void collide_dev(float (&v)[L::Q], float omega, float omega_minus,
                                            float rho0) {
  using P = PairsOf<L>;
  constexpr float S = Codec<FMT>::S;
  const DevMoments<L> m(v);
  const float R = fmaf(S, rho0, m.dv);  // S rho
  const float inv = fast_rcp(R);
  float u[L::D];
  static_for<L::D>([&](auto D) { u[LB_I(D)] = m.j[LB_I(D)] * inv; });
  float usq = u[0] * u[0];
  static_for<L::D - 1>([&](auto D) { usq = fmaf(u[LB_I(D) + 1], u[LB_I(D) + 1], usq); });
  const float base = fmaf(-1.5f * R, usq, m.dv);  // E of the rest population
  const float ob = omega * base;
  const float o45 = (4.5f * omega) * R;
  const float o3 = (3.0f * (CT == kTRT ? omega_minus : omega)) * R;
  const float a = CT == kTRT ? 0.5f * (omega_minus - omega) : 1.0f - omega;
  v[0] = fmaf(1.0f - omega, v[0], ob);
  static_for<P::count>([&](auto PP) {
    constexpr int i = P::lo(LB_I(PP)), o = P::hi(LB_I(PP));
    const float cu = c_dot<L, i>(u);
    const float oe = fmaf(o45 * cu, cu, ob);  // omega E_i = omega E_o
    const float vi = v[i], vo = v[o];
    if constexpr (CT == kTRT) {
      v[i] = fmaf(a, vo, fmaf(o3, cu, oe));
      v[o] = fmaf(a, vi, fmaf(o3, -cu, oe));
    } else {
      v[i] = fmaf(a, vi, fmaf(o3, cu, oe));
      v[o] = fmaf(a, vo, fmaf(o3, -cu, oe));
    }
  });
}

// Velocity u = j / rho of deviation variables v (the moments of collide_dev).
template <class L, int FMT>
__device__ __forceinline__ void dev_velocity(const float (&v)[L::Q], float rho0, float (&u)[L::D]) {
  constexpr float S = Codec<FMT>::S;
  const DevMoments<L> m(v);
  const float inv = fast_rcp(fmaf(S, rho0, m.dv));
  static_for<L::D>([&](auto D) { u[LB_I(D)] = m.j[LB_I(D)] * inv; });
}

// ---- MRT on deviation variables (D2Q9, D3Q19) -----------------------------------
// The reference MRT (collide_mrt_d2q9, lattice_mrt.hpp:586-603; collide_mrt_d3q19,
// :971-1009) relaxes the orthogonal moments m = M f towards m_eq and maps back
// with M^-1 = M^T D^-1 (D = diag |M_k|^2). In deviation form, with
// mu_k = S (m_k - rho0 m_k(rest)) = sum_j M_kj w_j v_j, the post-collision
// moments are mu_k (conserved), mu_eq_k (rate 1), 0 (rate 1 to a zero
// equilibrium: the D3Q19 ghost modes 14-18, :981-1001) or
// mu_eq_k + (1 - s_k)(mu_k - mu_eq_k), so that
//   v_i' = G_i + sum_k (1 - s_k) N_ik (mu_k - mu_eq_k),
//   G_i  = (1 / w_i) sum_k (M_ki / D_k) mu_eq_k,    N_ik = M_ki / (D_k w_i),
// the second sum over the moments relaxed at a rate other than 1. mu_eq is
// linear in the basis B = (dv, j_a, R u_a u_b) (R = S rho, j = R u), read off the
// reference's equilibrium moments:
//   D2Q9  (:548-569)  e: -2 dv + 3 R u.u   eps: dv - 3 R u.u   q: -j
//                     p_xx: R (ux^2 - uy^2)  p_xy: R ux uy; rates 1.63, 1.14, 1.92, omega
//   D3Q19 (:908-947)  e: -11 dv + 19 R u.u  eps: 3 dv - 5.5 R u.u  q: -2/3 j
//                     3p_xx: 3 R (2ux^2 - uy^2 - uz^2)  p_ww: R (uy^2 - uz^2)
//                     p_xy, p_yz, p_xz: R u_a u_b; rates: omega on 9-13, 1 on the rest
// so G_i = sum_q CG_iq B_q with compile-time coefficients. Both G and N split
// into a part even and a part odd in c_i, shared by the two populations of a
// pair. Algebraically this is the reference operator, evaluated in FP32 on the
// stored deviations.
template <class L>
struct DevMrt;

// Basis of the equilibrium moments: 0 = dv, 1..D = j_a, then R u_a u_b for
// (a, b) in QA / QB order.
template <int D>
struct QuadBasis;
template <>
struct QuadBasis<2> {
  static constexpr int n = 3;
  static constexpr int a[3] = {0, 1, 0}, b[3] = {0, 1, 1};
};
template <>
struct QuadBasis<3> {
  static constexpr int n = 6;
  static constexpr int a[6] = {0, 1, 2, 0, 1, 0}, b[6] = {0, 1, 2, 1, 2, 2};
};

// kinds: 0 conserved, 1 relaxed with rate 1 (to mu_eq), 2 relaxed with rate s,
// 3 relaxed with rate 1 to an equilibrium of 0
template <>
struct DevMrt<D2Q9> {
  using Mx = Mrt9;
  static constexpr int kind[9] = {0, 2, 2, 0, 2, 0, 2, 2, 2};
  __device__ __forceinline__ static float rate(int k, float omega) {
    return k == 1 ? 1.63f : k == 2 ? 1.14f : (k == 4 || k == 6) ? 1.92f : omega;
  }
  // eq[k][q]: basis (dv, jx, jy, Rxx, Ryy, Rxy)
  static constexpr double eq[9][6] = {
      {1, 0, 0, 0, 0, 0},  {-2, 0, 0, 3, 3, 0}, {1, 0, 0, -3, -3, 0},
      {0, 1, 0, 0, 0, 0},  {0, -1, 0, 0, 0, 0}, {0, 0, 1, 0, 0, 0},
      {0, 0, -1, 0, 0, 0}, {0, 0, 0, 1, -1, 0}, {0, 0, 0, 0, 0, 1}};
};

template <>
struct DevMrt<D3Q19> {
  using Mx = Mrt19;
  static constexpr int kind[19] = {0, 1, 1, 0, 1, 0, 1, 0, 1, 2, 2, 2, 2, 2, 3, 3, 3, 3, 3};
  __device__ __forceinline__ static float rate(int, float omega) { return omega; }
  // eq[k][q]: basis (dv, jx, jy, jz, Rxx, Ryy, Rzz, Rxy, Ryz, Rxz)
  static constexpr double eq[19][10] = {
      {1, 0, 0, 0, 0, 0, 0, 0, 0, 0},         {-11, 0, 0, 0, 19, 19, 19, 0, 0, 0},
      {3, 0, 0, 0, -5.5, -5.5, -5.5, 0, 0, 0}, {0, 1, 0, 0, 0, 0, 0, 0, 0, 0},
      {0, -2.0 / 3.0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 1, 0, 0, 0, 0, 0, 0, 0},
      {0, 0, -2.0 / 3.0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 1, 0, 0, 0, 0, 0, 0},
      {0, 0, 0, -2.0 / 3.0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 6, -3, -3, 0, 0, 0},
      {0, 0, 0, 0, 0, 1, -1, 0, 0, 0},         {0, 0, 0, 0, 0, 0, 0, 1, 0, 0},
      {0, 0, 0, 0, 0, 0, 0, 0, 1, 0},         {0, 0, 0, 0, 0, 0, 0, 0, 0, 1},
      {0, 0, 0, 0, 0, 0, 0, 0, 0, 0},         {0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
      {0, 0, 0, 0, 0, 0, 0, 0, 0, 0},         {0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
      {0, 0, 0, 0, 0, 0, 0, 0, 0, 0}};
};

// Compile-time coefficients of the deviation MRT of lattice L.
template <class L>
struct DevMrtCoef {
  using MR = DevMrt<L>;
  using Mx = typename MR::Mx;
  static constexpr int NB = 1 + L::D + QuadBasis<L::D>::n;
  // G_i = sum_q g(i, q) B_q
  __host__ __device__ static constexpr double g(int i, int q) {
    double acc = 0.0;
    for (int k = 0; k < L::Q; ++k)
      if (MR::kind[k] != 3) acc += (double)Mx::M.m[k][i] * MR::eq[k][q] / (double)Mx::M.norm[k];
    return acc / L::w[i];
  }
  __host__ __device__ static constexpr double n(int i, int k) {
    return (double)Mx::M.m[k][i] / ((double)Mx::M.norm[k] * L::w[i]);
  }
  // coefficients that cancel exactly may leave a double rounding residue
  __host__ __device__ static constexpr bool nonzero(double x) { return x > 1e-9 || x < -1e-9; }
  // basis element q (or moment k) is odd under c -> -c
  __host__ __device__ static constexpr bool odd_basis(int q) { return q >= 1 && q <= L::D; }
  __host__ __device__ static constexpr bool even_moment(int k) {
    for (int i = 0; i < L::Q; ++i)
      if (Mx::M.m[k][i] != Mx::M.m[k][L::opp[i]]) return false;
    return true;
  }
  __host__ __device__ static constexpr bool odd_moment(int k) {
    for (int i = 0; i < L::Q; ++i)
      if (Mx::M.m[k][i] != -Mx::M.m[k][L::opp[i]]) return false;
    return true;
  }
  __host__ __device__ static constexpr bool well_formed() {
    for (int k = 0; k < L::Q; ++k)
      if (!even_moment(k) && !odd_moment(k)) return false;
    return true;
  }
  static_assert(well_formed(), "every moment is even or odd in c");
};

template <class L, int FMT>
__device__ __forceinline__ void collide_dev_mrt(float (&v)[L::Q], float omega, float rho0) {
  using MR = DevMrt<L>;
  using Mx = typename MR::Mx;
  using C = DevMrtCoef<L>;
  using P = PairsOf<L>;
  using QB = QuadBasis<L::D>;
  constexpr float S = Codec<FMT>::S;
  const DevMoments<L> m(v);
  const float R = fmaf(S, rho0, m.dv);
  const float inv = fast_rcp(R);
  float B[C::NB];
  B[0] = m.dv;
  float u[L::D], Ru[L::D];
  static_for<L::D>([&](auto D) {
    constexpr int a = LB_I(D);
    B[1 + a] = m.j[a];
    u[a] = m.j[a] * inv;
    Ru[a] = m.j[a];  // R u_a = j_a
  });
  static_for<QB::n>([&](auto QQ) {
    constexpr int q = LB_I(QQ);
    constexpr int qa = QB::a[q], qb = QB::b[q];
    B[1 + L::D + q] = Ru[qa] * u[qb];
  });
  // (1 - s_k) (mu_k - mu_eq_k) of the moments relaxed at a rate other than 1
  float nd[L::Q];
  static_for<L::Q>([&](auto KK) {
    constexpr int k = LB_I(KK);
    if constexpr (MR::kind[k] == 2) {
      float mu = 0.0f;
      bool first = true;
      if constexpr (C::even_moment(k) && Mx::M.m[k][0] != 0) {
        constexpr float c0w = (float)(Mx::M.m[k][0] * L::w[0]);
        accumulate(mu, first, c0w * v[0]);
      }
      static_for<P::count>([&](auto PP) {
        constexpr int p = LB_I(PP);
        constexpr int coef = Mx::M.m[k][P::lo(p)];
        constexpr float cw = (float)(coef * L::w[P::lo(p)]);
        if constexpr (coef != 0) {
          const float x = C::even_moment(k) ? m.s[p] : m.d[p];
          mu = first ? cw * x : fmaf(cw, x, mu);
          first = false;
        }
      });
      float e = 0.0f;
      bool efirst = true;
      static_for<C::NB>([&](auto QQ) {
        constexpr double cq = MR::eq[k][LB_I(QQ)];
        if constexpr (cq != 0.0) {
          e = efirst ? (float)cq * B[LB_I(QQ)] : fmaf((float)cq, B[LB_I(QQ)], e);
          efirst = false;
        }
      });
      nd[k] = (1.0f - MR::rate(k, omega)) * (mu - e);
    }
  });
  // G_i + sum_k N_ik nd_k, split into the parts even (E) and odd (O) in c_i
  auto part = [&](auto II, auto ODD) {
    constexpr int i = LB_I(II);
    constexpr bool odd = decltype(ODD)::value;
    float acc = 0.0f;
    bool first = true;
    static_for<C::NB>([&](auto QQ) {
      constexpr int q = LB_I(QQ);
      constexpr float cg = (float)C::g(i, q);
      if constexpr (C::odd_basis(q) == odd && C::nonzero(C::g(i, q))) {
        acc = first ? cg * B[q] : fmaf(cg, B[q], acc);
        first = false;
      }
    });
    static_for<L::Q>([&](auto KK) {
      constexpr int k = LB_I(KK);
      constexpr float cn = (float)C::n(i, k);
      if constexpr (MR::kind[k] == 2 && C::odd_moment(k) == odd && Mx::M.m[k][i] != 0) {
        acc = first ? cn * nd[k] : fmaf(cn, nd[k], acc);
        first = false;
      }
    });
    return acc;
  };
  v[0] = part(std::integral_constant<int, 0>{}, std::false_type{});
  static_for<P::count>([&](auto PP) {
    constexpr int i = P::lo(LB_I(PP)), o = P::hi(LB_I(PP));
    const float E = part(std::integral_constant<int, i>{}, std::false_type{});
    const float O = part(std::integral_constant<int, i>{}, std::true_type{});
    v[i] = E + O;
    v[o] = E - O;
  });
}

}  // namespace lbcube
