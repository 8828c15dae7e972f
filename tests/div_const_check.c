/* Test helper: compares the division-free FP32 quotient x / D of the D3Q27
 * population transform (div_exact_const in lb-cube_b200/csrc/collide.cuh:
 * q0 = RN(x * RN(1/D)), r = fma(-q0, D, x), q = fma(r, RN(1/D), q0)) with the
 * IEEE quotient, bit for bit, over FP32 bit patterns [lo, hi] of both signs.
 * The host's fmaf and float multiply are the same IEEE operations as the
 * device's __fmaf_rn and __fmul_rn (round to nearest even, subnormals kept).
 *
 * usage: div_const_check D lo hi      (lo, hi: magnitude bit patterns, hex)
 * prints: "<evaluated> <mismatches> <mismatches with finite nonzero x and
 *          |x| >= 2^-124> <largest |x| of a finite nonzero mismatch>"
 *
 * FP64 (no exhaustive check possible): div_const_check D f64 N seed draws N
 * random bit patterns over every exponent and N dividends whose quotient lies
 * within an ulp fraction of a rounding midpoint (x = RN(D * odd * 2^e), the
 * hardest cases for rounding), and prints "<evaluated> <mismatches with
 * finite x, |x| >= 2^-960>".
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static float f_of(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static uint32_t u_of(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

static uint64_t next(uint64_t* s) {  /* xorshift64* */
  *s ^= *s >> 12; *s ^= *s << 25; *s ^= *s >> 27;
  return *s * 0x2545F4914F6CDD1DULL;
}

static int check64(double x, double d) {
  const double z = 1.0 / d;
  const double q0 = x * z;
  const double r = fma(-q0, d, x);
  const double q = fma(r, z, q0);
  const double ref = x / d;
  uint64_t a, b;
  memcpy(&a, &q, 8); memcpy(&b, &ref, 8);
  return a == b || !(isfinite(x) && fabs(x) >= 0x1p-960);
}

static int main64(double d, long long count, uint64_t seed) {
  unsigned long long n = 0, bad = 0;
#pragma omp parallel for reduction(+ : n, bad) schedule(static)
  for (long long i = 0; i < count; ++i) {
    uint64_t s = seed * 0x9E3779B97F4A7C15ULL + (uint64_t)i * 0xBF58476D1CE4E5B9ULL + 1;
    next(&s);
    uint64_t bits = next(&s);
    double x;
    memcpy(&x, &bits, 8);
    bad += !check64(x, d);
    /* near a midpoint: the quotient is odd * 2^(e-1) with a 54-bit odd significand */
    const uint64_t odd = (next(&s) >> 10) | 1u | (1ULL << 53);
    const int e = (int)(next(&s) % 2000) - 1000;
    x = ldexp((double)((__int128)odd * (__int128)(long long)d), e - 1);
    if ((next(&s) & 1u) != 0) x = -x;
    bad += !check64(x, d);
    n += 2;
  }
  printf("%llu %llu\n", n, bad);
  return 0;
}

int main(int argc, char** argv) {
  if (argc == 5 && strcmp(argv[2], "f64") == 0)
    return main64((double)atoi(argv[1]), atoll(argv[3]), (uint64_t)strtoull(argv[4], NULL, 10));
  if (argc != 4) return 2;
  const float d = (float)atoi(argv[1]);
  const uint32_t lo = (uint32_t)strtoul(argv[2], NULL, 16), hi = (uint32_t)strtoul(argv[3], NULL, 16);
  const float z = 1.0f / d;
  const float lim = 0x1p-124f;
  unsigned long long n = 0, bad = 0, bad_range = 0;
  float worst = 0.0f;
#pragma omp parallel for reduction(+ : n, bad, bad_range) reduction(max : worst) schedule(static)
  for (int64_t m = (int64_t)lo; m <= (int64_t)hi; ++m) {
    for (int s = 0; s < 2; ++s) {
      const float x = f_of((uint32_t)m | (s ? 0x80000000u : 0u));
      const float q0 = x * z;
      const float r = fmaf(-q0, d, x);
      const float q = fmaf(r, z, q0);
      const float ref = x / d;
      const int same = u_of(q) == u_of(ref) || (q != q && ref != ref);
      const int counted = !same && x == x && fabsf(x) != INFINITY && x != 0.0f;
      n += 1;
      bad += !same;
      bad_range += counted && fabsf(x) >= lim;
      if (counted && fabsf(x) > worst) worst = fabsf(x);
    }
  }
  printf("%llu %llu %llu %a\n", n, bad, bad_range, worst);
  return 0;
}
