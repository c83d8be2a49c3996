/*
 * esl_math.h: exp, log and pow for the bias-dependent device-model code.
 *
 * One implementation, compiled both into the CUDA lane kernels and into the
 * C restatement the kernels are checked against, so that a lane's model
 * evaluations are bitwise the same on both sides. CUDA's own exp/log/pow and
 * the host C library's differ in the last unit in the last place on some
 * arguments; a Newton gate sitting near its threshold then passes on one
 * side and fails on the other, and the two solves take different iteration
 * counts. With these functions the only floating-point operations are IEEE
 * double multiplies, adds, subtracts and divides, each rounded to nearest
 * (explicit __d*_rn intrinsics on the device; the host compiles this file
 * with floating-point contraction off), so both sides round every step the
 * same way.
 *
 * Methods (textbook ones, written from the mathematics):
 * - exp: Cody-Waite reduction x = k ln2 + r with ln2 split into a 32-bit
 *   head (k * head is exact for |k| < 2^21) and a tail, |r| <= ln2 / 2; then
 *   exp(r) = 1 + r + r^2 (1/2! + r/3! + ... + r^11/13!) (Taylor to degree
 *   13: truncation below 5e-18 relative on |r| <= 0.347; the polynomial by
 *   Estrin's scheme for a short dependency chain) and the scale 2^k applied
 *   by exponent arithmetic. Error about 1 ulp.
 * - log: x = 2^e m with m in [sqrt(2)/2, sqrt(2)], f = m - 1 (exact),
 *   s = f / (2 + f), log m = 2 atanh s = 2 s (1 + s^2/3 + s^4/5 + ...)
 *   to s^24/25 (|s| <= 0.172: truncation below 1e-18 relative), plus e ln2
 *   with the same head/tail split. Error about 1 ulp.
 * - pow(x, y) = exp(y log x) for x > 0 (relative error about 2 |y log x| ulp:
 *   the models raise junction and geometry factors near 1 to exponents of
 *   order 1), y = 2 and 3 as products; x = 0, x < 0 with an integral y, and
 *   the special values as C's pow returns them.
 * Accuracy against the host C library is checked by the tests
 * (tests/test_esl_math.py: within 2 ulp on exp and log over their ranges).
 */
#ifndef ESL_MATH_H
#define ESL_MATH_H

#include <stdint.h>
#include <string.h>

/* ESL_MATH_FN: the building blocks, inlined. ESL_MATH_ENTRY: esl_exp,
 * esl_log and esl_pow themselves; on the device they are compiled out of
 * line (a call with one or two arguments in registers), which keeps the
 * model code that calls them small enough to stay inlined in the lane
 * kernels. */
#if defined(__CUDACC__)
#define ESL_MATH_FN static __host__ __device__ __forceinline__
#define ESL_MATH_ENTRY static __host__ __device__ __noinline__
#else
#define ESL_MATH_FN static inline
#define ESL_MATH_ENTRY static inline
#endif

#if defined(__CUDA_ARCH__)
#define EM_MUL(a, b) __dmul_rn((a), (b))
#define EM_ADD(a, b) __dadd_rn((a), (b))
#define EM_SUB(a, b) __dsub_rn((a), (b))
#define EM_DIV(a, b) __ddiv_rn((a), (b))
#else
#define EM_MUL(a, b) ((a) * (b))
#define EM_ADD(a, b) ((a) + (b))
#define EM_SUB(a, b) ((a) - (b))
#define EM_DIV(a, b) ((a) / (b))
#endif

ESL_MATH_FN uint64_t em_bits(double x) {
#if defined(__CUDA_ARCH__)
  return (uint64_t)__double_as_longlong(x);
#else
  uint64_t u;
  memcpy(&u, &x, sizeof u);
  return u;
#endif
}

ESL_MATH_FN double em_from_bits(uint64_t u) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)u);
#else
  double x;
  memcpy(&x, &u, sizeof x);
  return x;
#endif
}

/* 2^k for -1022 <= k <= 1023 */
ESL_MATH_FN double em_pow2(int k) { return em_from_bits((uint64_t)(k + 1023) << 52); }

#define EM_LN2_HI 0.6931471806019545      /* ln 2 to 32 significant bits */
#define EM_LN2_LO -4.2009150726810846e-11 /* ln 2 - EM_LN2_HI */
#define EM_INV_LN2 1.4426950408889634
#define EM_SHIFTER 6755399441055744.0 /* 1.5 * 2^52: (t + S) - S rounds t to an integer */

ESL_MATH_FN double em_exp(double x) {
  if (x != x) return EM_ADD(x, x);
  if (x > 709.782712893384) return em_from_bits(0x7ff0000000000000ull);
  if (x < -745.1332191019412) return 0.0;
  const double kd = EM_SUB(EM_ADD(EM_MUL(x, EM_INV_LN2), EM_SHIFTER), EM_SHIFTER);
  const double r = EM_SUB(EM_SUB(x, EM_MUL(kd, EM_LN2_HI)), EM_MUL(kd, EM_LN2_LO));
  /* exp(r) = 1 + (r + r^2 P(r)), P(r) = sum_{k=0}^{11} r^k / (k + 2)!,
     evaluated by Estrin's scheme (pairs, then powers r^2, r^4, r^8): a
     dependency chain of about 9 operations instead of Horner's 24 */
  const double r2 = EM_MUL(r, r), r4 = EM_MUL(r2, r2), r8 = EM_MUL(r4, r4);
  const double q0 = EM_ADD(0.5, EM_MUL(r, 0.16666666666666666));
  const double q1 = EM_ADD(0.041666666666666664, EM_MUL(r, 0.008333333333333333));
  const double q2 = EM_ADD(0.001388888888888889, EM_MUL(r, 0.0001984126984126984));
  const double q3 = EM_ADD(2.48015873015873e-05, EM_MUL(r, 2.7557319223985893e-06));
  const double q4 = EM_ADD(2.755731922398589e-07, EM_MUL(r, 2.505210838544172e-08));
  const double q5 = EM_ADD(2.08767569878681e-09, EM_MUL(r, 1.6059043836821613e-10));
  const double s0 = EM_ADD(q0, EM_MUL(r2, q1)), s1 = EM_ADD(q2, EM_MUL(r2, q3)), s2 = EM_ADD(q4, EM_MUL(r2, q5));
  const double p = EM_ADD(EM_ADD(s0, EM_MUL(r4, s1)), EM_MUL(r8, s2));
  const double y = EM_ADD(1.0, EM_ADD(r, EM_MUL(r2, p)));
  const int k = (int)kd;
  if (k >= -1020 && k <= 1020) return EM_MUL(y, em_pow2(k));
  /* near overflow or into the subnormals: two exact-range scalings, the
     second the only one that rounds */
  const int k1 = k / 2;
  return EM_MUL(EM_MUL(y, em_pow2(k1)), em_pow2(k - k1));
}

ESL_MATH_FN double em_log(double x) {
  if (x != x) return EM_ADD(x, x);
  if (x == 0.0) return -em_from_bits(0x7ff0000000000000ull);
  if (x < 0.0) return em_from_bits(0x7ff8000000000000ull);
  if (x == em_from_bits(0x7ff0000000000000ull)) return x;
  uint64_t b = em_bits(x);
  int e = 0;
  if (b < 0x0010000000000000ull) { /* subnormal: into the normal range first */
    x = EM_MUL(x, 18014398509481984.0); /* 2^54 */
    b = em_bits(x);
    e = -54;
  }
  e += (int)(b >> 52) - 1023;
  double m = em_from_bits((b & 0x000fffffffffffffull) | 0x3ff0000000000000ull);
  if (m > 1.4142135623730951) {
    m = EM_MUL(m, 0.5);
    e += 1;
  }
  const double f = EM_SUB(m, 1.0);
  const double s = EM_DIV(f, EM_ADD(2.0, f));
  const double z = EM_MUL(s, s);
  /* log m = 2 s + 2 s z Q(z), Q(z) = sum_{k=0}^{11} z^k / (2k + 3), by
     Estrin's scheme as in exp */
  const double z2 = EM_MUL(z, z), z4 = EM_MUL(z2, z2), z8 = EM_MUL(z4, z4);
  const double q0 = EM_ADD(0.3333333333333333, EM_MUL(z, 0.2));
  const double q1 = EM_ADD(0.14285714285714285, EM_MUL(z, 0.1111111111111111));
  const double q2 = EM_ADD(0.09090909090909091, EM_MUL(z, 0.07692307692307693));
  const double q3 = EM_ADD(0.06666666666666667, EM_MUL(z, 0.058823529411764705));
  const double q4 = EM_ADD(0.05263157894736842, EM_MUL(z, 0.047619047619047616));
  const double q5 = EM_ADD(0.043478260869565216, EM_MUL(z, 0.04));
  const double s0 = EM_ADD(q0, EM_MUL(z2, q1)), s1 = EM_ADD(q2, EM_MUL(z2, q3)), s2 = EM_ADD(q4, EM_MUL(z2, q5));
  const double p = EM_ADD(EM_ADD(s0, EM_MUL(z4, s1)), EM_MUL(z8, s2));
  const double logm = EM_ADD(EM_ADD(s, s), EM_MUL(EM_ADD(s, s), EM_MUL(z, p)));
  const double ed = (double)e;
  return EM_ADD(EM_MUL(ed, EM_LN2_HI), EM_ADD(logm, EM_MUL(ed, EM_LN2_LO)));
}

ESL_MATH_ENTRY double esl_exp(double x) { return em_exp(x); }

ESL_MATH_ENTRY double esl_log(double x) { return em_log(x); }

/* sin x: x = k pi/2 + r with pi/2 split in three (33, 33 and 53 bits: the
 * first two products exact for |k| < 2^20), |r| <= pi/4, then by the
 * quadrant k mod 4 the Taylor series of sin r (to r^17/17!) or cos r (to
 * r^18/18!), each below 1e-19 truncation on |r| <= pi/4, by Estrin's scheme
 * in r^2. Error about 1 ulp for |x| below 1e6 (a source's 2 pi f t). */
#define EM_PIO2_1 1.5707963267341256
#define EM_PIO2_2 6.077100506303966e-11
#define EM_PIO2_3 2.0222662487959506e-21
#define EM_TWO_OVER_PI 0.6366197723675814

ESL_MATH_FN double em_sin(double x) {
  if (x != x || x - x != 0.0) return EM_SUB(x, x); /* NaN for NaN and infinities */
  const double kd = EM_SUB(EM_ADD(EM_MUL(x, EM_TWO_OVER_PI), EM_SHIFTER), EM_SHIFTER);
  const double r = EM_SUB(EM_SUB(EM_SUB(x, EM_MUL(kd, EM_PIO2_1)), EM_MUL(kd, EM_PIO2_2)), EM_MUL(kd, EM_PIO2_3));
  const double z = EM_MUL(r, r), z2 = EM_MUL(z, z), z4 = EM_MUL(z2, z2);
  const int64_t k = (int64_t)kd;
  double out;
  if ((k & 1) == 0) {
    /* sin r = r + r z P(z), P = -1/3! + z/5! - ... + z^7/17! */
    const double a0 = EM_ADD(-0.16666666666666666, EM_MUL(z, 0.008333333333333333));
    const double a1 = EM_ADD(-0.0001984126984126984, EM_MUL(z, 2.7557319223985893e-06));
    const double a2 = EM_ADD(-2.505210838544172e-08, EM_MUL(z, 1.6059043836821613e-10));
    const double a3 = EM_ADD(-7.647163731819816e-13, EM_MUL(z, 2.8114572543455206e-15));
    const double p = EM_ADD(EM_ADD(a0, EM_MUL(z2, a1)), EM_MUL(z4, EM_ADD(a2, EM_MUL(z2, a3))));
    out = EM_ADD(r, EM_MUL(EM_MUL(r, z), p));
  } else {
    /* cos r = 1 + z Q(z), Q = -1/2! + z/4! - ... + z^8/18! */
    const double b0 = EM_ADD(-0.5, EM_MUL(z, 0.041666666666666664));
    const double b1 = EM_ADD(-0.001388888888888889, EM_MUL(z, 2.48015873015873e-05));
    const double b2 = EM_ADD(-2.755731922398589e-07, EM_MUL(z, 2.08767569878681e-09));
    const double b3 = EM_ADD(-1.1470745597729725e-11, EM_MUL(z, 4.779477332387385e-14));
    const double z8 = EM_MUL(z4, z4);
    const double q = EM_ADD(EM_ADD(EM_ADD(b0, EM_MUL(z2, b1)), EM_MUL(z4, EM_ADD(b2, EM_MUL(z2, b3)))),
                            EM_MUL(z8, -1.5619206968586225e-16));
    out = EM_ADD(1.0, EM_MUL(z, q));
  }
  return (k & 2) ? -out : out;
}

ESL_MATH_ENTRY double esl_sin(double x) { return em_sin(x); }

ESL_MATH_ENTRY double esl_pow(double x, double y) {
  if (y == 0.0 || x == 1.0) return 1.0;
  if (x != x || y != y) return EM_ADD(x, y);
  /* squares and cubes (the diode's reverse-bias cube) as products */
  if (y == 2.0) return EM_MUL(x, x);
  if (y == 3.0) return EM_MUL(EM_MUL(x, x), x);
  if (x > 0.0) return em_exp(EM_MUL(y, em_log(x)));
  const double inf = em_from_bits(0x7ff0000000000000ull);
  const double ay = y < 0.0 ? -y : y;
  /* y an integer (every double of magnitude 2^52 or more is), odd or even */
  const int integral = ay >= 4503599627370496.0 || (double)(int64_t)ay == ay;
  const int odd = integral && ay < 9007199254740992.0 && ((int64_t)ay & 1);
  if (x == 0.0) {
    const double r = y > 0.0 ? 0.0 : inf;
    return (odd && em_bits(x) >> 63) ? -r : r;
  }
  if (!integral) return em_from_bits(0x7ff8000000000000ull);
  const double r = em_exp(EM_MUL(y, em_log(-x)));
  return odd ? -r : r;
}

#endif
