/*
 * trn_libm.h — the project's own double-precision log, exp and pow.
 *
 * Why this exists: the adaptation round takes topological decisions by
 * comparing FP64 values against thresholds (metric length > sqrt(2),
 * quality ties, ...). Two correct-to-1-ulp libraries (glibc on the host,
 * CUDA's libdevice on the GPU) do not return identical bits, so they can
 * flip a decision. Every side that must agree bit for bit — the CUDA
 * kernels, the C oracle and the shimmed build of the reference — calls the
 * functions below instead.
 *
 * Only IEEE-754 correctly rounded +, -, *, / and exact bit manipulation are
 * used, and no expression may be contracted into an FMA (host: compile with
 * -ffp-contract=off; device: nvcc --fmad=false), so host and device produce
 * identical results for identical inputs.
 *
 * Methods (textbook, Cody & Waite, "Software Manual for the Elementary
 * Functions", 1980):
 *   exp(x): x = k ln2 + r with ln2 split in a 32-bit head (k*head exact) and
 *           a tail; exp(r), |r| <= ln2/2, by its Taylor series to degree 14,
 *           evaluated by Estrin's scheme (short dependency chains: the GPU
 *           kernels that call it are latency-bound); scale by 2^k built from
 *           the exponent bits.
 *   log(x): x = 2^e m with m in [sqrt(1/2), sqrt(2)); log(m) = 2 atanh(s),
 *           s = (m-1)/(m+1), |s| <= 0.1716, odd series to s^25 (Estrin);
 *           log(x) = e*ln2_head + (e*ln2_tail + log(m)).
 *   pow(x,y): y == 2 -> x*x, y == 3 -> (x*x)*x (the reference only raises to
 *           these integer powers and to one fractional exponent, -1/(2p+2));
 *           otherwise exp(y*log(x)) for x > 0.
 * Accuracy against glibc is checked by tests/test_libm.py (a few ulp; the
 * bound is stated there).
 */
#ifndef TRN_LIBM_H
#define TRN_LIBM_H

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define TRN_HD __host__ __device__ __forceinline__
#else
#define TRN_HD static inline
#endif

TRN_HD uint64_t trn_bits(double x) {
#if defined(__CUDA_ARCH__)
  return (uint64_t)__double_as_longlong(x);
#else
  uint64_t u;
  memcpy(&u, &x, sizeof u);
  return u;
#endif
}

TRN_HD double trn_from_bits(uint64_t u) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)u);
#else
  double x;
  memcpy(&x, &u, sizeof x);
  return x;
#endif
}

/* 2^k for -1022 <= k <= 1023 */
TRN_HD double trn_pow2i(int k) {
  return trn_from_bits((uint64_t)(k + 1023) << 52);
}

#define TRN_LN2_HI  0x1.62e42fee00000p-1
#define TRN_LN2_LO  0x1.a39ef35793c76p-33
#define TRN_INV_LN2 0x1.71547652b82fep+0
#define TRN_SQRT2   0x1.6a09e667f3bcdp+0

TRN_HD double trn_exp(double x) {
  if (x != x) return x;                       /* NaN */
  if (x > 709.782712893384) return trn_from_bits(0x7ff0000000000000ULL);
  if (x < -745.2) return 0.0;
  double t = x * TRN_INV_LN2;
  int k = (int)(t + (t >= 0.0 ? 0.5 : -0.5)); /* round half away from zero */
  double kd = (double)k;
  double r = (x - kd * TRN_LN2_HI) - kd * TRN_LN2_LO;
  /* Taylor coefficients 1/n!, n = 0..14 (correctly rounded), evaluated by
   * Estrin's scheme: pairs, then pairs of pairs in r^2, r^4, r^8, so that the
   * chain of dependent operations is 8 long instead of Horner's 28 */
  const double r2 = r * r, r4 = r2 * r2, r8 = r4 * r4;
  const double a0 = 1.0 + r;
  const double a1 = 0x1.0000000000000p-1 + 0x1.5555555555555p-3 * r;
  const double a2 = 0x1.5555555555555p-5 + 0x1.1111111111111p-7 * r;
  const double a3 = 0x1.6c16c16c16c17p-10 + 0x1.a01a01a01a01ap-13 * r;
  const double a4 = 0x1.a01a01a01a01ap-16 + 0x1.71de3a556c734p-19 * r;
  const double a5 = 0x1.27e4fb7789f5cp-22 + 0x1.ae64567f544e4p-26 * r;
  const double a6 = 0x1.1eed8eff8d898p-29 + 0x1.6124613a86d09p-33 * r;
  const double a7 = 0x1.93974a8c07c9dp-37;
  const double b0 = a0 + a1 * r2, b1 = a2 + a3 * r2, b2 = a4 + a5 * r2, b3 = a6 + a7 * r2;
  const double d0 = b0 + b1 * r4, d1 = b2 + b3 * r4;
  const double p = d0 + d1 * r8;
  /* scale by 2^k, in two steps when 2^k alone is not a normal number */
  if (k > 1023) return (p * trn_pow2i(1023)) * trn_pow2i(k - 1023);
  if (k < -1022) return (p * trn_pow2i(-1022)) * trn_pow2i(k + 1022 < -1022 ? -1022 : k + 1022);
  return p * trn_pow2i(k);
}

TRN_HD double trn_log(double x) {
  uint64_t u = trn_bits(x);
  if (x != x) return x;                                   /* NaN */
  if (x < 0.0) return trn_from_bits(0x7ff8000000000000ULL); /* NaN */
  if (x == 0.0) return -trn_from_bits(0x7ff0000000000000ULL);
  if ((u >> 52) == 0x7ff) return x;                       /* +inf */
  int e = 0;
  if ((u >> 52) == 0) {                                    /* subnormal */
    x = x * 0x1p54;
    u = trn_bits(x);
    e = -54;
  }
  e += (int)(u >> 52) - 1023;
  double m = trn_from_bits((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
  if (m > TRN_SQRT2) {
    m = m * 0.5;
    e += 1;
  }
  double f = m - 1.0;
  double s = f / (2.0 + f);
  double z = s * s;
  /* 1/(2n+1), n = 1..12, as a polynomial in z, by Estrin's scheme (a chain
   * of 8 dependent operations instead of 22) */
  const double z2 = z * z, z4 = z2 * z2, z8 = z4 * z4;
  const double a0 = 0x1.5555555555555p-2 + 0x1.999999999999ap-3 * z;
  const double a1 = 0x1.2492492492492p-3 + 0x1.c71c71c71c71cp-4 * z;
  const double a2 = 0x1.745d1745d1746p-4 + 0x1.3b13b13b13b14p-4 * z;
  const double a3 = 0x1.1111111111111p-4 + 0x1.e1e1e1e1e1e1ep-5 * z;
  const double a4 = 0x1.af286bca1af28p-5 + 0x1.8618618618618p-5 * z;
  const double a5 = 0x1.642c8590b2164p-5 + 0x1.47ae147ae147bp-5 * z;
  const double b0 = a0 + a1 * z2, b1 = a2 + a3 * z2, b2 = a4 + a5 * z2;
  const double q = (b0 + b1 * z4) + b2 * z8;
  double two_s = s + s;
  double logm = two_s + two_s * (z * q);
  double ed = (double)e;
  return ed * TRN_LN2_HI + (ed * TRN_LN2_LO + logm);
}

TRN_HD double trn_pow(double x, double y) {
  if (y == 2.0) return x * x;
  if (y == 3.0) return (x * x) * x;
  if (y == 1.0) return x;
  if (y == 0.0) return 1.0;
  if (x > 0.0) return trn_exp(y * trn_log(x));
  if (x == 0.0) return y > 0.0 ? 0.0 : trn_from_bits(0x7ff0000000000000ULL);
  return trn_from_bits(0x7ff8000000000000ULL); /* negative base, non-integer use */
}

#endif /* TRN_LIBM_H */
