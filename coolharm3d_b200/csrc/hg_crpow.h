/* hg_crpow.h -- pow(x, y) rounded correctly, the same bits on the host and
 * on the GPU.
 *
 * The entropy fix of recover_primitives() (fixup.c:335-454,
 * utoprim_1d_ee.c, utoprim_1d_ee2.c) raises densities to the power gam-1
 * and 1-gam and feeds the results into Newton solves that amplify their last
 * bit.  Neither glibc's pow() nor CUDA's is correctly rounded, and they
 * round differently, so a device pow() cannot reproduce the reference's
 * results.  This one returns the double nearest to x^y (round to nearest
 * even) for every x > 0 and y whose result is a normal number, up to inputs
 * whose exact result lies within about 2^-92 (relative) of a point halfway
 * between two doubles.  It is built from +, -, *, / and fma() only, each
 * correctly rounded in IEEE double on both sides, with no library math
 * function on the path, so host and device compute identical bits and a CPU
 * restatement of the step that uses it agrees with the device bit for bit.
 * Where glibc's pow() is itself correctly rounded (all but roughly one call
 * in a thousand), the reference's results are reproduced too.
 *
 * Method: double-double arithmetic (Dekker 1971: exact sums and products
 * from two_sum and an fma, ~106-bit pairs hi + lo).
 *   log x = e log 2 + log c + 2 atanh((m - c)/(m + c)),  x = 2^e m,
 *           m in [1/sqrt 2, sqrt 2), c = 1 + k/256 the nearest table point,
 *           so |(m-c)/(m+c)| < 2^-9.4 and the atanh series converges fast;
 *   exp E = 2^q 2^(j/256) exp(r),  E = (256 q + j) log(2)/256 + r,
 *           |r| <= log(2)/512, exp(r) by its Taylor series.
 * The leading terms of both series are carried in double-double, the tail
 * in double; the tables log(1 + k/256) and 2^(j/256) are double-double
 * values computed with 80-digit decimal arithmetic (gen_pow_tables.py).
 * Other inputs (x <= 0, subnormal or infinite x, NaN, |y log x| >= 700) go
 * to the platform's pow(); the step never produces them.
 *
 * Works as C (the CPU restatement of the step) and as CUDA (host and device). */
#ifndef HG_CRPOW_H
#define HG_CRPOW_H

#include <math.h>
#include <stdint.h>
#include <string.h>

#include "hg_pow_tables.h"

#ifdef __CUDACC__
#define HG_PHD static __host__ __device__ __forceinline__
#else
#define HG_PHD static inline
#endif

static const double hg_pow_logc_h[2 * HG_POW_NLOGC] = HG_POW_LOGC_TABLE;
static const double hg_pow_exp2_h[2 * 256] = HG_POW_EXP2_TABLE;
#ifdef __CUDACC__
static __device__ const double hg_pow_logc_d[2 * HG_POW_NLOGC] = HG_POW_LOGC_TABLE;
static __device__ const double hg_pow_exp2_d[2 * 256] = HG_POW_EXP2_TABLE;
#endif

typedef struct {
  double hi, lo;
} hg_dd;

HG_PHD hg_dd hg_dd_make(double hi, double lo)
{
  hg_dd r;
  r.hi = hi;
  r.lo = lo;
  return r;
}

/* a + b exactly as s + e (any magnitudes) */
HG_PHD hg_dd hg_dd_two_sum(double a, double b)
{
  const double s = a + b;
  const double bb = s - a;
  const double e = (a - (s - bb)) + (b - bb);
  return hg_dd_make(s, e);
}

/* a + b exactly as s + e, for |a| >= |b| (or a == 0) */
HG_PHD hg_dd hg_dd_fast_sum(double a, double b)
{
  const double s = a + b;
  return hg_dd_make(s, b - (s - a));
}

/* a * b exactly as p + e */
HG_PHD hg_dd hg_dd_prod(double a, double b)
{
  const double p = a * b;
  return hg_dd_make(p, fma(a, b, -p));
}

HG_PHD hg_dd hg_dd_add(hg_dd x, hg_dd y)
{
  hg_dd s = hg_dd_two_sum(x.hi, y.hi);
  const hg_dd t = hg_dd_two_sum(x.lo, y.lo);
  s.lo = s.lo + t.hi;
  s = hg_dd_fast_sum(s.hi, s.lo);
  s.lo = s.lo + t.lo;
  return hg_dd_fast_sum(s.hi, s.lo);
}

HG_PHD hg_dd hg_dd_mul(hg_dd x, hg_dd y)
{
  hg_dd p = hg_dd_prod(x.hi, y.hi);
  p.lo = fma(x.hi, y.lo, fma(x.lo, y.hi, p.lo));
  return hg_dd_fast_sum(p.hi, p.lo);
}

HG_PHD hg_dd hg_dd_mul_d(hg_dd x, double d)
{
  hg_dd p = hg_dd_prod(x.hi, d);
  p.lo = fma(x.lo, d, p.lo);
  return hg_dd_fast_sum(p.hi, p.lo);
}

HG_PHD uint64_t hg_pow_bits(double x)
{
  uint64_t u;
  memcpy(&u, &x, 8);
  return u;
}

HG_PHD double hg_pow_from_bits(uint64_t u)
{
  double x;
  memcpy(&x, &u, 8);
  return x;
}

HG_PHD hg_dd hg_pow_logc(int i)
{
#ifdef __CUDA_ARCH__
  return hg_dd_make(__ldg(hg_pow_logc_d + 2 * i), __ldg(hg_pow_logc_d + 2 * i + 1));
#else
  return hg_dd_make(hg_pow_logc_h[2 * i], hg_pow_logc_h[2 * i + 1]);
#endif
}

HG_PHD hg_dd hg_pow_exp2(int j)
{
#ifdef __CUDA_ARCH__
  return hg_dd_make(__ldg(hg_pow_exp2_d + 2 * j), __ldg(hg_pow_exp2_d + 2 * j + 1));
#else
  return hg_dd_make(hg_pow_exp2_h[2 * j], hg_pow_exp2_h[2 * j + 1]);
#endif
}

/* log(x) as a double-double, x a positive normal double. */
HG_PHD hg_dd hg_dd_log(double x)
{
  const uint64_t bits = hg_pow_bits(x);
  int e = (int)(bits >> 52) - 1023;
  double m = hg_pow_from_bits((bits & 0x000fffffffffffffull) | 0x3ff0000000000000ull); /* [1, 2) */
  if (m > 0x1.6a09e667f3bcdp+0) { /* sqrt(2) */
    m = 0.5 * m;
    e = e + 1;
  }
  const int k = (int)floor((m - 1.0) * 256.0 + 0.5); /* -75 .. 106 */
  const double c = 1.0 + (double)k * (1.0 / 256.0);
  const double num = m - c; /* exact: c/2 <= m <= 2c */
  const hg_dd den = hg_dd_two_sum(m, c);
  /* r = num / den to double-double accuracy */
  const double q1 = num / den.hi;
  double rem = fma(-q1, den.hi, num);
  rem = fma(-q1, den.lo, rem);
  const hg_dd r = hg_dd_fast_sum(q1, rem / den.hi);
  /* 2 atanh(r) = 2r (1 + U),  U = s/3 + s^2/5 + s^3/7 + s^4/9 + s^5/11,  s = r^2 < 2^-18.9 */
  const hg_dd s = hg_dd_mul(r, r);
  const double sh = s.hi;
  const double tail = (sh * sh) * (HG_POW_INV5 + sh * (HG_POW_INV7 + sh * (HG_POW_INV9 + sh * HG_POW_INV11)));
  const hg_dd U = hg_dd_add(hg_dd_mul(s, hg_dd_make(HG_POW_THIRD_HI, HG_POW_THIRD_LO)), hg_dd_make(tail, 0.0));
  const hg_dd r2 = hg_dd_make(2.0 * r.hi, 2.0 * r.lo);
  const hg_dd at = hg_dd_add(r2, hg_dd_mul(r2, U));
  const hg_dd lm = hg_dd_add(hg_pow_logc(k + HG_POW_K0), at);
  const hg_dd el2 = hg_dd_mul_d(hg_dd_make(HG_POW_LN2_HI, HG_POW_LN2_LO), (double)e);
  return hg_dd_add(el2, lm);
}

/* exp(E) rounded to the nearest double, for |E.hi| < 700. */
HG_PHD double hg_dd_exp_rn(hg_dd E)
{
  const double nd = floor(E.hi * HG_POW_INV_LN2_256 + 0.5);
  const int n = (int)nd;
  const int j = n & 255;
  const int q = (n - j) / 256;
  /* r = E - n log(2)/256: nd*C1 is exact and E.hi - nd*C1 cancels exactly */
  const double t1 = E.hi - nd * HG_POW_C1;
  const hg_dd nc2 = hg_dd_prod(nd, HG_POW_C2);
  hg_dd r = hg_dd_two_sum(t1, -nc2.hi);
  r.lo = r.lo + ((E.lo - nc2.lo) - nd * HG_POW_C3);
  r = hg_dd_two_sum(r.hi, r.lo);
  /* exp(r) - 1 = r + r^2/2 + r^3/6 + r^4 (1/24 + r/120 + r^2/720 + r^3/5040 + r^4/40320), |r| < 2^-9.5 */
  const hg_dd rr = hg_dd_mul(r, r);
  const hg_dd r3 = hg_dd_mul(rr, r);
  const double rh = r.hi;
  const double tail = (rr.hi * rr.hi) *
                      (HG_POW_INV24 + rh * (HG_POW_INV120 + rh * (HG_POW_INV720 + rh * (HG_POW_INV5040 + rh * HG_POW_INV40320))));
  hg_dd p = hg_dd_add(r, hg_dd_make(0.5 * rr.hi, 0.5 * rr.lo));
  p = hg_dd_add(p, hg_dd_mul(r3, hg_dd_make(HG_POW_SIXTH_HI, HG_POW_SIXTH_LO)));
  p = hg_dd_add(p, hg_dd_make(tail, 0.0));
  const hg_dd T = hg_pow_exp2(j);
  const hg_dd res = hg_dd_add(T, hg_dd_mul(T, p)); /* res.hi = the double nearest to res.hi + res.lo */
  return res.hi * hg_pow_from_bits((uint64_t)(q + 1023) << 52);
}

/* x^y rounded to nearest (see the file comment for the domain). */
HG_PHD double hg_cr_pow(double x, double y)
{
  if (y == 1.0) return x;
  if (y == 0.0) return 1.0;
  if (!(x >= 0x1p-1022) || !(x < INFINITY) || y != y) return pow(x, y);
  if (x == 1.0) return 1.0;
  if (y == -1.0) return 1.0 / x;
  if (y == 0.5) return sqrt(x);
  const hg_dd E = hg_dd_mul_d(hg_dd_log(x), y);
  if (!(fabs(E.hi) < 700.0)) return pow(x, y);
  return hg_dd_exp_rn(E);
}

#endif /* HG_CRPOW_H */
