/*
 * FP64 elementary functions shared bit-for-bit by the CUDA kernels and the
 * CPU oracles (compiled as __host__ __device__ by nvcc, as plain C by gcc).
 *
 * Why: the tracking path calls sin/cos/asin/tan in every CSBEND substep
 * (csbend.c:1566-1574) and sin in RFCA (simple_rfca.c:560-573).  Library
 * implementations on the host (glibc) and on the device differ by an ulp now
 * and then, and over 1,000 turns those ulps grow.  With one implementation on
 * both sides the GPU reproduces the CPU oracle bit-for-bit; the oracle built
 * with glibc instead measures how far this implementation drifts from libm.
 *
 * Methods (all from the mathematics, coefficients derived here):
 *  - sin/cos: Cody & Waite (1980) additive range reduction by pi/2 split into
 *    three doubles (the first product is exact under fma), then the Taylor
 *    series of sin and cos on |r| <= pi/4 truncated where the remainder is
 *    below 2^-60 relative -- on |r| <= 2^-4 that is four terms of each
 *    series, beyond it ten; 1 - r^2/2 is evaluated with the compensated
 *    splitting used by Sun's fdlibm kernel cosine.
 *  - asin: Taylor series  asin(x) = sum C(2n,n) x^(2n+1) / (4^n (2n+1))  on
 *    |x| <= 1/2 (4 terms for |x| <= 2^-6, 10 for |x| <= 1/8, 28 beyond), and
 *    asin(x) = pi/2 - 2 asin(sqrt((1-x)/2)) for 1/2 < |x| <= 1.
 *  - tan = sin/cos from the shared reduction.
 *  - pow(x, y) for the exponents the CSR code evaluates per bin (1./3, 2./3,
 *    4./3, 2): a double-double cube root by Newton iteration, squared or
 *    multiplied by x in double-double, times the correction for the
 *    exponent's own rounding (y - p/3 = -(p/3) 2^-54: the factor
 *    1 - (p/3) 2^-54 ln x).
 *  - log: ln(1 + f) = f - (f^2/2 - s (f^2/2 + R(s^2))), s = f/(2 + f), with
 *    f = m - 1 exact for m in [1/sqrt2, sqrt2) and R the Taylor series of
 *    2 atanh(s) - 2 s (12 terms, |s| <= 0.1716), plus e ln2 with ln2 split
 *    into a 42-bit head (exact product) and a tail.
 * All polynomial evaluation uses explicit fma, so the result does not depend
 * on the compiler's contraction setting.
 */
#ifndef B2E_MATH_H
#define B2E_MATH_H

#ifdef __CUDACC__
#define B2E_HD __host__ __device__ __forceinline__
#else
#include <math.h>
#define B2E_HD static inline
#endif

/* pi/2 = B2E_PIO2_1 + B2E_PIO2_2 + B2E_PIO2_3 (successive 53-bit pieces) */
#define B2E_PIO2_1 0x1.921fb54442d18p+0
#define B2E_PIO2_2 0x1.1a62633145c07p-54
#define B2E_PIO2_3 (-0x1.f1976b7ed8fbcp-110)
#define B2E_TWO_OVER_PI 0x1.45f306dc9c883p-1
#define B2E_PIO4 0x1.921fb54442d18p-1

B2E_HD double b2e_fma(double a, double b, double c) { return fma(a, b, c); }

/* sin(r) for |r| <= pi/4: r + r^3 * sum_{n>=1} (-1)^n r^(2n-2) / (2n+1)!  (to r^19) */
B2E_HD double b2e_sin_kernel(double r) {
  double w = r * r, p;
  p = -1.0 / 121645100408832000.0;          /* -1/19! */
  p = b2e_fma(p, w, 1.0 / 355687428096000.0); /* 1/17! */
  p = b2e_fma(p, w, -1.0 / 1307674368000.0);  /* -1/15! */
  p = b2e_fma(p, w, 1.0 / 6227020800.0);      /* 1/13! */
  p = b2e_fma(p, w, -1.0 / 39916800.0);       /* -1/11! */
  p = b2e_fma(p, w, 1.0 / 362880.0);          /* 1/9! */
  p = b2e_fma(p, w, -1.0 / 5040.0);           /* -1/7! */
  p = b2e_fma(p, w, 1.0 / 120.0);             /* 1/5! */
  p = b2e_fma(p, w, -1.0 / 6.0);              /* -1/3! */
  return b2e_fma(r * w, p, r);
}

/* cos(r) for |r| <= pi/4: 1 - r^2/2 + r^4 * sum_{n>=0} (-1)^n r^(2n) / (2n+4)!  (to r^20) */
B2E_HD double b2e_cos_kernel(double r) {
  double w = r * r, q, hw, t;
  q = 1.0 / 2432902008176640000.0;             /* 1/20! */
  q = b2e_fma(q, w, -1.0 / 6402373705728000.0); /* -1/18! */
  q = b2e_fma(q, w, 1.0 / 20922789888000.0);    /* 1/16! */
  q = b2e_fma(q, w, -1.0 / 87178291200.0);      /* -1/14! */
  q = b2e_fma(q, w, 1.0 / 479001600.0);         /* 1/12! */
  q = b2e_fma(q, w, -1.0 / 3628800.0);          /* -1/10! */
  q = b2e_fma(q, w, 1.0 / 40320.0);             /* 1/8! */
  q = b2e_fma(q, w, -1.0 / 720.0);              /* -1/6! */
  q = b2e_fma(q, w, 1.0 / 24.0);                /* 1/4! */
  hw = 0.5 * w;
  t = 1.0 - hw;
  /* (1 - t) - hw recovers the rounding error of t exactly */
  return t + (((1.0 - t) - hw) + (w * w) * q);
}

/* The same series truncated for |r| <= 2^-4, where the first dropped term is
 * below 2^-60 relative: sin to r^9 (next: r^10/11! < 2.3e-20), cos to r^8
 * (next: r^10/10! < 2.6e-19). */
B2E_HD double b2e_sin_kernel_small(double r) {
  double w = r * r, p;
  p = 1.0 / 362880.0;                /* 1/9! */
  p = b2e_fma(p, w, -1.0 / 5040.0);  /* -1/7! */
  p = b2e_fma(p, w, 1.0 / 120.0);    /* 1/5! */
  p = b2e_fma(p, w, -1.0 / 6.0);     /* -1/3! */
  return b2e_fma(r * w, p, r);
}

B2E_HD double b2e_cos_kernel_small(double r) {
  double w = r * r, q, hw, t;
  q = 1.0 / 40320.0;               /* 1/8! */
  q = b2e_fma(q, w, -1.0 / 720.0); /* -1/6! */
  q = b2e_fma(q, w, 1.0 / 24.0);   /* 1/4! */
  hw = 0.5 * w;
  t = 1.0 - hw;
  return t + (((1.0 - t) - hw) + (w * w) * q);
}

B2E_HD double b2e_sin_r(double r) { return fabs(r) <= 0x1p-4 ? b2e_sin_kernel_small(r) : b2e_sin_kernel(r); }
B2E_HD double b2e_cos_r(double r) { return fabs(r) <= 0x1p-4 ? b2e_cos_kernel_small(r) : b2e_cos_kernel(r); }

/* Reduce x to r in [-pi/4, pi/4] and the quadrant k mod 4. */
B2E_HD double b2e_reduce_pio2(double x, int *quadrant) {
  double k, r;
  if (fabs(x) <= B2E_PIO4) {
    *quadrant = 0;
    return x;
  }
  k = rint(x * B2E_TWO_OVER_PI);
  r = b2e_fma(-k, B2E_PIO2_1, x); /* exact */
  r = b2e_fma(-k, B2E_PIO2_2, r);
  r = b2e_fma(-k, B2E_PIO2_3, r);
  *quadrant = (int)((long long)k & 3);
  return r;
}

/* For |x| <= 2^-4 the general path below takes quadrant 0, r = x and the
 * short kernels; the entry points test that case first and return the same
 * values without the reduction, quadrant and NaN logic (the bend integrator's
 * angles are nearly always that small). */
B2E_HD void b2e_sincos(double x, double *s, double *c) {
  if (fabs(x) <= 0x1p-4) {
    *s = b2e_sin_kernel_small(x);
    *c = b2e_cos_kernel_small(x);
    return;
  }
  int q;
  double r = b2e_reduce_pio2(x, &q), sr, cr;
  sr = b2e_sin_r(r);
  cr = b2e_cos_r(r);
  switch (q) {
  case 0:
    *s = sr;
    *c = cr;
    break;
  case 1:
    *s = cr;
    *c = -sr;
    break;
  case 2:
    *s = -sr;
    *c = -cr;
    break;
  default:
    *s = -cr;
    *c = sr;
    break;
  }
  if (x != x) { /* NaN in, NaN out */
    *s = x;
    *c = x;
  }
}

/* Single-result variants: same reduction and kernels as b2e_sincos, so each
 * returns bit-for-bit the corresponding member of the pair. */
B2E_HD double b2e_sin(double x) {
  if (fabs(x) <= 0x1p-4)
    return b2e_sin_kernel_small(x);
  int q;
  double r = b2e_reduce_pio2(x, &q), v;
  if (x != x)
    return x;
  v = (q & 1) ? b2e_cos_r(r) : b2e_sin_r(r);
  return (q & 2) ? -v : v;
}

B2E_HD double b2e_cos(double x) {
  if (fabs(x) <= 0x1p-4)
    return b2e_cos_kernel_small(x);
  int q;
  double r = b2e_reduce_pio2(x, &q), v;
  if (x != x)
    return x;
  v = (q & 1) ? b2e_sin_r(r) : b2e_cos_r(r);
  return (q == 1 || q == 2) ? -v : v;
}

B2E_HD double b2e_tan(double x) {
  double s, c;
  b2e_sincos(x, &s, &c);
  return s / c;
}

/* asin(x) - x = x^3 * P(x^2) for |x| <= 2^-6 to n = 4 (next term below
 * 2^-60 relative: 0.0224 x^10 < 2e-20) */
B2E_HD double b2e_asin_tiny(double x) {
  double w = x * x, p;
  p = (70.0 / 9.0) * 0x1p-8;                 /* n=4 */
  p = b2e_fma(p, w, (20.0 / 7.0) * 0x1p-6);  /* n=3 */
  p = b2e_fma(p, w, (6.0 / 5.0) * 0x1p-4);   /* n=2 */
  p = b2e_fma(p, w, (2.0 / 3.0) * 0x1p-2);   /* n=1 */
  return b2e_fma(x * w, p, x);
}

/* asin(x) - x = x^3 * P(x^2) for |x| <= 1/8; coefficients C(2n,n)/((2n+1) 4^n), n = 1..10 */
B2E_HD double b2e_asin_small(double x) {
  double w = x * x, p;
  p = (184756.0 / 21.0) * 0x1p-20;           /* n=10 */
  p = b2e_fma(p, w, (48620.0 / 19.0) * 0x1p-18); /* n=9 */
  p = b2e_fma(p, w, (12870.0 / 17.0) * 0x1p-16); /* n=8 */
  p = b2e_fma(p, w, (3432.0 / 15.0) * 0x1p-14);  /* n=7 */
  p = b2e_fma(p, w, (924.0 / 13.0) * 0x1p-12);   /* n=6 */
  p = b2e_fma(p, w, (252.0 / 11.0) * 0x1p-10);   /* n=5 */
  p = b2e_fma(p, w, (70.0 / 9.0) * 0x1p-8);     /* n=4 */
  p = b2e_fma(p, w, (20.0 / 7.0) * 0x1p-6);     /* n=3 */
  p = b2e_fma(p, w, (6.0 / 5.0) * 0x1p-4);       /* n=2 */
  p = b2e_fma(p, w, (2.0 / 3.0) * 0x1p-2);       /* n=1 */
  return b2e_fma(x * w, p, x);
}

/* Same series to n = 28 for 1/8 < |x| <= 1/2 (remainder < 2^-58 relative). */
B2E_HD double b2e_asin_mid(double x) {
  /* C(2n,n)/(2n+1) for n = 1..28; the 4^-n factor is applied by scaling w. */
  const double c[28] = {
    2.0 / 3.0, 6.0 / 5.0, 20.0 / 7.0, 70.0 / 9.0, 252.0 / 11.0, 924.0 / 13.0, 3432.0 / 15.0,
    12870.0 / 17.0, 48620.0 / 19.0, 184756.0 / 21.0, 705432.0 / 23.0, 2704156.0 / 25.0,
    10400600.0 / 27.0, 40116600.0 / 29.0, 155117520.0 / 31.0, 601080390.0 / 33.0,
    2333606220.0 / 35.0, 9075135300.0 / 37.0, 35345263800.0 / 39.0, 137846528820.0 / 41.0,
    538257874440.0 / 43.0, 2104098963720.0 / 45.0, 8233430727600.0 / 47.0,
    32247603683100.0 / 49.0, 126410606437752.0 / 51.0, 495918532948104.0 / 53.0,
    1946939425648112.0 / 55.0, 7648690600760440.0 / 57.0};
  double w = 0.25 * x * x, p;
  int n;
  /* terms: c[n-1] * 4^-n * x^(2n) = c[n-1] * (x^2/4)^n */
  p = c[27];
  for (n = 26; n >= 0; n--)
    p = b2e_fma(p, w, c[n]);
  return b2e_fma(x * w, p, x);
}

/* ln(x) to ~1e-8 relative, for the tiny exponent correction in b2e_pow13:
 * x = m 2^e, ln m = 2 atanh(s), s = (m-1)/(m+1), series to s^13. */
B2E_HD double b2e_log_coarse(double x) {
  int e;
  double m = frexp(x, &e), s, w, p;
  s = (m - 1.0) / (m + 1.0);
  w = s * s;
  p = b2e_fma(w, 1.0 / 13.0, 1.0 / 11.0);
  p = b2e_fma(p, w, 1.0 / 9.0);
  p = b2e_fma(p, w, 1.0 / 7.0);
  p = b2e_fma(p, w, 1.0 / 5.0);
  p = b2e_fma(p, w, 1.0 / 3.0);
  p = b2e_fma(p, w, 1.0);
  return e * 0x1.62e42fefa39efp-1 + 2.0 * s * p; /* ln 2 */
}

/* Cube root of x to double-double accuracy: x = m 2^(3q), m in [1/2, 4),
 * cbrt(m) = y + c.  Returns y, sets *c, *m and *q. */
B2E_HD double b2e_cbrt_dd(double x, double *c, double *mout, int *qout) {
  int e, q, r;
  double m, y, p_hi, p_lo, t_hi, t_lo, res;
  m = frexp(x, &e); /* x = m 2^e, m in [1/2, 1) */
  q = e >= 0 ? e / 3 : -((2 - e) / 3);
  r = e - 3 * q; /* 0, 1, 2 */
  m = ldexp(m, r); /* in [1/2, 4) */
  y = 0.65 + 0.25 * m - 0.0185 * m * m; /* within 6% on [1/2, 4) */
  for (int i = 0; i < 6; i++)
    y = y - (y * y * y - m) / (3.0 * y * y);
  /* residual m - y^3 with y^3 as an unevaluated sum */
  p_hi = y * y;
  p_lo = b2e_fma(y, y, -p_hi);
  t_hi = p_hi * y;
  t_lo = b2e_fma(p_hi, y, -t_hi) + p_lo * y;
  res = (m - t_hi) - t_lo;
  *c = res / (3.0 * y * y);
  *mout = m;
  *qout = q;
  return y;
}

/* pow(x, 1./3.): C's pow with the double nearest 1/3, as the CSR code calls
 * it (csbend.c:2379, :2575, :2590).  The cube root is computed to double-
 * double accuracy by Newton iteration with an exact fma residual; the
 * exponent's own rounding, 1/3 - 1./3. = 2^-54/3, enters as the factor
 * (1 - 2^-54/3 ln x).  One final rounding, so the result is the correctly
 * rounded value except in exceedingly rare near-tie cases. */
B2E_HD double b2e_pow13(double x) {
  int q;
  double m, c, y, corr;
  if (x != x || x < 0)
    return (x - x) / (x - x);
  if (x == 0 || x > 1.7976931348623157e308)
    return x;
  y = b2e_cbrt_dd(x, &c, &m, &q);
  corr = -(0x1p-54 / 3.0) * b2e_log_coarse(x);
  return ldexp(y + (c + y * corr), q);
}

/* pow(x, 2./3.) = (y + c)^2 2^(2q) (1 - (2/3) 2^-54 ln x), for x > 0 */
B2E_HD double b2e_pow23(double x) {
  int q;
  double m, c, y, hi, lo, corr;
  if (x != x || x < 0)
    return (x - x) / (x - x);
  if (x == 0 || x > 1.7976931348623157e308)
    return x;
  y = b2e_cbrt_dd(x, &c, &m, &q);
  hi = y * y;
  lo = b2e_fma(y, y, -hi) + 2.0 * y * c;
  corr = -(0x1p-54 * (2.0 / 3.0)) * b2e_log_coarse(x);
  return ldexp(hi + (lo + hi * corr), 2 * q);
}

/* pow(x, 4./3.) = m (y + c) 2^(4q) (1 - (4/3) 2^-54 ln x), for x > 0 */
B2E_HD double b2e_pow43(double x) {
  int q;
  double m, c, y, hi, lo, corr;
  if (x != x || x < 0)
    return (x - x) / (x - x);
  if (x == 0 || x > 1.7976931348623157e308)
    return x;
  y = b2e_cbrt_dd(x, &c, &m, &q);
  hi = m * y;
  lo = b2e_fma(m, y, -hi) + m * c;
  corr = -(0x1p-54 * (4.0 / 3.0)) * b2e_log_coarse(x);
  return ldexp(hi + (lo + hi * corr), 4 * q);
}

/* pow(x, y) for the exponents evaluated per bin (1./3, 2./3, 4./3, 2); any
 * other exponent only occurs in host-side setup, where the library pow is
 * used as in the reference. */
B2E_HD double b2e_pow(double x, double y) {
  if (y == 1.0 / 3.0)
    return b2e_pow13(x);
  if (y == 2.0 / 3.0)
    return b2e_pow23(x);
  if (y == 4.0 / 3.0)
    return b2e_pow43(x);
  if (y == 2.0)
    return x * x;
  return pow(x, y);
}

/* natural logarithm (see the header comment); x <= 0, inf and NaN as C's log */
#define B2E_LN2_HI 0x1.62e42fefa3800p-1 /* ln 2 to 42 bits: e * B2E_LN2_HI is exact */
#define B2E_LN2_LO 0x1.ef35793c76730p-45
B2E_HD double b2e_log(double x) {
  int e;
  double m, f, s, z, R, hfsq, lg;
  if (x != x)
    return x;
  if (x < 0)
    return (x - x) / (x - x);
  if (x == 0)
    return -1.0 / 0.0;
  if (x > 1.7976931348623157e308)
    return x;
  m = frexp(x, &e); /* handles subnormal x */
  if (m < 0.70710678118654752440) {
    m = 2.0 * m;
    e -= 1;
  }
  f = m - 1.0; /* exact */
  s = f / (2.0 + f);
  z = s * s;
  /* R = 2 z/3 + 2 z^2/5 + ... + 2 z^12/25 */
  R = 2.0 / 25.0;
  R = b2e_fma(R, z, 2.0 / 23.0);
  R = b2e_fma(R, z, 2.0 / 21.0);
  R = b2e_fma(R, z, 2.0 / 19.0);
  R = b2e_fma(R, z, 2.0 / 17.0);
  R = b2e_fma(R, z, 2.0 / 15.0);
  R = b2e_fma(R, z, 2.0 / 13.0);
  R = b2e_fma(R, z, 2.0 / 11.0);
  R = b2e_fma(R, z, 2.0 / 9.0);
  R = b2e_fma(R, z, 2.0 / 7.0);
  R = b2e_fma(R, z, 2.0 / 5.0);
  R = b2e_fma(R, z, 2.0 / 3.0);
  R = R * z;
  hfsq = 0.5 * f * f;
  lg = hfsq - s * (hfsq + R); /* ln(1 + f) = f - lg */
  {
    /* (e ln2_hi + f) as an exact two-sum (Knuth), then the small terms, so the
     * cancellation of e ln2 against f costs no extra rounding */
    const double a = e * B2E_LN2_HI, sum = a + f, bb = sum - a;
    const double err = (a - (sum - bb)) + (f - bb);
    return sum + (err + (e * B2E_LN2_LO - lg));
  }
}

B2E_HD double b2e_asin(double x) {
  double a = fabs(x), r;
  if (a <= 0x1p-6)
    return b2e_asin_tiny(x);
  if (a <= 0.125)
    return b2e_asin_small(x);
  if (a <= 0.5)
    return b2e_asin_mid(x);
  if (a > 1.0 || x != x)
    return (x - x) / (x - x); /* NaN */
  {
    double z = sqrt(0.5 * (1.0 - a)); /* 1 - a exact for a in [1/2, 1] */
    double t = 2.0 * b2e_asin_mid(z);
    r = (B2E_PIO2_1 - t) + B2E_PIO2_2;
  }
  return x < 0 ? -r : r;
}

#endif
