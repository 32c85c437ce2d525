/*
 * Real discrete Fourier transform pair for the CSR histogram filters.
 *
 * applyLHPassFilters (csbend.c:4611-4703) transforms the c*t histogram with
 * the SDDS toolkit's realFFT2, scales frequency pairs by a linear ramp (low
 * pass from HIGH_FREQUENCY_CUTOFF0..1, high pass from LOW_FREQUENCY_CUTOFF0..1,
 * in units of Nyquist) and transforms back.  realFFT2 is not part of the
 * reference tree, so this file defines the transform for this project, for
 * any bin count n (not only powers of two):
 *
 *   forward, k = 0 .. n/2 (layout re_0, im_0, re_1, im_1, ..., n + 2 values):
 *       re_k = sum_j x_j cos(2 pi j k / n),   im_k = -sum_j x_j sin(2 pi j k / n)
 *   inverse, j = 0 .. n-1:
 *       x_j = ( re_0 + sum_{k=1}^{(n-1)/2} 2 (re_k cos - im_k sin)(2 pi j k / n)
 *               [+ re_{n/2} cos(pi j) for even n] ) / n
 *
 * Each value is one serial sum in ascending order over a twiddle table
 * c[t], s[t] = cos, sin(2 pi t / n) built from the shared elementary functions
 * (b2e_math.h); the table index j k mod n is stepped in integers.  So the
 * device (one thread per output value), the C restatement and the shim that
 * gives elegant's own applyLHPassFilters its realFFT2 produce the same bits.
 * O(n^2) per transform: at most 4096 bins, once per kick, with the filters
 * off by default.
 */
#ifndef B2E_FFT_H
#define B2E_FFT_H
#include "b2e_math.h"

#ifdef __CUDACC__
#define B2E_FFT_FN __host__ __device__ static inline
#else
#define B2E_FFT_FN static inline
#endif

#define B2E_TWO_PI 6.283185307179586

B2E_FFT_FN void b2e_dft_twiddle(long n, long t, double *c, double *s) {
  const double a = B2E_TWO_PI * (double)t / (double)n;
  *c = b2e_cos(a);
  *s = b2e_sin(a);
}

/* forward pair k of x[0..n) */
B2E_FFT_FN void b2e_rdft_pair(const double *x, long n, long k, const double *c, const double *s, double *re,
                              double *im) {
  double r = 0, i = 0;
  long j, t = 0;
  for (j = 0; j < n; j++) {
    r += x[j] * c[t];
    i -= x[j] * s[t];
    t += k;
    if (t >= n)
      t -= n;
  }
  *re = r;
  *im = i;
}

/* inverse sample j from the n + 2 values ri */
B2E_FFT_FN double b2e_rdft_sample(const double *ri, long n, long j, const double *c, const double *s) {
  double v = ri[0];
  long k, t = 0;
  for (k = 1; k <= (n - 1) / 2; k++) {
    t += j;
    if (t >= n)
      t -= n;
    v += 2 * (ri[2 * k] * c[t] - ri[2 * k + 1] * s[t]);
  }
  if (n % 2 == 0)
    v += ri[n] * c[(j % 2) * (n / 2)];
  return v / n;
}

/* the ramps of applyLHPassFilters (csbend.c:4630-4685) on the pairs ri,
 * frequencies = n/2 + 1; serial, as the fraction is accumulated */
B2E_FFT_FN void b2e_lh_ramps(double *ri, long frequencies, double startHP, double endHP, double startLP,
                             double endLP) {
  long i, i1, i2;
  double fraction, dfraction;
  if (endLP < startLP)
    endLP = startLP;
  if (endHP < startHP)
    endHP = startHP;
  if (startLP > 0) {
    i1 = (long)(startLP * frequencies);
    if (i1 < 0)
      i1 = 0;
    if (i1 > frequencies - 1)
      i1 = frequencies - 1;
    i2 = (long)(endLP * frequencies);
    if (i2 < 0)
      i2 = 0;
    if (i2 > frequencies - 1)
      i2 = frequencies - 1;
    dfraction = i1 == i2 ? 0 : 1. / (i2 - i1);
    fraction = 1;
    for (i = i1; i <= i2; i++) {
      ri[2 * i] *= fraction;
      ri[2 * i + 1] *= fraction;
      if ((fraction -= dfraction) < 0)
        fraction = 0;
    }
    for (; i < frequencies; i++) {
      ri[2 * i] = 0;
      ri[2 * i + 1] = 0;
    }
  }
  if (startHP > 0) {
    i1 = (long)(startHP * frequencies);
    if (i1 < 0)
      i1 = 0;
    if (i1 > frequencies - 1)
      i1 = frequencies - 1;
    i2 = (long)(endHP * frequencies);
    if (i2 < 0)
      i2 = 0;
    if (i2 > frequencies - 1)
      i2 = frequencies - 1;
    dfraction = i1 == i2 ? 0 : 1. / (i2 - i1);
    fraction = 0;
    for (i = 0; i < i1; i++) {
      ri[2 * i] = 0;
      ri[2 * i + 1] = 0;
    }
    for (i = i1; i <= i2; i++) {
      ri[2 * i] *= fraction;
      ri[2 * i + 1] *= fraction;
      if ((fraction += dfraction) > 1)
        fraction = 1;
    }
  }
}

#endif
