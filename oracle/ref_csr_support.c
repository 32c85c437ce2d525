/*
 * Restated support routines that the reference's CSR path calls but that live
 * outside the compiled subset: final_props.c (rms_emittance, approximateBeamWidth)
 * and the SDDS toolkit's mdbmth (fill_double_array, index_min_max,
 * SavitzyGolaySmooth, zeroNewton, zeroInterp, realFFT2).  The Savitzky-Golay convention is the one this project
 * defines for both the oracle and the CUDA path (b2e_sg.h); the toolkit's own
 * edge treatment is not in the reference tree, so CSR parity at that boundary
 * is against this shared definition; the same holds for the two root finders
 * of SolveForPhiStupakov (b2e_roots.h) and the real transform behind
 * applyLHPassFilters (b2e_fft.h).  Test infrastructure only.
 */
#include "mdb.h"
#include "track.h"
#include "b2e_sg.h"
#include "b2e_roots.h"
#include "b2e_fft.h"

#define ANALYSIS_BINS 10000 /* final_props.c:21 */

void fill_double_array(double *array, long n, double value) {
  long i;
  for (i = 0; i < n; i++)
    array[i] = value;
}

/* Indices of the first minimum and first maximum of an array. */
long index_min_max(int64_t *imin, int64_t *imax, double *list, int64_t n) {
  int64_t i;
  double vmin, vmax;
  if (n <= 0)
    return 0;
  *imin = *imax = 0;
  vmin = vmax = list[0];
  for (i = 1; i < n; i++) {
    if (list[i] < vmin) {
      vmin = list[i];
      *imin = i;
    }
    if (list[i] > vmax) {
      vmax = list[i];
      *imax = i;
    }
  }
  return 1;
}

double rms_emittance(double **coord, long i1, long i2, long n, double *s11Return, double *s12Return,
                     double *s22Return, double *c1Return, double *c2Return) {
  /* final_props.c:844-880: centroids, then second moments, sequential sums */
  double s11, s12, s22, x, xp, xc, xpc;
  long i;
  if (!n)
    return 0.0;
  for (i = 0, xc = xpc = 0; i < n; i++) {
    xc += coord[i][i1];
    xpc += coord[i][i2];
  }
  xc /= n;
  xpc /= n;
  if (c1Return)
    *c1Return = xc;
  if (c2Return)
    *c2Return = xpc;
  for (i = 0, s11 = s12 = s22 = 0; i < n; i++) {
    x = coord[i][i1] - xc;
    xp = coord[i][i2] - xpc;
    s11 += sqr(x);
    s22 += sqr(xp);
    s12 += x * xp;
  }
  if (s11Return)
    *s11Return = s11 / n;
  if (s22Return)
    *s22Return = s22 / n;
  if (s12Return)
    *s12Return = s12 / n;
  x = s11 * s22 - sqr(s12);
  return (x > 0 ? sqrt(x) : 0) / n;
}

double approximateBeamWidth(double fraction, double **part, long nPart, long iCoord) {
  /* final_props.c:1258-1310: 1.01-expanded histogram into ANALYSIS_BINS bins,
   * cumulative distribution, then the index span holding `fraction` of the
   * particles around the median, times the bin size. */
  double *hist, *cdf;
  long maxBins = ANALYSIS_BINS, bins = ANALYSIS_BINS, i50, iLo, iHi, i;
  double xMin = 0, xMax = 0, dx = 0;
  hist = tmalloc(sizeof(*hist) * bins);
  binParticleCoordinate(&hist, &maxBins, &xMin, &xMax, &dx, &bins, 1.01, part, nPart, iCoord);
  cdf = hist;
  for (i = 1; i < bins; i++)
    cdf[i] += cdf[i - 1];
  i50 = bins / 2;
  for (i = 0; i < bins; i++) {
    cdf[i] /= cdf[bins - 1];
    if (cdf[i] < 0.50)
      i50 = i;
  }
  iLo = iHi = i50;
  for (i = i50; i < bins; i++) {
    if ((cdf[i] - 0.5) < fraction / 2)
      iHi = i;
    else
      break;
  }
  for (i = i50; i >= 0; i--) {
    if ((0.5 - cdf[i]) < fraction / 2)
      iLo = i;
    else
      break;
  }
  free(hist);
  return (iHi - iLo) * dx;
}

long SavitzyGolaySmooth(double *data, long rows, long order, long nLeft, long nRight, long derivativeOrder) {
  return b2e_sg_apply_host(data, rows, order, nLeft, nRight, derivativeOrder);
}

/* mdbmth's root finders as SolveForPhiStupakov (csbend.c:4189-4195) calls
 * them, on the shared definitions of b2e_roots.h */
double zeroNewton(double (*fn)(double), double value, double x_i, double dx, long n_passes, double _zero) {
  return b2e_zero_newton(fn, value, x_i, dx, n_passes, _zero);
}

double zeroInterp(double (*fn)(double), double value, double x_i, double x_f, double dx, double _zero) {
  return b2e_zero_interp(fn, value, x_i, x_f, dx, _zero);
}

/* realFFT2 as applyLHPassFilters (csbend.c:4631, :4687) calls it: forward
 * (flags 0) from n real values to n/2 + 1 (re, im) pairs, or back
 * (INVERSE_FFT), on the shared transform of b2e_fft.h; input and output may
 * be the same array */
long realFFT2(double *output, double *input, long n, unsigned long flags) {
  double *c, *s, *in;
  long i;
  if (n < 1)
    return 0;
  c = malloc(sizeof(double) * n);
  s = malloc(sizeof(double) * n);
  in = malloc(sizeof(double) * (n + 2));
  for (i = 0; i < n; i++)
    b2e_dft_twiddle(n, i, &c[i], &s[i]);
  if (flags & INVERSE_FFT) {
    memcpy(in, input, sizeof(double) * (n + 2));
    for (i = 0; i < n; i++)
      output[i] = b2e_rdft_sample(in, n, i, c, s);
  } else {
    memcpy(in, input, sizeof(double) * n);
    for (i = 0; i < n / 2 + 1; i++)
      b2e_rdft_pair(in, n, i, c, s, &output[2 * i], &output[2 * i + 1]);
  }
  free(c);
  free(s);
  free(in);
  return 1;
}
