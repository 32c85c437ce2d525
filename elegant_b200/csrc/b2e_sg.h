/*
 * Savitzky-Golay smoothing / differentiation of a 1-D histogram, as used by
 * the CSR step (csbend.c:2569-2581 calls SavitzyGolaySmooth on the line
 * density and its derivative).  The toolkit routine the reference links is not
 * in its source tree, so this file defines the convention for this project:
 *
 *   - Savitzky & Golay (1964): the value (derivativeOrder 0) or first
 *     derivative (derivativeOrder 1, per bin index) at a point is that of the
 *     least-squares polynomial of degree `order` fitted over a window of
 *     nLeft + nRight + 1 consecutive bins;
 *   - interior points use the window [i - nLeft, i + nRight];
 *   - near either end the window keeps its width and is shifted inwards, and
 *     the fitted polynomial is evaluated at the point's own offset inside it
 *     (no padding, no reflection);
 *   - arrays shorter than the window are fitted as a whole with the degree
 *     reduced to at most rows - 1.
 *
 * Coefficients are computed in double precision by the same code for every
 * user (oracle, reference driver, CUDA host), so all of them smooth with
 * bitwise identical weights; the filter is applied as an ascending-offset sum.
 * Plain C: compiled by gcc for the oracles and by nvcc for the host side of
 * the CUDA path.
 */
#ifndef B2E_SG_H
#define B2E_SG_H
#include <stdlib.h>
#include <string.h>

#define B2E_SG_MAX_WIDTH 65
#define B2E_SG_MAX_ORDER 6

/* the weight and window helpers also compile as device functions under nvcc */
#ifdef __CUDACC__
#define B2E_SG_FN __host__ __device__ static inline
#else
#define B2E_SG_FN static inline
#endif

/* Weights w[0..width-1] for the window offsets k = kLo .. kLo+width-1 relative
 * to the evaluation point, for a degree-`order` fit and derivative `deriv`.
 * Solves the (order+1)^2 normal equations by Gauss-Jordan elimination with
 * partial pivoting.  Returns 0 on success. */
B2E_SG_FN int b2e_sg_weights(double *w, long width, long kLo, long order, long deriv) {
  double a[B2E_SG_MAX_ORDER + 1][B2E_SG_MAX_ORDER + 1];
  double inv[B2E_SG_MAX_ORDER + 1][B2E_SG_MAX_ORDER + 1];
  long m = order + 1, i, j, k, r;
  double fact = 1;
  if (order < 0 || order > B2E_SG_MAX_ORDER || width < 1 || width > B2E_SG_MAX_WIDTH || deriv < 0 || deriv > order)
    return 1;
  /* normal matrix sum_k k^(i+j) */
  for (i = 0; i < m; i++)
    for (j = 0; j < m; j++) {
      double s = 0;
      for (k = 0; k < width; k++) {
        double t = 1, kk = (double)(kLo + k);
        long p;
        for (p = 0; p < i + j; p++)
          t *= kk;
        s += t;
      }
      a[i][j] = s;
      inv[i][j] = (i == j) ? 1 : 0;
    }
  for (i = 0; i < m; i++) {
    double piv;
    long best = i;
    for (r = i + 1; r < m; r++)
      if ((a[r][i] < 0 ? -a[r][i] : a[r][i]) > (a[best][i] < 0 ? -a[best][i] : a[best][i]))
        best = r;
    if (a[best][i] == 0)
      return 2;
    if (best != i)
      for (j = 0; j < m; j++) {
        double t = a[i][j];
        a[i][j] = a[best][j];
        a[best][j] = t;
        t = inv[i][j];
        inv[i][j] = inv[best][j];
        inv[best][j] = t;
      }
    piv = a[i][i];
    for (j = 0; j < m; j++) {
      a[i][j] /= piv;
      inv[i][j] /= piv;
    }
    for (r = 0; r < m; r++) {
      double f;
      if (r == i)
        continue;
      f = a[r][i];
      if (f == 0)
        continue;
      for (j = 0; j < m; j++) {
        a[r][j] -= f * a[i][j];
        inv[r][j] -= f * inv[i][j];
      }
    }
  }
  for (i = 2; i <= deriv; i++)
    fact *= i;
  /* coefficient `deriv` of the fitted polynomial, times deriv!, evaluated at 0 */
  for (k = 0; k < width; k++) {
    double kk = (double)(kLo + k), t = 1, s = 0;
    for (j = 0; j < m; j++) {
      s += inv[deriv][j] * t;
      t *= kk;
    }
    w[k] = s * fact;
  }
  return 0;
}

/* Window placement for point i: returns the first bin of the window and its width. */
B2E_SG_FN long b2e_sg_window(long i, long rows, long nLeft, long nRight, long *width) {
  long w = nLeft + nRight + 1, lo;
  if (w > rows)
    w = rows;
  lo = i - nLeft;
  if (lo < 0)
    lo = 0;
  if (lo + w > rows)
    lo = rows - w;
  *width = w;
  return lo;
}

/* In-place smoothing on the host.  Returns 1 on success, 0 on bad arguments
 * (the toolkit routine's convention). */
static inline long b2e_sg_apply_host(double *data, long rows, long order, long nLeft, long nRight, long deriv) {
  double *out, w[B2E_SG_MAX_WIDTH];
  long i, k, width, ord;
  if (rows < 1 || nLeft < 0 || nRight < 0 || nLeft + nRight + 1 > B2E_SG_MAX_WIDTH)
    return 0;
  out = (double *)malloc(sizeof(double) * rows);
  if (!out)
    return 0;
  for (i = 0; i < rows; i++) {
    long lo = b2e_sg_window(i, rows, nLeft, nRight, &width);
    double s = 0;
    ord = order < width - 1 ? order : width - 1;
    if (deriv > ord) {
      out[i] = 0;
      continue;
    }
    if (b2e_sg_weights(w, width, lo - i, ord, deriv)) {
      free(out);
      return 0;
    }
    for (k = 0; k < width; k++)
      s += w[k] * data[lo + k];
    out[i] = s;
  }
  memcpy(data, out, sizeof(double) * rows);
  free(out);
  return 1;
}

#endif
