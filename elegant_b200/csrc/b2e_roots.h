/*
 * One-dimensional root finders for the CSRDRIFT Stupakov wake.
 *
 * SolveForPhiStupakov (csbend.c:4169-4202) solves
 *     24 ds = phi^3 (phi + 4x) / (phi + x)
 * with two routines of the SDDS toolkit's mdbmth library, zeroNewton and
 * zeroInterp, which are not part of the reference tree.  This file defines
 * them for this project from the methods their names and call sites describe:
 *
 *   b2e_zero_newton(fn, value, x_i, dx, n_passes, tol)
 *       Newton's method on g(x) = fn(x) - value with a forward-difference
 *       slope (g(x + dx) - g(x)) / dx.  Each pass evaluates g at the iterate
 *       and returns it when |g| < tol; the last pass that does not converge
 *       returns the midpoint of the iterate and the previous difference point
 *       (the caller checks the answer and falls back to b2e_zero_interp).
 *
 *   b2e_zero_interp(fn, value, x_i, x_f, dx, tol)
 *       Scans x_i, x_i + dx, ... up to x_f for a sign change of g between
 *       two finite values (or a point with |g| < tol), then refines the bracket by false position with the
 *       Illinois correction, at most B2E_ROOT_MAX_REFINE steps.  Without a
 *       bracket it returns x_f + dx, outside the scanned interval, which the
 *       caller treats as no solution.
 *
 * Every caller -- the CUDA kernels, the C restatement and the shim that links
 * elegant's own csbend.c -- uses this one body, so all of them solve to the
 * same bits.  Plain C for gcc; a template over the function object under C++
 * (nvcc host and device code).  Loops are bounded by iteration counts, so no
 * input makes them spin.
 */
#ifndef B2E_ROOTS_H
#define B2E_ROOTS_H
#include <math.h>
#include <float.h>

#define B2E_ROOT_MAX_SCAN 100000
#define B2E_ROOT_MAX_REFINE 200

#ifdef __cplusplus
#ifdef __CUDACC__
#define B2E_ROOT_HD __host__ __device__
#else
#define B2E_ROOT_HD
#endif
#define B2E_ROOT_DEF(ret) template <typename B2eRootFn> B2E_ROOT_HD static inline ret
#define B2E_ROOT_FN_T B2eRootFn
#else
typedef double (*b2e_root_fn)(double);
#define B2E_ROOT_DEF(ret) static inline ret
#define B2E_ROOT_FN_T b2e_root_fn
#endif

B2E_ROOT_DEF(double)
b2e_zero_newton(B2E_ROOT_FN_T fn, double value, double x_i, double dx, long n_passes, double tol) {
  double x = x_i, x_diff = x_i, g, g_diff, slope;
  long pass;
  for (pass = 0; pass < n_passes; pass++) {
    g = fn(x) - value;
    if (fabs(g) < tol)
      return x;
    if (pass == n_passes - 1)
      return (x + x_diff) / 2;
    x_diff = x + dx;
    g_diff = fn(x_diff) - value;
    slope = (g_diff - g) / dx;
    x = x - g / slope;
  }
  return DBL_MAX;
}

B2E_ROOT_DEF(double)
b2e_zero_interp(B2E_ROOT_FN_T fn, double value, double x_i, double x_f, double dx, double tol) {
  double xa = x_i, xb, xm, ga, gb, gm;
  long step, k;
  int side = 0;
  if (!(dx > 0))
    return x_f + fabs(dx) + 1;
  ga = fn(xa) - value;
  if (fabs(ga) < tol)
    return xa;
  for (step = 0;; step++) {
    xb = xa + dx;
    if (xb > x_f || step >= B2E_ROOT_MAX_SCAN)
      return x_f + dx;
    gb = fn(xb) - value;
    if (fabs(gb) < tol)
      return xb;
    if (ga == ga && gb == gb && (ga < 0) != (gb < 0))
      break;
    xa = xb;
    ga = gb;
  }
  xm = xa;
  for (k = 0; k < B2E_ROOT_MAX_REFINE; k++) {
    xm = xa - ga * (xb - xa) / (gb - ga);
    gm = fn(xm) - value;
    if (fabs(gm) < tol)
      return xm;
    if ((gm < 0) == (ga < 0)) {
      xa = xm;
      ga = gm;
      if (side == -1)
        gb = gb / 2;
      side = -1;
    } else {
      xb = xm;
      gb = gm;
      if (side == 1)
        ga = ga / 2;
      side = 1;
    }
  }
  return xm;
}

#endif
