/*
 * Per-particle element maps on the device.  Each function follows the
 * reference routine's floating-point operation order (cited per function),
 * because the goal is bit-identical results against the CPU oracle built
 * with the same elementary functions (b2e_math.h).  The file is compiled
 * with --fmad=false: no multiply-add contraction except the explicit fma()
 * inside b2e_math.h.
 *
 * All functions return 0 while the particle survives, or a nonzero loss code.
 */
#ifndef B2E_ELEMENTS_CUH
#define B2E_ELEMENTS_CUH
#include <float.h>
#include "b2e_rng.h"
#include "b2e_engine.h"
#include "b2e_math.h"

#define B2E_C_MKS 2.99792458e8
#define B2E_PI 3.141592653589793238462643383279502884

enum { LOSS_NONE = 0, LOSS_APERTURE = 1, LOSS_LIMIT = 2, LOSS_SLOPE = 3, LOSS_NAN = 4, LOSS_ENERGY = 5 };

struct Part {
  double x, xp, y, yp, s, dp;
};

__device__ __forceinline__ double b2e_ipow(double x, int n) {
  /* integer power by repeated multiplication (the toolkit's ipow) */
  double r;
  int i;
  if (n == 2) /* the elliptical apertures' exponent: the loop's one product */
    return x * x;
  if (n == 0)
    return 1.0;
  r = x;
  for (i = 1; i < n; i++)
    r *= x;
  return r;
}

/* checkMultAperture (multipole.c:1786-1832) for a MAXAMP-derived aperture:
 * returns true when (x, y) is inside. */
__device__ __forceinline__ bool mult_aperture_ok(double xIn, double yIn, const DevAperture *ap, const DevElem &e) {
  double x, y;
  if (!ap)
    return true;
  x = xIn - 0.0; /* xCen = 0 without aperture files */
  y = yIn - 0.0;
  if (e.flags & EF_REVERSE_TILT) {
    double x0 = x, y0 = y;
    x = x0 * e.rev_cos + y0 * e.rev_sin;
    y = -x0 * e.rev_sin + y0 * e.rev_cos;
  }
  if (ap->elliptical == 0 || ap->x_max <= 0 || ap->y_max <= 0) {
    if ((ap->x_max > 0 && fabs(x) > ap->x_max) || (ap->y_max > 0 && fabs(y) > ap->y_max))
      return false;
  } else {
    /* |x| <= x_max/4 and |y| <= y_max/4 (exact comparisons) give rounded
     * quotients of magnitude <= 1/4, powers (exponent >= 1) <= 1/4 and a sum
     * <= 1/2: inside, the answer the divisions below would give */
    if (ap->xe >= 1 && ap->ye >= 1 && fabs(x) <= 0.25 * ap->x_max && fabs(y) <= 0.25 * ap->y_max)
      return true;
    double xa = x / ap->x_max, yb = y / ap->y_max;
    if ((b2e_ipow(xa, ap->xe) + b2e_ipow(yb, ap->ye)) >= 1)
      return false;
  }
  return true;
}

/* ---- DRIF: second-order drift matrix through track_particles ---------
 * drift_matrix (compute_matrices.c:391-412) has C[4]=L, R[0][1]=R[2][3]=L,
 * T[4][1][1]=T[4][3][3]=L/2; the order-2 contraction (matrix.c:390-419)
 * sums j = 5..0, so s picks up the yp^2 term before the xp^2 term. */
/* track_particles (matrix.c:294-469) forms every output as a sum over all
 * six inputs, so a non-finite coordinate anywhere (0 * NaN, 0 * inf) makes the
 * outputs non-finite and the particle is lost after the element; with finite
 * inputs the zero matrix entries add nothing and only the terms below remain. */
__device__ __forceinline__ bool matrix_inputs_finite(const Part &p) {
  return isfinite(p.x) && isfinite(p.xp) && isfinite(p.y) && isfinite(p.yp) && isfinite(p.s) && isfinite(p.dp);
}

__device__ __forceinline__ void drif_o2(Part &p, const DevElem &e) {
  if (!matrix_inputs_finite(p)) {
    p.x = p.y = NAN;
    return;
  }
  const double L = e.c[DR_L], LH = e.c[DR_LH];
  double xn = L * p.xp + p.x;
  double yn = L * p.yp + p.y;
  double sn = (L + p.s) + (LH * p.yp) * p.yp;
  sn = sn + (LH * p.xp) * p.xp;
  p.x = xn;
  p.y = yn;
  p.s = sn;
}

__device__ __forceinline__ void drif_o1(Part &p, const DevElem &e) {
  if (!matrix_inputs_finite(p)) {
    p.x = p.y = NAN;
    return;
  }
  const double L = e.c[DR_L];
  p.x = L * p.xp + p.x;
  p.y = L * p.yp + p.y;
  p.s = L + p.s;
}

/* ---- EDRIFT: exactDrift (csbend.c:3767-3790) ---- */
__device__ __forceinline__ void edrift(Part &p, double L) {
  p.x = p.x + p.xp * L;
  p.y = p.y + p.yp * L;
  p.s = p.s + L * sqrt((1 + p.xp * p.xp) + p.yp * p.yp);
}

/* convertMomentaToSlopes (multipole.h:261-280, expandHamiltonian = 0) */
__device__ __forceinline__ bool momenta_to_slopes(double &xp, double &yp, double qx, double qy, double dp) {
  double denom = ((1 + dp) * (1 + dp) - qx * qx) - qy * qy;
  if (denom <= 0)
    return false;
  denom = sqrt(denom);
  xp = qx / denom;
  yp = qy / denom;
  return true;
}

/* offsetBeamCoordinatesForMisalignment (malign_mat.c:172-182) */
__device__ __forceinline__ void offset_misalign(Part &p, double dx, double dy, double dz) {
  p.s = p.s + dz * sqrt((1 + p.xp * p.xp) + p.yp * p.yp);
  p.x = (p.x - dx) + dz * p.xp;
  p.y = (p.y - dy) + dz * p.yp;
}

/* rotateBeamCoordinatesForMisalignment (tilt_matrices.c:156-183), cos/sin precomputed */
__device__ __forceinline__ void rotate_misalign(Part &p, double ca, double sa) {
  double x = p.x, xp = p.xp, y = p.y, yp = p.yp;
  p.x = x * ca + y * sa;
  p.y = -x * sa + y * ca;
  p.xp = xp * ca + yp * sa;
  p.yp = -xp * sa + yp * ca;
}

/* a/b correctly rounded from y = RN(1/b) computed once (Markstein, "Computation
 * of elementary functions on the IBM RISC System/6000 processor", IBM J. Res.
 * Dev. 34, 1990: with y within half an ulp of 1/b and q = RN(a y) within one
 * ulp of a/b, the remainder r = a - b q is exact under FMA and RN(q + r y) is
 * RN(a/b)).  An exact quotient (r = 0, signed zeros included) and a
 * non-finite q are returned as they are.  For divisors fixed per element, away
 * from overflow and the subnormal range; checked against division on the
 * device by b2e_selftest_division. */
__device__ __forceinline__ double div_rn_recip(double a, double b, double y) {
  const double q = a * y;
  const double r = fma(-q, b, a);
  if (r == 0 || !isfinite(q))
    return q;
  return fma(r, y, q);
}

/* ---- KQUAD / KSEXT: multipole_tracking2 (multipole.c:693-1117) with
 * integrate_kick_multipole_ordn (multipole.c:1122-1410).  The reference
 * always runs its radiation bookkeeping block (isr_coef is negated, not
 * zeroed, when ISR is off, multipole.c:781-784), which divides and
 * re-multiplies the canonical momenta by (1+delta) after each kick; that
 * round trip is reproduced because it can move the last bit. */
/* where an ISR deviate comes from (b2e_rng.h): the particle and the place */
struct RadSite {
  int64_t id;
  int32_t pass, elem;
  uint64_t seed;
  double limit;
  const double *rc; /* the element's radiation constants (DevRad) */
};

/* radiation after a kick (multipole.c:1320-1349): the momenta scaled by
 * 1/(1+delta), F2 from this substep's kick and the steering kicks, the
 * classical loss with SYNCH_RAD and a Gaussian ISR kick with ISR */
__device__ __forceinline__ void kmult_radiation(double &qx, double &qy, double &dp, double dqx, double dqy,
                                                double xp, double yp, const double *c, int step, int nSub,
                                                unsigned flags, const RadSite &rs, int slice) {
  const double drift = rs.rc[RK_DRIFT], kfrac = rs.rc[RK_KFRAC0 + step];
  double deltaFactor, F2, dsFactor, dsISRFactor;
  qx = qx / (1 + dp);
  qy = qy / (1 + dp);
  deltaFactor = (1 + dp) * (1 + dp);
  dqx = dqx / kfrac;
  dqy = dqy / kfrac;
  {
    const double a = dqx / drift - rs.rc[RK_XKICK] / drift, b = dqy / drift + rs.rc[RK_YKICK] / drift;
    F2 = a * a + b * b;
  }
  dsFactor = sqrt((1 + xp * xp) + yp * yp);
  dsISRFactor = (dsFactor * drift) / (nSub - 1);
  dsFactor = dsFactor * (drift * kfrac);
  if (flags & EF_SR)
    dp = dp - ((rs.rc[RK_RAD] * deltaFactor) * F2) * dsFactor;
  if (flags & EF_ISR)
    dp = dp - (((rs.rc[RK_ISR] * deltaFactor) * b2e_isr_pow34(F2)) * sqrt(dsISRFactor)) *
                  b2e_isr_gauss(rs.seed, rs.id, rs.pass, rs.elem, slice, step, rs.limit);
  qx = qx * (1 + dp);
  qy = qy * (1 + dp);
}

/* kick `step` of a slice of the kick integrator (multipole.c:1264-1351):
 * the canonical multipole kick of the element's order, the KSEXT K1/J1
 * terms, momenta back to slopes and the radiation block. */
template <bool RAD>
__device__ __forceinline__ int kmult_kick(double x, double y, double &xp, double &yp, double &qx, double &qy,
                                          double &dp, const DevElem &e, int order, int step, int nSub, int slice,
                                          const RadSite &rs) {
  const double *c = e.c;
  const double kick = c[KM_KICK0 + step];
  double sumFx, sumFy, dqx = 0, dqy = 0;
  /* apply_canonical_multipole_kicks (multipole.h:213-245): coefficients
   * (x+iy)^n/n! with signs; order 1: Fx=y, Fy=x; order 2: Fx=x*y,
   * Fy=x^2/2-y^2/2, each accumulated from 0 in the reference's order. */
  if (order == 1) {
    sumFx = (1.0 * 1.0) * y;
    sumFy = (1.0 * x) * 1.0;
  } else {
    double x2 = (1.0 * x) * x, y2 = (1.0 * y) * y;
    sumFx = (1.0 * x) * y;
    sumFy = (0.5 * x2) * 1.0;
    sumFy = sumFy + (-0.5 * 1.0) * y2;
  }
  qx = qx - kick * sumFy;
  qy = qy + kick * sumFx;
  if (RAD) {
    /* delta_qx, delta_qy of apply_canonical_multipole_kicks (multipole.h:237-240) */
    dqx = dqx - kick * sumFy;
    dqy = dqy + kick * sumFx;
  }
  if (e.flags & (EF_QUAD_ORDER2 | EF_SKEW_ORDER2)) {
    /* KSEXT K1/J1 terms: quadrupole order, normal then skew (multipole.c:1272-1275) */
    if (e.flags & EF_QUAD_ORDER2) {
      const double k1 = c[KM_KICK1_0 + step];
      const double fy = (1.0 * x) * 1.0, fx = (1.0 * 1.0) * y;
      qx = qx - k1 * fy;
      qy = qy + k1 * fx;
      if (RAD) {
        dqx = dqx - k1 * fy;
        dqy = dqy + k1 * fx;
      }
    }
    if (e.flags & EF_SKEW_ORDER2) {
      const double j1 = c[KM_SKEW0 + step];
      /* skew: swap(Fx, Fy), Fx = -Fx */
      double fx = -((1.0 * x) * 1.0), fy = (1.0 * 1.0) * y;
      qx = qx - j1 * fy;
      qy = qy + j1 * fx;
      if (RAD) {
        dqx = dqx - j1 * fy;
        dqy = dqy + j1 * fx;
      }
    }
  }
  if (RAD && (e.flags & EF_STEERING)) {
    /* HKICK/VKICK as order-0 canonical kicks, normal then skew
     * (multipole.c:1281-1284): sum_Fy = 1, sum_Fx = 0; skew swaps them and
     * negates, so the vertical kick enters qy through -1 */
    const double kfrac = rs.rc[RK_KFRAC0 + step], xk = rs.rc[RK_XKICK], yk = rs.rc[RK_YKICK];
    if (xk != 0) {
      const double k = -xk * kfrac;
      qx = qx - k * 1.0;
      qy = qy + k * 0.0;
    }
    if (yk != 0) {
      const double k = -yk * kfrac;
      qx = qx - k * 0.0;
      qy = qy + k * -1.0;
    }
  }
  if (!momenta_to_slopes(xp, yp, qx, qy, dp))
    return LOSS_SLOPE;
  if (e.flags & EF_RADBLOCK) {
    if (RAD && (e.flags & (EF_SR | EF_ISR))) {
      kmult_radiation(qx, qy, dp, dqx, dqy, xp, yp, c, step, nSub, e.flags, rs, slice);
    } else {
      qx = qx / (1 + dp);
      qy = qy / (1 + dp);
      qx = qx * (1 + dp);
      qy = qy * (1 + dp);
    }
    if (!momenta_to_slopes(xp, yp, qx, qy, dp))
      return LOSS_SLOPE;
  }
  return LOSS_NONE;
}

/* KQUAD fringe field of one face (quadFringe, fringe.c:24-175): slopes to
 * momenta, the linear map of the first partial fringe matrix, the leading
 * nonlinear generator (edge effects 2) scaled by the nonlinear factor, the
 * second matrix, back to slopes (DBL_MAX where that fails).  At the entrance
 * the two matrices trade places with their diagonals swapped (:50-60). */
__device__ __forceinline__ void quad_fringe(Part &p, const double *rc, int in, int order, bool linear, double nlf) {
  const double *A = rc + (in < 0 ? RK_QF_M2 : RK_QF_M1), *B = rc + (in < 0 ? RK_QF_M1 : RK_QF_M2);
  double a00 = A[0], a11 = A[3], a22 = A[4], a33 = A[7], b00 = B[0], b11 = B[3], b22 = B[4], b33 = B[7];
  if (in < 0) {
    double t = a00;
    a00 = a11;
    a11 = t;
    t = a22;
    a22 = a33;
    a33 = t;
    t = b00;
    b00 = b11;
    b11 = t;
    t = b22;
    b22 = b33;
    b33 = t;
  }
  const double delta = p.dp, xp = p.xp, yp = p.yp;
  const double denom = sqrt((1 + xp * xp) + yp * yp);
  const double v1 = (1 + delta) * xp / denom, v3 = (1 + delta) * yp / denom;
  double x, px, y, py;
  if (linear) {
    x = a00 * p.x + A[1] * v1;
    px = A[2] * p.x + a11 * v1;
    y = a22 * p.y + A[5] * v3;
    py = A[6] * p.y + a33 * v3;
  } else {
    x = p.x;
    px = v1;
    y = p.y;
    py = v3;
  }
  const double a = -in * rc[RK_QF_K1] / (12 * (1 + delta));
  double dx = 0, dpx = 0, dy = 0, dpy = 0, ds = 0;
  if (order > 1) {
    const double x2 = x * x, x3 = x2 * x, y2 = y * y, y3 = y2 * y;
    dpx = 3 * a * (-px * x2 + 2 * py * x * y - px * y2);
    dpy = 3 * a * (py * x2 - 2 * px * x * y + py * y2);
    dx = a * (x3 + 3 * x * y2);
    dy = a * (-3 * x2 * y - y3);
    ds = (a / (1 + delta)) * (3 * py * y * x2 - px * x3 - 3 * px * x * y2 + py * y3);
  }
  x += nlf * dx;
  px += nlf * dpx;
  y += nlf * dy;
  py += nlf * dpy;
  double qx, qy;
  if (linear) {
    p.x = b00 * x + B[1] * px;
    qx = B[2] * x + b11 * px;
    p.y = b22 * y + B[5] * py;
    qy = B[6] * y + b33 * py;
  } else {
    p.x = x;
    qx = px;
    p.y = y;
    qy = py;
  }
  p.s -= nlf * ds;
  const double d2 = (1 + delta) * (1 + delta) - qx * qx - qy * qy;
  if (d2 > 0) {
    const double r = sqrt(d2);
    p.xp = qx / r;
    p.yp = qy / r;
  } else {
    p.xp = p.yp = DBL_MAX;
  }
}

/* The slice loop stays rolled: unrolled instances for 4 substeps measured
 * slower in the fused ring kernel (more registers live across the unrolled
 * body, more spills). */
template <bool RAD>
__device__ __forceinline__ int kmult(Part &p, const DevElem &e, const DevAperture *ap, const DevGlobals &g,
                                     const RadSite &rs) {
  const double *c = e.c;
  const int order = (int)c[KM_ORDER], nSlices = (int)c[KM_NSLICES], nSub = (int)c[KM_NSUB];
  const double dx = c[KM_DX], dy = c[KM_DY];
  double x, xp, y, yp, s, dp, qx, qy, denom;
  int i_kick, lost;

  /* entrance misalignment, offsetParticlesForMisalignment mode 0 face 1 (malign_mat.c:491-497) */
  if (e.flags & EF_ENTRANCE_OFFSET)
    offset_misalign(p, dx, dy, c[KM_DZ]);
  if (e.flags & EF_ENTRANCE_ROTATE)
    rotate_misalign(p, c[KM_COS_TILT], c[KM_SIN_TILT]);
  if (RAD && (e.flags & EF_END_DRIFT)) /* multipole.c:1028-1030 */
    edrift(p, c[KM_LEND]);
  if (RAD && (e.flags & EF_QFRINGE1)) /* multipole.c:1031-1037 */
    quad_fringe(p, rs.rc, -1, (int)rs.rc[RK_QF_EDGE1], rs.rc[RK_QF_LIN1] != 0, rs.rc[RK_QF_NLF1]);

  x = p.x;
  xp = p.xp;
  y = p.y;
  yp = p.yp;
  s = 0;
  dp = p.dp;
  if (isnan(x) || isnan(xp) || isnan(y) || isnan(yp))
    return LOSS_NAN;
  if (fabs(x) > g.coord_limit || fabs(y) > g.coord_limit || fabs(xp) > g.slope_limit || fabs(yp) > g.slope_limit)
    return LOSS_LIMIT;
  /* convertSlopesToMomenta (multipole.h:250-259) */
  denom = sqrt((1 + xp * xp) + yp * yp);
  qx = ((1 + dp) * xp) / denom;
  qy = ((1 + dp) * yp) / denom;
  if (!momenta_to_slopes(xp, yp, qx, qy, dp))
    return LOSS_SLOPE;

  for (i_kick = 0; i_kick < nSlices; i_kick++) {
    if (!mult_aperture_ok(x + dx, y + dy, ap, e)) {
      p.x = x;
      p.y = y;
      return LOSS_APERTURE;
    }
#pragma unroll 1
    for (int step = 0; step < nSub; step++) {
      const double dsh = c[KM_DSH0 + step];
      x = x + xp * dsh;
      y = y + yp * dsh;
      s = s + dsh * sqrt((1 + xp * xp) + yp * yp);
      if (step == nSub - 1) /* kickFrac[last] == 0 ends the slice */
        break;
      if ((lost = kmult_kick<RAD>(x, y, xp, yp, qx, qy, dp, e, order, step, nSub, i_kick, rs)))
        return lost;
    }
  }
  if (!mult_aperture_ok(x + dx, y + dy, ap, e)) {
    p.x = x;
    p.y = y;
    return LOSS_APERTURE;
  }
  if (!momenta_to_slopes(xp, yp, qx, qy, dp))
    return LOSS_SLOPE;
  p.x = x;
  p.xp = xp;
  p.y = y;
  p.yp = yp;
  if (RAD && (e.flags & EF_SR)) {
    /* path length at the changed velocity (multipole.c:1391-1394) */
    const double p0 = g.p_central * (1 + p.dp), beta0 = p0 / sqrt(p0 * p0 + 1);
    const double p1 = g.p_central * (1 + dp), beta1 = p1 / sqrt(p1 * p1 + 1);
    p.s = beta1 * (p.s / beta0 + (2 * s) / (beta0 + beta1));
  } else
    p.s = p.s + s;
  p.dp = dp;
  if (isnan(x) || isnan(xp) || isnan(y) || isnan(yp))
    return LOSS_NAN;
  if (fabs(x) > g.coord_limit || fabs(y) > g.coord_limit || fabs(xp) > g.slope_limit || fabs(yp) > g.slope_limit)
    return LOSS_LIMIT;
  if (RAD && (e.flags & EF_QFRINGE2)) /* multipole.c:1088-1094 */
    quad_fringe(p, rs.rc, 1, (int)rs.rc[RK_QF_EDGE2], rs.rc[RK_QF_LIN2] != 0, rs.rc[RK_QF_NLF2]);
  if (RAD && (e.flags & EF_END_DRIFT)) /* multipole.c:1098-1100 */
    edrift(p, c[KM_LEND]);
  /* exit misalignment, face 2 (malign_mat.c:498-503) */
  if (e.flags & EF_EXIT_MISALIGN) {
    if (e.flags & EF_ENTRANCE_ROTATE)
      rotate_misalign(p, c[KM_COS_TILT], -c[KM_SIN_TILT]);
    if (e.flags & EF_ENTRANCE_OFFSET)
      offset_misalign(p, -dx, -dy, -c[KM_DZ]);
  }
  return LOSS_NONE;
}

/* ---- CSBEND body: integrate_csbend_ordn (csbend.c:1434-1693) for the
 * pure-dipole field (Fx = 0, Fy = 1, csbend.c:106-110).  Q = (X, QX, Y, QY,
 * dist, DPoP).  `isr_block` reproduces the (QX/(1+d))*(1+d) round trip of
 * the radiation block that the negated isrConstant always enables. */

/* drift substep j of a slice (csbend.c:1555-1581) */
__device__ __forceinline__ int bend_drift(double &X, double &QX, double &Y, double QY, double &dist, double DPoP,
                                          double rho0, double dsh_rho0) {
  double f, sin_phi, phi, sine, cosi, tang, cos_phi, factor, arg;
  f = (1 + DPoP) * (1 + DPoP) - QY * QY;
  if (f <= 0)
    return LOSS_SLOPE;
  f = sqrt(f);
  if (fabs(QX / f) > 1)
    return LOSS_SLOPE;
  sin_phi = QX / f;
  phi = b2e_asin(sin_phi);
  arg = dsh_rho0 + phi;
  b2e_sincos(arg, &sine, &cosi);
  if (cosi == 0)
    return LOSS_SLOPE;
  tang = sine / cosi;
  cos_phi = b2e_cos(phi);
  QX = f * sine;
  factor = (((rho0 + X) * cos_phi) / f) * (tang - sin_phi / cos_phi);
  Y = Y + QY * factor;
  dist = dist + factor * (1 + DPoP);
  f = cos_phi / cosi;
  X = rho0 * (f - 1) + f * X;
  return LOSS_NONE;
}

/* Scaled fields of a bend with K1/K2 (computeCSBENDFields, the TURBO_MODE
 * form of csbend.c:101-150, normal terms, expansion order 4): the sums over
 * x^i y^j in the reference's order, i outer, each term (F*x^i)*y^j with the
 * powers as repeated products.  F: the 15 coefficients of bend_field_terms. */
__device__ __forceinline__ void bend_fields(double x, double y, const double *F, double fx0, double &Fx,
                                            double &Fy) {
  const double y2 = y * y, y3 = y2 * y, y4 = y3 * y;
  const double x2 = x * x, x3 = x2 * x, x4 = x3 * x;
  double sx = fx0, sy = 0;
  sx = sx + F[0] * y;
  sx = sx + F[1] * y3;
  sy = sy + F[6];
  sy = sy + F[7] * y2;
  sy = sy + F[8] * y4;
  sx = sx + (F[2] * x) * y;
  sx = sx + (F[3] * x) * y3;
  sy = sy + F[9] * x;
  sy = sy + (F[10] * x) * y2;
  sx = sx + (F[4] * x2) * y;
  sy = sy + F[11] * x2;
  sy = sy + (F[12] * x2) * y2;
  sx = sx + (F[5] * x3) * y;
  sy = sy + F[13] * x3;
  sy = sy + F[14] * x4;
  Fx = sx;
  Fy = sy;
}

/* EDGE_EFFECTS 3 (applySimpleDipoleEdgeKick, csbend.c:5639-5665; no kick
 * limit, unexpanded Hamiltonian): the linear edge kick applied to the
 * canonical momenta */
__device__ __forceinline__ void bend_edge_simple(double &xp, double &yp, double x, double y, double dp,
                                                 double rho, double tan_e, double e, double psi) {
  double f = (1 + dp) / sqrt((1 + xp * xp) + yp * yp);
  double qx = xp * f, qy = yp * f;
  const double dqx = (tan_e / rho) * x;
  const double dqy = (-b2e_tan(e - psi / (1 + dp)) / rho) * y;
  qx = qx + dqx;
  qy = qy + dqy;
  f = 1 / sqrt(((1 + dp) * (1 + dp) - qx * qx) - qy * qy);
  xp = qx * f;
  yp = qy * f;
}

/* kick j of a slice (csbend.c:1591-1638) */
template <bool RAD>
__device__ __forceinline__ void bend_kick(double X, double Y, double &QX, double &QY, double &DPoP, const double *c,
                                          int i, int j, int nSub, bool isr_block, const DevElem &e,
                                          const RadSite &rs) {
  const double rho_actual = c[CB_RHO_ACTUAL];
  const double ds = c[CB_DS0 + j];
  const double x_rho0 = div_rn_recip(X, c[CB_RHO0], c[CB_INV_RHO0]);
  double Fx = 0, Fy = 1;
  if (RAD && (e.flags & EF_FIELD)) {
    /* QX += -ds*(1+X/rho0)*Fy/rho_actual; QY += ds*(1+X/rho0)*Fx/rho_actual */
    bend_fields(X, Y, rs.rc + RB_FIELD0, (e.flags & EF_SKEW_KICK) ? rs.rc[RB_SKEW0] : 0.0, Fx, Fy);
    QX = QX + div_rn_recip((((-ds) * (1 + x_rho0)) * Fy), rho_actual, c[CB_INV_RHO_ACTUAL]);
    QY = QY + div_rn_recip(((ds * (1 + x_rho0)) * Fx), rho_actual, c[CB_INV_RHO_ACTUAL]);
  } else {
    /* Fy = 1, Fx = 0 */
    QX = QX + div_rn_recip((((-ds) * (1 + x_rho0)) * 1.0), rho_actual, c[CB_INV_RHO_ACTUAL]);
    /* (t * Fx) / rho_actual with Fx = 0 is a signed zero (NaN for a
     * non-finite t): the sign of t * 0.0 flipped by rho_actual's, which
     * is finite and nonzero in a bend -- the same value without the
     * division */
    const double z = ((ds) * (1 + x_rho0)) * 0.0;
    QY = QY + (rho_actual < 0 ? -z : z);
  }
  if (RAD && (e.flags & (EF_SR | EF_ISR))) {
    /* radiation after the kick (csbend.c:1603-1622) */
    const double a = 1 + X * rs.rc[RB_INV_RHO0];
    const double f = a / sqrt(((1 + DPoP) * (1 + DPoP) - QX * QX) - QY * QY);
    const double xp = QX * f, yp = QY * f;
    const double dsFactor = sqrt((a * a + xp * xp) + yp * yp);
    const double F2 = Fx * Fx + Fy * Fy;
    const double deltaFactor = (1 + DPoP) * (1 + DPoP);
    const double dsISR = rs.rc[RB_SLICE] / (nSub - 1);
    QX = QX / (1 + DPoP);
    QY = QY / (1 + DPoP);
    if (e.flags & EF_SR)
      DPoP = DPoP - (((rs.rc[RB_RAD] * deltaFactor) * F2) * ds) * dsFactor;
    if (e.flags & EF_ISR)
      DPoP = DPoP - (((rs.rc[RB_ISR] * deltaFactor) * b2e_isr_pow34(F2)) * sqrt(dsISR * dsFactor)) *
                        b2e_isr_gauss(rs.seed, rs.id, rs.pass, rs.elem, i, j, rs.limit);
    QX = QX * (1 + DPoP);
    QY = QY * (1 + DPoP);
  } else if (isr_block) {
    QX = QX / (1 + DPoP);
    QY = QY / (1 + DPoP);
    QX = QX * (1 + DPoP);
    QY = QY * (1 + DPoP);
  }
}

/* NSUB > 0: the substep count is a compile-time constant (4 for the default
 * INTEGRATION_ORDER=4) and the slice is unrolled (the CSR slice kernel: 5 %
 * less time per kick); NSUB = 0 takes nSub from the element.  The same
 * operations in the same order either way. */
template <bool RAD, int NSUB = 0>
__device__ __forceinline__ int csbend_integrate(double &X, double &QX, double &Y, double &QY, double &dist,
                                                double &DPoP, const double *c, int nSlices, int nSub_rt,
                                                bool isr_block, const DevAperture *ap, const DevElem &e,
                                                const RadSite &rs) {
  const double rho0 = c[CB_RHO0];
  const int nSub = NSUB > 0 ? NSUB : nSub_rt;
  int lost;
  dist = 0;
  for (int i = 0; i < nSlices; i++) {
    if (!mult_aperture_ok(X, Y, ap, e))
      return LOSS_APERTURE;
    if constexpr (NSUB > 0) {
#pragma unroll
      for (int j = 0; j < NSUB; j++) {
        if ((lost = bend_drift(X, QX, Y, QY, dist, DPoP, rho0, c[CB_DSH0 + j])))
          return lost;
        if (j < NSUB - 1) /* kickFrac[last] == 0 ends the slice */
          bend_kick<RAD>(X, Y, QX, QY, DPoP, c, i, j, nSub, isr_block, e, rs);
      }
    } else {
#pragma unroll 1
      for (int j = 0; j < nSub; j++) {
        if ((lost = bend_drift(X, QX, Y, QY, dist, DPoP, rho0, c[CB_DSH0 + j])))
          return lost;
        if (j == nSub - 1) /* kickFrac[last] == 0 ends the slice */
          break;
        bend_kick<RAD>(X, Y, QX, QY, DPoP, c, i, j, nSub, isr_block, e, rs);
      }
    }
  }
  if (!mult_aperture_ok(X, Y, ap, e))
    return LOSS_APERTURE;
  return LOSS_NONE;
}

/* ---- CSBEND: track_through_csbend (csbend.c:665-1409), malignMethod 0,
 * edge method 1 at edge order 1, no synchrotron radiation. */
/* dp_prime * x * tan(e) of the radiation edge corrections (csbend.c:1211-1216,
 * :1265-1276), with the fields at (x, y) */
__device__ __forceinline__ double bend_edge_radiation(double x, double y, double xp, double yp, double dp,
                                                      double tan_e, const double *c, const double *rc,
                                                      unsigned flags) {
  double Fx = 0, Fy = 1;
  if (flags & EF_FIELD)
    bend_fields(x, y, rc + RB_FIELD0, (flags & EF_SKEW_KICK) ? rc[RB_SKEW0] : 0.0, Fx, Fy);
  const double a = 1 + x / c[CB_RHO0];
  const double dp_prime = ((-rc[RB_RAD]) * (Fx * Fx + Fy * Fy)) * ((1 + dp) * (1 + dp)) *
                          sqrt((a * a + xp * xp) + yp * yp);
  return (dp_prime * x) * tan_e;
}

/* Second-order dipole edge (K. L. Brown's non-symplectic map; csbend.c:4266-4307)
 * for EDGE_ORDER >= 2: which = -1 at the entrance, +1 at the exit; rho is
 * (1+delta)*rho_actual and psi the fringe angle times (1+delta).  The pole-face
 * curvature term (H1/H2) is zero in this engine. */
static __device__ __noinline__ void bend_edge_order2(double &x, double &xp, double &y, double &yp, double rho, double psi,
                                              double tan_b, double beta, double sec2, double n, int which) {
  const double w = (double)which, mw = (double)(-which);
  const double h = 1 / rho, h2 = h * h, tan2 = tan_b * tan_b;
  const double R21 = h * tan_b, R43 = -h * b2e_tan(beta - psi);
  const double T111 = ((w * h) / 2) * tan2;
  const double T133 = ((mw * h) / 2) * sec2;
  const double T211 = which == -1 ? ((-n) * h2) * tan_b : ((-h2) * (n + tan2 / 2)) * tan_b;
  const double T221 = (mw * h) * tan2, T331 = T221, T441 = -T221;
  const double T233 = which == -1 ? (h2 * ((n + .5) + tan2)) * tan_b : (h2 * (n - tan2 / 2)) * tan_b;
  const double T243 = (w * h) * tan2;
  const double T431 = (h2 * (2 * n + (which == 1 ? sec2 : 0))) * tan_b;
  const double T432 = (w * h) * sec2;
  const double x0 = x, xp0 = xp, y0 = y, yp0 = yp;
  x = (x0 + T111 * (x0 * x0)) + T133 * (y0 * y0);
  xp = ((((xp0 + R21 * x0) + T211 * (x0 * x0)) + (T221 * x0) * xp0) + T233 * (y0 * y0)) + (T243 * y0) * yp0;
  y = y0 + (T331 * x0) * y0;
  yp = (((yp0 + R43 * y0) + (T441 * yp0) * x0) + (T431 * x0) * y0) + (T432 * xp0) * y0;
}

template <bool RAD>
__device__ __forceinline__ int csbend(Part &p, const DevElem &e, const DevAperture *ap, const DevGlobals &g,
                                      const RadSite &rs) {
  const double *c = e.c;
  const double ct = c[CB_COS_TT], st = c[CB_SIN_TT];
  const int nSlices = (int)c[CB_NSLICES], nSub = (int)c[CB_NSUB];
  double x, y, xp, yp, s, dp, dp0, Q0, Q1, Q2, Q3, Q4, f, rho;
  int lost;

  /* element offsets and tilt (csbend.c:1108-1118) */
  p.s = p.s + c[CB_DZI] * sqrt((1 + p.xp * p.xp) + p.yp * p.yp);
  p.x = (p.x + c[CB_DXI]) + c[CB_DZI] * p.xp;
  p.y = (p.y + c[CB_DYI]) + c[CB_DZI] * p.yp;
  x = p.x * ct + p.y * st;
  y = -p.x * st + p.y * ct;
  xp = p.xp * ct + p.yp * st;
  yp = -p.xp * st + p.yp * ct;
  s = p.s;
  dp = dp0 = p.dp;

  if (e.flags & EF_EDGE1) {
    double delta_xp;
    rho = (1 + dp) * c[CB_RHO_ACTUAL];
    /* EF_EDGE_ORDER2, EF_EDGE1_SIMPLE and EF_ETILT lattices run the RAD
     * instantiation, which has the DevRad table with the BendExtra constants */
    if (RAD && (e.flags & EF_EDGE1_SIMPLE)) {
      bend_edge_simple(xp, yp, x, y, dp, c[CB_RHO_ACTUAL], c[CB_TAN_E1], c[CB_E1], c[CB_PSI1]);
    } else if (RAD && (e.flags & EF_EDGE_ORDER2)) {
      const double *bx = rs.rc + RB_EXTRA0;
      bend_edge_order2(x, xp, y, yp, rho, c[CB_PSI1] * (1 + dp), c[CB_TAN_E1], c[CB_E1], bx[BX_SEC2_E1],
                       bx[BX_EDGE_N], -1);
    } else {
      delta_xp = (c[CB_TAN_E1] / rho) * x;
      xp = xp + delta_xp;
      yp = yp - (b2e_tan(c[CB_E1] - c[CB_PSI1] / (1 + dp)) / rho) * y;
    }
  }

  /* anticipate the radiation error of integrating the sector (csbend.c:1211-1216) */
  if (RAD && (e.flags & EF_EDGE1) && (e.flags & EF_SR) && c[CB_E1] != 0)
    dp = dp - bend_edge_radiation(x, y, xp, yp, dp, c[CB_TAN_E1], c, rs.rc, e.flags);

  /* convertToDipoleCanonicalCoordinates (csbend.c:1411-1419) */
  f = (1 + dp) / sqrt((1 + xp * xp) + yp * yp);
  Q0 = x;
  Q1 = xp * f;
  Q2 = y;
  Q3 = yp * f;

  /* rolled here: in the fused ring kernel the unrolled slice measured
   * slower (register pressure); the CSR slice kernel takes the unrolled one */
  lost = csbend_integrate<RAD>(Q0, Q1, Q2, Q3, Q4, dp, c, nSlices, nSub, (e.flags & EF_RADBLOCK) != 0, ap, e, rs);

  /* convertFromDipoleCanonicalCoordinates (csbend.c:1421-1429) */
  f = 1 / sqrt(((1 + dp) * (1 + dp) - Q1 * Q1) - Q3 * Q3);
  Q1 = Q1 * f;
  Q3 = Q3 * f;
  if (lost) {
    p.x = Q0;
    p.xp = Q1;
    p.y = Q2;
    p.yp = Q3;
    if (RAD)
      p.dp = dp;
    return lost;
  }
  /* correct the radiation error of the sector at the exit (csbend.c:1265-1276) */
  if (RAD && (e.flags & EF_EDGE2) && (e.flags & EF_SR) && c[CB_E2] != 0)
    dp = dp - bend_edge_radiation(Q0, Q2, Q1, Q3, dp, c[CB_TAN_E2], c, rs.rc, e.flags);

  if (e.flags & EF_RADBLOCK) {
    /* time-of-flight velocity fix (csbend.c:1278-1288) */
    double p0 = g.p_central * (1 + dp0), beta0 = p0 / sqrt(p0 * p0 + 1);
    double p1 = g.p_central * (1 + dp), beta1 = p1 / sqrt(p1 * p1 + 1);
    s = (beta1 * s) / beta0 + Q4;
  } else
    s = s + Q4;
  x = Q0;
  xp = Q1;
  y = Q2;
  yp = Q3;

  if (e.flags & EF_EDGE2) {
    double delta_xp;
    rho = (1 + dp) * c[CB_RHO_ACTUAL];
    if (RAD && (e.flags & EF_EDGE2_SIMPLE)) {
      bend_edge_simple(xp, yp, x, y, dp, c[CB_RHO_ACTUAL], c[CB_TAN_E2], c[CB_E2], c[CB_PSI2]);
    } else if (RAD && (e.flags & EF_EDGE_ORDER2)) {
      const double *bx = rs.rc + RB_EXTRA0;
      bend_edge_order2(x, xp, y, yp, rho, c[CB_PSI2] * (1 + dp), c[CB_TAN_E2], c[CB_E2], bx[BX_SEC2_E2],
                       bx[BX_EDGE_N], 1);
    } else {
      delta_xp = (c[CB_TAN_E2] / rho) * x;
      xp = xp + delta_xp;
      yp = yp - (b2e_tan(c[CB_E2] - c[CB_PSI2] / (1 + dp)) / rho) * y;
    }
  }

  /* back to the lab frame, plus the ETILT exit offsets (csbend.c:1359-1364;
   * zero without ETILT) */
  if (RAD && (e.flags & EF_ETILT)) {
    const double *bx = rs.rc + RB_EXTRA0;
    p.x = (x * ct - y * st) + bx[BX_ETILT0];
    p.y = (x * st + y * ct) + bx[BX_ETILT0 + 2];
    p.xp = (xp * ct - yp * st) + bx[BX_ETILT0 + 1];
    p.yp = (xp * st + yp * ct) + bx[BX_ETILT0 + 3];
    p.s = s + bx[BX_ETILT0 + 4];
  } else {
    p.x = (x * ct - y * st) + 0.0;
    p.y = (x * st + y * ct) + 0.0;
    p.xp = (xp * ct - yp * st) + 0.0;
    p.yp = (xp * st + yp * ct) + 0.0;
    p.s = s + 0.0;
  }
  p.dp = dp;
  p.x = p.x + (c[CB_DXF] + c[CB_DZF] * p.xp);
  p.y = p.y + (c[CB_DYF] + c[CB_DZF] * p.yp);
  p.s = p.s + c[CB_DZF] * sqrt((1 + p.xp * p.xp) + p.yp * p.yp);
  return LOSS_NONE;
}

/* ---- MALIGN: offset_beam (do_tracking.c:3243-3300) for one particle ---- */
__device__ __forceinline__ void malign(Part &p, const double *c, double p_central) {
  double ds, pc, beta, t;
  if (c[MA_DZ] != 0)
    ds = c[MA_DZ] * sqrt((1 + p.xp * p.xp) + p.yp * p.yp);
  else
    ds = 0;
  p.x = p.x + (c[MA_DX] + c[MA_DZ] * p.xp);
  p.xp = p.xp + c[MA_DXP];
  p.y = p.y + (c[MA_DY] + c[MA_DZ] * p.yp);
  p.yp = p.yp + c[MA_DYP];
  p.s = p.s + ds;
  if (c[MA_DT] != 0 || c[MA_DP] != 0 || c[MA_DE] != 0) {
    double gamma;
    pc = p_central * (1 + p.dp);
    beta = pc / (gamma = sqrt(1 + pc * pc));
    t = p.s / (beta * c[MA_C]) + c[MA_DT];
    if (c[MA_DP] != 0) {
      p.dp = p.dp + c[MA_DP];
      pc = p_central * (1 + p.dp);
      beta = pc / sqrt(1 + pc * pc);
    }
    if (c[MA_DE] != 0) {
      gamma = gamma + c[MA_DE] * gamma;
      pc = sqrt(gamma * gamma - 1);
      beta = pc / gamma;
      p.dp = (pc - p_central) / p_central;
    }
    p.s = (t * beta) * c[MA_C];
  }
}

/* ---- RFCA: trackRfCavityWithWakes (simple_rfca.c:295-985) without wakes,
 * change_t, Q, linearisation or end focusing (rejected at load): the
 * zero-length kick (one section), the drift-kick-drift sections of N_KICKS
 * > 0 (:569-700), or the matrix method (:823-945), then the final
 * removeInvalidParticles sweep (limit_amplitudes.c:274-315). */
__device__ __forceinline__ void rf_half_drift(Part &p, double length) {
  p.x = p.x + (p.xp * length) / 2;
  p.y = p.y + (p.yp * length) / 2;
  p.s = p.s + (length / 2) * sqrt((1 + p.xp * p.xp) + p.yp * p.yp);
}

/* add_to_particle_energy (simple_rfca.c:987-1006) */
__device__ __forceinline__ void rf_add_energy(Part &p, double t, double Po, double dgamma) {
  double P, gamma, gamma1, P1, Pz, Pz1, PRatio;
  P = Po * (1 + p.dp);
  gamma1 = (gamma = sqrt(P * P + 1)) + dgamma;
  if (gamma1 <= 1)
    gamma1 = 1 + 1e-7;
  P1 = sqrt(gamma1 * gamma1 - 1);
  p.dp = (P1 - Po) / Po;
  p.s = ((t * B2E_C_MKS) * P1) / gamma1;
  Pz = P / sqrt((1 + p.xp * p.xp) + p.yp * p.yp);
  Pz1 = sqrt((Pz * Pz + gamma1 * gamma1) - gamma * gamma);
  PRatio = Pz / Pz1;
  p.xp = p.xp * PRatio;
  p.yp = p.yp * PRatio;
}

__device__ __forceinline__ int rfca(Part &p, const DevElem &e, const DevRfState &rs, const DevGlobals &g) {
  const double *c = e.c;
  const double Po = g.p_central;
  const double length = c[RF_LENGTH];
  if (c[RF_DRIFT_ONLY] != 0) {
    /* zero voltage: the exact drift over the whole length (simple_rfca.c:380-392) */
    const double L = length * c[RF_NKICKS];
    if (L != 0) {
      p.x = p.x + p.xp * L;
      p.y = p.y + p.yp * L;
      p.s = p.s + L * sqrt((1 + p.xp * p.xp) + p.yp * p.yp);
    }
    return LOSS_NONE;
  }
  const int nKicks = (int)c[RF_NKICKS];
  p.x = p.x - c[RF_DX];
  p.y = p.y - c[RF_DY];
  for (int ik = 0; ik < nKicks; ik++) {
    if (c[RF_MATRIX] == 0) {
      /* a section: half drift, energy kick at its centre's time, half drift */
      if (p.dp != -1) {
        double P, gamma, beta_i, t, dgamma, dc4;
        dc4 = length != 0 ? (length / 2) * sqrt((1 + p.xp * p.xp) + p.yp * p.yp) : 0;
        P = Po * (1 + p.dp);
        gamma = sqrt(P * P + 1);
        beta_i = P / gamma;
        t = (p.s + dc4) / (B2E_C_MKS * beta_i) - 0.0;
        dgamma = (c[RF_VOLT] * b2e_sin(c[RF_OMEGA] * ((t - 0.0) - ik * c[RF_DTLIGHT]) + rs.phase)) * 1.0;
        if (length != 0)
          rf_half_drift(p, length);
        rf_add_energy(p, t, Po, dgamma);
        if (gamma + dgamma <= 1)
          p.dp = -1;
      }
      if (length != 0)
        rf_half_drift(p, length); /* the final drift takes every particle */
    } else {
      /* matrix method, momentum-based body focusing (simple_rfca.c:855-945) */
      double P, gamma, beta_i, t, dgamma, dP, ds1, R12, R22, x, xp;
      const double R11 = 1, R21 = 0;
      P = Po * (1 + p.dp);
      gamma = sqrt(P * P + 1);
      beta_i = P / gamma;
      ds1 = (length / 2) * sqrt((1 + p.xp * p.xp) + p.yp * p.yp);
      t = (p.s + ds1) / (B2E_C_MKS * beta_i) - 0.0;
      {
        const double arg = c[RF_OMEGA] * ((t - 0.0) - ik * c[RF_DTLIGHT]) + rs.phase;
        const double sin_phase = b2e_sin(arg);
        dgamma = c[RF_VOLT] * sin_phase;
      }
      dP = sqrt((gamma + dgamma) * (gamma + dgamma) - 1) - P;
      R22 = 1 / (1 + dP / P);
      if (fabs(dP / P) > 1e-14)
        R12 = length * ((P / dP) * b2e_log(1 + dP / P));
      else
        R12 = length;
      p.s = p.s + ds1;
      x = p.x;
      xp = p.xp;
      p.x = x * R11 + xp * R12;
      p.xp = x * R21 + xp * R22;
      x = p.y;
      xp = p.yp;
      p.y = x * R11 + xp * R12;
      p.yp = x * R21 + xp * R22;
      p.s = p.s + (length / 2) * sqrt((1 + p.xp * p.xp) + p.yp * p.yp);
      p.dp = ((P + dP) - Po) / Po;
      if ((gamma = gamma + dgamma) <= 1)
        p.dp = -1;
      p.s = (((P + dP) / gamma) * p.s) / beta_i;
    }
  }
  p.x = p.x + c[RF_DX];
  p.y = p.y + c[RF_DY];
  if (isnan(p.x) || isnan(p.xp) || isnan(p.y) || isnan(p.yp) || isnan(p.s) || isnan(p.dp) || p.dp <= -1)
    return LOSS_ENERGY;
  return LOSS_NONE;
}

/* ---- apertures after each element (do_tracking.c:2455-2475) ----------
 * mode 1: limit_amplitudes (limit_amplitudes.c:193-272), rectangular;
 * mode 2: elimit_amplitudes (limit_amplitudes.c:472-600), super-elliptical.
 * The host resolves elegant's fallbacks (elliptical with a zero half-axis
 * falls back to rectangular; all-nonpositive half-axes check nothing). */
__device__ __forceinline__ bool maxamp_ok(const Part &p, const DevAperture &a) {
  if (a.mode == 1) {
    bool out = (a.x_max > 0 && fabs(p.x) > a.x_max) || (a.y_max > 0 && fabs(p.y) > a.y_max);
    if (isinf(p.x) || isinf(p.y) || isnan(p.x) || isnan(p.y))
      out = true;
    return !out;
  }
  if (a.mode == 2) {
    if (isinf(p.x) || isinf(p.y) || isnan(p.x) || isnan(p.y))
      return false;
    /* |x| <= x_max/4, |y| <= y_max/4: with exponents 1..8 and half-axes in
     * [2^-100, 2^100] every rounded power is that of x_max/4 or less, i.e.
     * at most 4^-n a2 (scaling by 1/4 is exact there), so each term is at
     * most 1/4 and the particle is inside, as the divisions below find */
    if (a.xe >= 1 && a.xe <= 8 && a.ye >= 1 && a.ye <= 8 && a.x_max >= 0x1p-100 && a.x_max <= 0x1p100 &&
        a.y_max >= 0x1p-100 && a.y_max <= 0x1p100 && fabs(p.x) <= 0.25 * a.x_max && fabs(p.y) <= 0.25 * a.y_max)
      return true;
    return !((b2e_ipow(p.x, a.xe) / a.a2 + b2e_ipow(p.y, a.ye) / a.b2) > 1);
  }
  return true;
}

__device__ __forceinline__ bool finite_xy(const Part &p) {
  /* limit_amplitudes(DBL_MAX, DBL_MAX): only inf/nan in x or y remove a particle */
  return !(isinf(p.x) || isinf(p.y) || isnan(p.x) || isnan(p.y));
}

#endif
