/*
 * CPU oracle: a plain-C restatement of elegant's particle-tracking hot path
 * for the element subset of the CUDA engine (test infrastructure only; the
 * product never calls this code).
 *
 * It follows the reference's own data layout and control flow: particles are
 * rows of doubles (x, xp, y, yp, s, delta, id, lossPass), lost particles are
 * swapped to the tail of the array as the reference does, and every
 * floating-point expression keeps the reference's operation order, so with
 * the same elementary functions it reproduces the reference bit for bit.
 *
 * Elementary functions: compiled with -DB2E_ORACLE_LIBM it calls glibc like
 * the reference; otherwise sin/cos/tan/asin are the shared implementations of
 * elegant_b200/csrc/b2e_math.h that the CUDA engine uses.
 *
 * Sources restated (file:line in the reference tree):
 *   do_tracking        do_tracking.c:488-2640 (pass/element loop, z bookkeeping
 *                      :1077-1084, sticky MAXAMP :1848-1858, aperture after
 *                      each element :2455-2475, NaN sweep :2629, loss record
 *                      :4584-4605, effort :2758-2764)
 *   track_particles    matrix.c:294-469 (order-2 contraction :390-419)
 *   drift_matrix       compute_matrices.c:391-412
 *   exactDrift         csbend.c:3767-3790
 *   multipole_tracking2 multipole.c:693-1117
 *   integrate_kick_multipole_ordn multipole.c:1122-1410
 *   apply_canonical_multipole_kicks, expansion_coefficients, fillPowerArray,
 *   convertSlopesToMomenta/MomentaToSlopes multipole.h:173-280
 *   checkMultAperture  multipole.c:1786-1832
 *   offsetBeamCoordinatesForMisalignment malign_mat.c:172-182
 *   offsetParticlesForMisalignment (mode 0) malign_mat.c:480-531
 *   rotateBeamCoordinatesForMisalignment tilt_matrices.c:156-183
 *   track_through_csbend csbend.c:665-1409; integrate_csbend_ordn csbend.c:1434-1693
 *   convert{To,From}DipoleCanonicalCoordinates csbend.c:1411-1429
 *   computeCSBENDFields (pure dipole fast path) csbend.c:101-110
 *   trackRfCavityWithWakes simple_rfca.c:295-985; findFiducialTime :62-262;
 *   add_to_particle_energy :987-1006; KahanPlus kahan.c:28-35
 *   limit_amplitudes / removeInvalidParticles / elimit_amplitudes
 *                      limit_amplitudes.c:193-315, :472-600
 *   swapParticles      elegant.c:2663-2670; beta_from_delta do_tracking.c:95
 */
#include <math.h>
#include <float.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "../include/elegant_b200.h"

#ifdef B2E_ORACLE_LIBM
#define M_SIN(x) sin(x)
#define M_COS(x) cos(x)
#define M_TAN(x) tan(x)
#define M_ASIN(x) asin(x)
#define M_LOG(x) log(x)
#define M_POW(x, y) pow(x, y)
#else
#include "../elegant_b200/csrc/b2e_math.h"
#define M_SIN(x) b2e_sin(x)
#define M_COS(x) b2e_cos(x)
#define M_TAN(x) b2e_tan(x)
#define M_ASIN(x) b2e_asin(x)
#define M_LOG(x) b2e_log(x)
#define M_POW(x, y) b2e_pow(x, y)
#endif

#define NPROP 8 /* x, xp, y, yp, s, delta, id, lossPass */
#define C_MKS 2.99792458e8
#define ME_MEV 0.51099895000
#define ME_MKS 9.1093837015e-31
#define E_MKS 1.602176634e-19
#define RE_MKS 2.8179403262e-15
#define PI_ 3.141592653589793238462643383279502884
#define BETA_ 1.25992104989487316477
#define SQR(x) ((x) * (x))

static double coord_limit = 10, slope_limit = 1;

/* ---- small helpers ------------------------------------------------------ */
static void swap_rows(double *a, double *b) {
  double t[NPROP];
  if (a == b)
    return;
  memcpy(t, a, sizeof(t));
  memcpy(a, b, sizeof(t));
  memcpy(b, t, sizeof(t));
}

static double ipow_(double x, long n) {
  double r = x;
  long i;
  if (n == 0)
    return 1;
  for (i = 1; i < n; i++)
    r *= x;
  return r;
}

static int fractions(int order, double *df, double *kf) {
  static const double d6[8] = {0.39225680523878,   0.5100434119184585,   -0.47105338540975655, 0.0687531682525181,
                               0.0687531682525181, -0.47105338540975655, 0.5100434119184585,   0.39225680523878};
  static const double k6[8] = {0.784513610477560,  0.235573213359357, -1.17767998417887, 1.3151863206839063,
                               -1.17767998417887, 0.235573213359357, 0.784513610477560, 0};
  int j;
  if (order == 2) {
    df[0] = df[1] = 0.5;
    kf[0] = 1.0;
    kf[1] = 0.0;
    return 2;
  }
  if (order == 4) {
    df[0] = 0.5 / (2 - BETA_);
    df[1] = (1 - BETA_) / (2 - BETA_) / 2;
    df[2] = (1 - BETA_) / (2 - BETA_) / 2;
    df[3] = 0.5 / (2 - BETA_);
    kf[0] = 1. / (2 - BETA_);
    kf[1] = -BETA_ / (2 - BETA_);
    kf[2] = 1 / (2 - BETA_);
    kf[3] = 0;
    return 4;
  }
  if (order == 6) {
    for (j = 0; j < 8; j++) {
      df[j] = d6[j];
      kf[j] = k6[j];
    }
    return 8;
  }
  return 0;
}

/* ---- apertures ---------------------------------------------------------- */
typedef struct {
  int present; /* a MAXAMP has been seen */
  double x_max, y_max;
  long elliptical, exponent, y_exponent;
} MaxAmp;

typedef struct {
  double xMax, yMax, reverseTilt, rc, rs;
  long elliptical, xe, ye;
} MultAp;

static void setup_mult_ap(MultAp *a, double reverseTilt, const MaxAmp *m) {
  a->reverseTilt = reverseTilt;
  a->rc = M_COS(reverseTilt);
  a->rs = M_SIN(reverseTilt);
  a->xMax = a->yMax = 0;
  a->elliptical = 0;
  a->xe = a->ye = 2;
  if (m && m->present) {
    a->xMax = m->x_max;
    a->yMax = m->y_max;
    a->elliptical = m->elliptical;
    a->xe = a->ye = m->exponent;
    if (m->y_exponent)
      a->ye = m->y_exponent;
  }
}

static int mult_ap_ok(double xIn, double yIn, const MultAp *a) {
  double x = xIn - 0.0, y = yIn - 0.0;
  if (a->reverseTilt) {
    double x0 = x, y0 = y;
    x = x0 * a->rc + y0 * a->rs;
    y = -x0 * a->rs + y0 * a->rc;
  }
  if (a->elliptical == 0 || a->xMax <= 0 || a->yMax <= 0) {
    if ((a->xMax > 0 && fabs(x) > a->xMax) || (a->yMax > 0 && fabs(y) > a->yMax))
      return 0;
  } else {
    double xa = x / a->xMax, yb = y / a->yMax;
    if ((ipow_(xa, a->xe) + ipow_(yb, a->ye)) >= 1)
      return 0;
  }
  return 1;
}

static long limit_amps(double **c, double xmax, double ymax, long np, double z, double Po, int extrap) {
  long ip, itop = np - 1;
  if (xmax < 0 && ymax < 0)
    return np;
  for (ip = 0; ip < np; ip++) {
    double *part = c[ip], dz = 0;
    long is_out = 0;
    if (xmax > 0 && fabs(part[0]) > xmax)
      is_out += 1;
    if (ymax > 0 && fabs(part[2]) > ymax)
      is_out += 2;
    if (isinf(part[0]) || isinf(part[2]) || isnan(part[0]) || isnan(part[2]))
      is_out += 4;
    if (is_out && !(is_out & 4) && extrap) {
      double dzx = -DBL_MAX, dzy = -DBL_MAX;
      if (is_out & 1 && part[1] != 0)
        dzx = (part[0] - (part[1] < 0 ? -1 : 1) * xmax) / part[1];
      if (is_out & 2 && part[3] != 0)
        dzy = (part[2] - (part[3] < 0 ? -1 : 1) * ymax) / part[3];
      dz = dzx > dzy ? -dzx : -dzy;
      if (dz == -DBL_MAX)
        dz = 0;
    }
    if (is_out) {
      if (ip != itop)
        swap_rows(c[ip], c[itop]);
      c[itop][0] += dz * c[itop][1];
      c[itop][2] += dz * c[itop][3];
      c[itop][4] = z + dz;
      c[itop][5] = Po * (1 + c[itop][5]);
      --itop;
      --ip;
      np--;
    }
  }
  return np;
}

static long elimit_amps(double **c, double xmax, double ymax, long np, double z, double Po, int extrap, long xe,
                        long ye) {
  long ip, itop = np - 1;
  double a2, b2;
  if (!ye)
    ye = xe;
  if (xmax <= 0 || ymax <= 0) {
    if (xmax > 0 || ymax > 0)
      return limit_amps(c, xmax, ymax, np, z, Po, extrap);
    return np;
  }
  a2 = ipow_(xmax, xe);
  b2 = ipow_(ymax, ye);
  for (ip = 0; ip < np; ip++) {
    double *part = c[ip], dz = 0;
    if (isinf(part[0]) || isinf(part[2]) || isnan(part[0]) || isnan(part[2])) {
      swap_rows(c[ip], c[itop]);
      c[itop][4] = z;
      c[itop][5] = sqrt(SQR(Po * (1 + c[itop][5])) + 1);
      --itop;
      --ip;
      np--;
      continue;
    }
    if (!((ipow_(part[0], xe) / a2 + ipow_(part[2], ye) / b2) > 1))
      continue;
    if (extrap && xe == 2 && ye == 2) {
      double c0 = SQR(part[0]) / a2 + SQR(part[2]) / b2 - 1;
      double c1 = 2 * (part[0] * part[1] / a2 + part[2] * part[3] / b2);
      double c2 = SQR(part[1]) / a2 + SQR(part[3]) / b2;
      double det = SQR(c1) - 4 * c0 * c2;
      if (z > 0 && c2 && det >= 0) {
        if ((dz = (-c1 + sqrt(det)) / (2 * c2)) > 0)
          dz = (-c1 - sqrt(det)) / (2 * c2);
        if ((z + dz) < 0)
          dz = -z;
        part[0] += dz * part[1];
        part[2] += dz * part[3];
      }
    }
    swap_rows(c[ip], c[itop]);
    c[itop][4] = z + dz;
    c[itop][5] = sqrt(SQR(Po * (1 + c[itop][5])) + 1);
    --itop;
    --ip;
    np--;
  }
  return np;
}

/* ---- DRIF: order-2 contraction of the drift matrix ------------------------ */
static void drift_track(double **c, long np, double L, int order) {
  /* C/R/T of drift_matrix; T stored lower-triangular T[i][j][k], k <= j */
  double C[6] = {0, 0, 0, 0, L, 0}, R[6][6], T[6][6][6];
  long ip, i, j, k;
  memset(R, 0, sizeof(R));
  memset(T, 0, sizeof(T));
  for (i = 0; i < 6; i++)
    R[i][i] = 1;
  R[0][1] = R[2][3] = L;
  if (order > 1)
    T[4][1][1] = T[4][3][3] = L / 2;
  for (ip = np - 1; ip >= 0; ip--) {
    double *ini = c[ip], tmp[6];
    for (i = 5; i >= 0; i--) {
      double sum = C[i];
      if (order >= 2) {
        for (j = 5; j >= 0; j--) {
          double cj = ini[j];
          if (cj) {
            double sum1 = R[i][j];
            for (k = j; k >= 0; k--)
              sum1 += T[i][j][k] * ini[k];
            sum += sum1 * cj;
          }
        }
      } else {
        for (j = 5; j >= 0; j--)
          sum += R[i][j] * ini[j];
      }
      tmp[i] = sum;
    }
    for (i = 5; i >= 0; i--)
      ini[i] = tmp[i];
  }
}

static void exact_drift(double **c, long np, double L) {
  long i;
  for (i = 0; i < np; i++) {
    double *x = c[i];
    x[0] += x[1] * L;
    x[2] += x[3] * L;
    x[4] += L * sqrt(1 + SQR(x[1]) + SQR(x[3]));
  }
}

/* ---- misalignment ----------------------------------------------------------- */
static void offset_beam(double **c, long np, double dx, double dy, double dz) {
  long ip;
  for (ip = np - 1; ip >= 0; ip--) {
    double *p = c[ip];
    p[4] += dz * sqrt(1 + SQR(p[1]) + SQR(p[3]));
    p[0] = p[0] - dx + dz * p[1];
    p[2] = p[2] - dy + dz * p[3];
  }
}

static void rotate_beam(double **c, long np, double angle) {
  double ca, sa;
  long i;
  if (!angle || fabs(fabs(angle) - 2 * PI_) < 1e-12)
    return;
  if (fabs(fabs(angle) - PI_) < 1e-12) {
    ca = -1;
    sa = 0;
  } else if (fabs(angle - PI_ / 2) < 1e-12) {
    ca = 0;
    sa = 1;
  } else if (fabs(angle + PI_ / 2) < 1e-12) {
    ca = 0;
    sa = -1;
  } else {
    ca = M_COS(angle);
    sa = M_SIN(angle);
  }
  for (i = 0; i < np; i++) {
    double *p = c[i], x = p[0], xp = p[1], y = p[2], yp = p[3];
    p[0] = x * ca + y * sa;
    p[2] = -x * sa + y * ca;
    p[1] = xp * ca + yp * sa;
    p[3] = -xp * sa + yp * ca;
  }
}

/* ---- synchrotron radiation ------------------------------------------------ */
#include "../elegant_b200/csrc/b2e_rng.h"
/* ISR deviates: the counter-based generator the engine uses, addressed by
 * (seed; particle ID, pass, element, slice, step); the reference's own serial
 * gauss_rn_lim(0, 1, srGaussianLimit, random_2) draws from the same
 * truncated Gaussian in a different sequence */
static uint64_t g_isr_seed = 0;
static double g_sr_limit = 3.0;
void b2e_oracle_set_isr(uint64_t seed, double limit) {
  g_isr_seed = seed;
  g_sr_limit = limit;
}
#define EPS0_MKS (1 / ((4 * PI_ * 1e-7) * C_MKS * C_MKS))
#define POW3(x) ((x) * (x) * (x))
#define POW5(x) (((x) * (x)) * ((x) * (x)) * (x))

/* ---- KQUAD / KSEXT ---------------------------------------------------------- */
static int m2s(double *xp, double *yp, double qx, double qy, double dp) {
  double d = SQR(1 + dp) - SQR(qx) - SQR(qy);
  if (d <= 0)
    return 0;
  d = sqrt(d);
  *xp = qx / d;
  *yp = qy / d;
  return 1;
}

static void canonical_kick(double *qx, double *qy, double *dqx, double *dqy, double x, double y, long order,
                           double KnL, int skew) {
  /* apply_canonical_multipole_kicks with expansion coefficients of (x+iy)^n/n! */
  double xpow[4], ypow[4], coef[4], sFx = 0, sFy = 0, fi = 1, fni;
  long i, m;
  xpow[0] = ypow[0] = 1;
  for (i = 1; i <= order; i++) {
    xpow[i] = xpow[i - 1] * x;
    ypow[i] = ypow[i - 1] * y;
  }
  for (i = 0; i <= order; i++) {
    fi = 1;
    for (m = 2; m <= i; m++)
      fi *= m;
    fni = 1;
    for (m = 2; m <= order - i; m++)
      fni *= m;
    coef[i] = (((i / 2) & 1) ? -1.0 : 1.0) / (fi * fni);
  }
  for (i = 1; i <= order; i += 2)
    sFx += coef[i] * xpow[order - i] * ypow[i];
  for (i = 0; i <= order; i += 2)
    sFy += coef[i] * xpow[order - i] * ypow[i];
  if (skew) {
    double t = sFx;
    sFx = sFy;
    sFy = t;
    sFx = -sFx;
  }
  *qx -= KnL * sFy;
  *qy += KnL * sFx;
  *dqx -= KnL * sFy;
  *dqy += KnL * sFx;
}

/* quadPartialFringeMatrix (fringe.c:229-271), inFringe = 1:
 * R00 R01 R10 R11 R22 R23 R32 R33 */
static void qf_matrix(double *R, double K1, const double *fi, int part) {
  double J1x, J2x, J3x, J1y, J2y, J3y, K1sqr = SQR(K1), ex, ey;
  if (part == 1) {
    J1x = 1 * (K1 * fi[1] - 2 * K1sqr * fi[3] / 3. - K1sqr * fi[0] * fi[2] / 2);
    J2x = 1 * K1 * fi[2];
    J3x = 1 * K1sqr * (fi[2] + fi[4] + fi[0] * fi[1]);
    K1 = -K1;
    J1y = 1 * (K1 * fi[1] - 2 * K1sqr * fi[3] / 3. - K1sqr * fi[0] * fi[2] / 2);
  } else {
    J1x = 1 * (K1 * fi[1] + K1sqr * fi[0] * fi[2] / 2);
    J2x = 1 * K1 * fi[2];
    J3x = 1 * K1sqr * (fi[4] - fi[0] * fi[1]);
    K1 = -K1;
    J1y = 1 * (K1 * fi[1] + K1sqr * fi[0] * fi[2] / 2);
  }
  J2y = -J2x;
  J3y = J3x;
  R[0] = ex = exp(J1x);
  R[1] = J2x / ex;
  R[2] = ex * J3x;
  R[3] = (1 + J2x * J3x) / ex;
  R[4] = ey = exp(J1y);
  R[5] = J2y / ey;
  R[6] = ey * J3y;
  R[7] = (1 + J2y * J3y) / ey;
}

/* quadFringe (fringe.c:24-175) for higherOrder 1 and 2, forward tracking */
static void qf_track(double **c, long np, double K1, const double *fiM, const double *fiP, int inFringe,
                     int higherOrder, int linearFlag, double nlf) {
  double M1[8], M2[8], *A = M1, *B = M2, t;
  long ip;
  if (linearFlag) {
    qf_matrix(M1, K1, fiM, 1);
    qf_matrix(M2, K1, fiP, 2);
    if (inFringe == -1) {
      t = M1[0], M1[0] = M1[3], M1[3] = t;
      t = M1[4], M1[4] = M1[7], M1[7] = t;
      t = M2[0], M2[0] = M2[3], M2[3] = t;
      t = M2[4], M2[4] = M2[7], M2[7] = t;
      A = M2;
      B = M1;
    }
  }
  for (ip = 0; ip < np; ip++) {
    double *v = c[ip], delta = v[5], xp = v[1], yp = v[3], denom, x, px, y, py, a;
    double dx = 0, dpx = 0, dy = 0, dpy = 0, ds = 0;
    denom = sqrt(1 + SQR(xp) + SQR(yp));
    v[1] = (1 + delta) * xp / denom;
    v[3] = (1 + delta) * yp / denom;
    if (linearFlag) {
      x = A[0] * v[0] + A[1] * v[1];
      px = A[2] * v[0] + A[3] * v[1];
      y = A[4] * v[2] + A[5] * v[3];
      py = A[6] * v[2] + A[7] * v[3];
    } else {
      x = v[0], px = v[1], y = v[2], py = v[3];
    }
    a = -inFringe * K1 / (12 * (1 + delta));
    if (higherOrder > 1) {
      double x2 = x * x, x3 = x2 * x, y2 = y * y, y3 = y2 * y;
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
    if (linearFlag) {
      v[0] = B[0] * x + B[1] * px;
      v[1] = B[2] * x + B[3] * px;
      v[2] = B[4] * y + B[5] * py;
      v[3] = B[6] * y + B[7] * py;
    } else {
      v[0] = x, v[1] = px, v[2] = y, v[3] = py;
    }
    v[4] -= nlf * ds;
    px = v[1];
    py = v[3];
    if ((denom = SQR(1 + delta) - SQR(px) - SQR(py)) > 0) {
      denom = sqrt(denom);
      v[1] = px / denom;
      v[3] = py / denom;
    } else
      v[1] = v[3] = DBL_MAX;
  }
}

static long kmult_track(double **c, long np, const b2e_element *e, double Po, double z_start, const MaxAmp *ma,
                        int pass, int elem) {
  const double *p = e->p;
  double KnL[3] = {0, 0, 0}, df[8], kf[8], drift, dx, dy, dz, tilt, rad_coef = 0, isr_coef, xkick, ykick, lEnd = 0;
  int doEndDrift = 0;
  long order[3] = {0, 0, 0}, nSlices, n_kicks, ip, itop;
  int skew[3] = {0, 0, 0}, integ, nSub, radblock;
  MultAp ap;
  double dzLoss = 0;
  drift = p[B2E_KMULT_L];
  if (e->type == B2E_KQUAD && p[B2E_KMULT_LEFFECTIVE] > 0) {
    /* multipole.c:766-770: the effective length, exact end drifts of the rest */
    drift = p[B2E_KMULT_LEFFECTIVE];
    lEnd = (p[B2E_KMULT_L] - drift) / 2;
    doEndDrift = 1;
  }
  integ = (int)p[B2E_KMULT_INTEGRATION_ORDER];
  nSlices = (long)p[B2E_KMULT_N_SLICES];
  n_kicks = (long)p[B2E_KMULT_N_KICKS];
  dx = p[B2E_KMULT_DX];
  dy = p[B2E_KMULT_DY];
  dz = p[B2E_KMULT_DZ];
  tilt = p[B2E_KMULT_TILT];
  /* multipole.c:771-773, :834-837: with a bore radius, the strength from the pole-tip field */
  if (e->type == B2E_KQUAD) {
    order[0] = 1;
    if (p[B2E_KMULT_BORE])
      KnL[0] = p[B2E_KMULT_B] / p[B2E_KMULT_BORE] * (E_MKS / (ME_MKS * C_MKS * Po)) * drift * (1 + p[B2E_KMULT_FSE]);
    else
      KnL[0] = p[B2E_KMULT_K] * drift * (1 + p[B2E_KMULT_FSE]);
  } else {
    order[0] = 2;
    if (p[B2E_KMULT_BORE])
      KnL[0] = 2 * p[B2E_KMULT_B] / SQR(p[B2E_KMULT_BORE]) * (E_MKS / (ME_MKS * C_MKS * Po)) * drift *
               (1 + p[B2E_KMULT_FSE]);
    else
      KnL[0] = p[B2E_KMULT_K] * drift * (1 + p[B2E_KMULT_FSE]);
    if (p[B2E_KMULT_K1_OF_KSEXT]) {
      KnL[1] = p[B2E_KMULT_K1_OF_KSEXT] * drift;
      order[1] = 1;
    }
    if (p[B2E_KMULT_J1_OF_KSEXT]) {
      KnL[2] = p[B2E_KMULT_J1_OF_KSEXT] * drift;
      order[2] = 1;
      skew[2] = 1;
    }
  }
  nSub = fractions(integ, df, kf);
  if (n_kicks > 0) {
    if (integ > 2) {
      if ((nSlices = (long)ceil(n_kicks / (1.0 * integ))) < 1)
        nSlices = 1;
    } else
      nSlices = n_kicks;
  }
  /* steering, per slice (multipole.c:785-786, :1190-1191) */
  xkick = p[B2E_KMULT_HKICK] * p[B2E_KMULT_HCALIBRATION] / nSlices;
  ykick = p[B2E_KMULT_VKICK] * p[B2E_KMULT_VCALIBRATION] / nSlices;
  setup_mult_ap(&ap, -tilt, ma);
  /* entrance misalignment, mode 0 face 1 */
  if (dx || dy || dz)
    offset_beam(c, np, dx, dy, dz);
  if (tilt)
    rotate_beam(c, np, tilt);
  if (doEndDrift)
    exact_drift(c, np, lEnd);
  /* KQUAD entrance fringe on every particle (multipole.c:1031-1037) */
  if (e->type == B2E_KQUAD && p[B2E_KMULT_EDGE1_EFFECTS] > 0)
    qf_track(c, np, p[B2E_KMULT_K], p + B2E_KMULT_I0M, p + B2E_KMULT_I0P, -1, (int)p[B2E_KMULT_EDGE1_EFFECTS],
             (int)p[B2E_KMULT_EDGE1_LINEAR], p[B2E_KMULT_EDGE1_NONLINEAR_FACTOR]);
  /* multipole.c:788-800 */
  if (p[B2E_KMULT_SYNCH_RAD])
    rad_coef = SQR(E_MKS) * POW3(Po) / (6 * PI_ * EPS0_MKS * SQR(C_MKS) * ME_MKS);
  isr_coef = RE_MKS * sqrt(55.0 / (24 * sqrt(3)) * POW5(Po) * 137.0359895);
  if (!p[B2E_KMULT_ISR])
    isr_coef *= -1;
  if (p[B2E_KMULT_L] < 1e-6 && (p[B2E_KMULT_ISR] || p[B2E_KMULT_SYNCH_RAD]))
    rad_coef = isr_coef = 0;
  radblock = rad_coef || isr_coef;
  itop = np - 1;
  for (ip = 0; ip <= itop; ip++) {
    double *coord = c[ip], x, xp, y, yp, s, dpv, qx, qy, denom, dr, beta0, pp;
    long i_kick, step, io;
    int lost = 0;
    dr = drift / nSlices;
    pp = Po * (1 + coord[5]);
    beta0 = pp / sqrt(SQR(pp) + 1);
    x = coord[0];
    xp = coord[1];
    y = coord[2];
    yp = coord[3];
    s = 0;
    dpv = coord[5];
    if (isnan(x) || isnan(xp) || isnan(y) || isnan(yp))
      lost = 1;
    else if (fabs(x) > coord_limit || fabs(y) > coord_limit || fabs(xp) > slope_limit || fabs(yp) > slope_limit)
      lost = 1;
    if (!lost) {
      denom = sqrt(1 + SQR(xp) + SQR(yp));
      qx = (1 + dpv) * xp / denom;
      qy = (1 + dpv) * yp / denom;
      if (!m2s(&xp, &yp, qx, qy, dpv))
        lost = 1;
    }
    if (!lost) {
      dzLoss = 0;
      for (i_kick = 0; i_kick < nSlices && !lost; i_kick++) {
        if (!mult_ap_ok(x + dx, y + dy, &ap)) {
          coord[0] = x;
          coord[2] = y;
          lost = 1;
          break;
        }
        for (step = 0; step < nSub; step++) {
          if (dr) {
            double dsh = dr * df[step];
            x += xp * dsh;
            y += yp * dsh;
            s += dsh * sqrt(1 + SQR(xp) + SQR(yp));
            dzLoss += dsh;
          }
          if (!kf[step])
            break;
          {
            double dqx = 0, dqy = 0;
            for (io = 0; io < 3; io++)
              if (KnL[io])
                canonical_kick(&qx, &qy, &dqx, &dqy, x, y, order[io], KnL[io] / nSlices * kf[step], skew[io]);
            {
              /* steering kicks, not part of delta_qx/delta_qy (multipole.c:1281-1284) */
              double ux = 0, uy = 0;
              if (xkick)
                canonical_kick(&qx, &qy, &ux, &uy, x, y, 0, -xkick * kf[step], 0);
              if (ykick)
                canonical_kick(&qx, &qy, &ux, &uy, x, y, 0, -ykick * kf[step], 1);
            }
            if (!m2s(&xp, &yp, qx, qy, dpv)) {
              lost = 1;
              break;
            }
            if (radblock && dr) {
              /* multipole.c:1320-1349 */
              double deltaFactor, F2, dsFactor, dsISRFactor;
              qx /= (1 + dpv);
              qy /= (1 + dpv);
              deltaFactor = SQR(1 + dpv);
              dqx /= kf[step];
              dqy /= kf[step];
              F2 = SQR(dqx / dr - xkick / dr) + SQR(dqy / dr + ykick / dr);
              dsFactor = sqrt(1 + SQR(xp) + SQR(yp));
              dsISRFactor = dsFactor * dr / (nSub - 1);
              dsFactor *= dr * kf[step];
              if (rad_coef)
                dpv -= rad_coef * deltaFactor * F2 * dsFactor;
              if (isr_coef > 0)
                dpv -= isr_coef * deltaFactor * b2e_isr_pow34(F2) * sqrt(dsISRFactor) *
                       b2e_isr_gauss(g_isr_seed, (int64_t)coord[6], pass, elem, (int)i_kick, (int)step, g_sr_limit);
              qx *= (1 + dpv);
              qy *= (1 + dpv);
              if (!m2s(&xp, &yp, qx, qy, dpv)) {
                lost = 1;
                break;
              }
            }
          }
        }
      }
      if (!lost && !mult_ap_ok(x + dx, y + dy, &ap)) {
        coord[0] = x;
        coord[2] = y;
        lost = 1;
      }
      if (!lost && !m2s(&xp, &yp, qx, qy, dpv))
        lost = 1;
      if (!lost) {
        coord[0] = x;
        coord[1] = xp;
        coord[2] = y;
        coord[3] = yp;
        if (rad_coef) {
          double p1 = Po * (1 + dpv), beta1 = p1 / sqrt(SQR(p1) + 1);
          coord[4] = beta1 * (coord[4] / beta0 + 2 * s / (beta0 + beta1));
        } else
          coord[4] += s;
        coord[5] = dpv;
        if (isnan(x) || isnan(xp) || isnan(y) || isnan(yp) || fabs(x) > coord_limit || fabs(y) > coord_limit ||
            fabs(xp) > slope_limit || fabs(yp) > slope_limit)
          lost = 1;
      }
    }
    if (lost) {
      swap_rows(c[ip], c[itop]);
      c[itop][4] = z_start + dzLoss;
      c[itop][5] = Po * (1 + c[itop][5]);
      itop--;
      ip--;
    }
  }
  /* KQUAD exit fringe (multipole.c:1088-1094) and the exit misalignment,
   * face 2, applied to all np rows like the reference */
  if (e->type == B2E_KQUAD && p[B2E_KMULT_EDGE2_EFFECTS] > 0)
    qf_track(c, np, p[B2E_KMULT_K], p + B2E_KMULT_I0M, p + B2E_KMULT_I0P, 1, (int)p[B2E_KMULT_EDGE2_EFFECTS],
             (int)p[B2E_KMULT_EDGE2_LINEAR], p[B2E_KMULT_EDGE2_NONLINEAR_FACTOR]);
  if (doEndDrift)
    exact_drift(c, np, lEnd);
  if (dx || dy || dz || tilt) {
    if (tilt)
      rotate_beam(c, np, -tilt);
    if (dx || dy || dz)
      offset_beam(c, np, -dx, -dy, -dz);
  }
  return itop + 1;
}

/* ---- CSBEND ------------------------------------------------------------- */
/* radiation of one bend for csbend_integrate: rad_coef, isrConstant, and
 * the address of the particle's ISR deviates */
typedef struct {
  double rad_coef, isr;
  int64_t id;
  int pass, elem;
  int fields;                /* K1/K2/XKICK/YKICK present: the expansion below is used */
  int skew;                  /* YKICK: Fx_xy[0][0] = c0, every (i, j) summed (hasSkew) */
  double Fx_xy[5][5], Fy_xy[5][5];
} BendRad;

/* computeCSBENDFieldCoefficients (csbend.c:186-663) for normal quadrupole and
 * sextupole terms (b[1] = K1 rho0, b[2] = K2 rho0, b[0] the dipole
 * correction), expansion order 4, the entries the field sums read. */
static void bend_field_table(BendRad *br, const double *b_in, double h1, int nonlinear) {
  double h[4], b[4];
  int i;
  memset(br->Fx_xy, 0, sizeof(br->Fx_xy));
  memset(br->Fy_xy, 0, sizeof(br->Fy_xy));
  h[0] = 1;
  for (i = 1; i < 4; i++)
    h[i] = h[i - 1] * h1;
  br->Fy_xy[0][0] = 1 - b_in[0];
  for (i = 0; i < 4; i++)
    b[i] = b_in[i + 1]; /* b[0] the quadrupole term from here on */
  br->Fx_xy[0][1] = b[0];
  br->Fy_xy[1][0] = b[0];
  if (!nonlinear)
    return;
  br->Fy_xy[0][2] = -(h[1] * b[0]) / 2 - b[1] / 2;
  br->Fy_xy[0][4] = (h[3] * b[0]) / 24 - (h[2] * b[1]) / 24 + (h[1] * b[2]) / 12 + b[3] / 24;
  br->Fy_xy[1][2] = (h[2] * b[0]) / 2 - (h[1] * b[1]) / 2 - b[2] / 2;
  br->Fy_xy[2][0] = b[1] / 2;
  br->Fy_xy[2][2] = -(h[3] * b[0]) / 2 + (h[2] * b[1]) / 2 - (h[1] * b[2]) / 4 - b[3] / 4;
  br->Fy_xy[3][0] = b[2] / 6;
  br->Fy_xy[4][0] = b[3] / 24;
  br->Fx_xy[1][1] = b[1];
  br->Fx_xy[0][3] = (h[2] * b[0]) / 6 - (h[1] * b[1]) / 6 - b[2] / 6;
  br->Fx_xy[1][3] = -(h[3] * b[0]) / 3 + (h[2] * b[1]) / 3 - (h[1] * b[2]) / 6 - b[3] / 6;
  br->Fx_xy[2][1] = b[2] / 2;
  br->Fx_xy[3][1] = b[3] / 6;
}

/* computeCSBENDFields, TURBO_MODE form (csbend.c:101-150), normal terms */
static void bend_fields_at(const BendRad *br, double x, double y, double *Fx, double *Fy) {
  double yp[5], xt = 1, sumFx = 0, sumFy = 0;
  int i, j;
  if (!br || !br->fields) {
    *Fx = 0;
    *Fy = 1;
    return;
  }
  yp[0] = 1;
  for (i = 1; i < 5; i++)
    yp[i] = yp[i - 1] * y;
  if (br->skew) {
    /* csbend.c:124-135: every j */
    for (i = 0; i < 5; i++) {
      for (j = 0; j < 5 - i; j++) {
        sumFx += br->Fx_xy[i][j] * xt * yp[j];
        sumFy += br->Fy_xy[i][j] * xt * yp[j];
      }
      xt *= x;
    }
    *Fx = sumFx;
    *Fy = sumFy;
    return;
  }
  for (i = 0; i < 5; i++) {
    for (j = 1; j < 5 - i; j += 2)
      sumFx += br->Fx_xy[i][j] * xt * yp[j];
    for (j = 0; j < 5 - i; j += 2)
      sumFy += br->Fy_xy[i][j] * xt * yp[j];
    xt *= x;
  }
  *Fx = sumFx;
  *Fy = sumFy;
}

static int csbend_integrate(double *Qf, const double *Qi, double s, long n, double rho0, double rho_actual,
                            const MultAp *ap, int integ, int isr_block, double *dz_lost, const BendRad *br) {
  double df[8], kf[8];
  int nSub = fractions(integ, df, kf), i, j;
  double dist = 0;
  memcpy(Qf, Qi, sizeof(double) * 6);
  s /= n;
  *dz_lost = 0;
  for (i = 0; i < n; i++) {
    if (!mult_ap_ok(Qf[0], Qf[2], ap))
      return 0;
    for (j = 0; j < nSub; j++) {
      double dsh = s * df[j], f, sin_phi, phi, sine, cosi, tang, cos_phi, factor, ds;
      f = SQR(1 + Qf[5]) - SQR(Qf[3]);
      if (f <= 0)
        return 0;
      f = sqrt(f);
      if (fabs(Qf[1] / f) > 1)
        return 0;
      sin_phi = Qf[1] / f;
      phi = M_ASIN(sin_phi);
      sine = M_SIN(dsh / rho0 + phi);
      cosi = M_COS(dsh / rho0 + phi);
      if (cosi == 0)
        return 0;
      tang = sine / cosi;
      cos_phi = M_COS(phi);
      Qf[1] = f * sine;
      factor = (rho0 + Qf[0]) * cos_phi / f * (tang - sin_phi / cos_phi);
      Qf[2] += Qf[3] * factor;
      dist += factor * (1 + Qf[5]);
      *dz_lost += dsh;
      f = cos_phi / cosi;
      Qf[0] = rho0 * (f - 1) + f * Qf[0];
      if (kf[j] == 0)
        break;
      ds = s * kf[j];
      {
        double Fx, Fy;
        bend_fields_at(br, Qf[0], Qf[2], &Fx, &Fy);
        Qf[1] += -ds * (1 + Qf[0] / rho0) * Fy / rho_actual;
        Qf[3] += ds * (1 + Qf[0] / rho0) * Fx / rho_actual;
      if (isr_block) {
        /* csbend.c:1603-1622 */
        double f = (1 + Qf[0] * (1. / rho0)) / sqrt(SQR(1 + Qf[5]) - SQR(Qf[1]) - SQR(Qf[3]));
        double xp = Qf[1] * f, yp = Qf[3] * f;
        double dsFactor = sqrt(SQR(1 + Qf[0] * (1. / rho0)) + SQR(xp) + SQR(yp));
        double F2 = SQR(Fx) + SQR(Fy);
        double deltaFactor = SQR(1 + Qf[5]);
        double dsISR = s / (nSub - 1);
        Qf[1] /= (1 + Qf[5]);
        Qf[3] /= (1 + Qf[5]);
        if (br && br->rad_coef)
          Qf[5] -= br->rad_coef * deltaFactor * F2 * ds * dsFactor;
        if (br && br->isr > 0)
          Qf[5] -= br->isr * deltaFactor * b2e_isr_pow34(F2) * sqrt(dsISR * dsFactor) *
                   b2e_isr_gauss(g_isr_seed, br->id, br->pass, br->elem, i, j, g_sr_limit);
        Qf[1] *= (1 + Qf[5]);
        Qf[3] *= (1 + Qf[5]);
      }
      }
    }
  }
  *dz_lost = n * s;
  if (!mult_ap_ok(Qf[0], Qf[2], ap))
    return 0;
  Qf[4] += dist;
  return 1;
}

/* applySimpleDipoleEdgeKick (csbend.c:5639-5665), EDGE_EFFECTS 3, no kick
 * limit, unexpanded Hamiltonian: the linear edge kick on the canonical
 * momenta */
static void simple_edge_kick(double *xp, double *yp, double x, double y, double delta, double rho, double ea,
                             double psi) {
  double f = (1 + delta) / sqrt(1 + SQR(*xp) + SQR(*yp)), qx = *xp * f, qy = *yp * f, dqx, dqy;
  dqx = M_TAN(ea) / rho * x;
  dqy = -M_TAN(ea - psi / (1 + delta)) / rho * y;
  qx += dqx;
  qy += dqy;
  f = 1 / sqrt(SQR(1 + delta) - SQR(qx) - SQR(qy));
  *xp = qx * f;
  *yp = qy * f;
}

static int same_bend(const b2e_element *a, const b2e_element *b) {
  return a->type == b->type && strncmp(a->name, b->name, sizeof(a->name)) == 0;
}

/* apply_edge_effects (csbend.c:4266-4307): K. L. Brown's second-order edge,
 * used for EDGE_ORDER >= 2; he (H1/H2) is zero here. */
static void edge_order2(double *x, double *xp, double *y, double *yp, double rho, double n, double beta,
                        double psi, long which_edge) {
  double h, tan_beta, tan2_beta, sec_beta, sec2_beta, h2, R21, R43;
  double T111, T133, T211, T441, T331, T221, T233, T243, T431, T432, x0, xp0, y0, yp0;
  h = 1 / rho;
  R21 = h * (tan_beta = M_TAN(beta));
  R43 = -h * M_TAN(beta - psi);
  h2 = SQR(h);
  T111 = which_edge * h / 2 * (tan2_beta = SQR(tan_beta));
  sec_beta = 1. / M_COS(beta);
  sec2_beta = SQR(sec_beta);
  T133 = -which_edge * h / 2 * sec2_beta;
  T211 = which_edge == -1 ? -n * h2 * tan_beta : -h2 * (n + tan2_beta / 2) * tan_beta;
  T441 = -(T331 = T221 = -which_edge * h * tan2_beta);
  T233 = which_edge == -1 ? h2 * (n + .5 + tan2_beta) * tan_beta : h2 * (n - tan2_beta / 2) * tan_beta;
  T243 = which_edge * h * tan2_beta;
  T431 = h2 * (2 * n + (which_edge == 1 ? sec2_beta : 0)) * tan_beta;
  T432 = which_edge * h * sec2_beta;
  x0 = *x;
  xp0 = *xp;
  y0 = *y;
  yp0 = *yp;
  *x = x0 + T111 * SQR(x0) + T133 * SQR(y0);
  *xp = xp0 + R21 * x0 + T211 * SQR(x0) + T221 * x0 * xp0 + T233 * SQR(y0) + T243 * y0 * yp0;
  *y = y0 + T331 * x0 * y0;
  *yp = yp0 + R43 * y0 + T441 * yp0 * x0 + T431 * x0 * y0 + T432 * xp0 * y0;
}

/* computeEtiltCentroidOffset (csbend.c:4723-4769) with the closing
 * rotateCoordinatesForMisalignment(-tilt) (tilt_matrices.c:123-150):
 * exit-face offsets of a bend rolled by ETILT. */
static void etilt_offsets(double *d, double rho0, double angle, double etilt, double tilt) {
  double q1a, q3a, qp1, qp2, qp3, k, tan_alpha, q1b, q2b, dz, x, xp, y, yp, ca, sa, rot;
  int i;
  for (i = 0; i < 6; i++)
    d[i] = 0;
  if (!etilt)
    return;
  etilt *= -1;
  q1a = (1 - M_COS(angle)) * rho0 * (M_COS(etilt) - 1);
  q3a = (1 - M_COS(angle)) * rho0 * M_SIN(etilt);
  qp1 = M_SIN(angle) * M_COS(etilt);
  qp2 = M_COS(angle);
  k = sqrt(SQR(qp1) + SQR(qp2));
  qp3 = M_SIN(angle) * M_SIN(etilt) / k;
  tan_alpha = 1. / M_TAN(angle) / M_COS(etilt);
  q1b = q1a * tan_alpha / (M_TAN(angle) + tan_alpha);
  q2b = -q1b * M_TAN(angle);
  dz = sqrt(SQR(q1b - q1a) + SQR(q2b - 0));
  d[0] = sqrt(SQR(q1b) + SQR(q2b));
  d[1] = M_TAN(atan(tan_alpha) - (PI_ / 2 - angle));
  d[2] = q3a + qp3 * dz;
  d[3] = qp3;
  d[4] = dz * sqrt(1 + SQR(qp3));
  rot = -tilt;
  if (!rot || fabs(fabs(rot) - 2 * PI_) < 1e-12)
    return;
  if (fabs(fabs(rot) - PI_) < 1e-12) {
    ca = -1;
    sa = 0;
  } else if (fabs(rot - PI_ / 2) < 1e-12) {
    ca = 0;
    sa = 1;
  } else if (fabs(rot + PI_ / 2) < 1e-12) {
    ca = 0;
    sa = -1;
  } else {
    ca = M_COS(rot);
    sa = M_SIN(rot);
  }
  x = d[0];
  xp = d[1];
  y = d[2];
  yp = d[3];
  d[0] = x * ca + y * sa;
  d[2] = -x * sa + y * ca;
  d[1] = xp * ca + yp * sa;
  d[3] = -xp * sa + yp * ca;
}

static long csbend_track(double **c, long np, const b2e_element *el, int idx, const b2e_element *all, int n_all,
                         double Po, double z_start, const MaxAmp *ma, int pass) {
  const double *p = el->p;
  double angle, e1, e2, tilt, rho0, rho_actual, fse, h, psi1, psi2, Kg1, Kg2, ttilt, ct, st;
  BendRad br;
  double dxi, dyi, dzi, dxf, dyf, dzf, det[6], n_index, length = p[B2E_BEND_L];
  int edge1 = 0, edge2 = 0, j, integ = (int)p[B2E_BEND_INTEGRATION_ORDER];
  long nSlices = (long)p[B2E_BEND_N_SLICES], ip, itop;
  MultAp ap;
  if (p[B2E_BEND_ANGLE] == 0) {
    exact_drift(c, np, length);
    return np;
  }
  /* determine_bend_flags (bend_matrix.c:1342-1391) */
  {
    int pre = 0, post = 0;
    for (j = idx - 1; j >= 0; j--) {
      if (same_bend(&all[j], el)) {
        pre = 1;
        break;
      }
      if (all[j].type != B2E_MARK)
        break;
    }
    for (j = idx + 1; j < n_all; j++) {
      if (same_bend(&all[j], el)) {
        post = 1;
        break;
      }
      if (all[j].type != B2E_MARK)
        break;
    }
    edge1 = p[B2E_BEND_EDGE1_EFFECTS] && !pre;
    edge2 = p[B2E_BEND_EDGE2_EFFECTS] && !post;
  }
  rho0 = length / p[B2E_BEND_ANGLE];
  if (p[B2E_BEND_ANGLE] < 0) {
    angle = -p[B2E_BEND_ANGLE];
    e1 = -p[B2E_BEND_E1];
    e2 = -p[B2E_BEND_E2];
    tilt = p[B2E_BEND_TILT] + PI_;
    rho0 = length / angle;
  } else {
    angle = p[B2E_BEND_ANGLE];
    e1 = p[B2E_BEND_E1];
    e2 = p[B2E_BEND_E2];
    tilt = p[B2E_BEND_TILT];
    rho0 = length / angle;
  }
  setup_mult_ap(&ap, -tilt, ma);
  fse = p[B2E_BEND_FSE] + 0.0;
  h = 1 / rho0;
  /* n = -b[1]/h with b[1] = K1*rho0, sign-flipped for a negative angle (csbend.c:825, :879-882, :929) */
  n_index = p[B2E_BEND_K1] * (length / p[B2E_BEND_ANGLE]);
  n_index *= (1 + p[B2E_BEND_FSE] + 0) / (1 + p[B2E_BEND_FSE] + 0);
  if (p[B2E_BEND_ANGLE] < 0)
    n_index *= -1;
  n_index = -n_index / h;
  if (fabs(fse + 1) < 1e-12)
    fse = -1 + 1e-12;
  rho_actual = 1 / ((1 + fse) * h);
  Kg1 = Kg2 = 2 * p[B2E_BEND_HGAP] * p[B2E_BEND_FINT] * (rho0 < 0 ? -1 : 1);
  psi1 = Kg1 / fabs(rho_actual) / M_COS(e1) * (1 + SQR(M_SIN(e1)));
  psi2 = Kg2 / fabs(rho_actual) / M_COS(e2) * (1 + SQR(M_SIN(e2)));
  if (length < 0) {
    psi1 *= -1;
    psi2 *= -1;
  }
  ttilt = tilt + p[B2E_BEND_ETILT];
  if (ttilt == 0) {
    ct = 1;
    st = 0;
  } else if (fabs(fabs(ttilt) - PI_) < 1e-12) {
    ct = -1;
    st = 0;
  } else if (fabs(ttilt - PI_ / 2) < 1e-12) {
    ct = 0;
    st = 1;
  } else if (fabs(ttilt + PI_ / 2) < 1e-12) {
    ct = 0;
    st = -1;
  } else {
    ct = M_COS(ttilt);
    st = M_SIN(ttilt);
  }
  dxi = -p[B2E_BEND_DX];
  dzi = p[B2E_BEND_DZ];
  dyi = -p[B2E_BEND_DY];
  dxf = p[B2E_BEND_DX] * M_COS(p[B2E_BEND_ANGLE]) + p[B2E_BEND_DZ] * M_SIN(p[B2E_BEND_ANGLE]);
  dzf = p[B2E_BEND_DX] * M_SIN(p[B2E_BEND_ANGLE]) - p[B2E_BEND_DZ] * M_COS(p[B2E_BEND_ANGLE]);
  dyf = p[B2E_BEND_DY];
  etilt_offsets(det, rho0, angle, p[B2E_BEND_ETILT], tilt);
  /* csbend.c:964-977 */
  br.rad_coef = 0;
  if (p[B2E_BEND_SYNCH_RAD])
    br.rad_coef = SQR(E_MKS) * POW3(Po) * SQR(1 + fse) / (6 * PI_ * EPS0_MKS * SQR(C_MKS) * ME_MKS * SQR(rho0));
  br.isr = RE_MKS * sqrt(55.0 / (24 * sqrt(3)) * POW5(Po) * 137.0359895 / POW3(fabs(rho_actual)));
  if (!p[B2E_BEND_ISR])
    br.isr *= -1;
  br.pass = pass;
  br.elem = idx;
  /* b[] of the field expansion (csbend.c:824-882): K*rho0 with the signed
   * angle, the FSE ratios, odd terms negated with a negative angle */
  br.fields = p[B2E_BEND_K1] != 0 || p[B2E_BEND_K2] != 0 || p[B2E_BEND_XKICK] != 0 || p[B2E_BEND_YKICK] != 0;
  br.skew = p[B2E_BEND_YKICK] != 0;
  if (br.fields) {
    double b[5] = {0, 0, 0, 0, 0}, rs = length / p[B2E_BEND_ANGLE];
    b[1] = p[B2E_BEND_K1] * rs;
    b[2] = p[B2E_BEND_K2] * rs;
    b[1] *= (1 + p[B2E_BEND_FSE] + 0) / (1 + p[B2E_BEND_FSE] + 0);
    b[2] *= (1 + p[B2E_BEND_FSE]) / (1 + p[B2E_BEND_FSE] + 0);
    b[0] = p[B2E_BEND_XKICK] / p[B2E_BEND_ANGLE]; /* csbend.c:867 */
    if (p[B2E_BEND_ANGLE] < 0) {
      b[1] *= -1;
      b[3] *= -1;
    }
    bend_field_table(&br, b, h, p[B2E_BEND_NONLINEAR] != 0);
    br.Fx_xy[0][0] = p[B2E_BEND_YKICK] / p[B2E_BEND_ANGLE]; /* c[0], csbend.c:227, :868 */
  }
  itop = np - 1;
  for (ip = 0; ip <= itop; ip++) {
    double *coord = c[ip], x, y, xp, yp, s, dp, dp0, Qi[6], Qf[6], rho, f, dz_lost;
    int lost;
    br.id = (int64_t)coord[6];
    coord[4] += dzi * sqrt(1 + SQR(coord[1]) + SQR(coord[3]));
    coord[0] = coord[0] + dxi + dzi * coord[1];
    coord[2] = coord[2] + dyi + dzi * coord[3];
    x = coord[0] * ct + coord[2] * st;
    y = -coord[0] * st + coord[2] * ct;
    xp = coord[1] * ct + coord[3] * st;
    yp = -coord[1] * st + coord[3] * ct;
    s = coord[4];
    dp = dp0 = coord[5];
    if (edge1 && p[B2E_BEND_EDGE1_EFFECTS] == 3)
      simple_edge_kick(&xp, &yp, x, y, dp, rho_actual, e1, psi1);
    else if (edge1) {
      rho = (1 + dp) * rho_actual;
      if (p[B2E_BEND_EDGE_ORDER] >= 2)
        edge_order2(&x, &xp, &y, &yp, rho, n_index, e1, psi1 * (1 + dp), -1);
      else {
        xp += M_TAN(e1) / rho * x;
        yp -= M_TAN(e1 - psi1 / (1 + dp)) / rho * y;
      }
    }
    Qi[0] = x;
    Qi[1] = xp;
    Qi[2] = y;
    Qi[3] = yp;
    Qi[4] = 0;
    Qi[5] = dp;
    if (edge1 && e1 != 0 && br.rad_coef) {
      /* csbend.c:1211-1216 */
      double Fx, Fy, dp_prime;
      bend_fields_at(&br, x, y, &Fx, &Fy);
      dp_prime = -br.rad_coef * (SQR(Fx) + SQR(Fy)) * SQR(1 + dp) * sqrt(SQR(1 + x / rho0) + SQR(xp) + SQR(yp));
      Qi[5] -= dp_prime * x * M_TAN(e1);
    }
    f = (1 + Qi[5]) / sqrt(1 + SQR(Qi[1]) + SQR(Qi[3]));
    Qi[1] *= f;
    Qi[3] *= f;
    lost = !csbend_integrate(Qf, Qi, length, nSlices, rho0, rho_actual, &ap, integ, 1, &dz_lost, &br);
    f = 1 / sqrt(SQR(1 + Qf[5]) - SQR(Qf[1]) - SQR(Qf[3]));
    Qf[1] *= f;
    Qf[3] *= f;
    if (lost) {
      /* the reference converts back to lab coordinates (convertFromCSBendCoords)
       * before recording; only the loss bookkeeping is reproduced here */
      memcpy(coord, Qf, sizeof(double) * 4);
      coord[5] = Qf[5];
      swap_rows(c[ip], c[itop]);
      c[itop][4] = z_start + dz_lost;
      c[itop][5] = Po * (1 + c[itop][5]);
      itop--;
      ip--;
      continue;
    }
    if (edge2 && e2 != 0 && br.rad_coef) {
      /* csbend.c:1265-1276 */
      double Fx, Fy, dp_prime;
      bend_fields_at(&br, Qf[0], Qf[2], &Fx, &Fy);
      dp_prime = -br.rad_coef * (SQR(Fx) + SQR(Fy)) * SQR(1 + Qf[5]) *
                 sqrt(SQR(1 + Qf[0] / rho0) + SQR(Qf[1]) + SQR(Qf[3]));
      Qf[5] -= dp_prime * Qf[0] * M_TAN(e2);
    }
    {
      double p0 = Po * (1 + dp0), beta0 = p0 / sqrt(SQR(p0) + 1);
      double p1 = Po * (1 + Qf[5]), beta1 = p1 / sqrt(SQR(p1) + 1);
      s = beta1 * s / beta0 + Qf[4];
    }
    x = Qf[0];
    xp = Qf[1];
    y = Qf[2];
    yp = Qf[3];
    dp = Qf[5];
    if (edge2 && p[B2E_BEND_EDGE2_EFFECTS] == 3)
      simple_edge_kick(&xp, &yp, x, y, dp, rho_actual, e2, psi2);
    else if (edge2) {
      rho = (1 + dp) * rho_actual;
      if (p[B2E_BEND_EDGE_ORDER] >= 2)
        edge_order2(&x, &xp, &y, &yp, rho, n_index, e2, psi2 * (1 + dp), 1);
      else {
        xp += M_TAN(e2) / rho * x;
        yp -= M_TAN(e2 - psi2 / (1 + dp)) / rho * y;
      }
    }
    coord[0] = x * ct - y * st + det[0];
    coord[2] = x * st + y * ct + det[2];
    coord[1] = xp * ct - yp * st + det[1];
    coord[3] = xp * st + yp * ct + det[3];
    coord[4] = s + det[4];
    coord[5] = dp;
    coord[0] += dxf + dzf * coord[1];
    coord[2] += dyf + dzf * coord[3];
    coord[4] += dzf * sqrt(1 + SQR(coord[1]) + SQR(coord[3]));
  }
  return itop + 1;
}

/* ---- MALIGN: offset_beam (do_tracking.c:3243-3300) ----------------------- */
static void malign_track(double **c, long np, const b2e_element *e, double Po) {
  const double *p = e->p;
  const double dx = p[B2E_MALIGN_DX], dxp = p[B2E_MALIGN_DXP], dy = p[B2E_MALIGN_DY], dyp = p[B2E_MALIGN_DYP];
  const double dz = p[B2E_MALIGN_DZ], dt = p[B2E_MALIGN_DT], dp = p[B2E_MALIGN_DP], de = p[B2E_MALIGN_DE];
  const long s_pid = (long)p[B2E_MALIGN_START_PID], e_pid = (long)p[B2E_MALIGN_END_PID];
  long i;
  for (i = np - 1; i >= 0; i--) {
    double *v = c[i], ds, pc, beta, gamma, t;
    if (!(s_pid == -1 && e_pid == -1) && (v[6] < s_pid || v[6] > e_pid))
      continue;
    ds = dz ? dz * sqrt(1 + SQR(v[1]) + SQR(v[3])) : 0;
    v[0] += dx + dz * v[1];
    v[1] += dxp;
    v[2] += dy + dz * v[3];
    v[3] += dyp;
    v[4] += ds;
    if (dt || dp || de) {
      pc = Po * (1 + v[5]);
      beta = pc / (gamma = sqrt(1 + pc * pc));
      t = v[4] / (beta * C_MKS) + dt;
      if (dp) {
        v[5] += dp;
        pc = Po * (1 + v[5]);
        beta = pc / sqrt(1 + pc * pc);
      }
      if (de) {
        gamma += de * gamma;
        pc = sqrt(gamma * gamma - 1);
        beta = pc / gamma;
        v[5] = (pc - Po) / Po;
      }
      v[4] = t * beta * C_MKS;
    }
  }
}

/* ---- RFCA: trackRfCavityWithWakes, simple_rfca.c:295-985 --------------------
 * the zero-length kick, drift-kick-drift sections for L > 0 with N_KICKS > 0
 * (:569-700), the matrix method for L > 0 with N_KICKS <= 0 (:823-945), and
 * VOLT = 0 as a plain drift (:380-392); no wakes, Q, change_t, end focus.
 * Fiducial modes of findFiducialTime (:62-257): TMEAN, LIGHT and PMAXIMUM
 * (FIRST ends every serial run, :103-111, and is rejected at load). */
typedef struct {
  int seen;
  double phase_fiducial;
} RfState;

static long rfca_track(double **c, long np, const b2e_element *e, RfState *rs, double Po, double zEnd) {
  const double *p = e->p;
  double omega = (2 * PI_) * p[B2E_RFCA_FREQ];
  double volt = p[B2E_RFCA_VOLT] / (1e6 * ME_MEV * 1);
  double length = p[B2E_RFCA_L], dtLight, phase, t0;
  long ip, itop, nKicks, ik;
  int matrixMethod = 0;
  if (np <= 0)
    return np;
  if (p[B2E_RFCA_VOLT] == 0) {
    if (length)
      for (ip = 0; ip < np; ip++) {
        c[ip][0] += c[ip][1] * length;
        c[ip][2] += c[ip][3] * length;
        c[ip][4] += length * sqrt(1 + SQR(c[ip][1]) + SQR(c[ip][3]));
      }
    return np;
  }
  nKicks = length ? (long)p[B2E_RFCA_N_KICKS] : 1;
  if (nKicks <= 0) {
    matrixMethod = 1;
    nKicks = 1;
  }
  length /= nKicks;
  volt /= nKicks;
  dtLight = length / C_MKS;
  if (!rs->seen) {
    if (p[B2E_RFCA_T_REFERENCE] != -1)
      t0 = p[B2E_RFCA_T_REFERENCE];
    else if (p[B2E_RFCA_FIDUCIAL] == B2E_FIDUCIAL_LIGHT)
      t0 = (zEnd - p[B2E_RFCA_L] + length / 2) / C_MKS;
    else if (p[B2E_RFCA_FIDUCIAL] == B2E_FIDUCIAL_PMAXIMUM) {
      double best = c[0][5], pp;
      long ibest = -1;
      for (ip = 0; ip < np; ip++)
        if (best < c[ip][5]) {
          best = c[ip][5];
          ibest = ip;
        }
      if (ibest < 0)
        return -1; /* "No available particle for RF cavity fiducialization" */
      pp = Po * (1 + c[ibest][5]);
      t0 = (c[ibest][4] + length / 2) / (C_MKS * (pp / sqrt(pp * pp + 1)));
    } else {
      double tsum = 0, error = 0;
      for (ip = 0; ip < np; ip++) {
        double pp = Po * (1 + c[ip][5]);
        double b = (c[ip][4] + length / 2) / (C_MKS * (pp / sqrt(pp * pp + 1)));
        double Y = b + error, sum = tsum + Y;
        error = Y - (sum - tsum);
        tsum = sum;
      }
      t0 = tsum / np;
    }
    rs->phase_fiducial = -omega * t0;
    rs->seen = 1;
  }
  phase = rs->phase_fiducial;
  phase += p[B2E_RFCA_PHASE] * PI_ / 180.0;
  for (ip = 0; ip < np; ip++) {
    c[ip][0] -= p[B2E_RFCA_DX];
    c[ip][2] -= p[B2E_RFCA_DY];
  }
  for (ik = 0; ik < nKicks; ik++) {
    if (!matrixMethod) {
      for (ip = 0; ip < np; ip++) {
        double *coord = c[ip], P, gamma, beta_i, t, dgamma, gamma1, P1, Pz, Pz1, dc4;
        if (coord[5] == -1)
          continue;
        dc4 = length ? length / 2 * sqrt(1 + SQR(coord[1]) + SQR(coord[3])) : 0;
        P = Po * (1 + coord[5]);
        beta_i = P / (gamma = sqrt(SQR(P) + 1));
        t = (coord[4] + dc4) / (C_MKS * beta_i) - 0;
        dgamma = volt * M_SIN(omega * (t - 0 - ik * dtLight) + phase) * 1;
        if (length) {
          coord[0] += coord[1] * length / 2;
          coord[2] += coord[3] * length / 2;
          coord[4] += length / 2 * sqrt(1 + SQR(coord[1]) + SQR(coord[3]));
        }
        /* add_to_particle_energy */
        P = Po * (1 + coord[5]);
        gamma1 = (gamma = sqrt(P * P + 1)) + dgamma;
        if (gamma1 <= 1)
          gamma1 = 1 + 1e-7;
        P1 = sqrt(gamma1 * gamma1 - 1);
        coord[5] = (P1 - Po) / Po;
        coord[4] = t * C_MKS * P1 / gamma1;
        Pz = P / sqrt(1 + SQR(coord[1]) + SQR(coord[3]));
        Pz1 = sqrt(Pz * Pz + gamma1 * gamma1 - gamma * gamma);
        coord[1] *= Pz / Pz1;
        coord[3] *= Pz / Pz1;
        if ((gamma1 = gamma + dgamma) <= 1)
          coord[5] = -1;
      }
      if (length)
        for (ip = 0; ip < np; ip++) {
          c[ip][0] += c[ip][1] * length / 2;
          c[ip][2] += c[ip][3] * length / 2;
          c[ip][4] += length / 2 * sqrt(1 + SQR(c[ip][1]) + SQR(c[ip][3]));
        }
    } else {
      for (ip = 0; ip < np; ip++) {
        double *coord = c[ip], P, gamma, beta_i, t, dgamma, dP, ds1, sin_phase, R11 = 1, R21 = 0, R12, R22, x, xp;
        P = Po * (1 + coord[5]);
        beta_i = P / (gamma = sqrt(SQR(P) + 1));
        ds1 = length / 2 * sqrt(1 + SQR(coord[1]) + SQR(coord[3]));
        t = (coord[4] + ds1) / (C_MKS * beta_i) - 0;
        sin_phase = M_SIN(omega * (t - 0 - ik * dtLight) + phase);
        dgamma = (volt * 1) * sin_phase;
        dP = sqrt(SQR(gamma + dgamma) - 1) - P;
        R22 = 1 / (1 + dP / P);
        if (fabs(dP / P) > 1e-14)
          R12 = length * (P / dP * M_LOG(1 + dP / P));
        else
          R12 = length;
        coord[4] += ds1;
        x = coord[0];
        xp = coord[1];
        coord[0] = x * R11 + xp * R12;
        coord[1] = x * R21 + xp * R22;
        x = coord[2];
        xp = coord[3];
        coord[2] = x * R11 + xp * R12;
        coord[3] = x * R21 + xp * R22;
        coord[4] += length / 2 * sqrt(1 + SQR(coord[1]) + SQR(coord[3]));
        coord[5] = (P + dP - Po) / Po;
        if ((gamma += dgamma) <= 1)
          coord[5] = -1;
        coord[4] = (P + dP) / gamma * coord[4] / beta_i;
      }
    }
  }
  itop = np - 1;
  for (ip = 0; ip < np; ip++) {
    c[ip][0] += p[B2E_RFCA_DX];
    c[ip][2] += p[B2E_RFCA_DY];
  }
  /* removeInvalidParticles */
  for (ip = 0; ip <= itop; ip++) {
    double *part = c[ip];
    int ic, out = 0;
    for (ic = 0; ic < 6; ic++)
      if (isnan(part[ic]))
        out = 1;
    if (part[5] <= -1)
      out = 1;
    if (out) {
      swap_rows(c[ip], c[itop]);
      c[itop][5] = Po * (1 + c[itop][5]);
      itop--;
      ip--;
    }
  }
  return itop + 1;
}

/* ---- CSR: CSRCSBEND and CSRDRIFT (mode 0 and Stupakov) -------------------- */
#ifdef B2E_ORACLE_LIBM
#define M_POW13(x) pow(x, 1. / 3.)
#else
#define M_POW13(x) b2e_pow13(x)
#endif
#include "../elegant_b200/csrc/b2e_sg.h"
#include "../elegant_b200/csrc/b2e_roots.h"
#include "../elegant_b200/csrc/b2e_fft.h"

/* the reference's file-static CSR state (csbend.h:27-63, csbend.c:1932) */
typedef struct {
  int valid, bins;
  double *dGamma, dctBin, s0, ds0, zLast, z0;
  double accumulatedAngle;
  double macroParticleCharge;
  double *wakes; /* per-kick dGamma log for the tests */
  long n_wakes, cap_wakes;
  /* what the last dipole leaves for a Stupakov CSRDRIFT (csbend.c:2991-3003) */
  double rho, bendingAngle, GSConstant, binRangeFactor;
  long sgHalf, sgOrder, sgdHalf, sgdOrder;
  int trapz;
  int lastMode;       /* 0 none yet, 1 mode 0, 2 Stupakov (csbend.c:3243-3264) */
  double phiLast;     /* SolveForPhiStupakov's static start value (csbend.c:4177) */
  double lowCut0, lowCut1, highCut0, highCut1; /* csrWake's filter cutoffs (csbend.c:2272-2276) */
  int clip;
  double revolutionLength;
} CsrWake;

/* applyLHPassFilters (csbend.c:4611-4703) with the transform of b2e_fft.h;
 * returns the number of bins clipped */
static long lh_pass_filters(double *hist, long bins, double startHP, double endHP, double startLP, double endLP,
                            int clip) {
  double *ri = malloc(sizeof(double) * (bins + 2)), *c = malloc(sizeof(double) * bins);
  double *s = malloc(sizeof(double) * bins), sum = 0, sum2, factor;
  long i, nz = 0, freq = bins / 2 + 1;
  for (i = 0; i < bins; i++)
    b2e_dft_twiddle(bins, i, &c[i], &s[i]);
  for (i = 0; i < freq; i++)
    b2e_rdft_pair(hist, bins, i, c, s, &ri[2 * i], &ri[2 * i + 1]);
  b2e_lh_ramps(ri, freq, startHP, endHP, startLP, endLP);
  for (i = 0; i < bins; i++)
    sum += hist[i];
  for (i = 0; i < bins; i++)
    hist[i] = b2e_rdft_sample(ri, bins, i, c, s);
  if (clip) {
    /* correctDistribution (csbend.c:4705-4721) */
    for (i = 0, sum2 = 0; i < bins; i++) {
      if (hist[i] < 0) {
        nz++;
        hist[i] = 0;
      }
      sum2 += hist[i];
    }
    if (sum2) {
      factor = sum / sum2;
      for (i = 0; i < bins; i++)
        hist[i] *= factor;
    }
  }
  free(ri);
  free(c);
  free(s);
  return nz;
}

/* binParticleCoordinate (csbend.c:3047-3113) on column `ic` of rows c[0..np) */
static long bin_coordinate(double *hist, long bins, double *lower, double *upper, double *dct, double factor,
                           double **c, long np, int ic) {
  long ip, ib, nb = 0;
  *upper = -(*lower = DBL_MAX);
  for (ip = 0; ip < np; ip++) {
    double v = c[ip][ic];
    if (v < *lower)
      *lower = v;
    if (v > *upper)
      *upper = v;
  }
  if (factor > 1) {
    double center = (*lower + *upper) / 2, range = (*upper - *lower) * factor;
    *lower = center - range / 2;
    *upper = center + range / 2;
  }
  *dct = (*upper - *lower) / bins;
  for (ib = 0; ib < bins; ib++)
    hist[ib] = 0;
  for (ip = 0; ip < np; ip++) {
    ib = (long)((c[ip][ic] - *lower) / (*dct));
    if (ib < 0 || ib > bins - 1)
      continue;
    hist[ib] += 1;
    nb++;
  }
  return nb;
}

static long csrcsbend_track(double **c, long np, const b2e_element *el, int idx, const b2e_element *all, int n_all,
                            double Po, double z_start, double z_end, const MaxAmp *ma, CsrWake *cw) {
  const double *p = el->p;
  const double length = p[B2E_BEND_L];
  long nBins = (long)p[B2E_BEND_BINS], nSlices = (long)p[B2E_BEND_N_SLICES], ip, itop, kick, iBin;
  int integ = (int)p[B2E_BEND_INTEGRATION_ORDER], edge1, edge2, j;
  long sgHalf = (long)p[B2E_BEND_SG_HALFWIDTH], sgOrder = (long)p[B2E_BEND_SG_ORDER];
  long sgdHalf = (long)p[B2E_BEND_SGDERIV_HALFWIDTH], sgdOrder = (long)p[B2E_BEND_SGDERIV_ORDER];
  double angle, e1, e2, tilt, rho0, rho_actual, fse, h, psi1, psi2, Kg, ttilt, ct, st;
  double dxi, dyi, dzi, dxf, dyf, dzf, det[6], n_index, CSRConstant, phiBend, ctLower = 0, ctUpper = 0, dct = 0;
  double brf = p[B2E_BEND_BIN_RANGE_FACTOR] < 1.1 ? 1.1 : p[B2E_BEND_BIN_RANGE_FACTOR];
  double *beta0, *ctHist, *ctHistDeriv, *denom, *T1, *T2;
  int more_than_one = np > 1, same_pre = 0;
  MultAp ap;
  long nBinned = 0;
  if (p[B2E_BEND_ANGLE] == 0) {
    exact_drift(c, np, length);
    return np;
  }
  /* edge flags and SAME_BEND_PRECEDES (determine_bend_flags) */
  {
    int pre = 0, post = 0;
    for (j = idx - 1; j >= 0; j--) {
      if (same_bend(&all[j], el)) {
        pre = 1;
        break;
      }
      if (all[j].type != B2E_MARK)
        break;
    }
    for (j = idx + 1; j < n_all; j++) {
      if (same_bend(&all[j], el)) {
        post = 1;
        break;
      }
      if (all[j].type != B2E_MARK)
        break;
    }
    edge1 = p[B2E_BEND_EDGE1_EFFECTS] && !pre;
    edge2 = p[B2E_BEND_EDGE2_EFFECTS] && !post;
    same_pre = pre;
  }
  if (!same_pre)
    cw->accumulatedAngle = 0;
  cw->valid = 0;
  cw->lastMode = 0; /* reset_driftCSR (csbend.c:3539-3548) */
  if (sgdHalf <= 0)
    sgdHalf = sgHalf;
  if (sgdHalf <= 0)
    sgdHalf = 1;
  if (sgdOrder <= 0)
    sgdOrder = sgOrder;
  if (sgdOrder <= 0)
    sgdOrder = 1;
  rho0 = length / p[B2E_BEND_ANGLE];
  if (p[B2E_BEND_ANGLE] < 0) {
    angle = -p[B2E_BEND_ANGLE];
    e1 = -p[B2E_BEND_E1];
    e2 = -p[B2E_BEND_E2];
    tilt = p[B2E_BEND_TILT] + PI_;
    rho0 = length / angle;
  } else {
    angle = p[B2E_BEND_ANGLE];
    e1 = p[B2E_BEND_E1];
    e2 = p[B2E_BEND_E2];
    tilt = p[B2E_BEND_TILT];
    rho0 = length / angle;
  }
  setup_mult_ap(&ap, -tilt, ma);
  h = 1 / rho0;
  /* n = -b[1]/h with b[1] = K1*rho0, sign-flipped for a negative angle (csbend.c:825, :879-882, :929) */
  n_index = p[B2E_BEND_K1] * (length / p[B2E_BEND_ANGLE]);
  if (p[B2E_BEND_ANGLE] < 0)
    n_index *= -1;
  n_index = -n_index / h;
  fse = p[B2E_BEND_FSE];
  rho_actual = fse > -1 ? 1 / ((1 + fse) * h) : 1e16 / h;
  Kg = 2 * p[B2E_BEND_HGAP] * p[B2E_BEND_FINT];
  psi1 = Kg / rho_actual / M_COS(e1) * (1 + SQR(M_SIN(e1)));
  psi2 = Kg / rho_actual / M_COS(e2) * (1 + SQR(M_SIN(e2)));
  if (length < 0) {
    psi1 *= -1;
    psi2 *= -1;
  }
  ttilt = tilt + p[B2E_BEND_ETILT];
  if (ttilt == 0) {
    ct = 1;
    st = 0;
  } else if (fabs(fabs(ttilt) - PI_) < 1e-12) {
    ct = -1;
    st = 0;
  } else if (fabs(ttilt - PI_ / 2) < 1e-12) {
    ct = 0;
    st = 1;
  } else if (fabs(ttilt + PI_ / 2) < 1e-12) {
    ct = 0;
    st = -1;
  } else {
    ct = M_COS(ttilt);
    st = M_SIN(ttilt);
  }
  dxi = -p[B2E_BEND_DX];
  dzi = p[B2E_BEND_DZ];
  dyi = -p[B2E_BEND_DY];
  dxf = p[B2E_BEND_DX] * M_COS(p[B2E_BEND_ANGLE]) + p[B2E_BEND_DZ] * M_SIN(p[B2E_BEND_ANGLE]);
  dzf = p[B2E_BEND_DX] * M_SIN(p[B2E_BEND_ANGLE]) - p[B2E_BEND_DZ] * M_COS(p[B2E_BEND_ANGLE]);
  dyf = p[B2E_BEND_DY];
  etilt_offsets(det, rho0, angle, p[B2E_BEND_ETILT], tilt);
  beta0 = malloc(sizeof(double) * (np ? np : 1));
  ctHist = calloc(nBins, sizeof(double));
  ctHistDeriv = calloc(nBins, sizeof(double));
  denom = calloc(nBins, sizeof(double));
  T1 = calloc(nBins, sizeof(double));
  T2 = calloc(nBins, sizeof(double));
  free(cw->dGamma);
  cw->dGamma = calloc(nBins, sizeof(double));
  cw->bins = nBins;
  cw->ds0 = length / nSlices;
  cw->zLast = cw->z0 = z_end;
  cw->highCut0 = p[B2E_BEND_HIGH_FREQUENCY_CUTOFF0];
  cw->highCut1 = p[B2E_BEND_HIGH_FREQUENCY_CUTOFF1];
  cw->lowCut0 = p[B2E_BEND_LOW_FREQUENCY_CUTOFF0];
  cw->lowCut1 = p[B2E_BEND_LOW_FREQUENCY_CUTOFF1];
  cw->clip = p[B2E_BEND_CLIP_NEGATIVE_BINS] != 0;
  /* entrance (csbend.c:2286-2377) */
  for (ip = 0; ip < np; ip++) {
    double *x = c[ip], X, Y, XP, YP, p0, rho;
    x[4] += dzi * sqrt(1 + SQR(x[1]) + SQR(x[3]));
    x[0] = x[0] + dxi + dzi * x[1];
    x[2] = x[2] + dyi + dzi * x[3];
    X = x[0] * ct + x[2] * st;
    Y = -x[0] * st + x[2] * ct;
    x[0] = X;
    x[2] = Y;
    XP = x[1] * ct + x[3] * st;
    YP = -x[1] * st + x[3] * ct;
    x[1] = XP;
    x[3] = YP;
    p0 = Po * (1 + x[5]);
    beta0[ip] = p0 / sqrt(p0 * p0 + 1);
    x[4] /= beta0[ip];
    if (edge1) {
      rho = (1 + x[5]) * rho_actual;
      if (p[B2E_BEND_EDGE_ORDER] >= 2)
        edge_order2(&x[0], &x[1], &x[2], &x[3], rho, n_index, e1, psi1 * (1 + x[5]), -1);
      else {
        x[1] += M_TAN(e1) / rho * x[0];
        x[3] -= M_TAN(e1 - psi1 / (1 + x[5])) / rho * x[2];
      }
    }
  }
  CSRConstant = 0;
  if (p[B2E_BEND_CSR] && more_than_one) {
    double eps0 = 1 / ((4 * PI_ * 1e-7) * C_MKS * C_MKS);
    CSRConstant = 2 * cw->macroParticleCharge * E_MKS / M_POW13(3 * rho0 * rho0) / (4 * PI_ * eps0 * ME_MKS * SQR(C_MKS));
  }
  phiBend = cw->accumulatedAngle;
  itop = np - 1;
  for (kick = 0; kick < nSlices; kick++) {
    for (ip = 0; ip <= itop; ip++) {
      double *x = c[ip], Qi[6], Qf[6], f, dz_lost;
      int lost;
      Qi[0] = x[0];
      Qi[1] = x[1];
      Qi[2] = x[2];
      Qi[3] = x[3];
      Qi[4] = 0;
      Qi[5] = x[5];
      f = (1 + Qi[5]) / sqrt(1 + SQR(Qi[1]) + SQR(Qi[3]));
      Qi[1] *= f;
      Qi[3] *= f;
      lost = !csbend_integrate(Qf, Qi, length / nSlices, 1, rho0, rho_actual, &ap, integ, 0, &dz_lost, NULL);
      f = 1 / sqrt(SQR(1 + Qf[5]) - SQR(Qf[1]) - SQR(Qf[3]));
      Qf[1] *= f;
      Qf[3] *= f;
      x[0] = Qf[0];
      x[1] = Qf[1];
      x[2] = Qf[2];
      x[3] = Qf[3];
      x[5] = Qf[5];
      if (lost) {
        /* the reference swaps the rows but not beta0[] (csbend.c:2417-2437),
         * so the row moved into slot ip continues with the lost particle's
         * beta0; kept as is */
        swap_rows(c[ip], c[itop]);
        c[itop][4] = z_start + dz_lost;
        c[itop][5] = Po * (1 + c[itop][5]);
        itop--;
        ip--;
      } else
        x[4] += Qf[4] / beta0[ip];
    }
    np = itop + 1;
    if (more_than_one) {
      long diS, diS4, ib;
      ctLower = ctUpper = dct = 0;
      nBinned = bin_coordinate(ctHist, nBins, &ctLower, &ctUpper, &dct, brf, c, np, 4);
      if (p[B2E_BEND_HIGH_FREQUENCY_CUTOFF0] > 0 || p[B2E_BEND_LOW_FREQUENCY_CUTOFF0] >= 0)
        lh_pass_filters(ctHist, nBins, p[B2E_BEND_LOW_FREQUENCY_CUTOFF0], p[B2E_BEND_LOW_FREQUENCY_CUTOFF1],
                        p[B2E_BEND_HIGH_FREQUENCY_CUTOFF0], p[B2E_BEND_HIGH_FREQUENCY_CUTOFF1],
                        p[B2E_BEND_CLIP_NEGATIVE_BINS] != 0);
      if (sgHalf > 0) {
        double sum = 0, factor;
        b2e_sg_apply_host(ctHist, nBins, sgOrder, sgHalf, sgHalf, 0);
        /* correctDistribution (csbend.c:4705-4721) */
        for (ib = 0; ib < nBins; ib++) {
          if (ctHist[ib] < 0)
            ctHist[ib] = 0;
          sum += ctHist[ib];
        }
        if (sum) {
          factor = 1.0 * nBinned / sum;
          for (ib = 0; ib < nBins; ib++)
            ctHist[ib] *= factor;
        }
      }
      for (ib = 0; ib < nBins; ib++) {
        denom[ib] = M_POW13(dct * ib);
        ctHistDeriv[ib] = (ctHist[ib] /= dct);
      }
      b2e_sg_apply_host(ctHistDeriv, nBins, sgdOrder, sgdHalf, sgdHalf, 1);
      phiBend += angle / nSlices;
      {
        double slip = fabs(rho0 * (phiBend * phiBend * phiBend) / 24.0), slip13 = M_POW13(slip);
        if (p[B2E_BEND_IGF]) {
          /* integrated Green's function (csbend.c:2593-2621), convolveArrays1
           * (:5484-5491) and the wake factor (:2676-2680) */
          double gamma2 = Po * Po + 1, gamma3 = M_POW(gamma2, 3. / 2), frac = 9.0 / 16.0;
          double const1 = 6.0 - M_LOG(27.0 / 4.0), const2, eps0 = 1 / ((4 * PI_ * 1e-7) * C_MKS * C_MKS);
          double *chik = T1, *grnk = T2;
          for (ib = 0; ib < nBins; ib++) {
            double z = ib * dct, xmu = 3.0 * gamma3 * z / (2.0 * rho0), a = sqrt(xmu * xmu + 1.0), b = a + xmu;
            if (xmu < 1e-3)
              chik[ib] = frac * const1 + 0.50 * (xmu * xmu) - (7.0 / 54.0) * ((xmu * xmu) * (xmu * xmu)) +
                         (140.0 / 2187.0) * ((xmu * xmu * xmu) * (xmu * xmu * xmu));
            else
              chik[ib] = frac * (3.0 * (-2.0 * xmu * M_POW(b, 1.0 / 3.0) + M_POW(b, 2.0 / 3.0) + M_POW(b, 4.0 / 3.0)) +
                                 M_LOG(M_POW((1 - M_POW(b, 2.0 / 3.0)) / xmu, 2) /
                                       (1 + M_POW(b, 2.0 / 3.0) + M_POW(b, 4.0 / 3.0))));
          }
          const2 = (16.0 / 27.0) * (E_MKS / (4 * PI_ * eps0)) / (gamma2 * dct);
          grnk[0] = const2 * (chik[1] - chik[0]);
          for (ib = 1; ib < nBins - 1; ib++)
            grnk[ib] = const2 * (chik[ib + 1] - 2.0 * chik[ib] + chik[ib - 1]);
          grnk[nBins - 1] = 0;
          for (ib = 0; ib < nBins; ib++) {
            long ib1;
            double out = 0;
            for (ib1 = ib; ib1 < nBins; ib1++)
              out += ctHist[ib1] * grnk[ib1 - ib];
            cw->dGamma[ib] = out * (-cw->macroParticleCharge / (ME_MKS * SQR(C_MKS)) * length / nSlices);
          }
          diS = diS4 = 0;
        } else {
        diS = (long)(slip / dct);
        diS4 = (long)(4 * slip / dct);
        for (ib = 0; ib < nBins; ib++) {
          double term1 = 0, term2 = 0;
          long count, jb;
          T1[ib] = T2[ib] = 0;
          if (CSRConstant) {
            if (p[B2E_BEND_STEADY_STATE]) {
              if (!p[B2E_BEND_TRAPAZOID_INTEGRATION]) {
                for (jb = ib + 1; jb < nBins; jb++)
                  T1[ib] += ctHistDeriv[jb] / denom[jb - ib];
              } else {
                if ((jb = ib + 1) < nBins)
                  term1 = ctHistDeriv[jb] / denom[jb - ib];
                for (count = 0, jb = ib + 1; jb < nBins; jb++, count++)
                  T1[ib] += (term2 = ctHistDeriv[jb] / denom[jb - ib]);
                if ((ib + 1) < nBins)
                  T1[ib] += 0.3 * SQR(denom[1]) * (2 * ctHistDeriv[ib + 1] + 3 * ctHistDeriv[ib]) / dct;
                if (count > 1)
                  T1[ib] -= (term1 + term2) / 2;
              }
            } else {
              if (!p[B2E_BEND_TRAPAZOID_INTEGRATION]) {
                for (jb = ib + 1; jb <= (ib + diS) && jb < nBins; jb++)
                  T1[ib] += ctHistDeriv[jb] / denom[jb - ib];
              } else {
                if ((jb = ib + 1) < nBins && jb <= (ib + diS))
                  term1 = ctHistDeriv[jb] / denom[jb - ib] / 2;
                for (count = 0, jb = ib + 1; jb <= (ib + diS) && jb < nBins; count++, jb++)
                  T1[ib] += (term2 = ctHistDeriv[jb] / denom[jb - ib]);
                if (diS > 0 && (ib + 1) < nBins)
                  T1[ib] += 0.3 * SQR(denom[1]) * (2 * ctHistDeriv[ib + 1] + 3 * ctHistDeriv[ib]) / dct;
                if (count > 1)
                  T1[ib] -= (term1 + term2) / 2;
              }
              if ((ib + diS) < nBins)
                T2[ib] += ctHist[ib + diS];
              if ((ib + diS4) < nBins)
                T2[ib] -= ctHist[ib + diS4];
            }
            T1[ib] *= CSRConstant * length / nSlices;
            T2[ib] *= -CSRConstant * length / nSlices / slip13;
          }
          cw->dGamma[ib] = T1[ib] + T2[ib];
        }
        }
      }
      if (cw->wakes) {
        if (cw->n_wakes + nBins > cw->cap_wakes) {
          cw->cap_wakes = 2 * (cw->n_wakes + nBins);
          cw->wakes = realloc(cw->wakes, sizeof(double) * cw->cap_wakes);
        }
        memcpy(cw->wakes + cw->n_wakes, cw->dGamma, sizeof(double) * nBins);
        cw->n_wakes += nBins;
      }
      if (CSRConstant) {
        for (ip = 0; ip < np; ip++) {
          double *x = c[ip], f;
          iBin = (long)(f = (x[4] - ctLower) / dct);
          f -= iBin;
          if (iBin >= 0 && iBin < nBins - 1)
            x[5] += ((1 - f) * cw->dGamma[iBin] + f * cw->dGamma[iBin + 1]) / Po * (1 + x[0] / rho0);
        }
      }
    }
  }
  /* exit (csbend.c:2810-2955) */
  if (more_than_one) {
    cw->dctBin = dct;
    ctLower = ctUpper = dct = 0;
    bin_coordinate(ctHist, nBins, &ctLower, &ctUpper, &dct, brf, c, np, 4);
    cw->s0 = ctLower + dzf;
  } else {
    ctLower = ctUpper = dct = 0;
    cw->dctBin = dct;
    cw->s0 = ctLower + dzf;
  }
  itop = np - 1;
  for (ip = 0; ip <= itop; ip++) {
    double *x = c[ip], p1, beta1, X, Y, XP, YP, rho;
    p1 = Po * (1 + x[5]);
    beta1 = p1 / sqrt(SQR(p1) + 1);
    x[4] = x[4] * beta1;
    if (p1 <= 0) {
      swap_rows(c[ip], c[itop]);
      c[itop][5] = Po * (1 + c[itop][5]);
      itop--;
      ip--;
      continue;
    }
    if (edge2) {
      rho = (1 + x[5]) * rho_actual;
      if (p[B2E_BEND_EDGE_ORDER] >= 2)
        edge_order2(&x[0], &x[1], &x[2], &x[3], rho, n_index, e2, psi2 * (1 + x[5]), 1);
      else {
        x[1] += M_TAN(e2) / rho * x[0];
        x[3] -= M_TAN(e2 - psi2 / (1 + x[5])) / rho * x[2];
      }
    }
    X = x[0] * ct - x[2] * st + det[0];
    Y = x[0] * st + x[2] * ct + det[2];
    XP = x[1] * ct - x[3] * st + det[1];
    YP = x[1] * st + x[3] * ct + det[3];
    x[0] = X;
    x[2] = Y;
    x[1] = XP;
    x[3] = YP;
    x[0] += dxf + dzf * x[1];
    x[2] += dyf + dzf * x[3];
    x[4] += dzf * sqrt(1 + SQR(x[1]) + SQR(x[3])) + det[4];
  }
  if (more_than_one) {
    cw->valid = 1;
    cw->rho = rho_actual;
    cw->bendingAngle = same_pre ? fabs(phiBend) : fabs(angle);
    cw->GSConstant = CSRConstant * M_POW13(3 * rho0 * rho0) / 2;
    cw->binRangeFactor = p[B2E_BEND_BIN_RANGE_FACTOR];
    cw->sgHalf = sgHalf;
    cw->sgOrder = sgOrder;
    cw->sgdHalf = sgdHalf;
    cw->sgdOrder = sgdOrder;
    cw->trapz = p[B2E_BEND_TRAPAZOID_INTEGRATION] != 0;
  }
  cw->accumulatedAngle += fabs(angle);
  free(beta0);
  free(ctHist);
  free(ctHistDeriv);
  free(denom);
  free(T1);
  free(T2);
  return itop + 1;
}

/* SolveForPhiStupakov (csbend.c:4161-4202): phi with
 * 24 ds = phi^3 (phi + 4x) / (phi + x); each solve starts from the last one */
static double stup_x, stup_4x;
static double stupakov_fn(double phi) { return phi * phi * phi * (phi + stup_4x) / (phi + stup_x); }

static double stupakov_phi(double x, double ds, double phim, double *phiLast) {
  double phi;
  if (ds < 0)
    return -1;
  if (ds == 0)
    return 0;
  ds *= 24;
  stup_x = x;
  stup_4x = 4 * x;
  if (*phiLast == -1)
    *phiLast = phim / 2;
  if (fabs(ds - stupakov_fn(phim)) < ds / 1e4) {
    *phiLast = phim;
    return phim;
  }
  phi = b2e_zero_newton(stupakov_fn, ds, *phiLast, phim / 1000, 3, ds / 1e4);
  if (phi < 0 || phi > phim || fabs(ds - stupakov_fn(phi)) > ds / 1e4)
    phi = b2e_zero_interp(stupakov_fn, ds, 0, phim * 1.01, phim / 100, ds / 1e4);
  if (phi < 0 || phi > phim)
    return -1;
  *phiLast = phi;
  return phi;
}

/* track_through_driftCSR_Stupakov (csbend.c:3803-4159) without LSC, output
 * files or filters */
static long csrdrift_stupakov(double **c, long np, const b2e_element *el, double Po, double zStart, CsrWake *cw) {
  const double *p = el->p;
  double length = p[B2E_CSRDRIFT_L], dz, dz0, dzFirst, zTravel, x, dsMax, ds, factor;
  double ctLower, ctUpper, dct, *ctHist, *ctHistDeriv, *phiSoln, theta = cw->bendingAngle, rho = cw->rho;
  long nKicks, iKick, ip, iBin, nBins = cw->bins, nBins1 = nBins - 1, nBinned, diBin;
  if (zStart != cw->zLast) {
    length += (dzFirst = zStart - cw->zLast);
    for (ip = 0; ip < np; ip++) {
      double *v = c[ip];
      v[0] -= dzFirst * v[1];
      v[2] -= dzFirst * v[3];
      v[4] -= dzFirst * sqrt(1 + SQR(v[1]) + SQR(v[3]));
    }
    zStart = cw->zLast;
  }
  if (p[B2E_CSRDRIFT_DZ] > 0) {
    if ((nKicks = (long)(length / p[B2E_CSRDRIFT_DZ] + 0.5)) < 1)
      nKicks = 1;
  } else
    nKicks = (long)p[B2E_CSRDRIFT_N_KICKS];
  dz = (dz0 = length / nKicks) / 2;
  zTravel = zStart - cw->z0;
  ctHist = calloc(nBins, sizeof(double));
  ctHistDeriv = calloc(nBins, sizeof(double));
  phiSoln = calloc(nBins, sizeof(double));
  for (iKick = 0; iKick < nKicks; iKick++) {
    if (iKick == 1)
      dz = dz0;
    zTravel += dz;
    x = zTravel / rho;
    dsMax = rho / 24 * M_POW(theta, 3) * (theta + 4 * x) / (theta + x);
    for (ip = 0; ip < np; ip++) {
      double *v = c[ip], pp, beta;
      v[0] += v[1] * dz;
      v[2] += v[3] * dz;
      pp = Po * (1 + v[5]);
      beta = pp / sqrt(pp * pp + 1);
      v[4] = (v[4] + dz * sqrt(1 + SQR(v[1]) + SQR(v[3]))) / beta;
    }
    ctLower = ctUpper = dct = 0;
    nBinned = bin_coordinate(ctHist, nBins, &ctLower, &ctUpper, &dct,
                             cw->binRangeFactor < 1.1 ? 1.1 : cw->binRangeFactor, c, np, 4);
    if (cw->highCut0 > 0 || cw->lowCut0 >= 0)
      lh_pass_filters(ctHist, nBins, cw->lowCut0, cw->lowCut1, cw->highCut0, cw->highCut1, cw->clip);
    if (cw->sgHalf > 0) {
      double sum = 0, f;
      b2e_sg_apply_host(ctHist, nBins, cw->sgOrder, cw->sgHalf, cw->sgHalf, 0);
      for (iBin = 0; iBin < nBins; iBin++) {
        if (ctHist[iBin] < 0)
          ctHist[iBin] = 0;
        sum += ctHist[iBin];
      }
      if (sum) {
        f = 1.0 * nBinned / sum;
        for (iBin = 0; iBin < nBins; iBin++)
          ctHist[iBin] *= f;
      }
    }
    for (iBin = 0; iBin < nBins; iBin++)
      ctHistDeriv[iBin] = (ctHist[iBin] /= dct);
    b2e_sg_apply_host(ctHistDeriv, nBins, cw->sgdOrder, cw->sgdHalf, cw->sgdHalf, 1);
    /* case C */
    for (iBin = 0; iBin < nBins; iBin++) {
      ds = rho / 6 * SQR(theta) * (theta + 3 * x);
      diBin = (long)(ds / dct);
      if (iBin + diBin < nBins)
        cw->dGamma[iBin] = -1 / (theta + 2 * x) * ctHist[iBin + diBin];
      else
        cw->dGamma[iBin] = 0;
    }
    /* case D */
    for (iBin = 0; iBin < nBins; iBin++) {
      phiSoln[iBin] = -1;
      if ((ds = iBin * dct) > dsMax)
        break;
      phiSoln[iBin] = stupakov_phi(x, iBin * dct / rho, theta, &cw->phiLast);
    }
    for (iBin = 0; iBin < nBins; iBin++) {
      long jBin, first = 1, count = 0;
      double term1 = 0, term2 = 0;
      diBin = (long)(dsMax / dct);
      if (iBin + diBin < nBins)
        cw->dGamma[iBin] += ctHist[iBin + diBin] / (theta + 2 * x);
      for (jBin = iBin; jBin < nBins; jBin++) {
        double phi;
        if ((phi = phiSoln[jBin - iBin]) >= 0) {
          if (phi > 0) {
            term2 = ctHistDeriv[jBin] / (phi + 2 * x);
            cw->dGamma[iBin] -= term2;
            if (first) {
              term1 = term2;
              first = 0;
            }
            count++;
          }
        } else
          break;
      }
      if (count > 1 && cw->trapz)
        cw->dGamma[iBin] += (term1 + term2) / 2;
    }
    factor = -4 / rho * cw->GSConstant * dz0;
    for (iBin = 0; iBin < nBins; iBin++)
      cw->dGamma[iBin] *= factor;
    for (ip = 0; ip < np; ip++) {
      double *v = c[ip], f, pp, beta;
      iBin = (long)(f = (v[4] - ctLower) / dct);
      f -= iBin;
      if (iBin >= 0 && iBin < nBins1)
        v[5] += ((1 - f) * cw->dGamma[iBin] + f * cw->dGamma[iBin + 1]) / Po;
      pp = (1 + v[5]) * Po;
      beta = pp / sqrt(pp * pp + 1);
      v[4] = beta * v[4];
    }
  }
  dz = dz0 / 2;
  for (ip = 0; ip < np; ip++) {
    double *v = c[ip];
    v[0] += v[1] * dz;
    v[2] += v[3] * dz;
    v[4] += dz * sqrt(1 + SQR(v[1]) + SQR(v[3]));
  }
  cw->zLast = zStart + length;
  free(ctHist);
  free(ctHistDeriv);
  free(phiSoln);
  return np;
}

static long csrdrift_track(double **c, long np, const b2e_element *el, double Po, double zStart, CsrWake *cw) {
  const double *p = el->p;
  double length = p[B2E_CSRDRIFT_L], dz, dz0, dzFirst, ct0 = 0, factor, dct;
  long nKicks, iKick, ip, nBins1;
  int mode = p[B2E_CSRDRIFT_USE_STUPAKOV] ? 2 : 1;
  if (np <= 1 || !cw->valid || !p[B2E_CSRDRIFT_CSR]) {
    exact_drift(c, np, length);
    return np;
  }
  /* csbend.c:3243-3264 */
  while ((zStart + 1e-12) < cw->zLast && cw->revolutionLength > 0)
    zStart += cw->revolutionLength;
  if (cw->lastMode && cw->lastMode != mode)
    fprintf(stderr, "CSRDRIFT mode changed between dipoles (the reference stops here)\n");
  cw->lastMode = mode;
  if (mode == 2)
    return csrdrift_stupakov(c, np, el, Po, zStart, cw);
  nBins1 = cw->bins - 1;
  dct = cw->dctBin;
  if (p[B2E_CSRDRIFT_DZ] > 0) {
    if ((nKicks = (long)(length / p[B2E_CSRDRIFT_DZ])) < 1)
      nKicks = 1;
  } else
    nKicks = (long)p[B2E_CSRDRIFT_N_KICKS];
  dz = (dz0 = length / nKicks) / 2;
  dzFirst = zStart - cw->zLast;
  for (iKick = 0; iKick < nKicks; iKick++) {
    if (iKick == 1)
      dz = dz0;
    for (ip = 0; ip < np; ip++) {
      double *x = c[ip], pp, beta;
      x[0] += x[1] * dz;
      x[2] += x[3] * dz;
      pp = Po * (1 + x[5]);
      beta = pp / sqrt(pp * pp + 1);
      x[4] = (x[4] + dz * sqrt(1 + SQR(x[1]) + SQR(x[3]))) / beta;
    }
    cw->s0 += dz + dzFirst;
    ct0 = cw->s0;
    factor = (dz0 + dzFirst) / cw->ds0;
    dzFirst = 0;
    for (ip = 0; ip < np; ip++) {
      double *x = c[ip], f, pp, beta;
      long iBin = (long)(f = (x[4] - ct0) / dct);
      f -= iBin;
      if (iBin >= 0 && iBin < nBins1)
        x[5] += ((1 - f) * cw->dGamma[iBin] + f * cw->dGamma[iBin + 1]) / Po * factor;
      pp = (1 + x[5]) * Po;
      beta = pp / sqrt(pp * pp + 1);
      x[4] = beta * x[4];
    }
  }
  dz = dz0 / 2;
  for (ip = 0; ip < np; ip++) {
    double *x = c[ip];
    x[0] += x[1] * dz;
    x[2] += x[3] * dz;
    x[4] += dz * sqrt(1 + SQR(x[1]) + SQR(x[3]));
  }
  cw->zLast = zStart + length;
  cw->s0 += dz;
  return np;
}

/* ---- do_tracking restated ------------------------------------------------ */
/* rows: np x 8 (x, xp, y, yp, s, delta, id, lossPass); lossPass must be -1 on
 * input.  Returns survivors (-1 when an RFCA finds no fiducial particle);
 * rows are left in the reference's array order.
 * wakes (optional): every CSRCSBEND kick's dGamma, in order. */
long b2e_oracle_track_csr(const b2e_element *el, int n_el, double p_central, int n_passes, int default_order,
                          double *rows, long np, double *effort, double *wakes, long wake_cap, long *n_wakes) {
  double **c = malloc(sizeof(double *) * (np ? np : 1));
  long i, nToTrack = np, nLeft;
  int pass, k;
  MaxAmp ma;
  CsrWake cw;
  RfState *rf = calloc(n_el ? n_el : 1, sizeof(RfState));
  /* cavities sharing a nonzero PHASE_REFERENCE use the first one's state
   * (get_phase_reference / set_phase_reference, simple_rfca.c:410-470) */
  int *rf_of = malloc(sizeof(int) * (n_el ? n_el : 1));
  for (k = 0; k < n_el; k++) {
    rf_of[k] = k;
    if (el[k].type == B2E_RFCA && el[k].p[B2E_RFCA_PHASE_REFERENCE] != 0) {
      int j;
      for (j = 0; j < k; j++)
        if (el[j].type == B2E_RFCA && el[j].p[B2E_RFCA_PHASE_REFERENCE] == el[k].p[B2E_RFCA_PHASE_REFERENCE]) {
          rf_of[k] = j;
          break;
        }
    }
  }
  memset(&ma, 0, sizeof(ma));
  memset(&cw, 0, sizeof(cw));
  cw.phiLast = -1;
  for (k = 0; k < n_el; k++)
    if (el[k].type == B2E_DRIF || el[k].type == B2E_EDRIFT || el[k].type == B2E_KQUAD || el[k].type == B2E_KSEXT ||
        el[k].type == B2E_CSBEND || el[k].type == B2E_RFCA || el[k].type == B2E_CSRCSBEND ||
        el[k].type == B2E_CSRDRIFT)
      cw.revolutionLength += el[k].p[0];
  if (wakes) {
    cw.cap_wakes = 1024;
    cw.wakes = malloc(sizeof(double) * cw.cap_wakes);
  }
  for (i = 0; i < np; i++)
    c[i] = rows + i * NPROP;
  *effort = 0;
  for (pass = 0; pass < n_passes; pass++) {
    double z = 0, last_z = 0;
    long start = nToTrack;
    for (k = 0; k < n_el && nToTrack; k++) {
      const b2e_element *e = &el[k];
      const double *p = e->p;
      int no_aperture = (e->type == B2E_MARK || e->type == B2E_CHARGE || e->type == B2E_WATCH);
      double L = 0;
      switch (e->type) {
      case B2E_DRIF:
      case B2E_EDRIFT:
      case B2E_KQUAD:
      case B2E_KSEXT:
      case B2E_CSBEND:
      case B2E_RFCA:
      case B2E_CSRCSBEND:
      case B2E_CSRDRIFT:
        L = p[0];
        break;
      default:
        break;
      }
      last_z = z;
      z += L;
      nLeft = nToTrack;
      if (start) {
        switch (e->type) {
        case B2E_DRIF:
          drift_track(c, nToTrack, L, p[B2E_DRIF_ORDER] ? (int)p[B2E_DRIF_ORDER] : default_order);
          break;
        case B2E_EDRIFT:
          exact_drift(c, nToTrack, L);
          break;
        case B2E_KQUAD:
        case B2E_KSEXT:
          nLeft = kmult_track(c, nToTrack, e, p_central, last_z, &ma, pass, k);
          break;
        case B2E_CSBEND:
          nLeft = csbend_track(c, nToTrack, e, k, el, n_el, p_central, last_z, &ma, pass);
          break;
        case B2E_RFCA:
          nLeft = rfca_track(c, nToTrack, e, &rf[rf_of[k]], p_central, z);
          if (nLeft < 0) {
            nToTrack = -1; /* no fiducial particle (FIDUCIAL=pmaximum): the reference stops */
            goto finish;
          }
          break;
        case B2E_MAXAMP:
          ma.present = 1;
          ma.x_max = p[B2E_MAXAMP_X_MAX];
          ma.y_max = p[B2E_MAXAMP_Y_MAX];
          ma.elliptical = (long)p[B2E_MAXAMP_ELLIPTICAL];
          ma.exponent = (long)p[B2E_MAXAMP_EXPONENT];
          ma.y_exponent = (long)p[B2E_MAXAMP_Y_EXPONENT];
          break;
        case B2E_CHARGE:
          /* do_tracking.c:1324-1360: charge per macro-particle on the first pass */
          if (pass == 0) {
            cw.macroParticleCharge = np ? p[B2E_CHARGE_TOTAL] / np : 0;
            if (p[B2E_CHARGE_PER_PARTICLE])
              cw.macroParticleCharge = p[B2E_CHARGE_PER_PARTICLE];
          }
          break;
        case B2E_CSRCSBEND:
          nLeft = csrcsbend_track(c, nToTrack, e, k, el, n_el, p_central, last_z, z, &ma, &cw);
          break;
        case B2E_CSRDRIFT:
          nLeft = csrdrift_track(c, nToTrack, e, p_central, last_z, &cw);
          break;
        case B2E_MALIGN:
          /* do_tracking.c:1818-1821 */
          if ((long)p[B2E_MALIGN_ON_PASS] == -1 || (long)p[B2E_MALIGN_ON_PASS] == pass)
            malign_track(c, nToTrack, e, p_central);
          break;
        default:
          break;
        }
      }
      if (!no_aperture && ma.present && (ma.x_max || ma.y_max)) {
        if (!ma.elliptical)
          nLeft = limit_amps(c, ma.x_max, ma.y_max, nLeft, z, p_central, e->type == B2E_DRIF);
        else
          nLeft = elimit_amps(c, ma.x_max, ma.y_max, nLeft, z, p_central, e->type == B2E_DRIF, ma.exponent,
                              ma.y_exponent);
      }
      nLeft = limit_amps(c, DBL_MAX, DBL_MAX, nLeft, z, p_central, 0);
      for (i = nLeft; i < nToTrack; i++)
        c[i][7] = pass;
      nToTrack = nLeft;
    }
    *effort += nToTrack;
  }
finish:
  if (n_wakes)
    *n_wakes = cw.n_wakes;
  if (wakes && cw.wakes)
    memcpy(wakes, cw.wakes, sizeof(double) * (cw.n_wakes < wake_cap ? cw.n_wakes : wake_cap));
  free(cw.wakes);
  free(cw.dGamma);
  free(rf);
  free(rf_of);
  free(c);
  return nToTrack;
}

long b2e_oracle_track(const b2e_element *el, int n_el, double p_central, int n_passes, int default_order,
                      double *rows, long np, double *effort) {
  return b2e_oracle_track_csr(el, n_el, p_central, n_passes, default_order, rows, np, effort, NULL, 0, NULL);
}

/* Elementary functions as this build sees them (for the maths tests). */
double b2e_oracle_sin(double x) { return M_SIN(x); }
double b2e_oracle_cos(double x) { return M_COS(x); }
double b2e_oracle_tan(double x) { return M_TAN(x); }
double b2e_oracle_asin(double x) { return M_ASIN(x); }
double b2e_oracle_log(double x) { return M_LOG(x); }
double b2e_oracle_pow(double x, double y) { return M_POW(x, y); }

/* Wake integral of one histogram in bin units (dct = 1) with the CSR
 * constant, length and kick count folded to 1 and no T2 term: the T1 part of
 * the CSRCSBEND kick wake above (csbend.c:2566-2673), for the wake network's
 * data set.  counts are real-valued; their sum plays nBinned. */
void b2e_oracle_wake_t1(const double *counts, long nBins, double slippage_bins, int sgHalf, int sgOrder, int sgdHalf,
                        int sgdOrder, int trapz, int steady, double *T1, double *hist_out, double *deriv_out) {
  double *ctHist = malloc(sizeof(double) * nBins), *ctHistDeriv = malloc(sizeof(double) * nBins),
         *denom = malloc(sizeof(double) * nBins);
  double nBinned = 0, dct = 1;
  long ib, jb, diS;
  if (sgdHalf <= 0)
    sgdHalf = sgHalf;
  if (sgdHalf <= 0)
    sgdHalf = 1;
  if (sgdOrder <= 0)
    sgdOrder = sgOrder;
  if (sgdOrder <= 0)
    sgdOrder = 1;
  for (ib = 0; ib < nBins; ib++) {
    ctHist[ib] = counts[ib];
    nBinned += counts[ib];
  }
  if (sgHalf > 0) {
    double sum = 0, factor;
    b2e_sg_apply_host(ctHist, nBins, sgOrder, sgHalf, sgHalf, 0);
    for (ib = 0; ib < nBins; ib++) {
      if (ctHist[ib] < 0)
        ctHist[ib] = 0;
      sum += ctHist[ib];
    }
    if (sum) {
      factor = 1.0 * nBinned / sum;
      for (ib = 0; ib < nBins; ib++)
        ctHist[ib] *= factor;
    }
  }
  for (ib = 0; ib < nBins; ib++) {
    denom[ib] = M_POW13(dct * ib);
    ctHistDeriv[ib] = (ctHist[ib] /= dct);
  }
  b2e_sg_apply_host(ctHistDeriv, nBins, sgdOrder, sgdHalf, sgdHalf, 1);
  diS = (long)(slippage_bins / dct);
  for (ib = 0; ib < nBins; ib++) {
    double term1 = 0, term2 = 0;
    long count;
    T1[ib] = 0;
    if (steady) {
      if (!trapz) {
        for (jb = ib + 1; jb < nBins; jb++)
          T1[ib] += ctHistDeriv[jb] / denom[jb - ib];
      } else {
        if ((jb = ib + 1) < nBins)
          term1 = ctHistDeriv[jb] / denom[jb - ib];
        for (count = 0, jb = ib + 1; jb < nBins; jb++, count++)
          T1[ib] += (term2 = ctHistDeriv[jb] / denom[jb - ib]);
        if ((ib + 1) < nBins)
          T1[ib] += 0.3 * SQR(denom[1]) * (2 * ctHistDeriv[ib + 1] + 3 * ctHistDeriv[ib]) / dct;
        if (count > 1)
          T1[ib] -= (term1 + term2) / 2;
      }
    } else {
      if (!trapz) {
        for (jb = ib + 1; jb <= (ib + diS) && jb < nBins; jb++)
          T1[ib] += ctHistDeriv[jb] / denom[jb - ib];
      } else {
        if ((jb = ib + 1) < nBins && jb <= (ib + diS))
          term1 = ctHistDeriv[jb] / denom[jb - ib] / 2;
        for (count = 0, jb = ib + 1; jb <= (ib + diS) && jb < nBins; count++, jb++)
          T1[ib] += (term2 = ctHistDeriv[jb] / denom[jb - ib]);
        if (diS > 0 && (ib + 1) < nBins)
          T1[ib] += 0.3 * SQR(denom[1]) * (2 * ctHistDeriv[ib + 1] + 3 * ctHistDeriv[ib]) / dct;
        if (count > 1)
          T1[ib] -= (term1 + term2) / 2;
      }
    }
    T1[ib] *= 1.0;
  }
  for (ib = 0; ib < nBins; ib++) {
    if (hist_out)
      hist_out[ib] = ctHist[ib];
    if (deriv_out)
      deriv_out[ib] = ctHistDeriv[ib];
  }
  free(ctHist);
  free(ctHistDeriv);
  free(denom);
}

/* The project's Savitzky-Golay filter (b2e_sg.h) on one array, in place, for
 * tests against independent implementations; returns 1 on success. */
long b2e_oracle_sg_apply(double *data, long rows, long order, long nLeft, long nRight, long deriv) {
  return b2e_sg_apply_host(data, rows, order, nLeft, nRight, deriv);
}

/* SolveForPhiStupakov restated, for unit tests of the root finders;
 * *phi_last is the carried start value (-1 before the first solve) */
double b2e_oracle_stupakov_phi(double x, double ds, double phim, double *phi_last) {
  return stupakov_phi(x, ds, phim, phi_last);
}

/* applyLHPassFilters restated, for unit tests of the transform */
long b2e_oracle_lh_pass_filters(double *hist, long bins, double startHP, double endHP, double startLP, double endLP,
                                int clip) {
  return lh_pass_filters(hist, bins, startHP, endHP, startLP, endLP, clip);
}

/* Philox4x32-10 of b2e_rng.h, for its known-answer test */
void b2e_oracle_philox(const uint32_t *ctr, const uint32_t *key, uint32_t *out) { b2e_philox4x32(ctr, key, out); }
