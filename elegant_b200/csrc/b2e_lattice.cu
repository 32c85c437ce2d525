/*
 * Lattice compilation on the host (see b2e_lattice.h).
 */
#include <math.h>
#include <string.h>
#include <map>
#include <string>
#include "b2e_lattice.h"
#include "b2e_rng.h"
#include "b2e_math.h"

namespace b2e {

static const double kPI = 3.141592653589793238462643383279502884;
static const double kME_MEV = 0.51099895000; /* electron rest energy, MeV (CODATA 2018) */
static const double kBETA = 1.25992104989487316477; /* 2^(1/3), multipole.c:1119, csbend.c:1431 */
/* CODATA 2018, the values the oracle's reference build uses */
static const double kC_MKS = 2.99792458e8, kE_MKS = 1.602176634e-19, kME_MKS = 9.1093837015e-31;
static const double kRE_MKS = 2.8179403262e-15;

/* the radiation coefficients' common factors, in the reference's expression
 * order (multipole.c:789-790, csbend.c:967-972): epsilon_o = 1/(mu_o c^2),
 * pow3/pow5 as repeated products */
static double eps0_mks() { return 1 / ((4 * kPI * 1e-7) * kC_MKS * kC_MKS); }
static double pow3_host(double x) { return (x * x) * x; }
static double pow5_host(double x) { return ((x * x) * (x * x)) * x; }

/* ISR options that the engine does not follow */
static std::string check_radiation(const double *p, int slot_isr, int slot_isr1, long nSlices) {
  if (p[slot_isr] != 0 && p[slot_isr1] == 0)
    return "ISR=1 with ISR1PART=0 is not supported by this engine";
  if (p[slot_isr] != 0 && nSlices > B2E_ISR_MAX_SLICES)
    return "ISR with more than 256 slices per element is not supported by this engine";
  return "";
}

/* Symplectic integrator step fractions: multipole.c:1140-1182, csbend.c:1453-1488. */
static int integrator_fractions(int order, double *drift, double *kick) {
  static const double d6[8] = {0.39225680523878,     0.5100434119184585, -0.47105338540975655, 0.0687531682525181,
                               0.0687531682525181,   -0.47105338540975655, 0.5100434119184585, 0.39225680523878};
  static const double k6[8] = {0.784513610477560, 0.235573213359357, -1.17767998417887, 1.3151863206839063,
                               -1.17767998417887, 0.235573213359357, 0.784513610477560, 0};
  int j;
  switch (order) {
  case 2:
    drift[0] = drift[1] = 0.5;
    kick[0] = 1.0;
    kick[1] = 0.0;
    return 2;
  case 4:
    drift[0] = 0.5 / (2 - kBETA);
    drift[1] = (1 - kBETA) / (2 - kBETA) / 2;
    drift[2] = (1 - kBETA) / (2 - kBETA) / 2;
    drift[3] = 0.5 / (2 - kBETA);
    kick[0] = 1. / (2 - kBETA);
    kick[1] = -kBETA / (2 - kBETA);
    kick[2] = 1 / (2 - kBETA);
    kick[3] = 0;
    return 4;
  case 6:
    for (j = 0; j < 8; j++) {
      drift[j] = d6[j];
      kick[j] = k6[j];
    }
    return 8;
  default:
    return 0;
  }
}

static double ipow_host(double x, long n) {
  double r = x;
  long i;
  if (n == 0)
    return 1;
  for (i = 1; i < n; i++)
    r *= x;
  return r;
}

/* rotateBeamCoordinatesForMisalignment's special angles (tilt_matrices.c:160-176) */
static void rotation_cs(double angle, double *c, double *s) {
  if (fabs(fabs(angle) - kPI) < 1e-12) {
    *c = -1;
    *s = 0;
  } else if (fabs(angle - kPI / 2) < 1e-12) {
    *c = 0;
    *s = 1;
  } else if (fabs(angle + kPI / 2) < 1e-12) {
    *c = 0;
    *s = -1;
  } else {
    *c = b2e_cos(angle);
    *s = b2e_sin(angle);
  }
}

void element_defaults(int type, double *p) {
  for (int i = 0; i < B2E_MAX_PARAMS; i++)
    p[i] = 0;
  switch (type) {
  case B2E_KQUAD:
  case B2E_KSEXT:
    p[B2E_KMULT_N_SLICES] = 1;          /* track_data.c:1234, :1130 */
    p[B2E_KMULT_INTEGRATION_ORDER] = 4; /* :1253, :1153 */
    p[B2E_KMULT_ISR1PART] = 1;          /* :1257, :1157 */
    p[B2E_KMULT_HCALIBRATION] = 1;      /* :1238, :1138 */
    p[B2E_KMULT_VCALIBRATION] = 1;      /* :1239, :1139 */
    if (type == B2E_KQUAD) {
      p[B2E_KMULT_EDGE1_LINEAR] = 1; /* :1272-1275 */
      p[B2E_KMULT_EDGE2_LINEAR] = 1;
      p[B2E_KMULT_EDGE1_NONLINEAR_FACTOR] = 1;
      p[B2E_KMULT_EDGE2_NONLINEAR_FACTOR] = 1;
    }
    break;
  case B2E_CSBEND:
  case B2E_CSRCSBEND:
    p[B2E_BEND_FINT] = 0.5;             /* DEFAULT_FINT, track.h:1214 */
    p[B2E_BEND_N_SLICES] = 4;           /* DEFAULT_N_SLICES, track.h:1229 */
    p[B2E_BEND_INTEGRATION_ORDER] = 4;
    p[B2E_BEND_EDGE1_EFFECTS] = 1;
    p[B2E_BEND_EDGE2_EFFECTS] = 1;
    p[B2E_BEND_EDGE_ORDER] = 1;
    p[B2E_BEND_NONLINEAR] = 1;          /* track_data.c:1927, :2008 */
    p[B2E_BEND_ISR1PART] = 1;           /* track_data.c:1966, :2039 */
    if (type == B2E_CSRCSBEND) {
      p[B2E_BEND_BIN_RANGE_FACTOR] = 1.2; /* csrcsbend_param, track_data.c:1982-2060 */
      p[B2E_BEND_SG_ORDER] = 1;
      p[B2E_BEND_TRAPAZOID_INTEGRATION] = 1;
      p[B2E_BEND_CSR] = 1;
      p[B2E_BEND_CLIP_NEGATIVE_BINS] = 1;
      p[B2E_BEND_LOW_FREQUENCY_CUTOFF0] = -1; /* track_data.c:2046-2049 */
      p[B2E_BEND_LOW_FREQUENCY_CUTOFF1] = -1;
      p[B2E_BEND_HIGH_FREQUENCY_CUTOFF0] = -1;
      p[B2E_BEND_HIGH_FREQUENCY_CUTOFF1] = -1;
    }
    break;
  case B2E_RFCA:
    p[B2E_RFCA_FREQ] = 500e6;           /* track_data.c:580 */
    p[B2E_RFCA_T_REFERENCE] = -1;
    break;
  case B2E_MAXAMP:
    p[B2E_MAXAMP_EXPONENT] = 2;         /* track_data.c:990-997 */
    break;
  case B2E_CSRDRIFT:
    p[B2E_CSRDRIFT_N_KICKS] = 1;
    p[B2E_CSRDRIFT_CSR] = 1;
    break;
  case B2E_MALIGN:
    p[B2E_MALIGN_ON_PASS] = -1;         /* track_data.c:935-938 */
    p[B2E_MALIGN_START_PID] = -1;
    p[B2E_MALIGN_END_PID] = -1;
    break;
  case B2E_WATCH:
    p[B2E_WATCH_END_PASS] = -1;         /* track_data.c:881-895 */
    p[B2E_WATCH_INTERVAL] = 1;
    p[B2E_WATCH_FRACTION] = 1;
    p[B2E_WATCH_START_PID] = -1;
    p[B2E_WATCH_END_PID] = -1;
    p[B2E_WATCH_SPARSE_INTERVAL] = 1;
    p[B2E_WATCH_X_DATA] = 1;
    p[B2E_WATCH_Y_DATA] = 1;
    p[B2E_WATCH_LONGIT_DATA] = 1;
    p[B2E_WATCH_FLUSH_INTERVAL] = 100;
    p[B2E_WATCH_REFERENCE_FREQUENCY] = -1;
    break;
  default:
    break;
  }
}

static bool is_bend(int t) { return t == B2E_CSBEND || t == B2E_CSRCSBEND; }

/* determine_bend_flags (bend_matrix.c:1342-1391): edges are skipped where an
 * identically named bend of the same type follows/precedes (MARK between is
 * transparent). */
static void bend_edge_flags(const b2e_element *el, int n, int i, bool *edge1, bool *edge2) {
  bool same_pre = false, same_post = false;
  for (int j = i - 1; j >= 0; j--) {
    if (el[j].type == el[i].type && strncmp(el[j].name, el[i].name, sizeof(el[i].name)) == 0) {
      same_pre = true;
      break;
    }
    if (el[j].type != B2E_MARK)
      break;
  }
  for (int j = i + 1; j < n; j++) {
    if (el[j].type == el[i].type && strncmp(el[j].name, el[i].name, sizeof(el[i].name)) == 0) {
      same_post = true;
      break;
    }
    if (el[j].type != B2E_MARK)
      break;
  }
  *edge1 = el[i].p[B2E_BEND_EDGE1_EFFECTS] != 0 && !same_pre;
  *edge2 = el[i].p[B2E_BEND_EDGE2_EFFECTS] != 0 && !same_post;
}

/* quadPartialFringeMatrix (fringe.c:229-271) with inFringe = 1, as quadFringe
 * forms it: part 1 from the I*M integrals, part 2 from the I*P integrals;
 * out = R00 R01 R10 R11 R22 R23 R32 R33 */
static void quad_fringe_matrix(double out[8], double K1, const double *fi, int part) {
  const double K1sqr = K1 * K1;
  double J1x, J2x, J3x, J1y, J2y, J3y;
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
  const double ex = exp(J1x), ey = exp(J1y);
  out[0] = ex;
  out[1] = J2x / ex;
  out[2] = ex * J3x;
  out[3] = (1 + J2x * J3x) / ex;
  out[4] = ey;
  out[5] = J2y / ey;
  out[6] = ey * J3y;
  out[7] = (1 + J2y * J3y) / ey;
}

static std::string compile_kmult(const b2e_element &el, double Po, DevElem &d, DevRad &r) {
  const double *p = el.p;
  double drift_frac[8], kick_frac[8];
  /* a KQUAD with LEFFECTIVE > 0 integrates over the effective length between
   * two exact drifts (multipole.c:766-770, :1028-1030, :1098-1100) */
  const double L = el.type == B2E_KQUAD && p[B2E_KMULT_LEFFECTIVE] > 0 ? p[B2E_KMULT_LEFFECTIVE] : p[B2E_KMULT_L];
  if (el.type != B2E_KQUAD && p[B2E_KMULT_LEFFECTIVE] != 0)
    return "LEFFECTIVE applies to KQUAD only";
  if (L != p[B2E_KMULT_L]) {
    d.c[KM_LEND] = (p[B2E_KMULT_L] - L) / 2;
    d.flags |= EF_END_DRIFT;
  }
  int integ = (int)p[B2E_KMULT_INTEGRATION_ORDER];
  long n_kicks = (long)p[B2E_KMULT_N_KICKS], nSlices = (long)p[B2E_KMULT_N_SLICES];
  int nSub = integrator_fractions(integ, drift_frac, kick_frac);
  double KnL, drift;
  if (!nSub)
    return "multipole INTEGRATION_ORDER must be 2, 4, or 6";
  if (n_kicks <= 0) {
    if (nSlices <= 0)
      return "N_KICKS<=0 and N_SLICES<=0 in multipole tracking";
  } else if (integ > 2) {
    if ((nSlices = (long)ceil(n_kicks / (1.0 * integ))) < 1)
      nSlices = 1;
  } else
    nSlices = n_kicks;
  d.kind = K_KMULT;
  d.c[KM_ORDER] = el.type == B2E_KQUAD ? 1 : 2;
  d.c[KM_NSLICES] = (double)nSlices;
  d.c[KM_NSUB] = nSub;
  if (p[B2E_KMULT_BORE] != 0) {
    /* strength from the pole-tip field (multipole.c:771-773, :834-836):
     * KnL = n! B(a)/a^n * L/(B rho) * (1+FSE), electrons (charge e_mks) */
    const double rigidity = kE_MKS / (kME_MKS * kC_MKS * Po), a = p[B2E_KMULT_BORE];
    if (el.type == B2E_KQUAD)
      KnL = ((p[B2E_KMULT_B] / a) * rigidity * L) * (1 + p[B2E_KMULT_FSE]);
    else
      KnL = ((2 * p[B2E_KMULT_B] / (a * a)) * rigidity * L) * (1 + p[B2E_KMULT_FSE]);
  } else
    KnL = (p[B2E_KMULT_K] * L) * (1 + p[B2E_KMULT_FSE]);
  drift = L / nSlices;
  for (int j = 0; j < 8; j++) {
    d.c[KM_DSH0 + j] = j < nSub ? drift * drift_frac[j] : 0;
    d.c[KM_KICK0 + j] = j < nSub ? KnL / nSlices * kick_frac[j] : 0;
  }
  /* a zero KnL kick is skipped by the reference ("if (KnL[iOrder])"); here it
   * subtracts an exact zero, which leaves the momenta unchanged */
  if (el.type == B2E_KSEXT) {
    if (p[B2E_KMULT_K1_OF_KSEXT] != 0) {
      double K1L = p[B2E_KMULT_K1_OF_KSEXT] * L;
      d.flags |= EF_QUAD_ORDER2;
      for (int j = 0; j < 8; j++)
        d.c[KM_KICK1_0 + j] = j < nSub ? K1L / nSlices * kick_frac[j] : 0;
    }
    if (p[B2E_KMULT_J1_OF_KSEXT] != 0) {
      double J1L = p[B2E_KMULT_J1_OF_KSEXT] * L;
      if (nSub > 6)
        return "KSEXT J1 with INTEGRATION_ORDER=6 is not supported";
      d.flags |= EF_SKEW_ORDER2;
      for (int j = 0; j < 6; j++)
        d.c[KM_SKEW0 + j] = j < nSub ? J1L / nSlices * kick_frac[j] : 0;
    }
  }
  d.c[KM_DX] = p[B2E_KMULT_DX];
  d.c[KM_DY] = p[B2E_KMULT_DY];
  d.c[KM_DZ] = p[B2E_KMULT_DZ];
  if (p[B2E_KMULT_DX] != 0 || p[B2E_KMULT_DY] != 0 || p[B2E_KMULT_DZ] != 0)
    d.flags |= EF_ENTRANCE_OFFSET | EF_EXIT_MISALIGN;
  if (p[B2E_KMULT_TILT] != 0) {
    d.flags |= EF_ENTRANCE_ROTATE | EF_EXIT_MISALIGN;
    rotation_cs(p[B2E_KMULT_TILT], &d.c[KM_COS_TILT], &d.c[KM_SIN_TILT]);
    /* setupMultApertureData(-tilt): reverseTiltCS = cos(-tilt), sin(-tilt) */
    d.flags |= EF_REVERSE_TILT;
    d.rev_cos = b2e_cos(-p[B2E_KMULT_TILT]);
    d.rev_sin = b2e_sin(-p[B2E_KMULT_TILT]);
  }
  /* radiation (multipole.c:788-800): rad_coef with SYNCH_RAD; isr_coef is
   * always nonzero and negated when ISR is off, so the radiation block runs
   * whenever the slice drift is nonzero (:1320); both are zeroed for a
   * radiating element shorter than 1e-6 m */
  {
    std::string re = check_radiation(p, B2E_KMULT_ISR, B2E_KMULT_ISR1PART, nSlices);
    if (!re.empty())
      return re;
    double rad_coef = 0, isr_coef;
    const bool sr = p[B2E_KMULT_SYNCH_RAD] != 0, isr = p[B2E_KMULT_ISR] != 0;
    if (sr)
      rad_coef = (kE_MKS * kE_MKS) * pow3_host(Po) / (6 * kPI * eps0_mks() * (kC_MKS * kC_MKS) * kME_MKS);
    isr_coef = kRE_MKS * sqrt(55.0 / (24 * sqrt(3)) * pow5_host(Po) * 137.0359895);
    if (!isr)
      isr_coef *= -1;
    if (p[B2E_KMULT_L] < 1e-6 && (isr || sr))
      rad_coef = isr_coef = 0;
    r.c[RK_RAD] = rad_coef;
    r.c[RK_ISR] = isr_coef;
    r.c[RK_DRIFT] = drift;
    /* steering (multipole.c:785-786, :1190-1191): applied as dipole kicks
     * -xkick*kickFrac[step] after the multipole kicks (:1281-1284), and
     * part of F2 in the radiation block (:1333) */
    r.c[RK_XKICK] = (p[B2E_KMULT_HKICK] * p[B2E_KMULT_HCALIBRATION]) / nSlices;
    r.c[RK_YKICK] = (p[B2E_KMULT_VKICK] * p[B2E_KMULT_VCALIBRATION]) / nSlices;
    if (r.c[RK_XKICK] != 0 || r.c[RK_YKICK] != 0)
      d.flags |= EF_STEERING;
    for (int j = 0; j < 8; j++)
      r.c[RK_KFRAC0 + j] = j < nSub ? kick_frac[j] : 0;
    if ((rad_coef != 0 || isr_coef != 0) && drift != 0)
      d.flags |= EF_RADBLOCK;
    if (rad_coef != 0 && drift != 0)
      d.flags |= EF_SR;
    if (isr_coef > 0 && drift != 0)
      d.flags |= EF_ISR;
  }
  /* KQUAD fringe fields (multipole.c:1031-1037, :1088-1094; quadFringe, fringe.c:24-175) */
  {
    const double e1 = p[B2E_KMULT_EDGE1_EFFECTS], e2 = p[B2E_KMULT_EDGE2_EFFECTS];
    if (el.type != B2E_KQUAD && (e1 != 0 || e2 != 0))
      return "EDGE_EFFECTS apply to KQUAD only";
    /* a value <= 0 turns the fringe off (multipole.c:1033, :1090) */
    for (double v : {e1, e2})
      if (v > 2 || v != floor(v))
        return "KQUAD EDGE[12]_EFFECTS above 2 (higher-order fringe terms) is not supported by this engine";
    if (e1 > 0 || e2 > 0) {
      r.c[RK_QF_K1] = p[B2E_KMULT_K];
      quad_fringe_matrix(r.c + RK_QF_M1, p[B2E_KMULT_K], p + B2E_KMULT_I0M, 1);
      quad_fringe_matrix(r.c + RK_QF_M2, p[B2E_KMULT_K], p + B2E_KMULT_I0P, 2);
      r.c[RK_QF_EDGE1] = e1;
      r.c[RK_QF_EDGE2] = e2;
      r.c[RK_QF_LIN1] = p[B2E_KMULT_EDGE1_LINEAR];
      r.c[RK_QF_LIN2] = p[B2E_KMULT_EDGE2_LINEAR];
      r.c[RK_QF_NLF1] = p[B2E_KMULT_EDGE1_NONLINEAR_FACTOR];
      r.c[RK_QF_NLF2] = p[B2E_KMULT_EDGE2_NONLINEAR_FACTOR];
      if (e1 > 0)
        d.flags |= EF_QFRINGE1;
      if (e2 > 0)
        d.flags |= EF_QFRINGE2;
    }
  }
  return "";
}

/* Field expansion of a sector bend with quadrupole and sextupole terms
 * (computeCSBENDFieldCoefficients, csbend.c:186-663): b0 the dipole
 * correction (XKICK/angle, a signed zero without XKICK), b1 = K1*rho0, b2 = K2*rho0,
 * normal terms only, h1 the curvature.  The field sums of a normal-only
 * expansion to order 4 read 15 coefficients; each is formed with the
 * expansion's own terms in their order, the zero octupole and decapole terms
 * (b3, b4) included, so that signed zeros round alike.  Without NONLINEAR
 * only the linear ones are set.  Layout: Fx(0,1) Fx(0,3) Fx(1,1) Fx(1,3)
 * Fx(2,1) Fx(3,1) Fy(0,0) Fy(0,2) Fy(0,4) Fy(1,0) Fy(1,2) Fy(2,0) Fy(2,2)
 * Fy(3,0) Fy(4,0), Fx(i,j) the coefficient of x^i y^j. */
static void bend_field_terms(double *F, double b0, double b1, double b2, double h1, bool nonlinear) {
  const double b3 = 0, b4 = 0;
  const double h2 = h1 * h1, h3 = h2 * h1;
  for (int k = 0; k < 15; k++)
    F[k] = 0;
  F[0] = b1;
  F[6] = 1 - b0;
  F[9] = b1;
  if (!nonlinear)
    return;
  F[1] = (h2 * b1) / 6 - (h1 * b2) / 6 - b3 / 6;
  F[2] = b2;
  F[3] = -(h3 * b1) / 3 + (h2 * b2) / 3 - (h1 * b3) / 6 - b4 / 6;
  F[4] = b3 / 2;
  F[5] = b4 / 6;
  F[7] = -(h1 * b1) / 2 - b2 / 2;
  F[8] = (h3 * b1) / 24 - (h2 * b2) / 24 + (h1 * b3) / 12 + b4 / 24;
  F[10] = (h2 * b1) / 2 - (h1 * b2) / 2 - b3 / 2;
  F[11] = b2 / 2;
  F[12] = -(h3 * b1) / 2 + (h2 * b2) / 2 - (h1 * b3) / 4 - b4 / 4;
  F[13] = b3 / 6;
  F[14] = b4 / 24;
}

/* ETILT: the bend is rolled by etilt about its entrance axis, so the exit
 * face's centre moves off the design orbit.  Offsets (x, x', y, y', s) of that
 * centre in the bend frame, then turned by -tilt into the frame the exit
 * rotation leaves the particles in (csbend.c:4723-4769, the turn is
 * tilt_matrices.c:123-150).  Zero when etilt is zero. */
static void etilt_exit_offsets(double out[5], double rho0, double angle, double etilt, double tilt) {
  for (int k = 0; k < 5; k++)
    out[k] = 0;
  if (etilt == 0)
    return;
  const double roll = -etilt; /* ETILT's sign convention is TILT's */
  const double sa = b2e_sin(angle), ca = b2e_cos(angle), ta = b2e_tan(angle);
  const double cr = b2e_cos(roll), sr = b2e_sin(roll);
  /* exit centre of the rolled arc (a) and the unit tangent's out-of-plane
   * part (uz); the in-plane parts are not needed */
  const double ax = ((1 - ca) * rho0) * (cr - 1), az = ((1 - ca) * rho0) * sr;
  const double norm = sqrt((sa * cr) * (sa * cr) + ca * ca);
  const double uz = (sa * sr) / norm;
  /* where the tangent line from a meets the design exit plane (b), the path
   * length along it (dz) and the slope of the line in the bend plane */
  const double tan_alpha = (1. / ta) / cr;
  const double bx = (ax * tan_alpha) / (ta + tan_alpha);
  const double by = -bx * ta;
  const double dz = sqrt((bx - ax) * (bx - ax) + by * by);
  out[0] = sqrt(bx * bx + by * by);
  out[1] = b2e_tan(atan(tan_alpha) - (kPI / 2 - angle));
  out[2] = az + uz * dz;
  out[3] = uz;
  out[4] = dz * sqrt(1 + uz * uz);
  /* into the tilted frame: a turn by -tilt, with the exact quarter turns */
  const double turn = -tilt;
  double c, s;
  if (turn == 0 || fabs(fabs(turn) - 2 * kPI) < 1e-12)
    return;
  if (fabs(fabs(turn) - kPI) < 1e-12) {
    c = -1;
    s = 0;
  } else if (fabs(turn - kPI / 2) < 1e-12) {
    c = 0;
    s = 1;
  } else if (fabs(turn + kPI / 2) < 1e-12) {
    c = 0;
    s = -1;
  } else {
    c = b2e_cos(turn);
    s = b2e_sin(turn);
  }
  const double x = out[0], xp = out[1], y = out[2], yp = out[3];
  out[0] = x * c + y * s;
  out[2] = -x * s + y * c;
  out[1] = xp * c + yp * s;
  out[3] = -xp * s + yp * c;
}

static std::string compile_csbend(const b2e_element &el, bool edge1, bool edge2, double Po, DevElem &d,
                                  DevRad &r) {
  const double *p = el.p;
  double drift_frac[8], kick_frac[8];
  const double length = p[B2E_BEND_L];
  double angle, e1, e2, tilt, etilt, rho0, h, fse, rho_actual, Kg, psi1, psi2, ttilt, ct, st, s;
  int integ = (int)p[B2E_BEND_INTEGRATION_ORDER], nSub, nSlices = (int)p[B2E_BEND_N_SLICES];
  if (p[B2E_BEND_ANGLE] == 0) {
    d.kind = K_EDRIFT;
    d.c[DR_L] = length;
    return "";
  }
  nSub = integrator_fractions(integ, drift_frac, kick_frac);
  if (!nSub)
    return "CSBEND integration_order is invalid--must be 2, 4, or 6";
  if (nSlices < 1)
    return "CSBEND N_SLICES must be >= 1";
  /* the expansion runs when any b[] is nonzero (hasNormal, csbend.c:205-210),
   * b0 = XKICK/ANGLE included */
  const bool fields =
      p[B2E_BEND_K1] != 0 || p[B2E_BEND_K2] != 0 || p[B2E_BEND_XKICK] != 0 || p[B2E_BEND_YKICK] != 0;
  if (fields && el.type == B2E_CSRCSBEND)
    return "CSRCSBEND with K1/K2/XKICK/YKICK field terms is not supported by this engine";
  /* method 1 (K. L. Brown's edge matrix, to first or second order) and, on
   * CSBEND, method 3 (applySimpleDipoleEdgeKick, csbend.c:5639-5665) */
  const bool simple1 = edge1 && p[B2E_BEND_EDGE1_EFFECTS] == 3 && el.type == B2E_CSBEND;
  const bool simple2 = edge2 && p[B2E_BEND_EDGE2_EFFECTS] == 3 && el.type == B2E_CSBEND;
  if ((edge1 && p[B2E_BEND_EDGE1_EFFECTS] != 1 && !simple1) || (edge2 && p[B2E_BEND_EDGE2_EFFECTS] != 1 && !simple2))
    return "CSBEND EDGE[12]_EFFECTS other than 0, 1 or 3 (3 on CSBEND only) is not supported by this engine";
  /* csbend.c:933-950: negative angle folded into a PI tilt */
  if (p[B2E_BEND_ANGLE] < 0) {
    angle = -p[B2E_BEND_ANGLE];
    e1 = -p[B2E_BEND_E1];
    e2 = -p[B2E_BEND_E2];
    etilt = p[B2E_BEND_ETILT] * 1; /* etiltSign = 1 */
    tilt = p[B2E_BEND_TILT] + kPI;
    rho0 = length / angle;
  } else {
    angle = p[B2E_BEND_ANGLE];
    e1 = p[B2E_BEND_E1];
    e2 = p[B2E_BEND_E2];
    etilt = p[B2E_BEND_ETILT] * 1;
    tilt = p[B2E_BEND_TILT];
    rho0 = length / angle;
  }
  if (fabs(rho0) > 1e6)
    return "CSBEND with radius > 1e6 is not supported (use EDRIFT)";
  fse = p[B2E_BEND_FSE] + 0.0;
  h = 1 / rho0;
  if (fabs(fse + 1) < 1e-12)
    fse = -1 + 1e-12;
  rho_actual = 1 / ((1 + fse) * h);
  /* fringe angles (csbend.c:985-991); FINT1/FINT2 default to FINT */
  Kg = 2 * p[B2E_BEND_HGAP] * p[B2E_BEND_FINT] * (rho0 < 0 ? -1 : 1);
  psi1 = Kg / fabs(rho_actual) / b2e_cos(e1) * (1 + b2e_sin(e1) * b2e_sin(e1));
  psi2 = Kg / fabs(rho_actual) / b2e_cos(e2) * (1 + b2e_sin(e2) * b2e_sin(e2));
  if (length < 0) {
    psi1 *= -1;
    psi2 *= -1;
  }
  /* total tilt (csbend.c:1051-1066) */
  ttilt = tilt + etilt;
  if (ttilt == 0) {
    ct = 1;
    st = 0;
  } else if (fabs(fabs(ttilt) - kPI) < 1e-12) {
    ct = -1;
    st = 0;
  } else if (fabs(ttilt - kPI / 2) < 1e-12) {
    ct = 0;
    st = 1;
  } else if (fabs(ttilt + kPI / 2) < 1e-12) {
    ct = 0;
    st = -1;
  } else {
    ct = b2e_cos(ttilt);
    st = b2e_sin(ttilt);
  }
  d.kind = el.type == B2E_CSBEND ? K_CSBEND : K_CSRCSBEND;
  d.c[CB_RHO0] = rho0;
  d.c[CB_RHO_ACTUAL] = rho_actual;
  d.c[CB_NSLICES] = nSlices;
  d.c[CB_NSUB] = nSub;
  s = length / nSlices; /* integrate_csbend_ordn: s /= n */
  if (el.type == B2E_CSRCSBEND)
    s = (length / nSlices) / 1; /* track_through_csbendCSR integrates one slice of length/nSlices per kick */
  for (int j = 0; j < 8; j++) {
    /* the integrator uses the drift only as dsh/rho0 (csbend.c:1566): the
     * same two roundings, done once */
    d.c[CB_DSH0 + j] = j < nSub ? (s * drift_frac[j]) / rho0 : 0;
    d.c[CB_DS0 + j] = j < nSub ? s * kick_frac[j] : 0;
  }
  d.c[CB_TAN_E1] = b2e_tan(e1);
  d.c[CB_E1] = e1;
  d.c[CB_PSI1] = psi1;
  d.c[CB_TAN_E2] = b2e_tan(e2);
  d.c[CB_E2] = e2;
  d.c[CB_PSI2] = psi2;
  d.c[CB_COS_TT] = ct;
  d.c[CB_SIN_TT] = st;
  /* malignMethod 0 offsets (csbend.c:1070-1082) */
  d.c[CB_DXI] = -p[B2E_BEND_DX];
  d.c[CB_DZI] = p[B2E_BEND_DZ];
  d.c[CB_DYI] = -p[B2E_BEND_DY];
  d.c[CB_DXF] = p[B2E_BEND_DX] * b2e_cos(p[B2E_BEND_ANGLE]) + p[B2E_BEND_DZ] * b2e_sin(p[B2E_BEND_ANGLE]);
  d.c[CB_DZF] = p[B2E_BEND_DX] * b2e_sin(p[B2E_BEND_ANGLE]) - p[B2E_BEND_DZ] * b2e_cos(p[B2E_BEND_ANGLE]);
  d.c[CB_DYF] = p[B2E_BEND_DY];
  double *bx = r.c + RB_EXTRA0;
  etilt_exit_offsets(bx + BX_ETILT0, rho0, angle, etilt, tilt);
  if (etilt != 0)
    d.flags |= EF_ETILT;
  d.c[CB_INV_RHO0] = 1 / rho0;
  d.c[CB_INV_RHO_ACTUAL] = 1 / rho_actual;
  if (edge1)
    d.flags |= EF_EDGE1;
  if (edge2)
    d.flags |= EF_EDGE2;
  if (simple1)
    d.flags |= EF_EDGE1_SIMPLE;
  if (simple2)
    d.flags |= EF_EDGE2_SIMPLE;
  if ((edge1 || edge2) && p[B2E_BEND_EDGE_ORDER] >= 2) {
    /* second-order edges (apply_edge_effects, csbend.c:4266-4307): the
     * per-element parts; b1 = K1*rho0 (csbend.c:825), sign-flipped with a
     * negative angle (:879-882), gives n = -b1/h (:929) */
    double b1 = p[B2E_BEND_K1] * (length / p[B2E_BEND_ANGLE]);
    if (el.type == B2E_CSBEND)
      b1 *= ((1 + p[B2E_BEND_FSE]) + 0) / ((1 + p[B2E_BEND_FSE]) + 0);
    if (p[B2E_BEND_ANGLE] < 0)
      b1 *= -1;
    const double sec1 = 1. / b2e_cos(e1), sec2 = 1. / b2e_cos(e2);
    d.flags |= EF_EDGE_ORDER2;
    bx[BX_SEC2_E1] = sec1 * sec1;
    bx[BX_SEC2_E2] = sec2 * sec2;
    bx[BX_EDGE_N] = -b1 / h;
  }
  if (-tilt != 0) {
    d.flags |= EF_REVERSE_TILT;
    d.rev_cos = b2e_cos(-tilt);
    d.rev_sin = b2e_sin(-tilt);
  }
  /* isrConstant is nonzero for CSBEND (negated when ISR is off,
   * csbend.c:972-975); CSRCSBEND sets it to 0 unless ISR is on (:2138-2142) */
  if (el.type == B2E_CSBEND) {
    std::string re = check_radiation(p, B2E_BEND_ISR, B2E_BEND_ISR1PART, nSlices);
    if (!re.empty())
      return re;
    double rad_coef = 0, isr_const;
    if (p[B2E_BEND_SYNCH_RAD] != 0)
      rad_coef = (kE_MKS * kE_MKS) * pow3_host(Po) * ((1 + fse) * (1 + fse)) /
                 (6 * kPI * eps0_mks() * (kC_MKS * kC_MKS) * kME_MKS * (rho0 * rho0));
    isr_const = kRE_MKS * sqrt(55.0 / (24 * sqrt(3)) * pow5_host(Po) * 137.0359895 / pow3_host(fabs(rho_actual)));
    if (p[B2E_BEND_ISR] == 0)
      isr_const *= -1;
    r.c[RB_RAD] = rad_coef;
    r.c[RB_ISR] = isr_const;
    r.c[RB_SLICE] = s;
    r.c[RB_INV_RHO0] = 1. / rho0;
    if (fields) {
      /* b[] as track_through_csbend forms it (csbend.c:824-882): K*rho0 with
       * the signed angle, the FSE ratios (1 + fse)/(1 + fse), the quadrupole
       * term negated with a negative angle; b0 = XKICK/angle (:867) */
      const double rho_signed = length / p[B2E_BEND_ANGLE];
      double b1 = p[B2E_BEND_K1] * rho_signed, b2 = p[B2E_BEND_K2] * rho_signed;
      b1 *= ((1 + p[B2E_BEND_FSE]) + 0) / ((1 + p[B2E_BEND_FSE]) + 0);
      b2 *= (1 + p[B2E_BEND_FSE]) / ((1 + p[B2E_BEND_FSE]) + 0);
      if (p[B2E_BEND_ANGLE] < 0)
        b1 *= -1;
      bend_field_terms(r.c + RB_FIELD0, p[B2E_BEND_XKICK] / p[B2E_BEND_ANGLE], b1, b2, h,
                       p[B2E_BEND_NONLINEAR] != 0);
      /* c0 = YKICK/angle (:868): with it the reference sums every (i, j) of
       * the expansion (hasSkew, csbend.c:124-135); the other skew entries are
       * zero, so the sums are the normal ones with c0 first in Fx */
      if (p[B2E_BEND_YKICK] != 0) {
        r.c[RB_SKEW0] = p[B2E_BEND_YKICK] / p[B2E_BEND_ANGLE];
        d.flags |= EF_SKEW_KICK;
      }
      d.flags |= EF_FIELD;
    }
    d.flags |= EF_RADBLOCK;
    if (rad_coef != 0)
      d.flags |= EF_SR;
    if (isr_const > 0)
      d.flags |= EF_ISR;
  } else if (p[B2E_BEND_SYNCH_RAD] != 0 || p[B2E_BEND_ISR] != 0) {
    return "CSRCSBEND with SYNCH_RAD or ISR is not supported by this engine";
  }
  return "";
}

static std::string compile_rfca(const b2e_element &el, int slot, DevElem &d) {
  const double *p = el.p;
  if (p[B2E_RFCA_FREQ] == 0)
    return "RFCA with zero frequency is not supported by this engine";
  if (p[B2E_RFCA_L] < 0)
    return "RFCA with negative length (backtracking) is not supported by this engine";
  const int fid = (int)p[B2E_RFCA_FIDUCIAL];
  if (fid != p[B2E_RFCA_FIDUCIAL] || fid < B2E_FIDUCIAL_TMEAN || fid > B2E_FIDUCIAL_PMAXIMUM)
    return "RFCA FIDUCIAL must be tmean, light or pmaximum (first ends every serial elegant run: "
           "simple_rfca.c:103-111)";
  d.kind = K_RFCA;
  /* nKicks = length ? N_KICKS : 1, the matrix method for nKicks <= 0;
   * length and volt per section (simple_rfca.c:403-409) */
  const double L = p[B2E_RFCA_L];
  long nKicks = L != 0 ? (long)p[B2E_RFCA_N_KICKS] : 1;
  int matrix = 0;
  if (nKicks <= 0) {
    matrix = 1;
    nKicks = 1;
  }
  const double length = L / nKicks;
  /* volt = VOLT/(1e6*particleMassMV*particleRelSign)/nKicks, omega = PIx2*FREQ (simple_rfca.c:384-394) */
  d.c[RF_VOLT] = p[B2E_RFCA_VOLT] / (1e6 * kME_MEV * 1) / nKicks;
  d.c[RF_OMEGA] = (2 * kPI) * p[B2E_RFCA_FREQ];
  d.c[RF_PHASE_DEG_RAD] = p[B2E_RFCA_PHASE] * kPI / 180.0;
  d.c[RF_DX] = p[B2E_RFCA_DX];
  d.c[RF_DY] = p[B2E_RFCA_DY];
  d.c[RF_T_REFERENCE] = p[B2E_RFCA_T_REFERENCE];
  d.c[RF_SOFFSET] = length / 2; /* findFiducialTime's sOffset (simple_rfca.c:431) */
  d.c[RF_SLOT] = slot;
  d.c[RF_LENGTH] = length;
  d.c[RF_NKICKS] = (double)nKicks;
  d.c[RF_MATRIX] = matrix;
  d.c[RF_DTLIGHT] = length / kC_MKS;
  /* VOLT = 0: an exact drift over L and nothing else (simple_rfca.c:380-392) */
  d.c[RF_DRIFT_ONLY] = p[B2E_RFCA_VOLT] == 0;
  d.c[RF_FID_MODE] = fid;
  d.c[RF_L_TOTAL] = L;
  return "";
}

/* One CSRCSBEND standing alone (both edges active as its parameters say),
 * compiled into `d` without any container; returns nullptr on success or a
 * static message. */
const char *compile_single_csr_bend(const b2e_element &el, DevElem &d, BendExtra &bx) {
  static thread_local char msg[256];
  if (el.type != B2E_CSRCSBEND)
    return "element is not a CSRCSBEND";
  memset(&d, 0, sizeof(d));
  d.ap_pass0 = d.ap_later = -1;
  DevRad rad;
  memset(&rad, 0, sizeof(rad));
  std::string e = compile_csbend(el, el.p[B2E_BEND_EDGE1_EFFECTS] != 0, el.p[B2E_BEND_EDGE2_EFFECTS] != 0, 0.0, d,
                                 rad);
  if (!e.empty()) {
    snprintf(msg, sizeof(msg), "%s", e.c_str());
    return msg;
  }
  memcpy(bx.c, rad.c + RB_EXTRA0, sizeof(bx.c));
  if (d.kind != K_CSRCSBEND)
    return "CSRCSBEND with zero angle is a drift; nothing to do here";
  d.z_end = el.p[B2E_BEND_L];
  return nullptr;
}

std::string compile_lattice(const b2e_element *el, int n, const b2e_run_options &opt, CompiledLattice &out) {
  out = CompiledLattice();
  out.elems.resize(n);
  out.rads.assign(n, DevRad());
  for (DevRad &r : out.rads)
    memset(&r, 0, sizeof(r));
  int last_ap = -1;
  double z = 0;
  std::map<long, int> phase_groups; /* PHASE_REFERENCE -> RF state slot of its first cavity */
  for (int i = 0; i < n; i++) {
    DevElem &d = out.elems[i];
    memset(&d, 0, sizeof(d));
    d.ap_pass0 = d.ap_later = -1;
    std::string err;
    const double *p = el[i].p;
    d.z_start = z;
    switch (el[i].type) {
    case B2E_DRIF: {
      int order = p[B2E_DRIF_ORDER] != 0 ? (int)p[B2E_DRIF_ORDER] : opt.default_order;
      d.kind = order >= 2 ? K_DRIF_O2 : K_DRIF_O1;
      d.c[DR_L] = p[B2E_DRIF_L];
      d.c[DR_LH] = p[B2E_DRIF_L] / 2;
      d.flags |= EF_EXTRAPOLATE;
      z += p[B2E_DRIF_L];
      break;
    }
    case B2E_EDRIFT:
      d.kind = K_EDRIFT;
      d.c[DR_L] = p[B2E_EDRIFT_L];
      z += p[B2E_EDRIFT_L];
      break;
    case B2E_KQUAD:
    case B2E_KSEXT:
      err = compile_kmult(el[i], opt.p_central, d, out.rads[i]);
      z += p[B2E_KMULT_L];
      break;
    case B2E_CSBEND:
    case B2E_CSRCSBEND: {
      bool e1, e2;
      bend_edge_flags(el, n, i, &e1, &e2);
      err = compile_csbend(el[i], e1, e2, opt.p_central, d, out.rads[i]);
      if (el[i].type == B2E_CSRCSBEND && d.kind == K_CSRCSBEND)
        out.csr_elements.push_back(i);
      z += p[B2E_BEND_L];
      break;
    }
    case B2E_RFCA:
      err = compile_rfca(el[i], out.n_rf, d);
      d.c[RF_LEADER] = -1;
      if (const long ref = (long)p[B2E_RFCA_PHASE_REFERENCE]) {
        auto it = phase_groups.find(ref);
        if (it != phase_groups.end())
          d.c[RF_LEADER] = it->second;
        else
          phase_groups[ref] = out.n_rf;
      }
      out.rf_elements.push_back(i);
      out.n_rf++;
      z += p[B2E_RFCA_L];
      break;
    case B2E_MAXAMP: {
      DevAperture a;
      memset(&a, 0, sizeof(a));
      int xe = (int)p[B2E_MAXAMP_EXPONENT], ye = (int)p[B2E_MAXAMP_Y_EXPONENT];
      a.x_max = p[B2E_MAXAMP_X_MAX];
      a.y_max = p[B2E_MAXAMP_Y_MAX];
      a.elliptical = p[B2E_MAXAMP_ELLIPTICAL] != 0;
      a.xe = xe;
      a.ye = ye ? ye : xe;
      if (a.x_max != 0 || a.y_max != 0) {
        if (!a.elliptical)
          a.mode = (a.x_max < 0 && a.y_max < 0) ? 0 : 1;
        else if (a.x_max <= 0 || a.y_max <= 0)
          a.mode = (a.x_max > 0 || a.y_max > 0) ? 1 : 0;
        else {
          if (a.xe < 2 || a.xe % 2 || a.ye < 2 || a.ye % 2)
            err = "MAXAMP exponent must be an even integer >= 2";
          a.mode = 2;
          a.a2 = ipow_host(a.x_max, a.xe);
          a.b2 = ipow_host(a.y_max, a.ye);
        }
      }
      last_ap = (int)out.aps.size();
      out.aps.push_back(a);
      d.kind = K_MAXAMP;
      break;
    }
    case B2E_MARK:
    case B2E_CHARGE:
      d.kind = K_NONE;
      d.flags |= EF_NO_APERTURE;
      break;
    case B2E_CSRDRIFT:
      d.kind = K_CSRDRIFT;
      d.c[0] = p[B2E_CSRDRIFT_L];
      out.csr_elements.push_back(i);
      z += p[B2E_CSRDRIFT_L];
      break;
    case B2E_MALIGN: {
      /* offset_beam's checks (do_tracking.c:3268-3271) */
      const long s_pid = (long)p[B2E_MALIGN_START_PID], e_pid = (long)p[B2E_MALIGN_END_PID];
      if (s_pid >= 0 && s_pid > e_pid)
        err = "MALIGN START_PID greater than END_PID";
      else if ((e_pid >= 0 && s_pid < 0) || (s_pid >= 0 && e_pid < 0))
        err = "MALIGN START_PID and END_PID must both be set or both be -1";
      d.kind = K_MALIGN;
      d.c[MA_DX] = p[B2E_MALIGN_DX];
      d.c[MA_DXP] = p[B2E_MALIGN_DXP];
      d.c[MA_DY] = p[B2E_MALIGN_DY];
      d.c[MA_DYP] = p[B2E_MALIGN_DYP];
      d.c[MA_DZ] = p[B2E_MALIGN_DZ];
      d.c[MA_DT] = p[B2E_MALIGN_DT];
      d.c[MA_DP] = p[B2E_MALIGN_DP];
      d.c[MA_DE] = p[B2E_MALIGN_DE];
      d.c[MA_ON_PASS] = (double)(long)p[B2E_MALIGN_ON_PASS];
      d.c[MA_START_PID] = (double)s_pid;
      d.c[MA_END_PID] = (double)e_pid;
      d.c[MA_C] = kC_MKS;
      break;
    }
    case B2E_WATCH: {
      /* a WATCH never changes the particles; NO_APERTURE (track_data.c:3941) */
      d.flags |= EF_NO_APERTURE;
      const long s_pid = (long)p[B2E_WATCH_START_PID], e_pid = (long)p[B2E_WATCH_END_PID];
      if (p[B2E_WATCH_DISABLE] != 0) {
        d.kind = K_NONE;
        break;
      }
      if (p[B2E_WATCH_MODE] != 0 && p[B2E_WATCH_MODE] != 1 && p[B2E_WATCH_MODE] != 2)
        err = "WATCH fft mode is not supported by this engine";
      else if (p[B2E_WATCH_FRACTION] != 1)
        err = "WATCH FRACTION other than 1 is not supported by this engine";
      else if (p[B2E_WATCH_SPARSE_INTERVAL] > 1)
        err = "WATCH SPARSE_INTERVAL other than 1 is not supported by this engine";
      else if ((long)p[B2E_WATCH_INTERVAL] < 1)
        err = "WATCH INTERVAL must be at least 1";
      /* dump_watch_particles' checks (sdds_support.c:755-758) */
      else if (s_pid >= 0 && s_pid > e_pid)
        err = "WATCH startPID>endPID";
      else if ((e_pid >= 0 && s_pid < 0) || (s_pid >= 0 && e_pid < 0))
        err = "WATCH invalid startPID, endPID";
      d.kind = K_WATCH;
      d.c[WA_START] = (double)(long)p[B2E_WATCH_START_PASS];
      d.c[WA_END] = (double)(long)p[B2E_WATCH_END_PASS];
      d.c[WA_INTERVAL] = (double)(long)p[B2E_WATCH_INTERVAL];
      d.c[WA_ORDINAL] = (double)out.watch_elements.size();
      out.watch_elements.push_back(i);
      break;
    }
    default:
      err = "unsupported element type";
    }
    if (!err.empty())
      return std::string("element ") + std::to_string(i) + " (" + std::string(el[i].name, strnlen(el[i].name, 32)) +
             "): " + err;
    d.ap_pass0 = last_ap;
    d.z_end = z;
  }
  /* sticky MAXAMP carries over into later passes (do_tracking keeps x_max etc.) */
  for (int i = 0; i < n; i++)
    out.elems[i].ap_later = out.elems[i].ap_pass0 >= 0 ? out.elems[i].ap_pass0 : last_ap;
  out.total_length = z;
  return "";
}

} // namespace b2e
