/*
 * Internal data layout of the tracking engine (host and device).
 *
 * HBM layout: particles are six FP64 columns (x, xp, y, yp, s, delta), one
 * int64 ID column and two int32 loss columns, each contiguous and 256-byte
 * aligned, so a warp's 32 consecutive particles are one 256-byte transaction
 * per column.  Batched ensembles store instance i's particles contiguously
 * in [offset[i], offset[i+1]); the launch tiles each instance separately so
 * a thread block never mixes instances.
 *
 * The lattice is "compiled" on the host into DevElem records: every constant
 * the reference computes once per element call (KnL/nSlices*kickFrac,
 * rho0, rho_actual, edge tangents, misalignment sines ...) is evaluated
 * there, with the same expressions and the same elementary functions the
 * reference uses, so the device only runs the per-particle arithmetic.  A
 * block stages its instance's records in shared memory once per launch.
 */
#ifndef B2E_ENGINE_H
#define B2E_ENGINE_H
#include <stdint.h>
#include "../../include/elegant_b200.h"

#define B2E_NC 40 /* constants per compiled element */

/* Compiled element kinds (device dispatch) */
enum {
  K_NONE = 0, /* MARK, CHARGE: no particle action */
  K_DRIF_O1,  /* first-order drift matrix */
  K_DRIF_O2,  /* second-order drift matrix (default_order 2) */
  K_EDRIFT,
  K_KMULT,    /* KQUAD / KSEXT, 4th-order (or 2nd) kick integrator */
  K_CSBEND,
  K_RFCA,
  K_MAXAMP,
  K_CSRCSBEND, /* collective: handled by the CSR driver, never in the ring kernel */
  K_CSRDRIFT,
  K_MALIGN,    /* offset_beam on one pass (or every pass) */
  K_WATCH      /* coordinate-mode WATCH: records the live particles on its passes */
};

/* Flags */
#define EF_ENTRANCE_OFFSET 0x1  /* KMULT: dx||dy||dz at entrance */
#define EF_ENTRANCE_ROTATE 0x2  /* KMULT: tilt at entrance */
#define EF_EXIT_MISALIGN 0x4    /* KMULT: exit transform needed */
#define EF_EDGE1 0x8            /* CSBEND: entrance edge (order 1, method 1) */
#define EF_EDGE2 0x10           /* CSBEND: exit edge */
#define EF_EXTRAPOLATE 0x20     /* aperture loss z-extrapolation (DRIF) */
#define EF_NO_APERTURE 0x40     /* element class has NO_APERTURE */
#define EF_RADBLOCK 0x80        /* the reference's radiation bookkeeping block runs (ISR coefficient nonzero) */
#define EF_SKEW_ORDER2 0x100    /* KSEXT J1 term present */
#define EF_QUAD_ORDER2 0x200    /* KSEXT K1 term present */
#define EF_REVERSE_TILT 0x400   /* nonzero reverse tilt in the internal aperture check */
#define EF_SR 0x800             /* KMULT / CSBEND: classical synchrotron radiation (SYNCH_RAD) */
#define EF_ISR 0x1000           /* KMULT / CSBEND: quantum excitation (ISR) */
#define EF_EDGE_ORDER2 0x2000   /* CSBEND: edges by the second-order map (EDGE_ORDER >= 2; BendExtra) */
#define EF_FIELD 0x4000         /* CSBEND: K1/K2 field terms (coefficients in the DevRad table) */
#define EF_ETILT 0x8000         /* CSBEND: ETILT exit offsets (BendExtra) */
#define EF_STEERING 0x10000     /* KMULT: HKICK/VKICK steering kicks (per-part kicks in the DevRad table) */
#define EF_QFRINGE1 0x20000     /* KQUAD: entrance fringe (quadFringe; matrices in the DevRad table) */
#define EF_QFRINGE2 0x40000     /* KQUAD: exit fringe */
#define EF_END_DRIFT 0x80000    /* KQUAD with LEFFECTIVE: exact end drifts (KM_LEND) */
#define EF_SKEW_KICK 0x100000   /* CSBEND with YKICK: the skew dipole term RB_SKEW0 in Fx */
#define EF_EDGE1_SIMPLE 0x200000 /* CSBEND EDGE1_EFFECTS 3: applySimpleDipoleEdgeKick */
#define EF_EDGE2_SIMPLE 0x400000 /* CSBEND EDGE2_EFFECTS 3 */

/* KMULT constant slots */
#define KM_ORDER 0       /* 1 quad, 2 sext */
#define KM_NSLICES 1
#define KM_NSUB 2        /* substeps per slice (4 for order-4 integration) */
#define KM_DSH0 3        /* drift*driftFrac[j], j = 0..7 -> 3..10 */
#define KM_KICK0 11      /* KnL/nSlices*kickFrac[j], j = 0..7 -> 11..18 (0 terminates) */
#define KM_KICK1_0 19    /* secondary K1 term per substep, 19..25 (KSEXT K1) */
#define KM_LEND 26       /* (L - LEFFECTIVE)/2, the end drifts of a KQUAD with LEFFECTIVE */
#define KM_DX 27
#define KM_DY 28
#define KM_DZ 29
#define KM_COS_TILT 30
#define KM_SIN_TILT 31
#define KM_REV_COS 32   /* reverse tilt cos/sin for the aperture check */
#define KM_REV_SIN 33
#define KM_SKEW0 34     /* J1 kick per substep 34..39 (first 6 substeps) */


/* CSBEND constant slots */
#define CB_RHO0 0
#define CB_RHO_ACTUAL 1
#define CB_NSLICES 2
#define CB_NSUB 3
#define CB_DSH0 4       /* (s*driftFrac[j])/rho0, 4..11: the drift angle of substep j */
#define CB_DS0 12       /* s*kickFrac[j], 12..19 (0 terminates) */
#define CB_TAN_E1 20
#define CB_E1 21
#define CB_PSI1 22
#define CB_TAN_E2 23
#define CB_E2 24
#define CB_PSI2 25
#define CB_COS_TT 26
#define CB_SIN_TT 27
#define CB_DXI 28
#define CB_DYI 29
#define CB_DZI 30
#define CB_DXF 31
#define CB_DYF 32
#define CB_DZF 33
#define CB_INV_RHO0 34  /* RN(1/rho0), for X/rho0 by div_rn_recip */
#define CB_INV_RHO_ACTUAL 35 /* RN(1/rho_actual) */

/* A bend's rarely used constants (ETILT, second-order edges), kept out of
 * the element record that the ring kernel stages in shared memory: in the
 * DevRad table for the ring kernel (RB_EXTRA0), as a kernel argument for the
 * CSR kernels. */
#define BX_ETILT0 0     /* exit offsets of ETILT (x, xp, y, yp, s), 0..4; zero without ETILT */
#define BX_SEC2_E1 5    /* sqr(1/cos(e1)), second-order edges */
#define BX_SEC2_E2 6    /* sqr(1/cos(e2)) */
#define BX_EDGE_N 7     /* field index n = -b1/h of the second-order edge map */
#define B2E_NBX 8
typedef struct {
  double c[B2E_NBX];
} BendExtra;


/* Radiation constants of a KMULT / CSBEND, a KMULT's steering kicks and a
 * CSBEND's field-expansion coefficients, in a table beside the element
 * records ([instance][element] DevRad): only lattices that radiate, steer
 * in a KQUAD/KSEXT or have bends with K1/K2 read it (the ring kernel's RAD
 * instantiation), so the records the ring kernel stages in shared memory
 * stay small. */
#define B2E_NRAD 36
#define RK_KFRAC0 0     /* KMULT: kickFrac[j], j = 0..7 */
#define RK_RAD 8        /* rad_coef (multipole.c:789) */
#define RK_ISR 9        /* isr_coef, > 0 only when ISR is applied (:790-795) */
#define RK_DRIFT 10     /* slice drift length (:1189) */
#define RK_XKICK 11     /* HKICK*HCALIBRATION/n_parts, the steering kick per slice (:785, :1190) */
#define RK_YKICK 12     /* VKICK*VCALIBRATION/n_parts (:786, :1191) */
#define RK_QF_K1 13     /* KQUAD fringe (fringe.c:24-175): K1 without FSE */
#define RK_QF_M1 14     /* quadPartialFringeMatrix part 1 (I*M): R00 R01 R10 R11 R22 R23 R32 R33, 14..21 */
#define RK_QF_M2 22     /* part 2 (I*P), 22..29 */
#define RK_QF_EDGE1 30  /* EDGE1_EFFECTS, EDGE2_EFFECTS */
#define RK_QF_EDGE2 31
#define RK_QF_LIN1 32   /* EDGE1_LINEAR, EDGE2_LINEAR */
#define RK_QF_LIN2 33
#define RK_QF_NLF1 34   /* EDGE1/2_NONLINEAR_FACTOR */
#define RK_QF_NLF2 35
#define RB_RAD 0        /* CSBEND: rad_coef (csbend.c:967-970) */
#define RB_ISR 1        /* isrConstant, > 0 only when ISR is applied (:972-975) */
#define RB_SLICE 2      /* s = length / N_SLICES, for dsISR (:1614) */
#define RB_INV_RHO0 3   /* 1. / rho0 (:1605) */
#define RB_FIELD0 12    /* CSBEND with K1/K2: the 15 field-expansion coefficients the
                         * field sums use, 12..26 (bend_fields has the order) */
#define RB_SKEW0 27     /* CSBEND: c0 = YKICK/angle, the only skew coefficient (Fx at x^0 y^0) */
#define RB_EXTRA0 28    /* the bend's BendExtra constants, 28..35 */

/* RFCA constant slots */
#define RF_VOLT 0       /* volt/(1e6*mc^2[MV]*sign)/nKicks */
#define RF_OMEGA 1
#define RF_PHASE_DEG_RAD 2 /* rfca->phase*PI/180.0 */
#define RF_DX 3
#define RF_DY 4
#define RF_T_REFERENCE 5
#define RF_SOFFSET 6    /* length/2 used by the fiducial sum */
#define RF_SLOT 7       /* index into the per-instance RF state table */
#define RF_LENGTH 8     /* length of one kick's section, L/nKicks */
#define RF_NKICKS 9
#define RF_MATRIX 10    /* 1: matrix method (nonzero L, N_KICKS <= 0) */
#define RF_DTLIGHT 11   /* RF_LENGTH / c */
#define RF_DRIFT_ONLY 12 /* VOLT = 0: an exact drift over L (nothing for L = 0) */
#define RF_FID_MODE 13  /* B2E_FIDUCIAL_* */
#define RF_L_TOTAL 14   /* L, for the light fiducial's zEnd - L */
#define RF_LEADER 15    /* RF state slot of the first cavity with the same PHASE_REFERENCE, -1: none */

/* WATCH constant slots */
#define WA_START 0      /* first pass recorded */
#define WA_END 1        /* last pass recorded, -1: no end */
#define WA_INTERVAL 2
#define WA_ORDINAL 3    /* index among the lattice's recording WATCH elements */

/* MALIGN constant slots */
#define MA_DX 0
#define MA_DXP 1
#define MA_DY 2
#define MA_DYP 3
#define MA_DZ 4
#define MA_DT 5
#define MA_DP 6
#define MA_DE 7
#define MA_ON_PASS 8    /* -1: every pass */
#define MA_START_PID 9  /* -1: every particle */
#define MA_END_PID 10
#define MA_C 11         /* c_mks */

/* DRIF / EDRIFT slots */
#define DR_L 0
#define DR_LH 1         /* L/2, the T[4][1][1] coefficient */

typedef struct {
  int32_t kind;
  int32_t flags;
  int32_t ap_pass0;   /* aperture record active during/after this element on pass 0 (-1: none) */
  int32_t ap_later;   /* same, on later passes */
  double z_start;     /* do_tracking last_z */
  double z_end;       /* do_tracking z after the element */
  double rev_cos, rev_sin; /* reverse tilt for internal aperture checks */
  double c[B2E_NC];
} DevElem;

typedef struct {
  double c[B2E_NRAD];
} DevRad;

typedef struct {
  double x_max, y_max;
  double a2, b2;        /* ipow(x_max, xe), ipow(y_max, ye) */
  int32_t elliptical, xe, ye;
  int32_t mode; /* check after the element: 0 none, 1 rectangular, 2 elliptical */
} DevAperture;

/* Per RFCA per instance: fiducial time and phase (phase_reference.c state). */
typedef struct {
  double phase_fiducial; /* -omega*t0 of the fiducial time (the phase reference other cavities may share) */
  double phase;   /* phase_fiducial + PHASE*PI/180 */
  int32_t set, pad;
} DevRfState;

/* Launch description of one tile: a block tracks particles [start, start+count) of instance inst. */
typedef struct {
  int64_t start;
  int32_t count;
  int32_t inst;
} DevTile;

typedef struct {
  double *x, *xp, *y, *yp, *s, *dp;
  int32_t *lost_pass;
  int32_t *lost_elem;
} DevParticles;

typedef struct {
  double p_central;
  double coord_limit;
  double slope_limit;
} DevGlobals;

#endif
