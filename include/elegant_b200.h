/*
 * elegant_b200 -- C ABI of the B200 particle-tracking engine.
 *
 * The engine replaces, for one GPU, the per-element tracking calls that
 * elegant's do_tracking() (do_tracking.c:144) makes for the hot-path element
 * subset.  In the reference those calls are, per element and per pass:
 *   track_particles (DRIF, matrix.c:294, called at do_tracking.c:1280)
 *   exactDrift (EDRIFT, csbend.c:3767, do_tracking.c:1997)
 *   multipole_tracking2 (KQUAD/KSEXT, multipole.c:693, do_tracking.c:2013, :2024)
 *   track_through_csbend (CSBEND, csbend.c:665, do_tracking.c:1949)
 *   simple_rf_cavity (RFCA, simple_rfca.c:264, do_tracking.c:1576)
 *   track_through_csbendCSR (CSRCSBEND, csbend.c:1899, do_tracking.c:1977)
 *   track_through_driftCSR (CSRDRIFT, csbend.c:3176, do_tracking.c:1984)
 *   limit_amplitudes / elimit_amplitudes (apertures, limit_amplitudes.c:193,
 *     :472, do_tracking.c:2459-2468)
 * and the GPU hooks gpuElegant adds inside each of them
 * (gpu_multipole_tracking2, gpu_track_through_csbend, ...; gpu_multipole.h,
 * gpu_csbend.h, gpu_simple_rfca.h:11, gpu_limit_amplitudes.h:14,29).
 * Here one call tracks a whole run (all passes, all elements) with the
 * particles resident in HBM, so the host makes one call instead of
 * elements x passes calls.
 *
 * Conventions
 *  - Particles are structure-of-arrays FP64 columns x, xp, y, yp, s, delta
 *    (elegant's coordinate order, track.h:81-86) plus an int64 particle ID.
 *  - Every entry point returns B2E_OK (0) or a negative B2E_ERR_* code and
 *    never exits the process; b2e_last_error() describes the last failure.
 *  - A context owns one CUDA stream and the device buffers; use one context
 *    per host thread.  No global state: the reference's file-static CSR
 *    state (csrWake, csbend.h:27-63) is per context.
 *  - Lattice parameters use elegant's element-parameter names; slots not
 *    given take the defaults of elegant's parameter tables (track_data.c).
 */
#ifndef ELEGANT_B200_H
#define ELEGANT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define B2E_OK 0
#define B2E_ERR_ARG (-1)      /* invalid argument (null pointer, bad size) */
#define B2E_ERR_LATTICE (-2)  /* unsupported element or parameter value */
#define B2E_ERR_CUDA (-3)     /* CUDA runtime error */
#define B2E_ERR_NOMEM (-4)    /* device allocation failed */
#define B2E_ERR_STATE (-5)    /* call out of order (e.g. track before upload) */
#define B2E_ERR_TIMEOUT (-6)  /* a bounded device wait gave up */
#define B2E_ERR_DEVICE (-7)   /* the device reported a numerical fault flag */

/* ---- element types (names follow elegant's entity_name table) -------- */
#define B2E_DRIF 1
#define B2E_EDRIFT 2
#define B2E_KQUAD 3
#define B2E_KSEXT 4
#define B2E_CSBEND 5
#define B2E_RFCA 6
#define B2E_MAXAMP 7
#define B2E_MARK 8
#define B2E_CHARGE 9
#define B2E_CSRCSBEND 10
#define B2E_CSRDRIFT 11
#define B2E_MALIGN 12
#define B2E_WATCH 13

#define B2E_MAX_PARAMS 40
#define B2E_RING_VARIANTS 17

/* Parameter slot indices, per element type.  Slot names are elegant's
 * parameter names (track_data.c tables cited per type). */
/* DRIF  (drift_param, track_data.c:450) */
#define B2E_DRIF_L 0
#define B2E_DRIF_ORDER 1
/* EDRIFT (edrift_param, track_data.c:3174) */
#define B2E_EDRIFT_L 0
/* KQUAD (kquad_param, track_data.c:1222) and KSEXT (ksext_param, :1120) share slots */
#define B2E_KMULT_L 0
#define B2E_KMULT_K 1 /* K1 for KQUAD, K2 for KSEXT */
#define B2E_KMULT_TILT 2
#define B2E_KMULT_DX 3
#define B2E_KMULT_DY 4
#define B2E_KMULT_DZ 5
#define B2E_KMULT_FSE 6
#define B2E_KMULT_N_KICKS 7
#define B2E_KMULT_N_SLICES 8
#define B2E_KMULT_INTEGRATION_ORDER 9
#define B2E_KMULT_K1_OF_KSEXT 10 /* KSEXT K1 (quadrupole error term) */
#define B2E_KMULT_J1_OF_KSEXT 11 /* KSEXT J1 (skew quadrupole error term) */
#define B2E_KMULT_SYNCH_RAD 12    /* classical synchrotron radiation (multipole.c:1320-1349) */
#define B2E_KMULT_ISR 13          /* incoherent synchrotron radiation (quantum excitation) */
#define B2E_KMULT_ISR1PART 14     /* ISR also for a one-particle beam (default 1; 0 is not supported) */
#define B2E_KMULT_HKICK 15        /* horizontal steering kick (rad), spread over the integrator's kicks */
#define B2E_KMULT_VKICK 16        /* vertical steering kick (rad) */
#define B2E_KMULT_HCALIBRATION 17 /* factor on HKICK (default 1) */
#define B2E_KMULT_VCALIBRATION 18 /* factor on VKICK (default 1) */
#define B2E_KMULT_BORE 19         /* bore radius (m); nonzero: the strength comes from the pole-tip field B */
#define B2E_KMULT_B 20            /* pole-tip field (T), used when BORE is nonzero */
/* KQUAD fringe fields (quadFringe, fringe.c:24-175): EDGE[12]_EFFECTS +-1 linear,
 * +-2 linear and third order (negative: without the x, y terms); the fringe
 * integrals I0..I3 and LAMBDA2 of each side, the linear part on/off, a factor
 * on the nonlinear part */
#define B2E_KMULT_EDGE1_EFFECTS 21
#define B2E_KMULT_EDGE2_EFFECTS 22
#define B2E_KMULT_EDGE1_LINEAR 23            /* default 1 */
#define B2E_KMULT_EDGE2_LINEAR 24            /* default 1 */
#define B2E_KMULT_EDGE1_NONLINEAR_FACTOR 25  /* default 1 */
#define B2E_KMULT_EDGE2_NONLINEAR_FACTOR 26  /* default 1 */
#define B2E_KMULT_I0P 27 /* I0P, I1P, I2P, I3P, LAMBDA2P: 27..31 */
#define B2E_KMULT_I0M 32 /* I0M, I1M, I2M, I3M, LAMBDA2M: 32..36 */
#define B2E_KMULT_LEFFECTIVE 37 /* KQUAD effective length (> 0: exact end drifts of (L - LEFFECTIVE)/2) */
/* CSBEND (csbend_param, track_data.c:1893) and CSRCSBEND (csrcsbend_param, :1982) */
#define B2E_BEND_L 0
#define B2E_BEND_ANGLE 1
#define B2E_BEND_E1 2
#define B2E_BEND_E2 3
#define B2E_BEND_TILT 4
#define B2E_BEND_ETILT 5
#define B2E_BEND_DX 6
#define B2E_BEND_DY 7
#define B2E_BEND_DZ 8
#define B2E_BEND_FSE 9
#define B2E_BEND_HGAP 10
#define B2E_BEND_FINT 11
#define B2E_BEND_N_SLICES 12 /* N_KICKS is an alias (track_data.c:1925, :2006) */
#define B2E_BEND_INTEGRATION_ORDER 13
#define B2E_BEND_EDGE1_EFFECTS 14
#define B2E_BEND_EDGE2_EFFECTS 15
#define B2E_BEND_EDGE_ORDER 16
#define B2E_BEND_K1 17
#define B2E_BEND_K2 18
#define B2E_BEND_NONLINEAR 19 /* CSBEND: 1 (default) includes the nonlinear expansion terms of K1/K2 */
/* CSRCSBEND-only slots */
#define B2E_BEND_BINS 20
#define B2E_BEND_BIN_RANGE_FACTOR 21
#define B2E_BEND_SG_HALFWIDTH 22
#define B2E_BEND_SG_ORDER 23
#define B2E_BEND_SGDERIV_HALFWIDTH 24
#define B2E_BEND_SGDERIV_ORDER 25
#define B2E_BEND_TRAPAZOID_INTEGRATION 26
#define B2E_BEND_STEADY_STATE 27
#define B2E_BEND_CSR 28
#define B2E_BEND_CLIP_NEGATIVE_BINS 29
#define B2E_BEND_IGF 30 /* integrated Green's function, steady state only (csbend.c:2593-2621) */
/* CSRCSBEND histogram filters (applyLHPassFilters, csbend.c:2557-2562,
 * :4611-4703), in units of the Nyquist frequency; elegant's defaults are -1
 * (off): b2e_element_defaults sets them, a zero LOW_FREQUENCY_CUTOFF0 turns
 * the filter path on */
#define B2E_BEND_LOW_FREQUENCY_CUTOFF0 31
#define B2E_BEND_LOW_FREQUENCY_CUTOFF1 32
#define B2E_BEND_HIGH_FREQUENCY_CUTOFF0 33
#define B2E_BEND_HIGH_FREQUENCY_CUTOFF1 34
/* CSBEND radiation (csbend.c:964-977, :1603-1622; edges :1211-1276); not on CSRCSBEND */
#define B2E_BEND_SYNCH_RAD 35
#define B2E_BEND_ISR 36
#define B2E_BEND_ISR1PART 37
#define B2E_BEND_XKICK 38 /* CSBEND bend-plane steering: the field term b0 = XKICK/ANGLE (csbend.c:867) */
#define B2E_BEND_YKICK 39 /* CSBEND non-bend-plane steering: the skew term c0 = YKICK/ANGLE (csbend.c:868) */
/* RFCA (rfca_param, track_data.c:576) */
#define B2E_RFCA_L 0
#define B2E_RFCA_VOLT 1
#define B2E_RFCA_PHASE 2
#define B2E_RFCA_FREQ 3
#define B2E_RFCA_DX 4
#define B2E_RFCA_DY 5
#define B2E_RFCA_T_REFERENCE 6
#define B2E_RFCA_N_KICKS 7 /* with L > 0: 0 = matrix method, else drift-kick-drift sections (simple_rfca.c:403-408) */
#define B2E_RFCA_FIDUCIAL 8 /* FIDUCIAL mode (simple_rfca.c:22-27, :62-257): B2E_FIDUCIAL_* */
#define B2E_RFCA_PHASE_REFERENCE 9 /* nonzero: cavities with the same number share the first one's fiducial
                                    * phase (get/set_phase_reference, simple_rfca.c:410-470) */
#define B2E_FIDUCIAL_TMEAN 0    /* mean arrival time, Kahan sum (the default) */
#define B2E_FIDUCIAL_LIGHT 1    /* (zEnd - L + L/2/nKicks)/c */
#define B2E_FIDUCIAL_PMAXIMUM 2 /* arrival time of the highest-momentum particle */
/* MAXAMP (maxamp_param, track_data.c:990) */
#define B2E_MAXAMP_X_MAX 0
#define B2E_MAXAMP_Y_MAX 1
#define B2E_MAXAMP_ELLIPTICAL 2
#define B2E_MAXAMP_EXPONENT 3
#define B2E_MAXAMP_Y_EXPONENT 4 /* elegant name: YEXPONENT; 0 = EXPONENT */
/* CHARGE (charge_param, track_data.c:2488) */
#define B2E_CHARGE_TOTAL 0
#define B2E_CHARGE_PER_PARTICLE 1
/* CSRDRIFT (csrdrift_param, track_data.c:2543) */
#define B2E_CSRDRIFT_L 0
#define B2E_CSRDRIFT_N_KICKS 1
#define B2E_CSRDRIFT_DZ 2
#define B2E_CSRDRIFT_CSR 3
#define B2E_CSRDRIFT_USE_STUPAKOV 4
/* MALIGN (malign_param, track_data.c:926-940; offset_beam, do_tracking.c:3243-3300;
 * applied on pass ON_PASS, or every pass for -1, do_tracking.c:1818-1821) */
#define B2E_MALIGN_DXP 0
#define B2E_MALIGN_DYP 1
#define B2E_MALIGN_DX 2
#define B2E_MALIGN_DY 3
#define B2E_MALIGN_DZ 4
#define B2E_MALIGN_DT 5
#define B2E_MALIGN_DP 6
#define B2E_MALIGN_DE 7
#define B2E_MALIGN_ON_PASS 8   /* default -1 */
#define B2E_MALIGN_START_PID 9 /* default -1: every particle */
#define B2E_MALIGN_END_PID 10  /* default -1 */
/* WATCH (watch_param, track_data.c:880-900): on every INTERVAL-th pass from
 * START_PASS to END_PASS (inclusive, -1: no end) the coordinates of the
 * particles alive at the element are recorded when b2e_set_watch enables it
 * (the element never changes them); the coordinate, parameter and centroid
 * modes all record coordinates (the caller reduces them, e.g.
 * elegant_b200.sdds.write_watch).  DISABLE = 1 makes it a marker.  The
 * engine rejects the fft mode, FRACTION != 1 and SPARSE_INTERVAL != 1;
 * START_PID/END_PID select rows of the output, not the recording. */
#define B2E_WATCH_START_PASS 0
#define B2E_WATCH_END_PASS 1      /* default -1 */
#define B2E_WATCH_INTERVAL 2      /* default 1 */
#define B2E_WATCH_DISABLE 3
#define B2E_WATCH_MODE 4          /* 0 = "coordinates", 1 = "parameter", 2 = "centroid", 3 = "fft" */
#define B2E_WATCH_FRACTION 5      /* default 1 */
#define B2E_WATCH_START_PID 6     /* default -1 */
#define B2E_WATCH_END_PID 7       /* default -1 */
#define B2E_WATCH_SPARSE_INTERVAL 8 /* default 1 */
/* shape only the output file, which the caller writes (the engine ignores them) */
#define B2E_WATCH_X_DATA 9        /* default 1 */
#define B2E_WATCH_Y_DATA 10       /* default 1 */
#define B2E_WATCH_LONGIT_DATA 11  /* default 1 */
#define B2E_WATCH_EXCLUDE_SLOPES 12
#define B2E_WATCH_FLUSH_INTERVAL 13 /* default 100 */
#define B2E_WATCH_USE_DISCONNECT 14
#define B2E_WATCH_INDEX_OFFSET 15
#define B2E_WATCH_REFERENCE_FREQUENCY 16 /* default -1 */
#define B2E_WATCH_AUTO_REFERENCE 17

typedef struct {
  int32_t type;             /* B2E_DRIF ... */
  int32_t reserved;
  char name[32];            /* element name; adjacent bends with equal names share edges */
  double p[B2E_MAX_PARAMS]; /* parameter slots, see indices above */
} b2e_element;

/* Per-instance parameter overrides for batched ensembles: instance i
 * replaces slot `slot` of element `element` with values[i]. */
typedef struct {
  int32_t element;
  int32_t slot;
  const double *values; /* n_instances values (host memory) */
} b2e_override;

/* Run options (elegant &run_setup / &track subset). */
typedef struct {
  double p_central;        /* reference momentum beta*gamma (run_setup p_central) */
  int32_t n_passes;        /* &track n_passes */
  int32_t default_order;   /* run_setup default_order for DRIF (2) */
  double coord_limit;      /* global_settings coord_limit (10 m) */
  double slope_limit;      /* global_settings slope_limit (1) */
  int32_t passes_per_launch; /* 0 = all passes of a step in one launch */
  int32_t ring_variant;    /* ring-kernel variant (occupancy target x warp barrier level):
                              0 = autotune on first use, 1..B2E_RING_VARIANTS = fixed
                              (all variants give identical results) */
  int32_t record_history;  /* nonzero: keep per-instance, per-pass survivors, centroids and
                              rms emittances (b2e_ensemble_history) */
  int32_t compact_every;   /* > 0: every this many passes (after pass 0), move each instance's
                              surviving particles to the front of its range and launch only
                              them; the order of rows changes, IDs travel with them.  Not with
                              record_history or device-owned columns. */
  double sr_gaussian_limit; /* global_settings SR_gaussian_limit: ISR deviates beyond this many
                               sigma are redrawn; 0 = elegant's default 3, < 0 = no cut */
  uint64_t isr_seed;        /* seed of the ISR deviates, which are addressed by (particle ID,
                               pass, element, slice, step): a run is reproducible and does not
                               depend on launch shape or compaction */
  int32_t record_tbt;       /* nonzero: keep every particle's x, x', y, y' at the start of a
                               call and after each of its passes (b2e_tbt, b2e_tbt_tunes).  Not
                               with compact_every, CSR elements or device-owned columns. */
  int32_t fiducial_particles; /* > 0: only the first this many rows of each instance set the
                                 RF phase reference on pass 0 (elegant's separate fiducial
                                 particle, e.g. frequencyMap.c:180-195); 0 = all particles */
} b2e_run_options;

typedef struct b2e_ctx b2e_ctx;

/* ---- lifecycle --------------------------------------------------------- */
int b2e_create(b2e_ctx **ctx, int device);
int b2e_destroy(b2e_ctx *ctx);
const char *b2e_last_error(const b2e_ctx *ctx);
int b2e_version(void);

/* ---- lattice ----------------------------------------------------------- */
/* Fill *element with elegant's parameter defaults for `type` (the tables of
 * track_data.c for the supported parameters; zero elsewhere) and set its
 * type; the name is left as it is.  A caller sets the parameters it gives on
 * top.  Returns B2E_ERR_ARG for an unknown type.  No device needed. */
int b2e_element_defaults(int32_t type, b2e_element *element);

/* Replaces the parsed element list that do_tracking walks (ELEMENT_LIST,
 * track.h:290-344) with a flat array.  Parameters are validated here. */
int b2e_load_lattice(b2e_ctx *ctx, const b2e_element *elements, int32_t n_elements,
                     const b2e_run_options *options);

/* ---- particles (host buffers) ----------------------------------------- */
/* Uploads n particles as columns x, xp, y, yp, s, delta (host pointers) and
 * their IDs.  Replaces the host->device copy that gpuElegant performs on
 * residency change (gpu_base.cu setElementGpuData). */
int b2e_upload_particles(b2e_ctx *ctx, const double *const columns[6], const int64_t *ids, int64_t n);

/* Tracks the resident particles for options->n_passes more passes
 * (elegant's do_tracking pass loop, do_tracking.c:488).  The first call after
 * b2e_upload_particles starts at pass 0; later calls continue the same run
 * (pass numbers, RFCA fiducials and loss records carry over).  *effort
 * receives the sum over this call's passes of the survivors at the end of
 * each pass (do_tracking.c:2758-2764). */
int b2e_track(b2e_ctx *ctx, double *effort);

/* The CUDA stream (cudaStream_t) all of the context's work is queued on. */
void *b2e_stream(b2e_ctx *ctx);

/* Number of kernels this context has launched so far (instrumentation). */
int64_t b2e_kernel_launches(const b2e_ctx *ctx);

/* Ring-kernel autotuning result: the variant in use (0 = not tuned yet) and
 * the time of one pass per variant in ms (B2E_RING_VARIANTS floats, may be NULL). */
int b2e_ring_tuning(const b2e_ctx *ctx, int32_t *chosen, float *ms_per_variant);

/* Downloads survivors and losses.  Columns receive all n particles in upload
 * order; lost_pass[i] is -1 for survivors or the pass on which particle i
 * was lost (elegant's lossPass column, track.h:89, do_tracking.c:4584);
 * lost_element[i] is the index of the element where it was lost (or -1). */
int b2e_download(b2e_ctx *ctx, double *const columns[6], int64_t *ids, int32_t *lost_pass,
                 int32_t *lost_element, int64_t *n_left);

/* One call for the whole drop-in path with host buffers: upload, track,
 * download.  This is what a host program linked in place of the per-element
 * calls invokes. */
int b2e_track_host(b2e_ctx *ctx, double *const columns[6], int64_t *ids, int64_t n, int32_t *lost_pass,
                   int32_t *lost_element, int64_t *n_left, double *effort);

/* ---- device-resident variant (no host copies) ------------------------- */
/* Columns are device pointers owned by the caller, tracked in place. */
int b2e_track_device(b2e_ctx *ctx, double *const dev_columns[6], const int64_t *dev_ids, int64_t n,
                     int32_t *dev_lost_pass, int32_t *dev_lost_element, double *effort);

/* ---- batched ensembles ------------------------------------------------- */
/* n_instances lattice copies; instance i owns particles
 * [offsets[i], offsets[i+1]).  overrides apply per instance.  Each instance
 * has its own RFCA fiducial.  Particles are host columns, as for
 * b2e_upload_particles. */
int b2e_load_ensemble(b2e_ctx *ctx, int32_t n_instances, const int64_t *offsets, const b2e_override *overrides,
                      int32_t n_overrides);

/* Per-instance diagnostics after each pass: survivors, centroids <x>, <y>,
 * and rms emittances ex, ey (rms_emittance, final_props.c:844).  Requires
 * record_history in the run options and a lattice without CSR elements.
 * Buffers are host arrays of n_instances * b2e_history_passes() values,
 * instance-major; any may be NULL.  The record covers every pass tracked
 * since the last b2e_upload_particles (b2e_track continuations append). */
int b2e_ensemble_history(b2e_ctx *ctx, int64_t *survivors, double *cx, double *cy, double *ex, double *ey);
/* Passes recorded so far, or -1 for a null context. */
int64_t b2e_history_passes(const b2e_ctx *ctx);

/* ---- turn-by-turn data and tunes --------------------------------------- */
/* Turn-by-turn coordinates of the last b2e_track / b2e_track_host call made
 * with record_tbt: host array [records][4][n] (x, x', y, y'), record 0 the
 * coordinates at the call's start, record j those after its j-th pass (rows
 * in the uploaded order; a lost particle's records after its loss are NaN).
 * *written = records * 4 * n; with host_out NULL only *written is set.
 * Replaces the per-turn bookkeeping of computeTunesFromTracking
 * (twiss.cc:3885-3925). */
int b2e_tbt(b2e_ctx *ctx, double *host_out, int64_t capacity, int64_t *written);

/* WATCH coordinate recording (dump_watch_particles, sdds_support.c:703-860,
 * called at do_tracking.c:1585-1635).  b2e_set_watch(max_bytes > 0) turns it
 * on: each b2e_track / b2e_track_host call then keeps, for every WATCH
 * element (lattice order) and every pass of the call it records, one record
 * of 7 columns x rows (the context's particle rows): x, x', y, y', s, delta
 * and the particle ID as a double, NaN in the rows of particles not alive
 * at the element.  A call whose records would exceed max_bytes fails with
 * B2E_ERR_ARG before tracking.  b2e_watch_records gives the number of
 * records, the row count and each record's element index and pass (up to
 * capacity entries); b2e_watch_data copies one record ([7][rows]) to host
 * memory.  A recording call launches the ring kernel at least once per pass
 * (it stops at each recording WATCH).  Not with per-instance overrides of
 * WATCH elements. */
int b2e_set_watch(b2e_ctx *ctx, int64_t max_bytes);
int b2e_watch_records(b2e_ctx *ctx, int32_t *n_records, int64_t *rows, int32_t *elements, int32_t *passes,
                      int32_t capacity);
int b2e_watch_data(b2e_ctx *ctx, int32_t record, double *host_out);

/* Tunes of every particle from records [first_record, first_record +
 * n_records) of the turn-by-turn data, as computeTunesFromTracking does
 * (twiss.cc:3942-4022): the strongest frequency of x, x', y and y' by NAFF
 * (one frequency, Hann window, refined to 1e-12 of a turn by golden-section
 * search; the toolkit's PerformNAFF is not in the reference tree, so the
 * method is this library's), then adjustTuneHalfPlane (twiss.cc:4036-4046)
 * from the phases of x and x' (y and y').  Host arrays of n values; a
 * particle lost before the window's last record gets -1 in nux/nuy.  Runs
 * on the device; needs 4 <= n_records <= 8192. */
int b2e_tbt_tunes(b2e_ctx *ctx, int32_t first_record, int32_t n_records, double *nux, double *nuy, double *ax,
                  double *ay);

/* NAFF of n_signals device-resident signals of n_points each (signal s at
 * dev_signals + s * n_points), the strongest frequency in [0, 0.5] cycles per
 * sample with its amplitude and phase, written to device arrays of
 * n_signals values; the same method as b2e_tbt_tunes. */
int b2e_naff(const double *dev_signals, int64_t n_signals, int32_t n_points, double *dev_frequency,
             double *dev_amplitude, double *dev_phase, void *stream);

/* ---- CSR (CSRCSBEND / CSRDRIFT) ---------------------------------------- */
/* Wake arrays of every CSR kick of the last b2e_track call: for each
 * CSRCSBEND kick, BINS values of dGamma (csbend.c:2673) in kick order. */
int b2e_csr_wakes(b2e_ctx *ctx, double *wakes, int64_t capacity, int64_t *written);

/* What CSRCSBEND's OUTPUT_FILE holds (csbend.c:2227-2249 layout, one page
 * per kick written at :2762-2806).  With recording on (off by default), every
 * plain-integral kick of the following runs keeps, per bunch, a record of
 * B2E_CSR_PAGE_HEADER values -- element index, kick, bunch, BINS, the binned
 * range ctLower and ctUpper, the bin width dct, the slippage length, the
 * accumulated bend angle phiBend, the kick length L/N_KICKS, pCentral, the
 * bunch's macro-particle charge -- followed by BINS values each of the smoothed line
 * density per unit c*t (ctHist), its derivative (ctHistDeriv), and the wake
 * terms T1 and T2 (csbend.c:2664-2667); a bunch without CSR on that kick
 * has element index -1 and undefined arrays.  The file's columns follow from these:
 * LinearDensity = ctHist * (q_macro c), LinearDensityDeriv = ctHistDeriv *
 * (q_macro c^2 / dct), DeltaGamma = T1 + T2, GammaDeriv = DeltaGamma /
 * (L/N_KICKS), s = ctLower - (ctLower + ctUpper)/2 + dct (i + 1/2) (the
 * reference's expressions; elegant_b200.sdds.write_csr_wake writes the
 * file).  b2e_csr_pages copies the records of the last run
 * (*written = values; NULL to query).  Not with the learned wake, whose kicks
 * record no page.  No counterpart as an API in the reference. */
/* Timing of the CSR wake stage: with timing on, each CSRCSBEND kick of the
 * following runs brackets its wake stage -- the plain wake kernel, or the
 * learned wake's filter, network and combine kernels -- with CUDA events on
 * the context's stream.  b2e_csr_timing waits for the last run's events and
 * returns their summed device time in ms, the timed kicks and how many of
 * them took the learned wake.  No counterpart in the reference. */
int b2e_set_csr_timing(b2e_ctx *ctx, int32_t on);
int b2e_csr_timing(b2e_ctx *ctx, double *wake_ms, int64_t *kicks, int64_t *learned_kicks);

#define B2E_CSR_PAGE_HEADER 12
int b2e_set_csr_pages(b2e_ctx *ctx, int32_t record);
int b2e_csr_pages(b2e_ctx *ctx, double *pages, int64_t capacity, int64_t *written);

/* ---- batched wake integral (wake-network data) ------------------------
 * For each of n_profiles histograms (dev_counts: [n_profiles][bins] real
 * counts, bin width 1) the CSRCSBEND wake pipeline of one kick
 * (csbend.c:2566-2673: Savitzky-Golay smoothing, correctDistribution,
 * derivative filter, transient or steady-state integral) with the slippage
 * dev_slippage_bins[p] in bins.  Outputs, all [n_profiles][bins] FP64:
 * dev_t1 = the integral term T1 alone (CSR constant 1, no T2 term),
 * dev_density = the smoothed density, dev_derivative = its derivative.  The
 * wake of a kick with bin width dct is then
 *   CSRConstant * L / N_KICKS * dct^(-4/3) * (T1 - (hist[i+diS] - hist[i+diS4]) / s^(1/3)).
 * No counterpart in the reference (it evaluates one wake per kick). */
int b2e_csr_wake_batch(const double *dev_counts, const double *dev_slippage_bins, int32_t n_profiles, int32_t bins,
                       int32_t sg_halfwidth, int32_t sg_order, int32_t sgd_halfwidth, int32_t sgd_order,
                       int32_t trapezoid, int32_t steady, double *dev_t1, double *dev_density, double *dev_derivative,
                       void *stream);

/* Network inputs and back-transform for batched profiles, as the tracking
 * path forms them per kick (one CTA per profile, no host glue):
 * b2e_wake_features reads dev_density and dev_derivative ([n][bins] FP64,
 * bin units, from b2e_csr_wake_batch) and the slippage in bins, and writes
 * dev_inputs [n][4][bins] FP32 -- density and derivative over their total,
 * times k = 1/rms(derivative/total) and the channel scales, the code
 * log2(diS)/log2(bins) with diS = clamp(floor(s), 1, bins), and the scaled
 * density at bin i + diS (zero past the end; all zero when shift is 0) --
 * and dev_scales [n][2] (total, k).  b2e_wake_t1_from_output turns the
 * network output dev_y [n][bins] back into T1 = y / target_scale / k * total
 * (zero for a slippage under one bin).  No counterpart in the reference. */
int b2e_wake_features(const double *dev_density, const double *dev_derivative, const double *dev_slippage_bins,
                      int32_t n_profiles, int32_t bins, double density_scale, double derivative_scale, int32_t shift,
                      float *dev_inputs, double *dev_scales, void *stream);
int b2e_wake_t1_from_output(const float *dev_y, const double *dev_scales, const double *dev_slippage_bins,
                            int32_t n_profiles, int32_t bins, double target_scale, double *dev_t1, void *stream);

/* ---- wake network (learned CSR wake integral) --------------------------
 * A 6-layer 1-D convolutional network (64 channels, 5 taps, per-layer
 * dilations, GELU) that maps a binned profile -- smoothed density, its
 * derivative, a slippage code and the density shifted by the slippage,
 * [n][4][bins] FP32 on the device -- to the
 * wake integral T1 of b2e_csr_wake_batch, [n][bins] FP32, in the scaled units
 * the caller trains it in.  BF16 weights and activations, FP32 accumulation
 * on the tensor cores; the optimiser is Adam on FP32 master weights.
 * Parameters are a flat FP32 array of b2e_wakenet_param_count() values:
 * weights [layer][tap][out][in] (6 x 5 x 64 x 64), then biases [layer][64].
 * The reference has no learned component; this is an addition. */
typedef struct b2e_wakenet b2e_wakenet;
int b2e_wakenet_create(b2e_wakenet **out, int32_t bins, int32_t max_batch, const int32_t *dilations, int32_t device);
int b2e_wakenet_destroy(b2e_wakenet *net);
const char *b2e_wakenet_last_error(const b2e_wakenet *net);
int64_t b2e_wakenet_param_count(void);
/* Replaces the parameters (and resets the optimiser state). */
int b2e_wakenet_set_params(b2e_wakenet *net, const float *host_params);
/* Copies parameters and/or the last gradients (either may be NULL). */
int b2e_wakenet_get_params(b2e_wakenet *net, float *host_params, float *host_grads);
/* Inference: dev_out[n][bins] from dev_inputs[n][4][bins]. */
int b2e_wakenet_forward(b2e_wakenet *net, const float *dev_inputs, int32_t n, float *dev_out, void *stream);
/* Forward + backward of the mean squared error against dev_targets[n][bins];
 * gradients are kept for b2e_wakenet_get_params; *loss (host, may be NULL). */
int b2e_wakenet_gradients(b2e_wakenet *net, const float *dev_inputs, const float *dev_targets, int32_t n,
                          double *loss, void *stream);
/* One Adam step (learning rate lr) on one batch; *loss as above (NULL skips
 * the host synchronisation). */
int b2e_wakenet_train_step(b2e_wakenet *net, const float *dev_inputs, const float *dev_targets, int32_t n, float lr,
                           double *loss, void *stream);

/* ---- CSR with a bunch spread over several GPUs -------------------------
 * Each rank holds part of every bunch (same bunch layout on every rank).  At
 * the reference's exchange points (csbend.c:2532-2550, findGlobalMinMax.c)
 * the engine calls `fn` on device buffers of its own stream: the min/max of
 * c*t per bunch (B2E_REDUCE_MIN_U64 / MAX_U64 on order-preserving keys), the
 * histogram counts per bunch (B2E_REDUCE_SUM_U32, bunch-major), and the
 * particle counts per bunch (B2E_REDUCE_SUM_U64: alive at an element, and at
 * the start of a run for the macro-particle charge).  The callback must leave
 * the all-rank result in the buffer before later work on `stream` reads it
 * (for example an NCCL all-reduce enqueued on that stream) and return 0.
 * Every rank then bins, smooths and integrates the same global histogram, so
 * each particle receives the kick it would receive on one GPU.  fn = NULL
 * switches back to single-GPU bunches. */
#define B2E_REDUCE_MIN_U64 0
#define B2E_REDUCE_MAX_U64 1
#define B2E_REDUCE_SUM_U32 2
#define B2E_REDUCE_SUM_U64 3
typedef int (*b2e_reduce_fn)(void *user, int32_t op, void *dev_buf, int64_t count, void *stream);
int b2e_set_csr_reducer(b2e_ctx *ctx, b2e_reduce_fn fn, void *user);

/* ---- learned CSR wake in tracking --------------------------------------
 * Binds a trained wake network to a tracking context (net = NULL unbinds).
 * For CSRCSBEND kicks with the transient integral and the trapezoid rule
 * (the defaults), BINS <= the network's bins and at most its batch of
 * bunches, the network replaces the T1 integral of the kick wake; the T2
 * term, the filters and the kick stay exact.  feature_scales = the density,
 * derivative and target scales the network was trained with.  Every kick is
 * checked: the plain integral is evaluated at every gate_stride-th bin (a
 * different offset each kick) and, if the relative rms error of the wake
 * there exceeds tolerance, the kick uses the plain wake (bit-identical to the
 * plain path).  The network must outlive its use by the context.  No
 * counterpart in the reference. */
int b2e_set_csr_surrogate(b2e_ctx *ctx, b2e_wakenet *net, const double feature_scales[3], double tolerance,
                          int32_t gate_stride);
/* Since the last run start: network wake evaluations (kicks x bunches),
 * fallbacks to the plain wake, and the gate's relative error of each
 * evaluation (in kick order, bunches within a kick; NULL to query *written). */
int b2e_csr_surrogate_stats(b2e_ctx *ctx, int64_t *evaluations, int64_t *fallbacks, double *gate_errors,
                            int64_t capacity, int64_t *written);

/* ---- tensor-core self-test ---------------------------------------------
 * Runs one UMMA tile on device buffers to check the operand layouts the wake
 * network uses.  mode 0: D[128][64] = A[128][64] . B[64][64]^T; mode 1:
 * D[m][n] = sum_k A[m/64][k][m%64] * B[k][n] with A [2][128][64], B [128][64].
 * A, B: BF16 row-major; D: FP32.  mode 2 is a drill of the bounded waits:
 * the kernel waits on a load that is never issued, gives up after a short
 * poll limit, frees its tensor memory and returns B2E_ERR_TIMEOUT (buffers
 * unused, may be NULL).  No counterpart in the reference. */
int b2e_umma_selftest(int mode, const void *dev_a, const void *dev_b, float *dev_d, void *stream);

/* ---- division self-test -------------------------------------------------
 * Compares, on the device, a / b with the engine's division by a stored
 * reciprocal (Markstein's correction step) for every divisor in host_b and
 * `samples` numerators each, drawn with magnitudes 2^-40..2^40 and both signs
 * from `seed`; *mismatches = the pairs whose bits differ.  No counterpart in
 * the reference. */
int b2e_selftest_division(const double *host_b, int32_t n_b, int64_t samples, uint64_t seed, int64_t *mismatches);

/* ---- allocation-free CSR dipole ---------------------------------------
 * No counterpart in the reference: an addition for callers that cannot
 * allocate device memory when they track (a program whose memory pool owns
 * the whole card, code running where cudaMalloc is not allowed, or a job that
 * must not fail for lack of memory mid-run).  Tracks n caller-owned device
 * particles (columns x, xp, y, yp, s, delta; lost_pass/lost_element int32,
 * -1 = alive) through one CSRCSBEND, exactly as b2e_track does for that
 * element (same kernels, same results), writing the per-kick wakes
 * (N_KICKS x BINS values) to dev_wakes when it is non-NULL.  It allocates
 * nothing: all working memory is one static device array of ~10.2 MB in the
 * library image, for up to B2E_STATIC_MAX_PARTICLES particles and
 * B2E_STATIC_MAX_BINS bins; larger requests are rejected with B2E_ERR_ARG and
 * a message in errbuf.  The first call on a device is its set-up: with that
 * device current it looks up the array's device address, which is also when
 * CUDA (lazy module loading, the default) gives the array and the kernels'
 * code their device memory; the array then stays until the process exits.  A
 * caller whose memory pool will own the whole card makes that first call
 * (n = 0 is enough, with NULL particle buffers) before the pool takes the
 * memory, or runs with
 * CUDA_MODULE_LOADING=EAGER; the first call also comes before any stream
 * capture.  The set-up is per primary context: do not call this on a device
 * after cudaDeviceReset.  A call only enqueues work on the stream and returns
 * without waiting for the GPU.  All calls share the array and each clears
 * what it needs; calls that overlap on the GPU race on it and must be
 * serialised by the caller.  stream is a cudaStream_t (NULL = legacy default
 * stream).  p_central is beta*gamma; macro_particle_charge is CHARGE TOTAL
 * divided by the particle count. */
#define B2E_STATIC_MAX_PARTICLES 1048576
#define B2E_STATIC_MAX_BINS 2048
int b2e_csr_bend_static(double *const dev_columns[6], int32_t *dev_lost_pass, int32_t *dev_lost_element, int64_t n,
                        const b2e_element *bend, double p_central, double macro_particle_charge, double *dev_wakes,
                        int64_t wake_capacity, void *stream, char *errbuf, int64_t errlen);

#ifdef __cplusplus
}
#endif

#endif
