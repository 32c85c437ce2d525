/*
 * b2e_adapter.c -- elegant's element list into the engine's C ABI (see
 * b2e_adapter.h for where do_tracking calls it).
 *
 * Parameters travel by elegant's own parameter tables: for every parameter
 * entity_description[type] lists (name, storage type, offset into the element
 * structure, default; track_data.c), the value is read from the element
 * structure at that offset.  A parameter with an engine slot is copied into
 * it; one without must still hold its table default, otherwise the line is
 * declined and stays on elegant's CPU path.  So the adapter never tracks an
 * element with a setting the engine would ignore, and it needs no per-field
 * code for the element structures.  The engine itself rejects values it does
 * not support in a slot it has (b2e_load_lattice), which also declines.
 */
#include "mdb.h"
#include "track.h"
#include "elegant_b200.h"
#include "b2e_adapter.h"
#include <string.h>

typedef struct {
  const char *name; /* elegant parameter name */
  int slot;         /* engine slot */
} b2e_param_map;

#define END_MAP {NULL, 0}
static const b2e_param_map map_drif[] = {{"L", B2E_DRIF_L}, {"ORDER", B2E_DRIF_ORDER}, END_MAP};
static const b2e_param_map map_edrift[] = {{"L", B2E_EDRIFT_L}, END_MAP};
#define KMULT_COMMON                                                                                              \
  {"L", B2E_KMULT_L}, {"TILT", B2E_KMULT_TILT}, {"DX", B2E_KMULT_DX}, {"DY", B2E_KMULT_DY}, {"DZ", B2E_KMULT_DZ}, \
      {"FSE", B2E_KMULT_FSE}, {"N_KICKS", B2E_KMULT_N_KICKS}, {"N_SLICES", B2E_KMULT_N_SLICES},                    \
      {"INTEGRATION_ORDER", B2E_KMULT_INTEGRATION_ORDER}, {"SYNCH_RAD", B2E_KMULT_SYNCH_RAD},                     \
      {"ISR", B2E_KMULT_ISR}, {"ISR1PART", B2E_KMULT_ISR1PART}, {"HKICK", B2E_KMULT_HKICK},                        \
      {"VKICK", B2E_KMULT_VKICK}, {"HCALIBRATION", B2E_KMULT_HCALIBRATION},                                       \
      {"VCALIBRATION", B2E_KMULT_VCALIBRATION}, {"BORE", B2E_KMULT_BORE}, {"B", B2E_KMULT_B},                     \
      /* read by no tracking code: optimizer flags, PITCH/YAW under MALIGN_METHOD 0 */                           \
      {"HSTEERING", -1}, {"VSTEERING", -1}, {"SQRT_ORDER", -1}, {"PITCH", -1}, {"YAW", -1}
static const b2e_param_map map_kquad[] = {KMULT_COMMON,
                                          {"K1", B2E_KMULT_K},
                                          {"SR_IN_ORDINARY_MATRIX", -1},
                                          {"TRACKING_MATRIX", -1},
                                          {"EDGE1_EFFECTS", B2E_KMULT_EDGE1_EFFECTS},
                                          {"EDGE2_EFFECTS", B2E_KMULT_EDGE2_EFFECTS},
                                          {"EDGE1_LINEAR", B2E_KMULT_EDGE1_LINEAR},
                                          {"EDGE2_LINEAR", B2E_KMULT_EDGE2_LINEAR},
                                          {"EDGE1_NONLINEAR_FACTOR", B2E_KMULT_EDGE1_NONLINEAR_FACTOR},
                                          {"EDGE2_NONLINEAR_FACTOR", B2E_KMULT_EDGE2_NONLINEAR_FACTOR},
                                          {"I0P", B2E_KMULT_I0P},
                                          {"I1P", B2E_KMULT_I0P + 1},
                                          {"I2P", B2E_KMULT_I0P + 2},
                                          {"I3P", B2E_KMULT_I0P + 3},
                                          {"LAMBDA2P", B2E_KMULT_I0P + 4},
                                          {"I0M", B2E_KMULT_I0M},
                                          {"I1M", B2E_KMULT_I0M + 1},
                                          {"I2M", B2E_KMULT_I0M + 2},
                                          {"I3M", B2E_KMULT_I0M + 3},
                                          {"LAMBDA2M", B2E_KMULT_I0M + 4},
                                          {"LEFFECTIVE", B2E_KMULT_LEFFECTIVE},
                                          END_MAP};
static const b2e_param_map map_ksext[] = {KMULT_COMMON,
                                          {"K2", B2E_KMULT_K},
                                          {"K1", B2E_KMULT_K1_OF_KSEXT},
                                          {"J1", B2E_KMULT_J1_OF_KSEXT},
                                          END_MAP};
#define BEND_COMMON                                                                                                \
  {"L", B2E_BEND_L}, {"ANGLE", B2E_BEND_ANGLE}, {"E1", B2E_BEND_E1}, {"E2", B2E_BEND_E2}, {"TILT", B2E_BEND_TILT}, \
      {"ETILT", B2E_BEND_ETILT}, {"DX", B2E_BEND_DX}, {"DY", B2E_BEND_DY}, {"DZ", B2E_BEND_DZ},                     \
      {"FSE", B2E_BEND_FSE}, {"HGAP", B2E_BEND_HGAP}, {"FINT", B2E_BEND_FINT}, {"N_SLICES", B2E_BEND_N_SLICES},   \
      {"N_KICKS", B2E_BEND_N_SLICES}, {"INTEGRATION_ORDER", B2E_BEND_INTEGRATION_ORDER},                         \
      {"EDGE1_EFFECTS", B2E_BEND_EDGE1_EFFECTS}, {"EDGE2_EFFECTS", B2E_BEND_EDGE2_EFFECTS},                        \
      {"EDGE_ORDER", B2E_BEND_EDGE_ORDER}, {"K1", B2E_BEND_K1}, {"K2", B2E_BEND_K2},                        \
      {"NONLINEAR", B2E_BEND_NONLINEAR}, {"XKICK", B2E_BEND_XKICK}, {"YKICK", B2E_BEND_YKICK}
static const b2e_param_map map_csbend[] = {
    BEND_COMMON, {"SYNCH_RAD", B2E_BEND_SYNCH_RAD}, {"ISR", B2E_BEND_ISR}, {"ISR1PART", B2E_BEND_ISR1PART}, END_MAP};
static const b2e_param_map map_csrcsbend[] = {BEND_COMMON,
                                              {"BINS", B2E_BEND_BINS},
                                              {"BIN_RANGE_FACTOR", B2E_BEND_BIN_RANGE_FACTOR},
                                              {"SG_HALFWIDTH", B2E_BEND_SG_HALFWIDTH},
                                              {"SG_ORDER", B2E_BEND_SG_ORDER},
                                              {"SGDERIV_HALFWIDTH", B2E_BEND_SGDERIV_HALFWIDTH},
                                              {"SGDERIV_ORDER", B2E_BEND_SGDERIV_ORDER},
                                              {"TRAPAZOID_INTEGRATION", B2E_BEND_TRAPAZOID_INTEGRATION},
                                              {"STEADY_STATE", B2E_BEND_STEADY_STATE},
                                              {"CSR", B2E_BEND_CSR},
                                              {"CLIP_NEGATIVE_BINS", B2E_BEND_CLIP_NEGATIVE_BINS},
                                              {"IGF", B2E_BEND_IGF},
                                              {"LOW_FREQUENCY_CUTOFF0", B2E_BEND_LOW_FREQUENCY_CUTOFF0},
                                              {"LOW_FREQUENCY_CUTOFF1", B2E_BEND_LOW_FREQUENCY_CUTOFF1},
                                              {"HIGH_FREQUENCY_CUTOFF0", B2E_BEND_HIGH_FREQUENCY_CUTOFF0},
                                              {"HIGH_FREQUENCY_CUTOFF1", B2E_BEND_HIGH_FREQUENCY_CUTOFF1},
                                              END_MAP};
/* PHASE_REFERENCE links cavities to one phase: the engine gives the later
 * cavities of a group the first one's fiducial phase, as elegant does. */
static const b2e_param_map map_rfca[] = {{"L", B2E_RFCA_L},         {"VOLT", B2E_RFCA_VOLT},
                                         {"PHASE", B2E_RFCA_PHASE}, {"FREQ", B2E_RFCA_FREQ},
                                         {"DX", B2E_RFCA_DX},       {"DY", B2E_RFCA_DY},
                                         {"T_REFERENCE", B2E_RFCA_T_REFERENCE}, {"N_KICKS", B2E_RFCA_N_KICKS},
                                         {"PHASE_REFERENCE", B2E_RFCA_PHASE_REFERENCE},
                                         END_MAP};
static const b2e_param_map map_maxamp[] = {{"X_MAX", B2E_MAXAMP_X_MAX},
                                           {"Y_MAX", B2E_MAXAMP_Y_MAX},
                                           {"ELLIPTICAL", B2E_MAXAMP_ELLIPTICAL},
                                           {"EXPONENT", B2E_MAXAMP_EXPONENT},
                                           {"YEXPONENT", B2E_MAXAMP_Y_EXPONENT},
                                           END_MAP};
static const b2e_param_map map_mark[] = {END_MAP};
static const b2e_param_map map_charge[] = {{"TOTAL", B2E_CHARGE_TOTAL}, {"PER_PARTICLE", B2E_CHARGE_PER_PARTICLE},
                                           END_MAP};
static const b2e_param_map map_csrdrift[] = {{"L", B2E_CSRDRIFT_L},     {"N_KICKS", B2E_CSRDRIFT_N_KICKS},
                                             {"DZ", B2E_CSRDRIFT_DZ},   {"CSR", B2E_CSRDRIFT_CSR},
                                             {"USE_STUPAKOV", B2E_CSRDRIFT_USE_STUPAKOV}, END_MAP};
static const b2e_param_map map_malign[] = {{"DXP", B2E_MALIGN_DXP},         {"DYP", B2E_MALIGN_DYP},
                                           {"DX", B2E_MALIGN_DX},           {"DY", B2E_MALIGN_DY},
                                           {"DZ", B2E_MALIGN_DZ},           {"DT", B2E_MALIGN_DT},
                                           {"DP", B2E_MALIGN_DP},           {"DE", B2E_MALIGN_DE},
                                           {"ON_PASS", B2E_MALIGN_ON_PASS}, {"START_PID", B2E_MALIGN_START_PID},
                                           {"END_PID", B2E_MALIGN_END_PID}, END_MAP};

/* elegant type -> engine type and parameter map; 0 = not in the engine's set */
static int engine_type(long type, const b2e_param_map **map) {
  switch (type) {
  case T_DRIF:
    *map = map_drif;
    return B2E_DRIF;
  case T_EDRIFT:
    *map = map_edrift;
    return B2E_EDRIFT;
  case T_KQUAD:
    *map = map_kquad;
    return B2E_KQUAD;
  case T_KSEXT:
    *map = map_ksext;
    return B2E_KSEXT;
  case T_CSBEND:
    *map = map_csbend;
    return B2E_CSBEND;
  case T_CSRCSBEND:
    *map = map_csrcsbend;
    return B2E_CSRCSBEND;
  case T_RFCA:
    *map = map_rfca;
    return B2E_RFCA;
  case T_MAXAMP:
    *map = map_maxamp;
    return B2E_MAXAMP;
  case T_MARK:
    *map = map_mark;
    return B2E_MARK;
  case T_CHARGE:
    *map = map_charge;
    return B2E_CHARGE;
  case T_CSRDRIFT:
    *map = map_csrdrift;
    return B2E_CSRDRIFT;
  case T_MALIGN:
    *map = map_malign;
    return B2E_MALIGN;
  case T_WATCH:
    /* a disabled WATCH only (see b2e_adapter_track): a marker */
    *map = map_mark;
    return B2E_MARK;
  default:
    return 0;
  }
}

static void say(char *why, long why_len, const char *fmt, const char *a, const char *b) {
  if (why && why_len > 0)
    snprintf(why, why_len, fmt, a, b);
}

/* The element's parameters into el->p; 0, or -1 (with a reason) when a
 * parameter without an engine slot is not at its table default. */
static int fill_parameters(b2e_element *el, const ELEMENT_LIST *eptr, const b2e_param_map *map, char *why,
                           long why_len) {
  const PARAMETER *par = entity_description[eptr->type].parameter;
  const char *p_elem = eptr->p_elem;
  long i;
  for (i = 0; i < entity_description[eptr->type].n_params; i++) {
    const char *where = p_elem + par[i].offset;
    const b2e_param_map *m = map;
    double value = 0;
    int is_default = 1;
    switch (par[i].type) {
    case IS_DOUBLE:
      value = *(const double *)where;
      is_default = value == par[i].number;
      break;
    case IS_LONG:
      value = (double)*(const long *)where;
      is_default = *(const long *)where == par[i].integer;
      break;
    case IS_SHORT:
      value = (double)*(const short *)where;
      is_default = *(const short *)where == (short)par[i].integer;
      break;
    case IS_STRING: {
      const char *s = *(char *const *)where;
      is_default = (!s && !par[i].string) || (s && par[i].string && strcmp(s, par[i].string) == 0);
      /* RFCA FIDUCIAL: elegant's own parser (parseFiducialMode, simple_rfca.c:35-48) picks the
       * mode; light, tmean and pmaximum go to the engine's slot, anything else declines */
      if (eptr->type == T_RFCA && strcmp(par[i].name, "FIDUCIAL") == 0) {
        const unsigned long mode = parseFiducialMode((char *)s);
        if (mode & FID_MODE_LIGHT)
          el->p[B2E_RFCA_FIDUCIAL] = B2E_FIDUCIAL_LIGHT;
        else if (mode & FID_MODE_PMAX)
          el->p[B2E_RFCA_FIDUCIAL] = B2E_FIDUCIAL_PMAXIMUM;
        else if (mode & FID_MODE_TMEAN)
          el->p[B2E_RFCA_FIDUCIAL] = B2E_FIDUCIAL_TMEAN;
        is_default = (mode & (FID_MODE_LIGHT | FID_MODE_PMAX | FID_MODE_TMEAN)) != 0;
      }
      break;
    }
    default:
      break;
    }
    while (m->name && strcmp(m->name, par[i].name) != 0)
      m++;
    if (m->name && par[i].type != IS_STRING) {
      if (m->slot >= 0)
        el->p[m->slot] = value;
    } else if (!is_default) {
      say(why, why_len, "%s: parameter %s is not supported by the engine", eptr->name, par[i].name);
      return -1;
    }
  }
  return 0;
}

static b2e_ctx *adapter_ctx = NULL;

void b2e_adapter_release(void) {
  if (adapter_ctx)
    b2e_destroy(adapter_ctx);
  adapter_ctx = NULL;
}

long b2e_adapter_track(double **coord, long np, ELEMENT_LIST *first, double P_central, long n_passes,
                       long default_order, double *effort_out, char *why, long why_len) {
  ELEMENT_LIST *eptr;
  long n = 0, i, j;
  b2e_element *el;
  b2e_run_options opt;
  double *cols[6] = {NULL, NULL, NULL, NULL, NULL, NULL}, effort = 0, *rows = NULL;
  int64_t *ids = NULL, n_left = 0;
  int32_t *lost_pass = NULL, *lost_elem = NULL;
  long status = -2;

  for (eptr = first; eptr; eptr = eptr->succ, n++) {
    const b2e_param_map *map;
    if (!engine_type(eptr->type, &map)) {
      say(why, why_len, "%s: element type %s is not supported by the engine", eptr->name, entity_name[eptr->type]);
      return -1;
    }
    /* elegant writes WATCH output itself (dump_watch_particles, at each
     * pass): a line with an active WATCH stays with elegant */
    if (eptr->type == T_WATCH && !((WATCH *)eptr->p_elem)->disable) {
      say(why, why_len, "%s: WATCH output is written by elegant%s", eptr->name, "");
      return -1;
    }
  }
  el = (b2e_element *)calloc(n ? n : 1, sizeof(*el));
  for (eptr = first, i = 0; eptr; eptr = eptr->succ, i++) {
    const b2e_param_map *map;
    const int code = engine_type(eptr->type, &map);
    b2e_element_defaults(code, &el[i]);
    strncpy(el[i].name, eptr->name, sizeof(el[i].name) - 1);
    if (eptr->type == T_WATCH)
      continue; /* disabled: its other parameters shape no output */
    if (fill_parameters(&el[i], eptr, map, why, why_len)) {
      free(el);
      return -1;
    }
  }

  if (!adapter_ctx && b2e_create(&adapter_ctx, 0) != B2E_OK) {
    say(why, why_len, "no CUDA device for the engine%s%s", "", "");
    b2e_adapter_release();
    free(el);
    return -2;
  }
  memset(&opt, 0, sizeof(opt));
  opt.p_central = P_central;
  opt.n_passes = (int32_t)n_passes;
  opt.default_order = (int32_t)default_order;
  opt.coord_limit = coordLimit;
  opt.slope_limit = slopeLimit;
  if (b2e_load_lattice(adapter_ctx, el, (int32_t)n, &opt) != B2E_OK) {
    say(why, why_len, "%s%s", b2e_last_error(adapter_ctx), "");
    free(el);
    return -1; /* a value the engine does not support: the CPU path takes the line */
  }
  free(el);

  /* rows -> columns */
  for (j = 0; j < 6; j++)
    if (!(cols[j] = (double *)malloc(sizeof(double) * (np ? np : 1))))
      goto done;
  ids = (int64_t *)malloc(sizeof(int64_t) * (np ? np : 1));
  lost_pass = (int32_t *)malloc(sizeof(int32_t) * (np ? np : 1));
  lost_elem = (int32_t *)malloc(sizeof(int32_t) * (np ? np : 1));
  rows = (double *)malloc(sizeof(double) * (np ? np : 1) * totalPropertiesPerParticle);
  if (!ids || !lost_pass || !lost_elem || !rows)
    goto done;
  for (i = 0; i < np; i++) {
    for (j = 0; j < 6; j++)
      cols[j][i] = coord[i][j];
    ids[i] = (int64_t)coord[i][particleIDIndex];
  }
  if (b2e_track_host(adapter_ctx, cols, ids, np, lost_pass, lost_elem, &n_left, &effort) != B2E_OK) {
    say(why, why_len, "%s%s", b2e_last_error(adapter_ctx), "");
    goto done;
  }
  /* columns -> rows: survivors first in their original order, then the lost
   * rows, with the loss pass where recordLostParticles puts it
   * (do_tracking.c:4584-4605) */
  {
    long top = 0, bottom = n_left;
    for (i = 0; i < np; i++) {
      double *r = rows + (size_t)(lost_pass[i] < 0 ? top++ : bottom++) * totalPropertiesPerParticle;
      memcpy(r, coord[i], sizeof(double) * totalPropertiesPerParticle);
      for (j = 0; j < 6; j++)
        r[j] = cols[j][i];
      r[lossPassIndex] = lost_pass[i] < 0 ? -1 : lost_pass[i];
    }
    for (i = 0; i < np; i++)
      memcpy(coord[i], rows + (size_t)i * totalPropertiesPerParticle, sizeof(double) * totalPropertiesPerParticle);
  }
  if (effort_out)
    *effort_out = effort;
  status = (long)n_left;
done:
  for (j = 0; j < 6; j++)
    free(cols[j]);
  free(ids);
  free(lost_pass);
  free(lost_elem);
  free(rows);
  return status;
}
