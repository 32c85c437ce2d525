/*
 * Driver around elegant's own hot-path routines, compiled unmodified from the
 * reference sources (see oracle/Makefile.ref).  It is the pinned CPU oracle:
 * the restatement in oracle/b2e_oracle.c and the CUDA path are both checked
 * against what this file produces.
 *
 * What is the reference's and what is restated here:
 *  - element physics: multipole_tracking2 (multipole.c:693), track_through_csbend
 *    (csbend.c:665), track_through_csbendCSR (csbend.c:1899),
 *    track_through_driftCSR (csbend.c:3176), simple_rf_cavity (simple_rfca.c:264),
 *    exactDrift (csbend.c:3767), track_particles (matrix.c:294),
 *    limit_amplitudes / elimit_amplitudes (limit_amplitudes.c:193, :472) -- all
 *    called as compiled from the reference;
 *  - element construction: parameter names, storage offsets and defaults come
 *    from the reference's own tables (track_data.c entity_description); this
 *    file only walks them (restating the default-setting of mad_parse.c);
 *  - the pass/element loop restates do_tracking.c:488-2640 for the supported
 *    element subset: z bookkeeping (:1077-1084), sticky MAXAMP (:1848-1858),
 *    aperture after each element (:2455-2475), NaN sweep and loss recording
 *    (:2629-2636, recordLostParticles :4584-4605), effort counter (:2758).
 *
 * Interface (ctypes): b2e_ref_track().  Particle rows are
 * (x, xp, y, yp, s, delta, id, lossPass, bunch, weight) as in track.h:81-100.
 */
#include "mdb.h"
#include "track.h"
#include "csbend.h"
#include <setjmp.h>
#include <ctype.h>

extern jmp_buf b2e_ref_trap;
extern int b2e_ref_trap_armed;
extern char b2e_ref_errmsg[512];
extern long b2e_ref_warning_count;
void b2e_ref_capture_reset(void);

typedef struct {
  const char *name;
  long type;
} B2E_REF_TYPE;

static const B2E_REF_TYPE b2e_ref_types[] = {
  {"DRIF", T_DRIF}, {"DRIFT", T_DRIF}, {"EDRIFT", T_EDRIFT}, {"KQUAD", T_KQUAD},
  {"KSEXT", T_KSEXT}, {"CSBEND", T_CSBEND}, {"SBEN", T_CSBEND}, {"RFCA", T_RFCA},
  {"MAXAMP", T_MAXAMP}, {"MARK", T_MARK}, {"CHARGE", T_CHARGE},
  {"CSRCSBEND", T_CSRCSBEND}, {"CSRDRIFT", T_CSRDRIFT}, {"MALIGN", T_MALIGN},
  /* built but not tracked by the restated loop: lets the adapter's tests
   * hand it an element type outside the engine's set */
  {"SEXT", T_SEXT}, {"WATCH", T_WATCH}, {NULL, 0}};

/* offset_beam (do_tracking.c:3243-3300) restated: do_tracking.c is not part
 * of the compiled subset */
static void b2e_ref_offset_beam(double **coord, long nToTrack, MALIGN *offset, double P_central) {
  long i_part, allParticles;
  double *part, pc, beta, gamma, t, ds;
  allParticles = (offset->startPID == -1) && (offset->endPID == -1);
  for (i_part = nToTrack - 1; i_part >= 0; i_part--) {
    part = coord[i_part];
    if (!allParticles && (part[6] < offset->startPID || part[6] > offset->endPID))
      continue;
    if (offset->dz)
      ds = offset->dz * sqrt(1 + sqr(part[1]) + sqr(part[3]));
    else
      ds = 0;
    part[0] += offset->dx + offset->dz * part[1];
    part[1] += offset->dxp;
    part[2] += offset->dy + offset->dz * part[3];
    part[3] += offset->dyp;
    part[4] += ds;
    if (offset->dt || offset->dp || offset->de) {
      pc = P_central * (1 + part[5]);
      beta = pc / (gamma = sqrt(1 + pc * pc));
      t = part[4] / (beta * c_mks) + offset->dt;
      if (offset->dp) {
        part[5] += offset->dp;
        pc = P_central * (1 + part[5]);
        beta = pc / sqrt(1 + pc * pc);
      }
      if (offset->de) {
        gamma += offset->de * gamma;
        pc = sqrt(gamma * gamma - 1);
        beta = pc / gamma;
        part[5] = (pc - P_central) / P_central;
      }
      part[4] = t * beta * c_mks;
    }
  }
}

static long lookup_type(const char *name) {
  long i;
  for (i = 0; b2e_ref_types[i].name; i++)
    if (strcmp(name, b2e_ref_types[i].name) == 0)
      return b2e_ref_types[i].type;
  return -1;
}

/* Fill an element structure with the defaults of its parameter table. */
static void set_defaults(char *p_elem, long type) {
  PARAMETER *par = entity_description[type].parameter;
  long i;
  for (i = 0; i < entity_description[type].n_params; i++) {
    char *where = p_elem + par[i].offset;
    switch (par[i].type) {
    case IS_DOUBLE:
      *(double *)where = par[i].number;
      break;
    case IS_LONG:
      *(long *)where = par[i].integer;
      break;
    case IS_SHORT:
      *(short *)where = (short)par[i].integer;
      break;
    case IS_STRING:
      *(char **)where = par[i].string ? strdup(par[i].string) : NULL;
      break;
    }
  }
}

static int set_parameter(char *p_elem, long type, const char *key, const char *value) {
  PARAMETER *par = entity_description[type].parameter;
  long i;
  for (i = 0; i < entity_description[type].n_params; i++) {
    if (strcmp(par[i].name, key) == 0) {
      char *where = p_elem + par[i].offset;
      switch (par[i].type) {
      case IS_DOUBLE:
        *(double *)where = strtod(value, NULL);
        break;
      case IS_LONG:
        *(long *)where = strtol(value, NULL, 10);
        break;
      case IS_SHORT:
        *(short *)where = (short)strtol(value, NULL, 10);
        break;
      case IS_STRING:
        *(char **)where = strdup(value);
        break;
      }
      return 1;
    }
  }
  return 0;
}

/* Parse "NAME:TYPE KEY=VALUE ...;NAME:TYPE ..." into an ELEMENT_LIST chain. */
static ELEMENT_LIST *build_line(const char *spec, long *n_out) {
  char *text = strdup(spec), *save1 = NULL, *item;
  ELEMENT_LIST *head = NULL, *tail = NULL;
  double pos = 0;
  long n = 0;
  for (item = strtok_r(text, ";\n", &save1); item; item = strtok_r(NULL, ";\n", &save1)) {
    char *save2 = NULL, *tok, *colon;
    ELEMENT_LIST *e;
    long type;
    while (isspace((unsigned char)*item))
      item++;
    if (!*item)
      continue;
    tok = strtok_r(item, " \t", &save2);
    e = calloc(1, sizeof(*e));
    colon = strchr(tok, ':');
    if (colon) {
      *colon = 0;
      e->name = strdup(tok);
      tok = colon + 1;
    } else {
      char buf[32];
      snprintf(buf, sizeof(buf), "E%ld", n);
      e->name = strdup(buf);
    }
    if ((type = lookup_type(tok)) < 0) {
      snprintf(b2e_ref_errmsg, sizeof(b2e_ref_errmsg), "unsupported element type %s", tok);
      free(text);
      return NULL;
    }
    e->type = type;
    e->p_elem = calloc(1, entity_description[type].structure_size + 64);
    set_defaults(e->p_elem, type);
    while ((tok = strtok_r(NULL, " \t", &save2))) {
      char *eq = strchr(tok, '=');
      if (!eq)
        continue;
      *eq = 0;
      if (!set_parameter(e->p_elem, type, tok, eq + 1)) {
        snprintf(b2e_ref_errmsg, sizeof(b2e_ref_errmsg), "unknown parameter %s for %s", tok, entity_name[type]);
        free(text);
        return NULL;
      }
    }
    switch (type) {
    case T_CSBEND:
      ((CSBEND *)e->p_elem)->e1Index = 0;
      ((CSBEND *)e->p_elem)->e2Index = 1;
      ((CSBEND *)e->p_elem)->etiltSign = 1;
      break;
    case T_CSRCSBEND:
      ((CSRCSBEND *)e->p_elem)->e1Index = 0;
      ((CSRCSBEND *)e->p_elem)->e2Index = 1;
      ((CSRCSBEND *)e->p_elem)->etiltSign = 1;
      break;
    default:
      break;
    }
    e->beg_pos = pos;
    if (entity_description[type].flags & HAS_LENGTH)
      pos += ((DRIFT *)e->p_elem)->length;
    e->end_pos = pos;
    e->occurence = 1;
    if (!head)
      head = e;
    else {
      tail->succ = e;
      e->pred = tail;
    }
    tail = e;
    n++;
  }
  free(text);
  *n_out = n;
  return head;
}

static void record_lost(double **coord, long nLeft, long nToTrack, long pass) {
  /* do_tracking.c:4584-4605 (recordLostParticles) */
  long i;
  for (i = nLeft; i < nToTrack; i++)
    coord[i][lossPassIndex] = pass;
}

/* CSR wake capture for parity tests: the reference keeps the last dipole wake
 * in the global csrWake (csbend.h); after each CSRCSBEND we copy dGamma out. */
static double *wake_out = NULL;
static long wake_cap = 0, wake_count = 0;

/* Fiducial time of the last zero-length RFCA fiducialised in a run: the same
 * findFiducialTime call, on the same particles, that simple_rf_cavity makes
 * on its first pass (simple_rfca.c:421-431 with length 0, so s0 = zEnd and
 * sOffset = 0).  A run split over particle slices passes it back as
 * T_REFERENCE (simple_rfca.c:428-429), so that every slice uses the phase of
 * the whole beam. */
static double last_fiducial_t0 = -1;

double b2e_ref_last_fiducial_t0(void) { return last_fiducial_t0; }

/* Optional per-pass history of the survivors: [pass][5] = survivors, <x>,
 * <y>, and the rms emittances sqrt(<dx^2><dx'^2> - <dx dx'>^2) per plane
 * (the form of rms_emittance, final_props.c:844-880), recorded after the
 * last element of every pass.  Two-pass sums in particle order. */
static double *history_out = NULL;
static long history_passes = 0;

/* WATCH capture (test infrastructure): at each coordinate-mode WATCH on the
 * passes dump_watch_particles writes (sdds_support.c:738-741), the rows it is
 * handed (the particles alive at the element, do_tracking.c:1626-1629) are
 * copied as (element index, pass, particleID, x, xp, y, yp, s, delta). */
static double *watch_buf = NULL;
static long watch_cap = 0, watch_count = 0;

void b2e_ref_set_watch(double *buffer, long capacity_rows) {
  watch_buf = buffer;
  watch_cap = capacity_rows;
  watch_count = 0;
}

long b2e_ref_watch_rows(void) { return watch_count; }

static void capture_watch(const WATCH *w, long elem_index, long pass, double **coord, long n) {
  long i, j;
  if (!watch_buf || w->disable)
    return;
  if (!(pass >= w->start_pass && (pass - w->start_pass) % w->interval == 0 && (w->end_pass < 0 || pass <= w->end_pass)))
    return;
  for (i = 0; i < n && watch_count < watch_cap; i++) {
    double *r = watch_buf + watch_count * 9;
    r[0] = elem_index;
    r[1] = pass;
    r[2] = coord[i][6];
    for (j = 0; j < 6; j++)
      r[3 + j] = coord[i][j];
    watch_count++;
  }
}

/* accumulate_beam_sums (compute_centroids.c:286-490) on rows [n][7] (x, xp,
 * y, yp, s, delta, particleID) as dump_watch_parameters calls it
 * (sdds_support.c:979-981): centroid[7] and the sparse sigma[7][7]. */
long b2e_ref_beam_sums(const double *rows, long n, double Po, long startPID, long endPID, double *centroid,
                       double *sigma) {
  double **coord = (double **)czarray_2d(sizeof(double), n ? n : 1, totalPropertiesPerParticle);
  BEAM_SUMS *sums;
  long i, j;
  for (i = 0; i < n; i++)
    for (j = 0; j < 7; j++)
      coord[i][j] = rows[i * 7 + j];
  sums = allocateBeamSums(0, 1);
  zero_beam_sums(sums, 1);
  accumulate_beam_sums(sums, coord, n, Po, 0.0, NULL, 0.0, 0.0, startPID, endPID,
                       BEAM_SUMS_SPARSE | BEAM_SUMS_NOMINMAX);
  for (i = 0; i < 7; i++) {
    centroid[i] = sums->centroid[i];
    for (j = 0; j < 7; j++)
      sigma[i * 7 + j] = sums->beamSums2->sigma[i][j];
  }
  j = sums->n_part;
  free_czarray_2d((void **)coord, n ? n : 1, totalPropertiesPerParticle);
  return j;
}

void b2e_ref_set_history(double *buffer, long n_passes) {
  history_out = buffer;
  history_passes = buffer ? n_passes : 0;
}

static void record_history(double **coord, long n, long pass) {
  double m[4] = {0, 0, 0, 0}, s[6] = {0, 0, 0, 0, 0, 0}, *h, ex, ey;
  long i, k;
  if (!history_out || pass >= history_passes)
    return;
  h = history_out + 5 * pass;
  h[0] = n;
  h[1] = h[2] = h[3] = h[4] = 0;
  if (!n)
    return;
  for (i = 0; i < n; i++)
    for (k = 0; k < 4; k++)
      m[k] += coord[i][k];
  for (k = 0; k < 4; k++)
    m[k] /= n;
  for (i = 0; i < n; i++) {
    double dx = coord[i][0] - m[0], dxp = coord[i][1] - m[1], dy = coord[i][2] - m[2], dyp = coord[i][3] - m[3];
    s[0] += dx * dx;
    s[1] += dxp * dxp;
    s[2] += dx * dxp;
    s[3] += dy * dy;
    s[4] += dyp * dyp;
    s[5] += dy * dyp;
  }
  for (k = 0; k < 6; k++)
    s[k] /= n;
  ex = s[0] * s[1] - s[2] * s[2];
  ey = s[3] * s[4] - s[5] * s[5];
  h[1] = m[0];
  h[2] = m[2];
  h[3] = ex > 0 ? sqrt(ex) : 0;
  h[4] = ey > 0 ? sqrt(ey) : 0;
}

long b2e_ref_track(const char *lattice, double p_central, double *rows_in, long np, long n_passes,
                   double *rows_out, long *n_left, double *effort, double *wake_buffer, long wake_capacity,
                   long *wake_written, char *errbuf, long errlen) {
  ELEMENT_LIST *line, *eptr;
  double **coord = NULL;
  long nElems = 0, nToTrack, nLeft, i_pass, i, j;
  double z, z_travel, last_z;
  MAXAMP *maxamp = NULL;
  double x_max = 0, y_max = 0;
  long elliptical = 0, maxampOpenCode = 0, maxampExponent = 0, maxampYExponent = 0;
  CHARGE *charge = NULL;
  APERTURE_DATA apertureData;
  double P_central = p_central;
  double revolution_length;
  long status = 0;

  static int offsets_done = 0;
  if (!offsets_done) {
    /* track_data.c:4066: parameter offsets are stored as addresses into the
     * *_example structures until compute_offsets() rebases them */
    compute_offsets();
    offsets_done = 1;
  }
  memset(&apertureData, 0, sizeof(apertureData));
  b2e_ref_capture_reset();
  b2e_ref_errmsg[0] = 0;
  sizeOfParticle = totalPropertiesPerParticle * sizeof(double);
  particleMass = me_mks;
  particleCharge = e_mks;
  particleMassMV = me_mev;
  particleRadius = re_mks;
  particleRelSign = 1;
  particleIsElectron = 1;
  wake_out = wake_buffer;
  wake_cap = wake_capacity;
  wake_count = 0;
  last_fiducial_t0 = -1;
  delete_phase_references(); /* each run starts as a new elegant run: no phase reference set */

  if (setjmp(b2e_ref_trap)) {
    b2e_ref_trap_armed = 0;
    if (errbuf && errlen > 0)
      snprintf(errbuf, errlen, "%s", b2e_ref_errmsg);
    return -1;
  }
  b2e_ref_trap_armed = 1;

  if (!(line = build_line(lattice, &nElems))) {
    b2e_ref_trap_armed = 0;
    if (errbuf && errlen > 0)
      snprintf(errbuf, errlen, "%s", b2e_ref_errmsg);
    return -2;
  }

  for (eptr = line, revolution_length = 0; eptr; eptr = eptr->succ)
    revolution_length = eptr->end_pos - line->beg_pos;

  coord = (double **)czarray_2d(sizeof(double), np ? np : 1, totalPropertiesPerParticle);
  for (i = 0; i < np; i++) {
    for (j = 0; j < 7; j++)
      coord[i][j] = rows_in[i * 7 + j];
    coord[i][lossPassIndex] = -1;
    coord[i][bunchIndex] = 0;
    coord[i][weightIndex] = 1;
  }
  nToTrack = nLeft = np;
  *effort = 0;

  for (i_pass = 0; i_pass < n_passes; i_pass++) {
    long nParticlesStartPass = nToTrack;
    long elem_index = -1;
    z = z_travel = last_z = line->beg_pos;
    eptr = line;
    while (eptr && nToTrack) {
      elem_index++;
      unsigned long classFlags = entity_description[eptr->type].flags;
      last_z = z;
      if (classFlags & HAS_LENGTH && eptr->p_elem) {
        z += ((DRIFT *)eptr->p_elem)->length;
        z_travel += ((DRIFT *)eptr->p_elem)->length;
      } else {
        z += eptr->end_pos - eptr->beg_pos;
        z_travel += eptr->end_pos - eptr->beg_pos;
      }
      setTrackingContext(eptr->name, eptr->occurence, eptr->type, "b2e", eptr);
      nLeft = nToTrack;
      if (classFlags & MATRIX_TRACKING) {
        if (!eptr->matrix) {
          DRIFT *drift = (DRIFT *)eptr->p_elem;
          /* default_order = 2 (elegant.nl run_setup default) */
          eptr->matrix = drift_matrix(drift->length, drift->order ? drift->order : 2);
        }
        if (nParticlesStartPass)
          track_particles(coord, eptr->matrix, coord, nToTrack);
      } else if (nParticlesStartPass) {
        switch (eptr->type) {
        case T_CHARGE:
          if (i_pass == 0) {
            charge = (CHARGE *)eptr->p_elem;
            charge->macroParticleCharge = 0;
            if (np)
              charge->macroParticleCharge = charge->charge / np;
            if (charge->chargePerParticle)
              charge->macroParticleCharge = charge->chargePerParticle;
          }
          break;
        case T_MARK:
          break;
        case T_WATCH:
          capture_watch((WATCH *)eptr->p_elem, elem_index, i_pass, coord, nToTrack);
          break;
        case T_MALIGN:
          /* do_tracking.c:1818-1821 */
          if (((MALIGN *)eptr->p_elem)->on_pass == -1 || ((MALIGN *)eptr->p_elem)->on_pass == i_pass)
            b2e_ref_offset_beam(coord, nToTrack, (MALIGN *)eptr->p_elem, P_central);
          break;
        case T_MAXAMP:
          maxamp = (MAXAMP *)eptr->p_elem;
          x_max = maxamp->x_max;
          y_max = maxamp->y_max;
          elliptical = maxamp->elliptical;
          maxampOpenCode = determineOpenSideCode(maxamp->openSide);
          maxampExponent = maxamp->exponent;
          maxampYExponent = maxamp->yExponent;
          break;
        case T_RFCA: {
          RFCA *rf = (RFCA *)eptr->p_elem;
          if (!rf->fiducial_seen && rf->tReference == -1 && rf->length == 0) {
            unsigned long mode = parseFiducialMode(rf->fiducial);
            if (mode)
              last_fiducial_t0 = findFiducialTime(coord, nToTrack, z_travel, 0.0, P_central, mode);
          }
          nLeft = simple_rf_cavity(coord, nToTrack, rf, NULL, &P_central, z_travel);
          break;
        }
        case T_EDRIFT:
          exactDrift(coord, nToTrack, ((EDRIFT *)eptr->p_elem)->length);
          break;
        case T_KQUAD:
        case T_KSEXT:
          nLeft = multipole_tracking2(coord, nToTrack, eptr, 0.0, P_central, NULL, last_z, maxamp, NULL,
                                      &apertureData, NULL, -1);
          break;
        case T_CSBEND: {
          CSBEND *cs = (CSBEND *)eptr->p_elem;
          cs->edgeFlags = determine_bend_flags(eptr, cs->edge_effects[cs->e1Index], cs->edge_effects[cs->e2Index]);
          nLeft = track_through_csbend(coord, nToTrack, cs, 0.0, P_central, NULL, last_z, NULL, "b2e", maxamp,
                                       NULL, &apertureData, -1, eptr);
          break;
        }
        case T_CSRCSBEND: {
          CSRCSBEND *cs = (CSRCSBEND *)eptr->p_elem;
          cs->edgeFlags = determine_bend_flags(eptr, cs->edge_effects[cs->e1Index], cs->edge_effects[cs->e2Index]);
          nLeft = track_through_csbendCSR(coord, nToTrack, cs, 0.0, P_central, NULL, last_z, z, charge, "b2e",
                                          maxamp, NULL, &apertureData, eptr);
          if (wake_out && csrWake.valid && csrWake.dGamma) {
            for (j = 0; j < csrWake.bins && wake_count < wake_cap; j++)
              wake_out[wake_count++] = csrWake.dGamma[j];
          }
          break;
        }
        case T_CSRDRIFT:
          nLeft = track_through_driftCSR(coord, nToTrack, (CSRDRIFT *)eptr->p_elem, P_central, NULL, last_z,
                                         revolution_length, charge, "b2e");
          break;
        default:
          bombElegant("element type not supported by the reference driver", NULL);
        }
      }
      if (!(classFlags & NO_APERTURE)) {
        if (x_max || y_max) {
          if (!elliptical)
            nLeft = limit_amplitudes(coord, x_max, y_max, nLeft, NULL, z, P_central, eptr->type == T_DRIF,
                                     maxampOpenCode, eptr);
          else
            nLeft = elimit_amplitudes(coord, x_max, y_max, nLeft, NULL, z, P_central, eptr->type == T_DRIF,
                                      maxampOpenCode, maxampExponent, maxampYExponent, eptr);
        }
      }
      nLeft = limit_amplitudes(coord, DBL_MAX, DBL_MAX, nLeft, NULL, z, P_central, 0, 0, eptr);
      if (nLeft != nToTrack)
        record_lost(coord, nLeft, nToTrack, i_pass);
      nToTrack = nLeft;
      eptr = eptr->succ;
    }
    *effort += nLeft;
    record_history(coord, nToTrack, i_pass);
  }

  for (i = 0; i < np; i++)
    for (j = 0; j < 8; j++)
      rows_out[i * 8 + j] = coord[i][j];
  *n_left = nToTrack;
  if (wake_written)
    *wake_written = wake_count;
  b2e_ref_trap_armed = 0;
  free_czarray_2d((void **)coord, np ? np : 1, totalPropertiesPerParticle);
  return status;
}

/* Report element-class flags so tests can check aperture bookkeeping. */
unsigned long b2e_ref_type_flags(const char *type_name) {
  long type = lookup_type(type_name);
  (void)compute_offsets;
  return type < 0 ? 0 : entity_description[type].flags;
}

#ifdef B2E_REF_WITH_ADAPTER
/* The drop-in adapter (elegant_b200/adapter) driven from an element list
 * built here from the reference's own tables, exactly as b2e_ref_track
 * builds it: the rows go through b2e_adapter_track (the engine on the GPU)
 * instead of the restated do_tracking loop.  Returns the adapter's status
 * (survivors, or -1 / -2). */
#include "b2e_adapter.h"

long b2e_ref_adapter_track(const char *lattice, double p_central, double *rows_in, long np, long n_passes,
                           double *rows_out, double *effort, char *errbuf, long errlen) {
  ELEMENT_LIST *line;
  double **coord;
  long nElems = 0, i, j, status;
  static int offsets_done = 0;
  if (!offsets_done) {
    compute_offsets();
    offsets_done = 1;
  }
  b2e_ref_errmsg[0] = 0;
  if (!(line = build_line(lattice, &nElems))) {
    if (errbuf && errlen > 0)
      snprintf(errbuf, errlen, "%s", b2e_ref_errmsg);
    return -3;
  }
  coord = (double **)czarray_2d(sizeof(double), np ? np : 1, totalPropertiesPerParticle);
  for (i = 0; i < np; i++) {
    for (j = 0; j < 7; j++)
      coord[i][j] = rows_in[i * 7 + j];
    coord[i][lossPassIndex] = -1;
    coord[i][bunchIndex] = 0;
    coord[i][weightIndex] = 1;
  }
  status = b2e_adapter_track(coord, np, line, p_central, n_passes, 2, effort, errbuf, errlen);
  for (i = 0; i < np; i++)
    for (j = 0; j < 8; j++)
      rows_out[i * 8 + j] = coord[i][j];
  free_czarray_2d((void **)coord, np ? np : 1, totalPropertiesPerParticle);
  return status;
}
#endif
