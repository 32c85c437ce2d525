/*
 * Link-time stand-ins for the symbols that elegant's hot-path sources reference
 * but that live outside the compiled subset (elegant.c, do_tracking.c,
 * final_props.c, the SDDS toolkit's mdblib/mdbmth/SDDS1 libraries).
 *
 * Symbols on the tracked path are restated here from the reference
 * (file:line cited) or from the published method they implement; everything
 * else reports a fatal "not on the hot path" error through the driver's
 * error trap, so a lattice that strays outside the supported subset fails
 * loudly instead of producing numbers.  Test infrastructure only.
 */
#include "mdb.h"
#include "track.h"
#include <stdarg.h>
#include <setjmp.h>

/* ---- error trap shared with ref_driver.c -------------------------------- */
jmp_buf b2e_ref_trap;
int b2e_ref_trap_armed = 0;
char b2e_ref_errmsg[512];
long b2e_ref_warning_count = 0;

static void b2e_ref_fail(const char *what) {
  snprintf(b2e_ref_errmsg, sizeof(b2e_ref_errmsg), "%s", what ? what : "(null)");
  if (b2e_ref_trap_armed)
    longjmp(b2e_ref_trap, 1);
  fprintf(stderr, "fatal (no trap armed): %s\n", b2e_ref_errmsg);
  abort();
}

#define NOT_ON_PATH(name) b2e_ref_fail("reference routine " #name " is not on the supported hot path")

/* ---- elegant.c / do_tracking.c routines used by the compiled subset ----- */
void swapParticles(double *p1, double *p2) {
  /* elegant.c:2663-2670: exchange two particle rows of sizeOfParticle bytes */
  double buffer[MAX_PROPERTIES_PER_PARTICLE];
  if (p1 == p2)
    return;
  memcpy(buffer, p1, sizeOfParticle);
  memcpy(p1, p2, sizeOfParticle);
  memcpy(p2, buffer, sizeOfParticle);
}

double beta_from_delta(double p, double delta) {
  /* do_tracking.c:95-98 */
  p *= 1 + delta;
  return (p / sqrt(p * p + 1));
}

void bombElegant(const char *error, const char *usage) { b2e_ref_fail(error); }
void bombTracking(const char *error) { b2e_ref_fail(error); }
void bombElegantVA(char *ptemplate, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, ptemplate);
  vsnprintf(buf, sizeof(buf), ptemplate, ap);
  va_end(ap);
  b2e_ref_fail(buf);
}
void exitElegant(long status) { b2e_ref_fail("exitElegant called"); }
void printWarningForTracking(char *text, char *detail) { b2e_ref_warning_count++; }

static TRACKING_CONTEXT b2e_ctx_store;
void getTrackingContext(TRACKING_CONTEXT *tc) { *tc = b2e_ctx_store; }
void setTrackingContext(char *name, long occurence, long type, char *rootname, ELEMENT_LIST *eptr) {
  memset(&b2e_ctx_store, 0, sizeof(b2e_ctx_store));
  if (name)
    strncpy(b2e_ctx_store.elementName, name, CONTEXT_BUFSIZE - 1);
  b2e_ctx_store.elementOccurrence = occurence;
  b2e_ctx_store.element = eptr;
}

/* No obstructions are defined in the supported subset (obstructionData absent). */
long insideObstruction(double *part, short mode, double dz, long segment, long nSegments) { return 0; }
long insideObstruction_xyz(double x, double xp, double y, double yp, long particleID, double *lossCoordinates,
                           double tilt, short mode, double dz, long segment, long nSegments) { return 0; }

VMATRIX *drift_matrix(double length, long order) {
  /* compute_matrices.c:391-412 */
  VMATRIX *M = tmalloc(sizeof(*M));
  M->order = (order > 2 ? 2 : order);
  initialize_matrices(M, M->order);
  M->C[4] = length;
  M->R[0][0] = M->R[1][1] = M->R[2][2] = M->R[3][3] = M->R[4][4] = M->R[5][5] = 1;
  M->R[0][1] = M->R[2][3] = length;
  if (order > 1)
    M->T[4][1][1] = M->T[4][3][3] = length / 2;
  return M;
}

/* ---- toolkit (mdblib / mdbmth) routines, restated from their definitions -- */
void *b2e_shim_tmalloc(size_t n) {
  void *p = calloc(1, n ? n : 1);
  if (!p)
    b2e_ref_fail("allocation failure");
  return p;
}
void *SDDS_Realloc(void *p, size_t n) { return realloc(p, n ? n : 1); }
void *SDDS_Malloc(size_t n) { return malloc(n ? n : 1); }
void *SDDS_Calloc(size_t n, size_t m) { return calloc(n ? n : 1, m ? m : 1); }
void SDDS_Bomb(char *msg) { b2e_ref_fail(msg); }

/* x^n by repeated multiplication (integer power) */
double ipow(double x, long n) {
  double r = 1;
  long i;
  if (n < 0) {
    for (i = 0; i < -n; i++)
      r *= x;
    return 1 / r;
  }
  if (n == 0)
    return 1;
  r = x;
  for (i = 1; i < n; i++)
    r *= x;
  return r;
}

/* n! as a double */
double dfactorial(long n) {
  double f = 1;
  long i;
  for (i = 2; i <= n; i++)
    f *= i;
  return f;
}

/* Unique-prefix string match against a table of options; returns the index or -1. */
long match_string(char *s, char **options, long n, long mode) {
  long i, hit = -1, len;
  if (!s)
    return -1;
  len = strlen(s);
  for (i = 0; i < n; i++) {
    if (strcmp(s, options[i]) == 0)
      return i;
  }
  for (i = 0; i < n; i++) {
    if (strncmp(s, options[i], len) == 0) {
      if (hit >= 0)
        return -1;
      hit = i;
    }
  }
  return hit;
}

/* Contiguous row-pointer 2-D array (one block for the data) */
void **czarray_2d(long size, long n1, long n2) {
  void **rows = calloc(n1 ? n1 : 1, sizeof(void *));
  char *block = calloc((size_t)(n1 ? n1 : 1) * (n2 ? n2 : 1), size);
  long i;
  for (i = 0; i < n1; i++)
    rows[i] = block + (size_t)i * n2 * size;
  return rows;
}
void free_czarray_2d(void **array, long n1, long n2) {
  if (array) {
    free(array[0]);
    free(array);
  }
}
void **zarray_2d(long size, long n1, long n2) { return czarray_2d(size, n1, n2); }
void free_zarray_2d(void **array, long n1, long n2) { free_czarray_2d(array, n1, n2); }

char *cp_str(char **s, char *t) {
  *s = t ? strdup(t) : NULL;
  return *s;
}
int SDDS_CopyString(char **target, const char *source) {
  *target = source ? strdup(source) : NULL;
  return 1;
}

/* Random numbers, reached with ISR (gauss_rn_lim(0, 1, srGaussianLimit,
 * random_2), multipole.c:1343, csbend.c:1619).  The toolkit's generators are
 * not in the tree; these are this project's: random_2 a SplitMix64 stream
 * (reseeded by a negative seed, as the toolkit's generators are), gauss_rn_lim
 * Box-Muller on it with deviates beyond `limit` sigma (limit > 0) redrawn.
 * The reference's ISR is therefore compared with the engine's in
 * distribution, not draw by draw. */
static uint64_t b2e_r2_state = 0x853c49e6748fea9bull;
double random_2(long iseed) {
  uint64_t z;
  if (iseed < 0)
    b2e_r2_state = (uint64_t)(-iseed) * 0x9E3779B97F4A7C15ull;
  z = (b2e_r2_state += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return ((double)(z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}
double gauss_rn_lim(double mean, double sigma, double limit, double (*urandom)(long)) {
  int tries;
  for (tries = 0; tries < 1000; tries++) {
    double u1 = urandom(0), u2 = urandom(0);
    double g = sqrt(-2.0 * log(u1)) * cos(2 * 3.141592653589793 * u2);
    if (!(limit > 0) || fabs(g) <= limit)
      return mean + sigma * g;
  }
  return mean;
}
double random_1(long iseed) { NOT_ON_PATH(random_1); return 0; }
double random_3(long iseed) { NOT_ON_PATH(random_3); return 0; }
double random_4(long iseed) { NOT_ON_PATH(random_4); return 0; }
double random_1_elegant(long iseed) { NOT_ON_PATH(random_1_elegant); return 0; }

void b2e_ref_offpath(const char *name) {
  char buf[256];
  snprintf(buf, sizeof(buf), "reference routine %s is not on the supported hot path", name);
  b2e_ref_fail(buf);
}

long determine_bend_flags(ELEMENT_LIST *elem, long edge1_effects, long edge2_effects) {
  /* bend_matrix.c:1342-1391: edge effects are skipped at a face that joins an
   * identically named bend of the same type (MARK/WATCH in between are
   * transparent); zero-length LSCDRIFT is not in the supported subset. */
  ELEMENT_LIST *other;
  long bend_flags = 0;
  for (other = elem->pred; other; other = other->pred) {
    if (other->type == elem->type && strcmp(other->name, elem->name) == 0) {
      bend_flags |= SAME_BEND_PRECEDES;
      break;
    }
    if (other->type != T_MARK && other->type != T_WATCH)
      break;
  }
  for (other = elem->succ; other; other = other->succ) {
    if (other->type == elem->type && strcmp(other->name, elem->name) == 0) {
      bend_flags |= SAME_BEND_FOLLOWS;
      break;
    }
    if (other->type != T_MARK && other->type != T_WATCH)
      break;
  }
  if (edge1_effects && !(bend_flags & SAME_BEND_PRECEDES))
    bend_flags |= BEND_EDGE1_EFFECTS;
  if (edge2_effects && !(bend_flags & SAME_BEND_FOLLOWS))
    bend_flags |= BEND_EDGE2_EFFECTS;
  bend_flags |= BEND_EDGE_DETERMINED;
  return bend_flags;
}

/* Number of set bits in a word (mdblib bitsSet; used by CSRDRIFT mode checks). */
long bitsSet(unsigned long data) {
  long n = 0;
  while (data) {
    n += (long)(data & 1UL);
    data >>= 1;
  }
  return n;
}

/* ---- beam sums (compute_centroids.c, compiled for the WATCH statistics) --- */
/* exactNormalizedEmittance (global_settings exact_normalized_emittance) is
 * defined in track_data.c: 0, elegant's default */
/* computeTimeCoordinates (trwake.c:532-590, serial branch): t = s sqrt(P^2+1)/(c P)
 * for every particle and their Kahan mean */
double computeTimeCoordinates(double *time, double Po, double **part, long np) {
  double tmean = 0, error = 0, P;
  long ip;
  for (ip = 0; ip < np; ip++) {
    P = Po * (part[ip][5] + 1);
    time[ip] = part[ip][4] * sqrt(sqr(P) + 1) / (c_mks * P);
    tmean = KahanPlus(tmean, time[ip], &error);
  }
  return np ? tmean / np : 0;
}

void computeTimeCoordinatesOnly(double *time, double Po, double **part, long np) {
  long ip;
  double P;
  for (ip = 0; ip < np; ip++) {
    P = Po * (part[ip][5] + 1);
    time[ip] = part[ip][4] * sqrt(sqr(P) + 1) / (c_mks * P);
  }
}
