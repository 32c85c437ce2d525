/*
 * In-memory stand-in for the SDDS writer calls that elegant's CSRCSBEND makes
 * when OUTPUT_FILE is set (csbend.c:2187-2226 layout, :2762-2806 one page
 * per kick).  Instead of writing a file, the columns of every page are
 * appended to per-column buffers that the tests read back: this is how the
 * per-kick wake arrays of the reference are obtained without modifying its
 * source.  Test infrastructure only.
 */
#include <stdarg.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "b2e_ref_shim.h"

#define B2E_CAPTURE_COLUMNS 7
static const char *capture_names[B2E_CAPTURE_COLUMNS] = {"DeltaGamma",   "LinearDensity", "LinearDensityDeriv",
                                                         "DeltaGammaT1", "DeltaGammaT2",  "s",
                                                         "GammaDeriv"};
/* the page parameters CSRCSBEND sets (csbend.c:2781-2785), in this order;
 * Pass is passed as an int, Kick as a long, the rest as doubles */
#define B2E_CAPTURE_PARAMS 9
static const char *param_names[B2E_CAPTURE_PARAMS] = {"Pass",  "Kick",           "dsKick",
                                                      "pCentral", "Angle",       "SlippageLength",
                                                      "TotalBunchLength", "BinSize", "DerbenevRatio"};
static double *param_buf;
static long param_len, param_cap;
static double *capture_buf[B2E_CAPTURE_COLUMNS];
static long capture_len[B2E_CAPTURE_COLUMNS], capture_cap[B2E_CAPTURE_COLUMNS];
static long capture_pages;

void b2e_ref_capture_reset(void) {
  int i;
  for (i = 0; i < B2E_CAPTURE_COLUMNS; i++)
    capture_len[i] = 0;
  capture_pages = 0;
  param_len = 0;
}

/* Copies up to `cap` captured parameter values (B2E_CAPTURE_PARAMS per page,
 * in param_names order); returns the number available. */
long b2e_ref_capture_params(double *out, long cap) {
  if (out)
    memcpy(out, param_buf, sizeof(double) * (param_len < cap ? param_len : cap));
  return param_len;
}

/* Copies up to `cap` captured values of column `which` (index into
 * capture_names); returns the number available. */
long b2e_ref_capture_get(int which, double *out, long cap) {
  long n;
  if (which < 0 || which >= B2E_CAPTURE_COLUMNS)
    return -1;
  n = capture_len[which];
  if (out)
    memcpy(out, capture_buf[which], sizeof(double) * (n < cap ? n : cap));
  return n;
}

long b2e_ref_capture_pages(void) { return capture_pages; }

char *compose_filename(char *templateString, char *root_name) { return strdup(templateString ? templateString : ""); }

int32_t SDDS_InitializeOutputElegant(SDDS_DATASET *ds, int32_t data_mode, int32_t lines_per_row,
                                     const char *description, const char *contents, const char *filename) {
  return 1;
}
int32_t SDDS_DefineParameter(SDDS_DATASET *ds, const char *name, const char *symbol, const char *units,
                             const char *description, const char *format_string, int32_t type, char *fixed_value) {
  return 0;
}
int32_t SDDS_DefineSimpleParameter(SDDS_DATASET *ds, const char *name, const char *unit, int32_t type) { return 1; }
int32_t SDDS_DefineColumn(SDDS_DATASET *ds, const char *name, const char *symbol, const char *units,
                          const char *description, const char *format_string, int32_t type, int32_t field_length) {
  return 0;
}
int32_t SDDS_DefineSimpleColumn(SDDS_DATASET *ds, const char *name, const char *unit, int32_t type) { return 1; }
int32_t SDDS_WriteLayout(SDDS_DATASET *ds) { return 1; }
int32_t SDDS_StartPage(SDDS_DATASET *ds, int64_t rows) { return 1; }
int32_t SDDS_SetParameters(SDDS_DATASET *ds, int32_t mode, ...) {
  va_list ap;
  const char *name;
  double values[B2E_CAPTURE_PARAMS];
  int i;
  for (i = 0; i < B2E_CAPTURE_PARAMS; i++)
    values[i] = 0;
  if (!((mode & SDDS_SET_BY_NAME) && (mode & SDDS_PASS_BY_VALUE)))
    return 1;
  va_start(ap, mode);
  while ((name = va_arg(ap, const char *))) {
    for (i = 0; i < B2E_CAPTURE_PARAMS && strcmp(name, param_names[i]) != 0; i++)
      ;
    if (i == 0)
      values[i] = va_arg(ap, int);
    else if (i == 1)
      values[i] = va_arg(ap, long);
    else if (i < B2E_CAPTURE_PARAMS)
      values[i] = va_arg(ap, double);
    else {
      va_end(ap);
      return 0; /* a parameter this capture does not know: its type is unknown */
    }
  }
  va_end(ap);
  if (param_len + B2E_CAPTURE_PARAMS > param_cap) {
    param_cap = 2 * (param_len + B2E_CAPTURE_PARAMS);
    param_buf = realloc(param_buf, sizeof(double) * param_cap);
  }
  memcpy(param_buf + param_len, values, sizeof(values));
  param_len += B2E_CAPTURE_PARAMS;
  return 1;
}
int32_t SDDS_WritePage(SDDS_DATASET *ds) {
  capture_pages++;
  return 1;
}
int32_t SDDS_DoFSync(SDDS_DATASET *ds) { return 1; }

int32_t SDDS_SetColumn(SDDS_DATASET *ds, int32_t mode, void *data, int64_t rows, ...) {
  va_list ap;
  const char *name = NULL;
  int i;
  va_start(ap, rows);
  if (mode & SDDS_SET_BY_NAME)
    name = va_arg(ap, const char *);
  va_end(ap);
  if (!name)
    return 1;
  for (i = 0; i < B2E_CAPTURE_COLUMNS; i++) {
    if (strcmp(name, capture_names[i]) == 0) {
      if (capture_len[i] + rows > capture_cap[i]) {
        capture_cap[i] = 2 * (capture_len[i] + rows);
        capture_buf[i] = realloc(capture_buf[i], sizeof(double) * capture_cap[i]);
      }
      memcpy(capture_buf[i] + capture_len[i], data, sizeof(double) * rows);
      capture_len[i] += rows;
    }
  }
  return 1;
}
