/*
 * Minimal stand-in for the un-vendored SDDS/EPICS toolkit headers, written for
 * compiling elegant's hot-path C sources (multipole.c, csbend.c, simple_rfca.c,
 * limit_amplitudes.c, matrix.c, malign_mat.c, tilt_matrices.c, kahan.c,
 * phase_reference.c) as the CPU oracle.  It declares only the types, macros and
 * constants those files reference; SDDS I/O, namelists and hash tables are
 * opaque.  Function bodies live in b2e_ref_stubs.c.  This is test
 * infrastructure: nothing in the product links it.
 */
#ifndef B2E_REF_SHIM_H
#define B2E_REF_SHIM_H
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <float.h>
#include <stdint.h>
#include <limits.h>

/* --- SDDS types (opaque) -------------------------------------------------- */
typedef struct { void *opaque; long n_rows; } SDDS_DATASET;
typedef SDDS_DATASET SDDS_TABLE;
typedef struct { char *name; long type; } SDDS_DEFINITION;
#define SDDS_DOUBLE 1
#define SDDS_FLOAT 2
#define SDDS_LONG 3
#define SDDS_SHORT 4
#define SDDS_STRING 5
#define SDDS_CHARACTER 6
#define SDDS_ULONG 7
#define SDDS_USHORT 8
#define SDDS_LONG64 9
#define SDDS_ULONG64 10
#define SDDS_LONGDOUBLE 11
#define SDDS_ANY_NUMERIC_TYPE 99
#define SDDS_ANY_FLOATING_TYPE 98
#define SDDS_ANY_INTEGER_TYPE 97
#define SDDS_CHECK_OK 0
#define SDDS_CHECK_NONEXISTENT 1
#define SDDS_CHECK_WRONGTYPE 2
#define SDDS_CHECK_WRONGUNITS 3
#define SDDS_VERBOSE_PrintErrors 1
#define SDDS_EXIT_PrintErrors 2
#define SDDS_SET_BY_NAME 1
#define SDDS_SET_BY_INDEX 2
#define SDDS_PASS_BY_VALUE 1
#define SDDS_PASS_BY_REFERENCE 2
#define SDDS_GET_BY_NAME 1
#define SDDS_GET_BY_INDEX 2
#define SDDS_ROW_MAJOR_DATA 1
#define SDDS_COLUMN_MAJOR_DATA 2
#define SDDS_BINARY 1
#define SDDS_ASCII 2
#define SDDS_ROW_MAJOR_ORDER 1
#define SDDS_COLUMN_MAJOR_ORDER 2
#define SDDS_PRINT_NOQUOTES 1
#define FLUSH_TABLE 1
#define INVERSE_FFT 1
#define SVN_VERSION "shim"

/* --- namelist / rpn / hash table / table (opaque) ------------------------- */
typedef struct { void *opaque; } NAMELIST_TEXT;
typedef struct htab_s htab;
typedef struct {
  double *c1, *c2, *s1, *s2;
  char *xlab, *ylab, *topline, *title;
  long n_data, flags;
} TABLE;

/* --- matlib MATRIX -------------------------------------------------------- */
typedef struct { double **a; long n, m; } MATRIX;

/* --- mdb.h macros --------------------------------------------------------- */
#ifndef PI
#define PI 3.141592653589793238462643383279502884
#endif
#define SQRT2 1.41421356237309504880
#define PIx2 (2*PI)
#define PIo2 (PI/2)
#define sqr(x) ((x)*(x))
#define SIGN(x) ((x)<0?-1:1)
#define FABS(x) fabs(x)
#define ODD(x) ((x)&1)
#define SWAP_DOUBLE(x, y) { double tmp_swap_d = (x); (x) = (y); (y) = tmp_swap_d; }
#define SWAP_LONG(x, y) { long tmp_swap_l = (x); (x) = (y); (y) = tmp_swap_l; }
#define SWAP_PTR(x, y) { void *tmp_swap_p = (x); (x) = (y); (y) = tmp_swap_p; }
#define ipow1(x) (x)
#define ipow2(x) ((x)*(x))
#define ipow3(x) ((x)*(x)*(x))
#define ipow4(x) (ipow2(x)*ipow2(x))
#define ipow5(x) (ipow4(x)*(x))
#define ipow6(x) (ipow3(x)*ipow3(x))
#define pow2(x) ipow2(x)
#define pow3(x) ipow3(x)
#define pow4(x) ipow4(x)
#define pow5(x) ipow5(x)
#define MAX(a,b) ((a)>(b)?(a):(b))
#define MIN(a,b) ((a)<(b)?(a):(b))
#define tmalloc(n) b2e_shim_tmalloc(n)
#define trealloc(p, n) realloc(p, n)
#define tfree(p) free(p)
#define log_entry(s)
#define log_exit(s)
#define TRUE 1
#define FALSE 0
#define DUMMY_RN_SEED 1
#ifndef STANDARD
#define STANDARD 1
#endif
#ifndef HASHTAB
#define HASHTAB 1
#endif
typedef int32_t int32;

/* --- physical constants (CODATA 2018; the toolkit's own values are not in
 * the tree).  The product uses the same numbers. */
#define c_mks 2.99792458e8
#define e_mks 1.602176634e-19
#define me_mks 9.1093837015e-31
#define mu_o (4*PI*1e-7)
#define epsilon_o (1/(mu_o*c_mks*c_mks))
#define hbar_mks 1.054571817e-34
#define re_mks 2.8179403262e-15
#define mp_mks 1.67262192369e-27
#define k_boltzmann_mks 1.380649e-23
#define h_mks 6.62607015e-34
#define me_mev 0.51099895000
#define mp_mev 938.27208816
#define NAvogadro 6.02214076e23

void *b2e_shim_tmalloc(size_t n);
long ipow_i(long x, long n);
double ipow(double x, long n);
double dfactorial(long n);
long match_string(char *s, char **options, long n, long mode);
double gauss_rn_lim(double mean, double sigma, double limit, double (*urandom)(long));
double random_2(long iseed);
double random_1(long iseed);
double random_3(long iseed);
double random_4(long iseed);
void **czarray_2d(long size, long n1, long n2);
void free_czarray_2d(void **array, long n1, long n2);
void **zarray_2d(long size, long n1, long n2);
void free_zarray_2d(void **array, long n1, long n2);
void *SDDS_Realloc(void *p, size_t n);
void *SDDS_Malloc(size_t n);
void *SDDS_Calloc(size_t n, size_t m);
void SDDS_Bomb(char *msg);
int SDDS_CopyString(char **target, const char *source);
char *cp_str(char **s, char *t);
double interp(double *f, double *x, long n, double xo, long warnings, long order, long *returnCode);
double zeroNewton(double (*fn)(double), double value, double x_i, double dx, long n_passes, double _zero);
double zeroInterp(double (*fn)(double), double value, double x_i, double x_f, double dx, double _zero);
long realFFT2(double *output, double *input, long n, unsigned long flags);
int double_cmpasc(const void *a, const void *b);
long binaryArraySearch(void *array, size_t elemSize, long nElems, void *key, int (*compare)(const void *, const void *), long bracket);
long SavitzyGolaySmooth(double *data, long rows, long order, long nLeft, long nRight, long derivativeOrder);
#define SavitzkyGolaySmooth SavitzyGolaySmooth
#endif
