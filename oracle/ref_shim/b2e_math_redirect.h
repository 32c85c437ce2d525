/*
 * Forced-include header for the shared-maths build of the reference oracle:
 * routes the reference's per-particle elementary functions to the
 * implementations the CUDA engine uses (elegant_b200/csrc/b2e_math.h), so the
 * reference's own tracking code and the GPU agree bit for bit.  sqrt,
 * division and the arithmetic operators are IEEE correctly rounded on both
 * sides and stay as they are.
 */
#ifndef B2E_MATH_REDIRECT_H
#define B2E_MATH_REDIRECT_H
#include <math.h>
#include "b2e_math.h"
#define sin(x) b2e_sin(x)
#define cos(x) b2e_cos(x)
#define tan(x) b2e_tan(x)
#define asin(x) b2e_asin(x)
#define pow(x, y) b2e_pow(x, y)
#define log(x) b2e_log(x)
#endif
