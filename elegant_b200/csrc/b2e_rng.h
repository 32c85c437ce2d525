/*
 * Counter-based Gaussian deviates for incoherent synchrotron radiation (ISR).
 *
 * The reference draws ISR deviates with gauss_rn_lim(0, 1, srGaussianLimit,
 * random_2) (multipole.c:1343, csbend.c:1619): one serial generator shared by
 * all particles in tracking order, which a parallel tracker cannot follow.
 * Here every deviate has an address instead -- (seed; particle ID, pass,
 * element, slice, integrator step, draw) -- and is a pure function of it:
 *
 *   Philox4x32-10 (Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as
 *   easy as 1, 2, 3", SC 2011): counter {id_lo, id_hi, pass, site}, key
 *   {seed_lo, seed_hi}; site = ((element * 256 + slice) * 8 + step) * 16 + draw;
 *   two 53-bit uniforms from the four output words; Box-Muller with the shared
 *   log/sin/cos (b2e_math.h): g = sqrt(-2 ln(1 - u1)) cos(2 pi u2);
 *   truncation as gauss_rn_lim: a deviate with |g| > limit (limit > 0) is
 *   redrawn with the next draw index, at most 16 draws (then 0).
 *   The amplitude's pow(F2, 0.75) is b2e_isr_pow34.
 *
 * So the device and the C restatement produce the same deviates bit for bit,
 * independent of launch shape, compaction or the order particles are tracked
 * in; the distribution is the reference's (a unit Gaussian cut at the limit),
 * its sequence is not.  Plain C for gcc; host+device under nvcc.
 */
#ifndef B2E_RNG_H
#define B2E_RNG_H
#include <stdint.h>
#include "b2e_math.h"

#ifdef __CUDACC__
#define B2E_RNG_FN __host__ __device__ static inline
#else
#define B2E_RNG_FN static inline
#endif

#define B2E_ISR_MAX_SLICES 256
#define B2E_ISR_MAX_ELEMENTS 131072
#define B2E_ISR_MAX_DRAWS 16

B2E_RNG_FN void b2e_mulhilo32(uint32_t a, uint32_t b, uint32_t *hi, uint32_t *lo) {
  const uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  *lo = (uint32_t)p;
}

/* Philox4x32 with 10 rounds */
B2E_RNG_FN void b2e_philox4x32(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3], k0 = key_in[0], k1 = key_in[1];
  int r;
  for (r = 0; r < 10; r++) {
    uint32_t hi0, lo0, hi1, lo1;
    b2e_mulhilo32(0xD2511F53u, c0, &hi0, &lo0);
    b2e_mulhilo32(0xCD9E8D57u, c2, &hi1, &lo1);
    c0 = hi1 ^ c1 ^ k0;
    c1 = lo1;
    c2 = hi0 ^ c3 ^ k1;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

/* 53-bit uniform in [0, 1) from two words */
B2E_RNG_FN double b2e_u53(uint32_t hi, uint32_t lo) {
  return ((double)(hi >> 5) * 67108864.0 + (double)(lo >> 6)) * (1.0 / 9007199254740992.0);
}

/* F2^(3/4) of the ISR amplitude (the reference's pow(F2, 0.75)) as
 * sqrt(F2) sqrt(sqrt(F2)): correctly rounded square roots only, so host and
 * device agree; within 2 ulp of pow */
B2E_RNG_FN double b2e_isr_pow34(double f2) {
  const double r = sqrt(f2);
  return r * sqrt(r);
}

/* the truncated unit Gaussian at one address */
B2E_RNG_FN double b2e_isr_gauss(uint64_t seed, int64_t id, int32_t pass, int32_t element, int32_t slice, int32_t step,
                                double limit) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  const uint32_t site0 = ((((uint32_t)element * B2E_ISR_MAX_SLICES + (uint32_t)slice) * 8u + (uint32_t)step) *
                          B2E_ISR_MAX_DRAWS);
  int draw;
  for (draw = 0; draw < B2E_ISR_MAX_DRAWS; draw++) {
    const uint32_t ctr[4] = {(uint32_t)(uint64_t)id, (uint32_t)((uint64_t)id >> 32), (uint32_t)pass,
                             site0 + (uint32_t)draw};
    uint32_t w[4];
    double u1, u2, g;
    b2e_philox4x32(ctr, key, w);
    u1 = 1.0 - b2e_u53(w[0], w[1]); /* (0, 1] */
    u2 = b2e_u53(w[2], w[3]);
    g = sqrt(-2.0 * b2e_log(u1)) * b2e_cos(6.283185307179586 * u2);
    if (!(limit > 0) || fabs(g) <= limit)
      return g;
  }
  return 0;
}

#endif
