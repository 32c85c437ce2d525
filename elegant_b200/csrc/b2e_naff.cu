/*
 * NAFF: the strongest frequency of sampled signals, one CTA per signal, and
 * the tunes of turn-by-turn data (computeTunesFromTracking, twiss.cc:3799-4032,
 * with adjustTuneHalfPlane, :4036-4046).
 *
 * The reference calls the SDDS toolkit's PerformNAFF with one frequency and a
 * 1e-12 frequency accuracy; that routine is not in the reference tree, so the
 * method here is this library's statement of Laskar's NAFF for one line:
 *   y_t = (x_t - mean(x)) w_t, w_t = 1 - cos(2 pi t / N) (Hann, mean 1);
 *   coarse: the largest |F(k/N)|^2, k = 1..N/2, F(nu) = sum_t y_t e^{-2 pi i nu t};
 *   fine: the maximum of |F(nu)|^2 on [(k-1)/N, (k+1)/N] within [0, 1/2],
 *         60 bisections on the sign of its derivative
 *         2 Re(conj(F) dF/dnu) (a zero crossing is located to rounding,
 *         where a search on |F|^2 itself stops at the square root of it);
 *   amplitude 2 |F(nu)| / N, phase arg F(nu).
 * Sums run over a twiddle table of the shared sin/cos (b2e_math.h) for the
 * grid and b2e_sincos for off-grid frequencies; CTA reductions are a fixed
 * tree, so results do not depend on scheduling.
 */
#include <math.h>
#include <algorithm>
#include <cuda_runtime.h>
#include "b2e_engine.h"
#include "b2e_kernels.h"
#include "b2e_math.h"
#include "b2e_fft.h"

namespace b2e {

#define NAFF_THREADS 256
#define NAFF_BISECTIONS 60

/* sum of a and b over the CTA (fixed order: lanes by shuffles, then warps in
 * index order on thread 0); the result is valid on every thread */
__device__ void naff_reduce2(double &a, double &b, double *red) {
  for (int off = 16; off > 0; off >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, off);
    b += __shfl_down_sync(0xffffffffu, b, off);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) {
    red[2 * warp] = a;
    red[2 * warp + 1] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sa = 0, sb = 0;
    for (int w = 0; w < nw; w++) {
      sa += red[2 * w];
      sb += red[2 * w + 1];
    }
    red[64] = sa;
    red[65] = sb;
  }
  __syncthreads();
  a = red[64];
  b = red[65];
}

/* sums of four values over the CTA, like naff_reduce2 */
__device__ void naff_reduce4(double v[4], double *red) {
  for (int off = 16; off > 0; off >>= 1)
    for (int k = 0; k < 4; k++)
      v[k] += __shfl_down_sync(0xffffffffu, v[k], off);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0)
    for (int k = 0; k < 4; k++)
      red[4 * warp + k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    double s[4] = {0, 0, 0, 0};
    for (int w = 0; w < nw; w++)
      for (int k = 0; k < 4; k++)
        s[k] += red[4 * w + k];
    for (int k = 0; k < 4; k++)
      red[128 + k] = s[k];
  }
  __syncthreads();
  for (int k = 0; k < 4; k++)
    v[k] = red[128 + k];
}

/* F(nu) = sum_t y_t e^{-2 pi i nu t} and dF/dnu (all threads get the sums);
 * returns d|F|^2/dnu */
__device__ double naff_slope(const double *y, int N, double nu, double *re, double *im, double *red) {
  double v[4] = {0, 0, 0, 0};
  for (int t = threadIdx.x; t < N; t += blockDim.x) {
    double sn, cs;
    b2e_sincos(6.283185307179586 * nu * t, &sn, &cs);
    const double w = 6.283185307179586 * t;
    v[0] += y[t] * cs;
    v[1] -= y[t] * sn;
    v[2] -= (y[t] * w) * sn;
    v[3] -= (y[t] * w) * cs;
  }
  naff_reduce4(v, red);
  *re = v[0];
  *im = v[1];
  return 2 * (v[0] * v[2] + v[1] * v[3]);
}

/* NAFF of x[t * stride], t < N, by the whole CTA; sm holds 3N doubles.
 * Returns through the pointers on thread 0; *bad = 1 for a non-finite sample. */
__device__ void naff_block(const double *x, int64_t stride, int N, double *freq, double *amp, double *phase,
                           int *bad, double *sm) {
  __shared__ double red[136];
  __shared__ int s_k;
  double *y = sm, *tc = sm + N, *ts = sm + 2 * N;
  double sum = 0, dummy = 0;
  int nonfinite = 0;
  for (int t = threadIdx.x; t < N; t += blockDim.x) {
    const double v = x[(int64_t)t * stride];
    y[t] = v;
    nonfinite |= !isfinite(v);
    sum += v;
    b2e_dft_twiddle(N, t, &tc[t], &ts[t]);
  }
  nonfinite = __syncthreads_or(nonfinite);
  naff_reduce2(sum, dummy, red);
  if (nonfinite) {
    if (threadIdx.x == 0) {
      *freq = *amp = *phase = 0;
      *bad = 1;
    }
    return;
  }
  const double mean = sum / N;
  for (int t = threadIdx.x; t < N; t += blockDim.x)
    y[t] = (y[t] - mean) * (1 - tc[t]);
  __syncthreads();
  /* coarse: the grid line of largest power, the lowest k on ties */
  double best = -1;
  int bestk = 1;
  for (int k = 1 + threadIdx.x; k <= N / 2; k += blockDim.x) {
    double r = 0, i = 0;
    int64_t idx = 0;
    for (int t = 0; t < N; t++) {
      r += y[t] * tc[idx];
      i -= y[t] * ts[idx];
      idx += k;
      if (idx >= N)
        idx -= N;
    }
    const double pw = r * r + i * i;
    if (pw > best) {
      best = pw;
      bestk = k;
    }
  }
  for (int off = 16; off > 0; off >>= 1) {
    const double ob = __shfl_down_sync(0xffffffffu, best, off);
    const int ok = __shfl_down_sync(0xffffffffu, bestk, off);
    if (ob > best || (ob == best && ok < bestk)) {
      best = ob;
      bestk = ok;
    }
  }
  __shared__ double wbest[32];
  __shared__ int wk[32];
  if ((threadIdx.x & 31) == 0) {
    wbest[threadIdx.x >> 5] = best;
    wk[threadIdx.x >> 5] = bestk;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = -1;
    int kk = 1;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++)
      if (wbest[w] > b || (wbest[w] == b && wk[w] < kk)) {
        b = wbest[w];
        kk = wk[w];
      }
    s_k = kk;
  }
  __syncthreads();
  /* fine: bisection on the sign of d|F|^2/dnu inside [(k-1)/N, (k+1)/N]
   * (every thread keeps the same bracket: the sums come back from the
   * reduction on all threads) */
  double a = (s_k - 1.0) / N, b = (s_k + 1.0) / N, re, im;
  if (a < 0)
    a = 0;
  if (b > 0.5)
    b = 0.5;
  for (int it = 0; it < NAFF_BISECTIONS; it++) {
    const double m = 0.5 * (a + b);
    if (naff_slope(y, N, m, &re, &im, red) > 0)
      a = m;
    else
      b = m;
  }
  const double nu = 0.5 * (a + b);
  naff_slope(y, N, nu, &re, &im, red);
  const double pw = re * re + im * im;
  if (threadIdx.x == 0) {
    *freq = nu;
    *amp = 2 * sqrt(pw) / N;
    *phase = atan2(im, re);
    *bad = 0;
  }
}

__global__ void __launch_bounds__(NAFF_THREADS) naff_kernel(const double *sig, int N, double *freq, double *amp,
                                                            double *phase) {
  extern __shared__ double sm[];
  int bad;
  naff_block(sig + (size_t)blockIdx.x * N, 1, N, freq + blockIdx.x, amp + blockIdx.x, phase + blockIdx.x, &bad,
             sm);
}

/* one CTA per (particle, coordinate): record r of coordinate c of particle i
 * at tbt[(r * 4 + c) * rows + i] */
__global__ void __launch_bounds__(NAFF_THREADS) tbt_naff_kernel(const double *tbt, int64_t rows, int first, int N,
                                                                double *out /* [4][3][rows] */, int *bad) {
  extern __shared__ double sm[];
  const int64_t i = blockIdx.x;
  const int c = blockIdx.y;
  int b = 0;
  naff_block(tbt + ((int64_t)first * 4 + c) * rows + i, 4 * rows, N, out + (c * 3 + 0) * rows + i,
             out + (c * 3 + 1) * rows + i, out + (c * 3 + 2) * rows + i, &b, sm);
  if (threadIdx.x == 0 && b)
    bad[i] = 1;
}

/* adjustTuneHalfPlane (twiss.cc:4036-4046) */
__device__ __forceinline__ double adjust_tune_half_plane(double frequency, double phase0, double phase1) {
  const double pi = 3.141592653589793, pix2 = 6.283185307179586;
  if (fabs(phase0 - phase1) > pi) {
    if (phase0 < phase1)
      phase0 += pix2;
    else
      phase1 += pix2;
  }
  if (phase0 < phase1)
    return frequency;
  return 1 - frequency;
}

__global__ void tbt_tunes_kernel(const double *out, const int *bad, int64_t rows, double *nu) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= rows)
    return;
  double nux = -1, nuy = -1, ax = 0, ay = 0;
  if (!bad[i]) {
    nux = adjust_tune_half_plane(out[(0 * 3 + 0) * rows + i], out[(0 * 3 + 2) * rows + i],
                                 out[(1 * 3 + 2) * rows + i]);
    nuy = adjust_tune_half_plane(out[(2 * 3 + 0) * rows + i], out[(2 * 3 + 2) * rows + i],
                                 out[(3 * 3 + 2) * rows + i]);
    ax = out[(0 * 3 + 1) * rows + i];
    ay = out[(2 * 3 + 1) * rows + i];
  }
  nu[i] = nux;
  nu[rows + i] = nuy;
  nu[2 * rows + i] = ax;
  nu[3 * rows + i] = ay;
}

cudaError_t launch_naff(const double *sig, int64_t n_signals, int N, double *freq, double *amp, double *phase,
                        cudaStream_t stream) {
  const size_t smem = sizeof(double) * 3 * N;
  cudaError_t e = cudaFuncSetAttribute(naff_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess)
    return e;
  for (int64_t s0 = 0; s0 < n_signals; s0 += 65535) {
    const int nb = (int)std::min<int64_t>(65535, n_signals - s0);
    naff_kernel<<<nb, NAFF_THREADS, smem, stream>>>(sig + s0 * N, N, freq + s0, amp + s0, phase + s0);
  }
  return cudaGetLastError();
}

cudaError_t launch_tbt_tunes(const double *tbt, int64_t rows, int first, int N, double *scratch, int *bad,
                             double *nu, cudaStream_t stream) {
  const size_t smem = sizeof(double) * 3 * N;
  cudaError_t e = cudaFuncSetAttribute(tbt_naff_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess)
    return e;
  for (int64_t i0 = 0; i0 < rows; i0 += 65535) {
    const int nb = (int)std::min<int64_t>(65535, rows - i0);
    tbt_naff_kernel<<<dim3(nb, 4), NAFF_THREADS, smem, stream>>>(tbt + i0, rows, first, N, scratch + i0, bad + i0);
  }
  tbt_tunes_kernel<<<(unsigned)((rows + 255) / 256), 256, 0, stream>>>(scratch, bad, rows, nu);
  return cudaGetLastError();
}

} // namespace b2e
