/*
 * CSR step on the device: CSRCSBEND (track_through_csbendCSR, csbend.c:1899-3044)
 * and CSRDRIFT mode 0 (track_through_driftCSR, csbend.c:3176-3533).
 * See b2e_csr.h for the kernel pipeline.  Every floating-point expression
 * keeps the reference's operation order; histogram counts are integers and
 * min/max are exact, so the pipeline reproduces the CPU oracle bit for bit
 * regardless of thread scheduling.
 */
#include <math.h>
#include <string.h>
#include <stdio.h>
#include <algorithm>
#include <mutex>
#include <type_traits>
#include <utility>
#include "b2e_csr.h"
#include "b2e_roots.h"
#include "b2e_fft.h"
#include "b2e_elements.cuh"
#include "b2e_kernels.h"
#include "b2e_sg.h"
#include "b2e_wakenet.h"

namespace b2e {

static const double kPI = 3.141592653589793238462643383279502884;
static const double kC = 2.99792458e8;
static const double kE = 1.602176634e-19;
static const double kME = 9.1093837015e-31;

struct CsrDevState {
  unsigned long long ct_min_key, ct_max_key; /* order-preserving keys of min/max c*t */
  double ctLower, ctUpper, dct;              /* binning of the current kick */
  double s0, dctBin;                         /* csrWake.s0, csrWake.dctBin */
  long long nBinned;
  double dGamma[B2E_CSR_MAX_BINS];           /* csrWake.dGamma: last dipole wake */
  double phi_last;                           /* SolveForPhiStupakov's start value */
};

/* Per-bunch view for the CSR kernels.  Bunches are contiguous particle ranges
 * [offs[b], offs[b+1]); each has its own binning and wake state, its own
 * CSRConstant (zero when the bunch has at most one particle at the element
 * entrance) and, in CSRDRIFT, its own choice between wake kicks and the exact
 * drift.  A single bunch is n = 1 (offs is then not read). */
struct CsrBunches {
  const int64_t *offs;
  int n;
  CsrDevState *st;
  const double *csr_const; /* [3][n]: CSRConstant, the IGF wake factor, GSConstant */
  const unsigned char *active; /* more than one particle alive at the element entrance */
  const unsigned char *mode;   /* CSRDRIFT: 1 = wake kicks, 0 = exact drift */
};

__device__ __forceinline__ int bunch_of(int64_t i, const CsrBunches &B) {
  if (B.n <= 1)
    return 0;
  int lo = 0, hi = B.n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (B.offs[mid] <= i)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

__device__ __forceinline__ unsigned long long key_of(double v) {
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double value_of(unsigned long long k) {
  unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)b);
}

/* binParticleCoordinate's range expansion (csbend.c:3079-3094) */
__device__ __forceinline__ void expand_range(double *lower, double *upper, double factor) {
  if (factor > 1) {
    double center = (*lower + *upper) / 2, range = (*upper - *lower) * factor;
    *lower = center - range / 2;
    *upper = center + range / 2;
  }
}

__device__ __forceinline__ void block_minmax(double v, bool valid, CsrDevState *st) {
  unsigned long long kmin = valid ? key_of(v) : ~0ull, kmax = valid ? key_of(v) : 0ull;
  for (int off = 16; off > 0; off >>= 1) {
    kmin = min(kmin, __shfl_down_sync(0xffffffffu, kmin, off));
    kmax = max(kmax, __shfl_down_sync(0xffffffffu, kmax, off));
  }
  if ((threadIdx.x & 31) == 0) {
    if (kmin != ~0ull)
      atomicMin(&st->ct_min_key, kmin);
    if (kmax != 0ull)
      atomicMax(&st->ct_max_key, kmax);
  }
}

/* min/max of c*t per bunch: a warp whose lanes all belong to one bunch
 * reduces first; a warp that straddles bunches updates lane by lane. */
__device__ __forceinline__ void bunch_minmax(double v, bool valid, int b, const CsrBunches &B) {
  const int b0 = __shfl_sync(0xffffffffu, b, 0);
  if (__all_sync(0xffffffffu, b == b0)) {
    block_minmax(v, valid, B.st + b0);
  } else if (valid) {
    atomicMin(&B.st[b].ct_min_key, key_of(v));
    atomicMax(&B.st[b].ct_max_key, key_of(v));
  }
}

/* CSR energy kick from the previous kick's wake (csbend.c:2692-2711) */
__device__ __forceinline__ double csr_kick(double CT, double X, double DP, const CsrDevState *st, int nBins,
                                           double Po, double rho0) {
  double f = (CT - st->ctLower) / st->dct;
  long long iBin = (long long)f;
  f -= iBin;
  if (iBin >= 0 && iBin < nBins - 1)
    DP += ((1 - f) * st->dGamma[iBin] + f * st->dGamma[iBin + 1]) / Po * (1 + X / rho0);
  return DP;
}

/* Programmatic dependent launch (sm_90 and later, PTX griddepcontrol): a
 * kernel of the kick chain launched with the programmatic-serialization
 * attribute may be scheduled while its predecessor's last CTAs still run.
 * Each such kernel first lets its own successor be scheduled (once all of its
 * CTAs have started), then waits until the predecessor grid has completed
 * and its memory is visible, before touching any memory.  In a kernel
 * launched without the attribute both instructions return at once. */
__device__ __forceinline__ void chain_enter() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

/* entrance: offsets, tilt, c*t = s/beta, entrance edge (csbend.c:2286-2377) */
__global__ void csr_entry_kernel(DevParticles P, int64_t n, double *beta0, const DevElem *ep, BendExtra bx,
                                 double Po) {
  chain_enter();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n || P.lost_pass[i] >= 0)
    return;
  const DevElem &e = *ep;
  const double *c = e.c;
  const double ct = c[CB_COS_TT], st = c[CB_SIN_TT];
  double x = P.x[i], xp = P.xp[i], y = P.y[i], yp = P.yp[i], s = P.s[i], dp = P.dp[i];
  double X, Y, XP, YP, p0, b0, rho;
  s = s + c[CB_DZI] * sqrt((1 + xp * xp) + yp * yp);
  x = (x + c[CB_DXI]) + c[CB_DZI] * xp;
  y = (y + c[CB_DYI]) + c[CB_DZI] * yp;
  X = x * ct + y * st;
  Y = -x * st + y * ct;
  XP = xp * ct + yp * st;
  YP = -xp * st + yp * ct;
  p0 = Po * (1 + dp);
  b0 = p0 / sqrt(p0 * p0 + 1);
  s = s / b0;
  if (e.flags & EF_EDGE1) {
    rho = (1 + dp) * c[CB_RHO_ACTUAL];
    if (e.flags & EF_EDGE_ORDER2) {
      bend_edge_order2(X, XP, Y, YP, rho, c[CB_PSI1] * (1 + dp), c[CB_TAN_E1], c[CB_E1], bx.c[BX_SEC2_E1],
                       bx.c[BX_EDGE_N], -1);
    } else {
      XP = XP + (c[CB_TAN_E1] / rho) * X;
      YP = YP - (b2e_tan(c[CB_E1] - c[CB_PSI1] / (1 + dp)) / rho) * Y;
    }
  }
  P.x[i] = X;
  P.xp[i] = XP;
  P.y[i] = Y;
  P.yp[i] = YP;
  P.s[i] = s;
  beta0[i] = b0;
}

/* one kick: optional wake kick of the previous kick, one integrator slice,
 * c*t update, min/max of c*t (csbend.c:2385-2450, :3066-3076) */
/* 64 registers (4 blocks of 256 per SM): twice the resident warps of the
 * unconstrained build, the FP64 chains' latency being what limits it */
__global__ void __launch_bounds__(256, 4) csr_slice_kernel(DevParticles P, int64_t n, const double *beta0, const DevElem *ep,
                                 const DevAperture *ap, CsrBunches B, int after_first_kick, int nBins, double Po,
                                 int pass, int elem_index) {
  chain_enter();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  bool alive = i < n && P.lost_pass[i] < 0;
  const int b = i < n ? bunch_of(i, B) : B.n - 1;
  const CsrDevState *st = B.st + b;
  const int apply_kick = after_first_kick && B.csr_const[b] != 0;
  double CT = 0;
  if (alive) {
    const DevElem &e = *ep;
    const double *c = e.c;
    double X = P.x[i], XP = P.xp[i], Y = P.y[i], YP = P.yp[i], DP = P.dp[i], f, Q1, Q3, Q4;
    CT = P.s[i];
    if (apply_kick)
      DP = csr_kick(CT, X, DP, st, nBins, Po, c[CB_RHO0]);
    f = (1 + DP) / sqrt((1 + XP * XP) + YP * YP);
    Q1 = XP * f;
    Q3 = YP * f;
    const RadSite no_rad = {0, 0, 0, 0, 0, nullptr};
    const int nsub = (int)c[CB_NSUB];
    int lost = nsub == 4 ? csbend_integrate<false, 4>(X, Q1, Y, Q3, Q4, DP, c, 1, nsub, false, ap, e, no_rad)
                         : csbend_integrate<false>(X, Q1, Y, Q3, Q4, DP, c, 1, nsub, false, ap, e, no_rad);
    f = 1 / sqrt(((1 + DP) * (1 + DP) - Q1 * Q1) - Q3 * Q3);
    Q1 = Q1 * f;
    Q3 = Q3 * f;
    P.x[i] = X;
    P.xp[i] = Q1;
    P.y[i] = Y;
    P.yp[i] = Q3;
    P.dp[i] = DP;
    if (lost) {
      P.lost_pass[i] = pass;
      P.lost_elem[i] = elem_index;
      alive = false;
    } else {
      CT = CT + Q4 / beta0[i];
      P.s[i] = CT;
    }
  }
  bunch_minmax(CT, alive, b, B);
}

/* histogram of c*t with the range of binParticleCoordinate (csbend.c:3047-3113):
 * shared-memory integer counts, then added to global counts. */
static const int kHistUnroll = 4;

/* Copies of the shared-memory counts per histogram CTA: warp w adds into
 * copy w % copies, so warps of a CTA do not queue on the central bins' counters
 * (integer counts: the sum over copies is the same in any order).  As many
 * as fit 48 KB, at most B2E_HIST_COPIES.  One by default: on the 1e6-particle
 * chicane (600 bins) 1, 4 and 8 copies measured 94.1, 94.2 and 94.5 us per
 * kick (the zeroing and the final sum over copies cost what the spread
 * saves); a compile-time option for beams with sharper peaks. */
#ifndef B2E_HIST_COPIES
#define B2E_HIST_COPIES 1
#endif
static inline size_t hist_smem(int nBins) {
  const size_t one = sizeof(unsigned int) * (size_t)nBins;
  size_t copies = (48 * 1024) / one;
  copies = copies < 1 ? 1 : (copies > B2E_HIST_COPIES ? B2E_HIST_COPIES : copies);
  return copies * one;
}

/* histogram CTAs (1024 threads) per bunch: one per 1024 particles, at most two
 * resident CTAs per SM over all bunches (each thread then takes up to
 * kHistUnroll particles per sweep) */
static inline int hist_blocks(int64_t per_bunch, int nbunch) {
  return (int)std::min<int64_t>(std::max<int64_t>(1, 148 * 2 / std::max(nbunch, 1)),
                                std::max<int64_t>(1, (per_bunch + 1023) / 1024));
}

/* launch with programmatic stream serialization (the kernel begins with
 * chain_enter) */
template <typename... KArgs, typename... Args>
static cudaError_t launch_chained(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                                  Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

__global__ void csr_hist_kernel(DevParticles P, int64_t n, CsrBunches B, unsigned int *counts_all, int nBins,
                                double factor) {
  extern __shared__ unsigned int scount[];
  chain_enter();
  const int bunch = blockIdx.y;
  if (!B.active[bunch])
    return;
  CsrDevState *st = B.st + bunch;
  unsigned int *counts = counts_all + (size_t)bunch * nBins;
  const int64_t first = B.n <= 1 ? 0 : B.offs[bunch], end = B.n <= 1 ? n : B.offs[bunch + 1];
  double lower = value_of(st->ct_min_key), upper = value_of(st->ct_max_key), dct;
  expand_range(&lower, &upper, factor);
  dct = (upper - lower) / nBins;
  /* the launch gives copies x nBins counters (hist_smem) */
  unsigned int smem_bytes;
  asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(smem_bytes));
  const int copies = (int)(smem_bytes / (sizeof(unsigned int) * nBins));
  unsigned int *mycount = scount + (size_t)((threadIdx.x >> 5) % copies) * nBins;
  for (int b = threadIdx.x; b < copies * nBins; b += blockDim.x)
    scount[b] = 0;
  __syncthreads();
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->ctLower = lower;
    st->ctUpper = upper;
    st->dct = dct;
  }
  /* kHistUnroll particles per thread and sweep, their loads issued together
   * (the loss word and c*t are read unconditionally within the range, so
   * neither waits on the other); the loop bounds are uniform over the block */
  /* (c*t - lower)/dct through the stored reciprocal, correctly rounded as the
   * division (div_rn_recip), while dct is a normal number well inside the
   * range where 1/dct and the remainder stay normal */
  const double inv_dct = 1.0 / dct;
  const bool recip_ok = dct > 1e-280 && dct < 1e280;
  /* chunks of blockDim.x particles, chunk c to CTA c mod gridDim.x */
  const int64_t G = gridDim.x, D = blockDim.x;
  for (int64_t c0 = blockIdx.x; first + c0 * D < end; c0 += G * kHistUnroll) {
    int32_t lp[kHistUnroll];
    double ct[kHistUnroll];
#pragma unroll
    for (int u = 0; u < kHistUnroll; u++) {
      const int64_t i = first + (c0 + u * G) * D + threadIdx.x;
      lp[u] = i < end ? P.lost_pass[i] : 0;
      ct[u] = i < end ? P.s[i] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kHistUnroll; u++) {
      const int64_t i = first + (c0 + u * G) * D + threadIdx.x;
      int bin = -1;
      if (i < end && lp[u] < 0) {
        const double a = ct[u] - lower;
        long long b = (long long)(recip_ok ? div_rn_recip(a, dct, inv_dct) : a / dct);
        if (b >= 0 && b <= nBins - 1)
          bin = (int)b;
      }
      /* one shared-memory atomic per particle, unless neighbouring lanes
       * share a bin (a beam stored in c*t order, where a warp's particles
       * would queue on one counter): then one atomic per distinct bin */
      const int lane = threadIdx.x & 31;
      const int prev = __shfl_up_sync(0xffffffffu, bin, 1);
      if (__any_sync(0xffffffffu, lane > 0 && bin >= 0 && bin == prev)) {
        const unsigned int peers = __match_any_sync(0xffffffffu, bin);
        if (bin >= 0 && lane == __ffs(peers) - 1)
          atomicAdd(&mycount[bin], (unsigned int)__popc(peers));
      } else if (bin >= 0) {
        atomicAdd(&mycount[bin], 1u);
      }
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < nBins; b += blockDim.x) {
    unsigned int c = 0;
    for (int k = 0; k < copies; k++)
      c += scount[(size_t)k * nBins + b];
    if (c)
      atomicAdd(&counts[b], c);
  }
}

struct WakeArgs {
  int nBins, sgHalf, sgdHalf, trapz, steady, correct;
  const double *sg_w, *sgd_w; /* [nBins][B2E_SG_MAX_WIDTH] */
  const int *sg_lo, *sg_n, *sgd_lo, *sgd_n;
  double slippage, slippage13, c1, c2, csr_constant;
  double length, nSlices;   /* element length and kicks: c1 and c2 of each bunch */
  double *wakelog;          /* nBins values per bunch for this kick, or null */
  /* page record (CSRCSBEND OUTPUT_FILE): B2E_CSR_PAGE_HEADER + 4 nBins values
   * per bunch for this kick, or null; the header's host-known fields */
  double *pagelog;
  double page_element, page_kick, page_angle, page_ds_kick, page_p_central, page_range_factor;
  /* integrated Green's function (csbend.c:2593-2621, :2676-2680) */
  int igf;
  double gamma2, gamma3, rho0, const1, q4pe, igf_factor;
  /* low/high-pass filters of the histogram (applyLHPassFilters): on when
   * HIGH_FREQUENCY_CUTOFF0 > 0 or LOW_FREQUENCY_CUTOFF0 >= 0 */
  int lh, clip;
  double startHP, endHP, startLP, endLP;
};

/* applyLHPassFilters (csbend.c:4611-4703) on hist[0..nb) in one CTA with the
 * transform of b2e_fft.h; scratch: ri = sm + nb (nb + 2 values), twiddles at
 * sm + 2 nb + 2 and sm + 3 nb + 2 (the filters' arrays are not yet in use) */
__device__ void lh_pass_filters(const WakeArgs &a, double *sm) {
  const int nb = a.nBins, freq = nb / 2 + 1;
  double *hist = sm, *ri = sm + nb, *tc = sm + 2 * nb + 2, *ts = sm + 3 * nb + 2;
  __shared__ double orig_sum;
  for (int t = threadIdx.x; t < nb; t += blockDim.x)
    b2e_dft_twiddle(nb, t, &tc[t], &ts[t]);
  __syncthreads();
  for (int k = threadIdx.x; k < freq; k += blockDim.x)
    b2e_rdft_pair(hist, nb, k, tc, ts, &ri[2 * k], &ri[2 * k + 1]);
  __syncthreads();
  if (threadIdx.x == 0) {
    b2e_lh_ramps(ri, freq, a.startHP, a.endHP, a.startLP, a.endLP);
    double sum = 0;
    for (int b = 0; b < nb; b++)
      sum += hist[b];
    orig_sum = sum;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < nb; j += blockDim.x)
    hist[j] = b2e_rdft_sample(ri, nb, j, tc, ts);
  __syncthreads();
  if (a.clip) {
    /* correctDistribution (csbend.c:4705-4721) to the unfiltered sum */
    __shared__ double factor;
    __shared__ int skip;
    if (threadIdx.x == 0) {
      double sum = 0;
      for (int b = 0; b < nb; b++) {
        if (hist[b] < 0)
          hist[b] = 0;
        sum += hist[b];
      }
      skip = !sum;
      factor = skip ? 1 : orig_sum / sum;
    }
    __syncthreads();
    if (!skip)
      for (int b = threadIdx.x; b < nb; b += blockDim.x)
        hist[b] = hist[b] * factor;
    __syncthreads();
  }
}

/* Savitzky-Golay pass with precomputed per-bin weights (b2e_sg.h convention);
 * lo/wn point into an interleaved (start, width) table, stride 2 per bin. */
__device__ void sg_apply(const double *in, double *out, int nBins, const double *w, const int *lo, const int *wn) {
  for (int b = threadIdx.x; b < nBins; b += blockDim.x) {
    double s = 0;
    const double *wb = w + (size_t)b * B2E_SG_MAX_WIDTH;
    const int start = lo[2 * b], width = wn[2 * b];
    for (int k = 0; k < width; k++)
      s += wb[k] * in[start + k];
    out[b] = s;
  }
}

/* ((v[0] + v[1]) + v[2]) + ... in index order, as a serial loop forms it;
 * the next eight values load while the current eight are added */
__device__ __forceinline__ double ordered_sum(const double *v, int n) {
  double s = 0;
  int b = 0;
  if (n >= 8) {
    double r[8];
#pragma unroll
    for (int k = 0; k < 8; k++)
      r[k] = v[k];
    for (b = 8; b + 8 <= n; b += 8) {
      double q[8];
#pragma unroll
      for (int k = 0; k < 8; k++)
        q[k] = v[b + k];
#pragma unroll
      for (int k = 0; k < 8; k++)
        s += r[k];
#pragma unroll
      for (int k = 0; k < 8; k++)
        r[k] = q[k];
    }
#pragma unroll
    for (int k = 0; k < 8; k++)
      s += r[k];
  }
  for (; b < n; b++)
    s += v[b];
  return s;
}

/* bring this thread's rows of both Savitzky-Golay tables toward L1 while the
 * counts load, so that the two filter passes do not wait on L2 */
__device__ __forceinline__ void prefetch_sg_rows(const WakeArgs &a) {
  for (int b = threadIdx.x; b < a.nBins; b += blockDim.x) {
    if (a.sgHalf > 0) {
      asm volatile("prefetch.global.L1 [%0];" ::"l"(a.sg_w + (size_t)b * B2E_SG_MAX_WIDTH));
      asm volatile("prefetch.global.L1 [%0];" ::"l"(a.sg_lo + 2 * b));
    }
    asm volatile("prefetch.global.L1 [%0];" ::"l"(a.sgd_w + (size_t)b * B2E_SG_MAX_WIDTH));
    asm volatile("prefetch.global.L1 [%0];" ::"l"(a.sgd_lo + 2 * b));
  }
}

/* Filters of one kick's wake (csbend.c:2566-2591) on one CTA: Savitzky-Golay
 * smoothing of the counts, correctDistribution, density per unit ct, its
 * derivative filter and the (dct*b)^(1/3) denominators.  Leaves hist = sm,
 * deriv = sm + nBins, denom = sm + 2 nBins (tmp = sm + 3 nBins is scratch). */
template <typename CountT, typename SumT>
__device__ void wake_filters(const CountT *counts, const WakeArgs &a, const double dct, double *sm, SumT *nbinned_out) {
  const int nb = a.nBins;
  double *hist = sm, *deriv = sm + nb, *denom = sm + 2 * nb, *tmp = sm + 3 * nb;
  __shared__ double nBinnedD;
  __shared__ int skip;
  __shared__ SumT warp_sums[32];
  prefetch_sg_rows(a);
  if constexpr (std::is_integral<SumT>::value) {
    /* integer counts: the total is exact in any order, so it is a block
     * reduction (per thread, warp shuffles, then the warps' totals) */
    SumT part = 0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
      const CountT v = counts[b];
      hist[b] = (double)v;
      part += v;
    }
    for (int o = 16; o > 0; o >>= 1)
      part += __shfl_down_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0)
      warp_sums[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
      SumT s = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++)
        s += warp_sums[w];
      nBinnedD = 1.0 * s;
      if (nbinned_out)
        *nbinned_out = s;
      skip = 0;
    }
  } else {
    /* real-valued counts: summed in bin order, as the reference's loop */
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
      hist[b] = (double)counts[b];
    __syncthreads();
    if (threadIdx.x == 0) {
      SumT s = ordered_sum(hist, nb);
      nBinnedD = 1.0 * s;
      if (nbinned_out)
        *nbinned_out = s;
      skip = 0;
    }
  }
  __syncthreads();
  if (a.lh)
    lh_pass_filters(a, sm);
  if (a.sgHalf > 0) {
    sg_apply(hist, tmp, nb, a.sg_w, a.sg_lo, a.sg_n);
    __syncthreads();
    /* correctDistribution (csbend.c:4705-4721): negative bins clipped in
     * parallel, then the sum in bin order, as the reference forms it */
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
      if (tmp[b] < 0)
        tmp[b] = 0;
    __syncthreads();
    /* thread 0 runs the serial sum while warps 1.. form the denominators */
    if (threadIdx.x == 0) {
      const double sum = ordered_sum(tmp, nb);
      if (!sum)
        skip = 1;
      else
        deriv[0] = nBinnedD / sum; /* factor, parked in deriv[0] */
    } else if (threadIdx.x >= 32) {
      for (int b = threadIdx.x - 32; b < nb; b += blockDim.x - 32)
        denom[b] = b2e_pow13(dct * b);
    }
    __syncthreads();
    const double factor = deriv[0];
    const int sk = skip;
    __syncthreads();
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
      hist[b] = sk ? tmp[b] : tmp[b] * factor;
  }
  const bool denom_done = a.sgHalf > 0 && blockDim.x > 32;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    if (!denom_done)
      denom[b] = b2e_pow13(dct * b);
    hist[b] = hist[b] / dct;
    deriv[b] = hist[b];
  }
  __syncthreads();
  sg_apply(deriv, tmp, nb, a.sgd_w, a.sgd_lo, a.sgd_n);
  __syncthreads();
  for (int b = threadIdx.x; b < nb; b += blockDim.x)
    deriv[b] = tmp[b];
  __syncthreads();
}

/* bins of slippage; clamped to [0, nb] so indexing stays in bounds for a
 * degenerate bin size (the comparisons below give the same result) */
__device__ __forceinline__ void slippage_bins(const WakeArgs &a, double dct, long long *diS, long long *diS4) {
  long long d = (long long)(a.slippage / dct), d4 = (long long)(4 * a.slippage / dct);
  *diS = d < 0 ? 0 : (d > a.nBins ? a.nBins : d);
  *diS4 = d4 < 0 ? 0 : (d4 > a.nBins ? a.nBins : d4);
}

/* T1 (integral) and T2 (slippage boundary) of bin ib before the c1/c2 factors
 * (csbend.c:2623-2662) */
__device__ __forceinline__ void wake_terms(int ib, const WakeArgs &a, const double dct, const double *hist,
                                           const double *deriv, const double *denom, long long diS, long long diS4,
                                           double *T1out, double *T2out) {
  const int nb = a.nBins;
  double T1 = 0, T2 = 0, term1 = 0, term2 = 0;
  long long count, j;
  if (a.steady) {
    if (!a.trapz) {
      for (j = ib + 1; j < nb; j++)
        T1 += deriv[j] / denom[j - ib];
    } else {
      if ((j = ib + 1) < nb)
        term1 = deriv[j] / denom[j - ib];
      for (count = 0, j = ib + 1; j < nb; j++, count++)
        T1 += (term2 = deriv[j] / denom[j - ib]);
      if ((ib + 1) < nb)
        T1 += 0.3 * (denom[1] * denom[1]) * (2 * deriv[ib + 1] + 3 * deriv[ib]) / dct;
      if (count > 1)
        T1 -= (term1 + term2) / 2;
    }
  } else {
    if (!a.trapz) {
      for (j = ib + 1; j <= (ib + diS) && j < nb; j++)
        T1 += deriv[j] / denom[j - ib];
    } else {
      if ((j = ib + 1) < nb && j <= (ib + diS))
        term1 = deriv[j] / denom[j - ib] / 2;
      for (count = 0, j = ib + 1; j <= (ib + diS) && j < nb; count++, j++)
        T1 += (term2 = deriv[j] / denom[j - ib]);
      if (diS > 0 && (ib + 1) < nb)
        T1 += 0.3 * (denom[1] * denom[1]) * (2 * deriv[ib + 1] + 3 * deriv[ib]) / dct;
      if (count > 1)
        T1 -= (term1 + term2) / 2;
    }
    if ((ib + diS) < nb)
      T2 += hist[ib + diS];
    if ((ib + diS4) < nb)
      T2 -= hist[ib + diS4];
  }
  *T1out = T1;
  *T2out = T2;
}

/* Steady-state wake by the integrated Green's function (csbend.c:2593-2621,
 * :2676-2680, convolveArrays1 :5484-5491): chi(z) per bin, its second
 * difference, the one-sided convolution with the density (per-bin serial
 * sums in the reference's order), times -q_macro/(m c^2) L/N_KICKS.  chik and
 * grnk are nBins scratch arrays in shared memory. */
__device__ void igf_wake(const WakeArgs &a, const double dct, const double *hist, double *chik, double *grnk,
                         double *dgamma) {
  const int nb = a.nBins;
  const double frac = 9.0 / 16.0;
  for (int ib = threadIdx.x; ib < nb; ib += blockDim.x) {
    const double z = ib * dct;
    const double xmu = 3.0 * a.gamma3 * z / (2.0 * a.rho0);
    const double aa = sqrt(xmu * xmu + 1.0);
    const double b = aa + xmu;
    double chi;
    if (xmu < 1e-3) {
      const double x2 = xmu * xmu, x3 = xmu * xmu * xmu;
      chi = frac * a.const1 + 0.50 * x2 - (7.0 / 54.0) * (x2 * x2) + (140.0 / 2187.0) * (x3 * x3);
    } else {
      const double b13 = b2e_pow13(b), b23 = b2e_pow23(b), b43 = b2e_pow43(b);
      const double q = (1 - b23) / xmu;
      chi = frac * (3.0 * (-2.0 * xmu * b13 + b23 + b43) + b2e_log((q * q) / (1 + b23 + b43)));
    }
    chik[ib] = chi;
  }
  __syncthreads();
  const double const2 = (16.0 / 27.0) * a.q4pe / (a.gamma2 * dct);
  for (int ib = threadIdx.x; ib < nb; ib += blockDim.x) {
    double g;
    if (ib == 0)
      g = const2 * (chik[1] - chik[0]);
    else if (ib < nb - 1)
      g = const2 * (chik[ib + 1] - 2.0 * chik[ib] + chik[ib - 1]);
    else
      g = 0;
    grnk[ib] = g;
  }
  __syncthreads();
  for (int ib = threadIdx.x; ib < nb; ib += blockDim.x) {
    double out = 0;
    for (int ib1 = ib; ib1 < nb; ib1++)
      out += hist[ib1] * grnk[ib1 - ib];
    const double dg = out * a.igf_factor;
    dgamma[ib] = dg;
    if (a.wakelog)
      a.wakelog[ib] = dg;
  }
}

/* Wake of one kick (csbend.c:2566-2673) on one CTA, from a histogram of
 * counts (unsigned counts in tracking, real-valued counts for batched
 * profiles).  sm holds 4*nBins + 8 doubles.  Writes dgamma[nBins], the wake log
 * when a.wakelog is set, the binned total when nbinned_out is set, and the
 * smoothed density (per unit ct) and its derivative when hist_out/deriv_out
 * are set. */
template <typename CountT, typename SumT>
__device__ void wake_body(const CountT *counts, const WakeArgs &a, const double dct, double *sm, double *dgamma,
                          SumT *nbinned_out, double *hist_out, double *deriv_out, double *page = nullptr) {
  const int nb = a.nBins;
  wake_filters<CountT, SumT>(counts, a, dct, sm, nbinned_out);
  const double *hist = sm, *deriv = sm + nb, *denom = sm + 2 * nb;
  double *page_t1 = page ? page + 2 * nb : nullptr, *page_t2 = page ? page + 3 * nb : nullptr;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    if (hist_out)
      hist_out[b] = hist[b];
    if (deriv_out)
      deriv_out[b] = deriv[b];
    if (page) {
      page[b] = hist[b];
      page[nb + b] = deriv[b];
      page_t1[b] = 0; /* the IGF path and an empty range leave T1 and T2 at zero */
      page_t2[b] = 0;
    }
  }
  long long diS, diS4;
  slippage_bins(a, dct, &diS, &diS4);
  if (!(dct > 0)) {
    for (int ib = threadIdx.x; ib < nb; ib += blockDim.x) {
      dgamma[ib] = 0;
      if (a.wakelog)
        a.wakelog[ib] = 0;
    }
    return;
  }
  if (a.igf) {
    igf_wake(a, dct, hist, sm + 3 * nb, sm + 2 * nb, dgamma);
    return;
  }
  for (int ib = threadIdx.x; ib < nb; ib += blockDim.x) {
    double T1 = 0, T2 = 0;
    if (a.csr_constant) {
      wake_terms(ib, a, dct, hist, deriv, denom, diS, diS4, &T1, &T2);
      T1 *= a.c1;
      T2 *= a.c2;
    }
    double dg = T1 + T2;
    dgamma[ib] = dg;
    if (a.wakelog)
      a.wakelog[ib] = dg;
    if (page) {
      page_t1[ib] = T1;
      page_t2[ib] = T2;
    }
  }
}

/* wake of one kick, one CTA per bunch; c1 and c2 from the bunch's CSRConstant
 * in the host expression's order (csbend.c:2664-2667).  With recycle set the
 * CTA also readies its bunch for the next binning pass once this one's inputs
 * are consumed: empty c*t range keys (the histogram kernel, the only reader,
 * has finished) and zero counts (after they are read into shared memory). */
__global__ void __launch_bounds__(1024, 1) csr_wake_kernel(CsrBunches B, unsigned int *counts_all, WakeArgs a,
                                                           int recycle) {
  extern __shared__ double sm[];
  chain_enter();
  const int bunch = blockIdx.x;
  /* the bunch's scalars load together with its active flag (all in bounds) */
  const int active = B.active[bunch];
  const double csr_constant = B.csr_const[bunch], igf_factor = B.csr_const[B.n + bunch];
  CsrDevState *st = B.st + bunch;
  const double dct = st->dct;
  double *page = nullptr;
  if (a.pagelog) {
    page = a.pagelog + (size_t)bunch * (B2E_CSR_PAGE_HEADER + 4 * a.nBins);
    if (threadIdx.x == 0) {
      /* the binning's range, as the histogram kernel formed it; a bunch
       * without CSR on this kick gets element index -1 and no arrays */
      double lower = value_of(st->ct_min_key), upper = value_of(st->ct_max_key);
      expand_range(&lower, &upper, a.page_range_factor);
      page[0] = active ? a.page_element : -1.0;
      page[1] = a.page_kick;
      page[2] = bunch;
      page[3] = a.nBins;
      page[4] = lower;
      page[5] = upper;
      page[6] = dct;
      page[7] = a.slippage;
      page[8] = a.page_angle;
      page[9] = a.page_ds_kick;
      page[10] = a.page_p_central;
      page[11] = B.csr_const[3 * B.n + bunch];
    }
    __syncthreads(); /* the keys are read before they are emptied below */
    page += B2E_CSR_PAGE_HEADER;
  }
  if (recycle && threadIdx.x == 0) {
    st->ct_min_key = ~0ull;
    st->ct_max_key = 0ull;
  }
  if (!active)
    return;
  WakeArgs w = a;
  w.csr_constant = csr_constant;
  w.c1 = csr_constant * a.length / a.nSlices;
  w.c2 = -csr_constant * a.length / a.nSlices / a.slippage13;
  w.igf_factor = igf_factor;
  w.wakelog = a.wakelog ? a.wakelog + (size_t)bunch * a.nBins : nullptr;
  unsigned int *counts = counts_all + (size_t)bunch * a.nBins;
  wake_body<unsigned int, long long>(counts, w, dct, sm, st->dGamma, &st->nBinned, nullptr, nullptr, page);
  if (recycle) /* the counts were copied to shared memory before the first barrier */
    for (int b = threadIdx.x; b < a.nBins; b += blockDim.x)
      counts[b] = 0;
}

/* deterministic sum over the CTA (blockDim.x a power of two, red >= blockDim.x doubles) */
__device__ double block_sum(double v, double *red) {
  red[threadIdx.x] = v;
  __syncthreads();
  for (int s = blockDim.x >> 1; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
      red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  const double r = red[0];
  __syncthreads();
  return r;
}

/* Learned wake, step 1 (one CTA per bunch): the kick's filters, then the
 * network inputs in bin units -- density and derivative normalised to unit
 * sum and by k = 1/rms(derivative) over the network's L bins, the slippage
 * code log2(diS)/log2(L), and the density at bin i + diS -- padded with zeros
 * to L bins.  The tables (density, derivative, denominators) and the
 * per-bunch scalars (sum, k, dct) are kept for step 3. */
__global__ void __launch_bounds__(1024, 1) csr_sur_filter_kernel(CsrBunches B, const unsigned int *counts_all, WakeArgs a, int L, float sc_dens,
                                      float sc_deriv, double *tab, double *scal, float *inputs) {
  extern __shared__ double sm[];
  const int b = blockIdx.x, nb = a.nBins;
  float *in = inputs + (size_t)b * 4 * L;
  if (!B.active[b]) {
    for (int i = threadIdx.x; i < 4 * L; i += blockDim.x)
      in[i] = 0.f;
    return;
  }
  CsrDevState *st = B.st + b;
  const double dct = st->dct;
  wake_filters<unsigned int, long long>(counts_all + (size_t)b * nb, a, dct, sm, &st->nBinned);
  const double *hist = sm, *deriv = sm + nb, *denom = sm + 2 * nb;
  double *red = sm + 3 * nb;
  double *t = tab + (size_t)b * 3 * B2E_CSR_MAX_BINS;
  double part = 0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    t[i] = hist[i];
    t[B2E_CSR_MAX_BINS + i] = deriv[i];
    t[2 * B2E_CSR_MAX_BINS + i] = denom[i];
    part += hist[i] * dct;
  }
  const double total = block_sum(part, red);
  part = 0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    const double d = deriv[i] * dct / total;
    part += d * d;
  }
  const double k = 1.0 / sqrt(block_sum(part, red) / L);
  long long diS, diS4;
  slippage_bins(a, dct, &diS, &diS4);
  const float code = (float)(log2((double)(diS < 1 ? 1 : (diS > L ? L : diS))) / log2((double)L));
  const double fd = k / total * sc_dens, fg = k / total * sc_deriv;
  const int dsh = (int)(diS < 1 ? 1 : diS);
  for (int i = threadIdx.x; i < L; i += blockDim.x) {
    in[i] = i < nb ? (float)(hist[i] * dct * fd) : 0.f;
    in[L + i] = i < nb ? (float)(deriv[i] * dct * fg) : 0.f;
    in[2 * L + i] = code;
    in[3 * L + i] = i + dsh < nb ? (float)(hist[i + dsh] * dct * fd) : 0.f;
  }
  if (threadIdx.x == 0) {
    scal[b * 4 + 0] = total;
    scal[b * 4 + 1] = k;
    scal[b * 4 + 2] = dct;
  }
}

/* Learned wake, step 3 (one CTA per bunch): the network's T1 (bin units) to
 * the kick's T1 (times dct^(-4/3)), the gate -- the plain T1 and T2 at every
 * stride-th bin from `start`, relative rms error of the wake c1 T1 + c2 T2
 * there -- and the kick's dGamma: the learned T1 with the exact T2, or, when
 * the error exceeds tol, the plain wake exactly as csr_wake_kernel forms it. */
__global__ void __launch_bounds__(1024, 1) csr_sur_combine_kernel(CsrBunches B, WakeArgs a, const double *tab, const double *scal, const float *y,
                                       int L, float sc_target, double tol, int stride, int start, double *gate_log,
                                       unsigned long long *counters) {
  extern __shared__ double sm[];
  const int b = blockIdx.x, nb = a.nBins;
  if (!B.active[b])
    return;
  CsrDevState *st = B.st + b;
  double *hist = sm, *deriv = sm + nb, *denom = sm + 2 * nb, *red = sm + 3 * nb;
  const double *t = tab + (size_t)b * 3 * B2E_CSR_MAX_BINS;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    hist[i] = t[i];
    deriv[i] = t[B2E_CSR_MAX_BINS + i];
    denom[i] = t[2 * B2E_CSR_MAX_BINS + i];
  }
  __syncthreads();
  const double csr_constant = B.csr_const[b];
  const double c1 = csr_constant * a.length / a.nSlices;
  const double c2 = -csr_constant * a.length / a.nSlices / a.slippage13;
  const double total = scal[b * 4 + 0], k = scal[b * 4 + 1], dct = scal[b * 4 + 2];
  double *wl = a.wakelog ? a.wakelog + (size_t)b * nb : nullptr;
  if (!(dct > 0) || !csr_constant) {
    for (int ib = threadIdx.x; ib < nb; ib += blockDim.x) {
      st->dGamma[ib] = 0;
      if (wl)
        wl[ib] = 0;
    }
    return;
  }
  long long diS, diS4;
  slippage_bins(a, dct, &diS, &diS4);
  const double unit = 1.0 / dct / b2e_pow13(dct); /* dct^(-4/3) */
  const float *yb = y + (size_t)b * L;
  /* gate */
  double e2 = 0, w2 = 0;
  if (diS > 0)
    for (int ib = start + threadIdx.x * stride; ib < nb; ib += blockDim.x * stride) {
      double T1p, T2;
      wake_terms(ib, a, dct, hist, deriv, denom, diS, diS4, &T1p, &T2);
      const double T1s = (double)yb[ib] / sc_target / k * total * unit;
      const double d = (T1s - T1p) * c1, wp = T1p * c1 + T2 * c2;
      e2 += d * d;
      w2 += wp * wp;
    }
  e2 = block_sum(e2, red);
  w2 = block_sum(w2, red);
  const double err = diS > 0 ? (w2 > 0 ? sqrt(e2 / w2) : (e2 > 0 ? INFINITY : 0.0)) : 0.0;
  const bool plain = !(err <= tol);
  for (int ib = threadIdx.x; ib < nb; ib += blockDim.x) {
    double T1, T2;
    if (plain) {
      wake_terms(ib, a, dct, hist, deriv, denom, diS, diS4, &T1, &T2);
    } else {
      T1 = diS > 0 ? (double)yb[ib] / sc_target / k * total * unit : 0.0;
      T2 = 0;
      if ((ib + diS) < nb)
        T2 += hist[ib + diS];
      if ((ib + diS4) < nb)
        T2 -= hist[ib + diS4];
    }
    T1 *= c1;
    T2 *= c2;
    const double dg = T1 + T2;
    st->dGamma[ib] = dg;
    if (wl)
      wl[ib] = dg;
  }
  if (threadIdx.x == 0) {
    gate_log[b] = err;
    atomicAdd(&counters[0], 1ull);
    if (plain)
      atomicAdd(&counters[1], 1ull);
  }
}

/* Batched wake integral of many profiles in bin units (dct = 1), one CTA per
 * profile: out = T1 (c1 = 1, no T2 term) for the profile's slippage in bins;
 * hist_out/deriv_out receive the smoothed density and its derivative. */
__global__ void wake_batch_kernel(const double *counts, const double *slippage_bins, WakeArgs a, double *t1_out,
                                  double *hist_out, double *deriv_out) {
  extern __shared__ double sm[];
  const size_t off = (size_t)blockIdx.x * a.nBins;
  WakeArgs w = a;
  w.slippage = slippage_bins[blockIdx.x];
  w.slippage13 = 1;
  w.c1 = 1;
  w.c2 = 0;
  w.csr_constant = 1;
  w.wakelog = nullptr;
  wake_body<double, double>(counts + off, w, 1.0, sm, t1_out + off, (double *)nullptr, hist_out + off,
                            deriv_out + off);
}

/* after the last kick: its wake kick and the min/max for the exit binning */
__global__ void csr_last_kick_kernel(DevParticles P, int64_t n, CsrBunches B, int nBins, double Po, double rho0) {
  chain_enter();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  bool alive = i < n && P.lost_pass[i] < 0;
  const int b = i < n ? bunch_of(i, B) : B.n - 1;
  double CT = 0;
  if (alive) {
    CT = P.s[i];
    if (B.active[b] && B.csr_const[b] != 0)
      P.dp[i] = csr_kick(CT, P.x[i], P.dp[i], B.st + b, nBins, Po, rho0);
  }
  bunch_minmax(CT, alive, b, B);
}

/* exit: c*t -> s at the final velocity, exit edge, back to the lab frame
 * (csbend.c:2810-2955); csrWake.s0 from the exit binning's lower edge. */
__global__ void csr_exit_kernel(DevParticles P, int64_t n, const DevElem *ep, BendExtra bx, CsrBunches B, double factor,
                                double Po,
                                int pass, int elem_index) {
  chain_enter();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const DevElem &e = *ep;
  const double *c = e.c;
  if (blockIdx.x == 0)
    for (int b = threadIdx.x; b < B.n; b += blockDim.x) {
      CsrDevState *st = B.st + b;
      const int do_bin = B.active[b];
      double lower = 0, upper = 0;
      st->dctBin = do_bin ? st->dct : 0;
      if (do_bin) {
        lower = value_of(st->ct_min_key);
        upper = value_of(st->ct_max_key);
        expand_range(&lower, &upper, factor);
      }
      st->s0 = lower + c[CB_DZF];
    }
  if (i >= n || P.lost_pass[i] >= 0)
    return;
  const double ct = c[CB_COS_TT], sn = c[CB_SIN_TT];
  double X = P.x[i], XP = P.xp[i], Y = P.y[i], YP = P.yp[i], CT = P.s[i], DP = P.dp[i];
  double p1 = Po * (1 + DP), beta1 = p1 / sqrt(p1 * p1 + 1), s, x, y, xp, yp, rho;
  s = CT * beta1;
  if (p1 <= 0) {
    P.lost_pass[i] = pass;
    P.lost_elem[i] = elem_index;
    return;
  }
  if (e.flags & EF_EDGE2) {
    rho = (1 + DP) * c[CB_RHO_ACTUAL];
    if (e.flags & EF_EDGE_ORDER2) {
      bend_edge_order2(X, XP, Y, YP, rho, c[CB_PSI2] * (1 + DP), c[CB_TAN_E2], c[CB_E2], bx.c[BX_SEC2_E2],
                       bx.c[BX_EDGE_N], 1);
    } else {
      XP = XP + (c[CB_TAN_E2] / rho) * X;
      YP = YP - (b2e_tan(c[CB_E2] - c[CB_PSI2] / (1 + DP)) / rho) * Y;
    }
  }
  /* the ETILT offsets are zero without ETILT */
  x = (X * ct - Y * sn) + bx.c[BX_ETILT0];
  y = (X * sn + Y * ct) + bx.c[BX_ETILT0 + 2];
  xp = (XP * ct - YP * sn) + bx.c[BX_ETILT0 + 1];
  yp = (XP * sn + YP * ct) + bx.c[BX_ETILT0 + 3];
  x = x + (c[CB_DXF] + c[CB_DZF] * xp);
  y = y + (c[CB_DYF] + c[CB_DZF] * yp);
  s = s + (c[CB_DZF] * sqrt((1 + xp * xp) + yp * yp) + bx.c[BX_ETILT0 + 4]);
  P.x[i] = x;
  P.xp[i] = xp;
  P.y[i] = y;
  P.yp[i] = yp;
  P.s[i] = s;
}

/* CSRDRIFT mode 0, one kick (csbend.c:3415-3502) */
__global__ void csr_drift_kick_kernel(DevParticles P, int64_t n, CsrBunches B, double dz, double s0_incr,
                                      double factor, int apply, int nBins, double Po) {
  chain_enter();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n || P.lost_pass[i] >= 0)
    return;
  const int b = bunch_of(i, B);
  if (!B.mode[b])
    return;
  const CsrDevState *st = B.st + b;
  double x = P.x[i], xp = P.xp[i], y = P.y[i], yp = P.yp[i], s = P.s[i], dp = P.dp[i], p, beta;
  x = x + xp * dz;
  y = y + yp * dz;
  p = Po * (1 + dp);
  beta = p / sqrt(p * p + 1);
  s = (s + dz * sqrt((1 + xp * xp) + yp * yp)) / beta;
  if (apply) {
    const double ct0 = st->s0 + s0_incr;
    double f = (s - ct0) / st->dctBin;
    long long iBin = (long long)f;
    f -= iBin;
    if (iBin >= 0 && iBin < nBins - 1)
      dp = dp + ((1 - f) * st->dGamma[iBin] + f * st->dGamma[iBin + 1]) / Po * factor;
  }
  p = (1 + dp) * Po;
  beta = p / sqrt(p * p + 1);
  P.x[i] = x;
  P.y[i] = y;
  P.s[i] = beta * s;
  P.dp[i] = dp;
}

/* ---- CSRDRIFT, Stupakov mode (csbend.c:3803-4159) ---------------------- */

/* phi_last starts at -1, the value SolveForPhiStupakov's static holds before
 * its first call (csbend.c:4177) */
__global__ void csr_init_state_kernel(CsrDevState *st, int n) {
  for (int b = threadIdx.x; b < n; b += blockDim.x)
    st[b].phi_last = -1;
}

/* one kick's drift: the particles move back by dz_back first (only on the
 * first kick when the drift does not start where the last CSR element ended,
 * csbend.c:3835-3848), then forward by dz; c*t = s/beta; min/max of c*t per
 * bunch (csbend.c:3876-3893) */
__global__ void stupakov_drift_kernel(DevParticles P, int64_t n, CsrBunches B, double dz_back, double dz, double Po) {
  chain_enter();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int b = i < n ? bunch_of(i, B) : B.n - 1;
  const bool mine = i < n && P.lost_pass[i] < 0 && B.mode[b];
  double ct = 0;
  if (mine) {
    double x = P.x[i], xp = P.xp[i], y = P.y[i], yp = P.yp[i], s = P.s[i];
    if (dz_back != 0) {
      x = x - dz_back * xp;
      y = y - dz_back * yp;
      s = s - dz_back * sqrt((1 + xp * xp) + yp * yp);
    }
    x = x + xp * dz;
    y = y + yp * dz;
    const double p = Po * (1 + P.dp[i]), beta = p / sqrt(p * p + 1);
    ct = (s + dz * sqrt((1 + xp * xp) + yp * yp)) / beta;
    P.x[i] = x;
    P.y[i] = y;
    P.s[i] = ct;
  }
  bunch_minmax(ct, mine, b, B);
}

/* fn of SolveForPhiStupakov (csbend.c:4163-4165) */
struct StupakovFn {
  double x, x4;
  __device__ double operator()(double phi) const { return phi * phi * phi * (phi + x4) / (phi + x); }
};

/* SolveForPhiStupakov (csbend.c:4169-4202); *phi_last carries the start
 * value from one solve to the next */
__device__ double stupakov_phi(double x, double ds, double phim, double *phi_last) {
  if (ds < 0)
    return -1;
  if (ds == 0)
    return 0;
  ds *= 24;
  StupakovFn fn;
  fn.x = x;
  fn.x4 = 4 * x;
  if (*phi_last == -1)
    *phi_last = phim / 2;
  if (fabs(ds - fn(phim)) < ds / 1e4) {
    *phi_last = phim;
    return phim;
  }
  double phi = b2e_zero_newton(fn, ds, *phi_last, phim / 1000, 3, ds / 1e4);
  if (phi < 0 || phi > phim || fabs(ds - fn(phi)) > ds / 1e4)
    phi = b2e_zero_interp(fn, ds, 0, phim * 1.01, phim / 100, ds / 1e4);
  if (phi < 0 || phi > phim)
    return -1;
  *phi_last = phi;
  return phi;
}

/* per-kick scalars, formed on the host as the reference writes them */
struct StupakovArgs {
  double x;      /* zTravel / rho */
  double dsMax;  /* rho/24 theta^3 (theta + 4x)/(theta + x) */
  double dsC;    /* rho/6 theta^2 (theta + 3x), case C */
  double theta, rho, dz0;
  int trapz;
};

/* bins of a distance, clamped to [0, nb] (the comparisons against nb give
 * the reference's result; a negative distance does not occur behind a dipole) */
__device__ __forceinline__ long long clamp_bins(double d, int nb) {
  if (!(d > 0))
    return 0;
  return d >= (double)nb ? nb : (long long)d;
}

/* wake of one Stupakov kick, one CTA per bunch (csbend.c:3950-4054): the
 * histogram filters of the last dipole, phi solutions (serial, each starting
 * from the previous one), then per bin case C, case D's boundary term and its
 * integral in the reference's order, times -4/rho GSConstant dz0.  Shared
 * memory: 4 nBins + 8 doubles for the filters, nBins for phi. */
__global__ void __launch_bounds__(1024, 1) stupakov_wake_kernel(CsrBunches B, const unsigned int *counts_all, WakeArgs a, StupakovArgs sa) {
  extern __shared__ double sm[];
  chain_enter();
  const int bunch = blockIdx.x;
  if (!B.mode[bunch])
    return;
  CsrDevState *st = B.st + bunch;
  const int nb = a.nBins;
  const double dct = st->dct;
  wake_filters<unsigned int, unsigned long long>(counts_all + (size_t)bunch * nb, a, dct, sm, nullptr);
  const double *hist = sm, *deriv = sm + nb;
  double *phi = sm + 4 * nb + 8;
  if (!(dct > 0)) {
    for (int ib = threadIdx.x; ib < nb; ib += blockDim.x)
      st->dGamma[ib] = 0;
    return;
  }
  if (threadIdx.x == 0) {
    double last = st->phi_last;
    for (int ib = 0; ib < nb; ib++) {
      phi[ib] = -1;
      if (ib * dct > sa.dsMax)
        break;
      phi[ib] = stupakov_phi(sa.x, ib * dct / sa.rho, sa.theta, &last);
    }
    st->phi_last = last;
  }
  __syncthreads();
  const long long diC = clamp_bins(sa.dsC / dct, nb), diD = clamp_bins(sa.dsMax / dct, nb);
  const double fC = -1 / (sa.theta + 2 * sa.x), factor = -4 / sa.rho * B.csr_const[2 * B.n + bunch] * sa.dz0;
  for (int ib = threadIdx.x; ib < nb; ib += blockDim.x) {
    double g = ib + diC < nb ? fC * hist[ib + diC] : 0, term1 = 0, term2 = 0;
    if (ib + diD < nb)
      g = g + hist[ib + diD] / (sa.theta + 2 * sa.x);
    int count = 0;
    for (int j = ib; j < nb; j++) {
      const double p = phi[j - ib];
      if (!(p >= 0))
        break;
      if (p > 0) {
        term2 = deriv[j] / (p + 2 * sa.x);
        g = g - term2;
        if (count == 0)
          term1 = term2;
        count++;
      }
    }
    if (count > 1 && sa.trapz)
      g = g + (term1 + term2) / 2;
    st->dGamma[ib] = g * factor;
  }
}

/* kick from the wake and c*t back to s at the new velocity (csbend.c:4078-4096) */
__global__ void stupakov_kick_kernel(DevParticles P, int64_t n, CsrBunches B, int nBins, double Po) {
  chain_enter();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n || P.lost_pass[i] >= 0)
    return;
  const int b = bunch_of(i, B);
  if (!B.mode[b])
    return;
  const CsrDevState *st = B.st + b;
  const double ct = P.s[i];
  double dp = P.dp[i], f = (ct - st->ctLower) / st->dct;
  const long long iBin = (long long)f;
  f -= iBin;
  if (iBin >= 0 && iBin < nBins - 1)
    dp = dp + ((1 - f) * st->dGamma[iBin] + f * st->dGamma[iBin + 1]) / Po;
  const double p = (1 + dp) * Po, beta = p / sqrt(p * p + 1);
  P.dp[i] = dp;
  P.s[i] = beta * ct;
}

/* empty min/max keys of every bunch before a binning pass */
__global__ void csr_reset_keys_kernel(CsrBunches B) {
  for (int b = threadIdx.x; b < B.n; b += blockDim.x) {
    B.st[b].ct_min_key = ~0ull;
    B.st[b].ct_max_key = 0ull;
  }
}

/* min/max keys of every bunch to a contiguous [2][n] buffer and back, around
 * an all-rank reduction */
__global__ void csr_keys_gather_kernel(CsrBunches B, unsigned long long *keys) {
  for (int b = threadIdx.x; b < B.n; b += blockDim.x) {
    keys[b] = B.st[b].ct_min_key;
    keys[B.n + b] = B.st[b].ct_max_key;
  }
}
__global__ void csr_keys_scatter_kernel(CsrBunches B, const unsigned long long *keys) {
  for (int b = threadIdx.x; b < B.n; b += blockDim.x) {
    B.st[b].ct_min_key = keys[b];
    B.st[b].ct_max_key = keys[B.n + b];
  }
}

__global__ void csr_s0_add_kernel(CsrBunches B, double incr) {
  chain_enter();
  for (int b = threadIdx.x; b < B.n; b += blockDim.x)
    if (B.mode[b])
      B.st[b].s0 = B.st[b].s0 + incr;
}

/* do_tracking's sweeps after a collective element (do_tracking.c:2455-2475,
 * :2629): MAXAMP aperture if one is active, then inf/NaN in x or y. */
__global__ void post_element_sweep_kernel(DevParticles P, int64_t n, const DevAperture *ap, int pass, int elem_index) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n || P.lost_pass[i] >= 0)
    return;
  Part p;
  p.x = P.x[i];
  p.y = P.y[i];
  bool lost = false;
  if (ap && ap->mode) {
    p.xp = P.xp[i];
    p.yp = P.yp[i];
    lost = !maxamp_ok(p, *ap);
  }
  if (!lost && !finite_xy(p))
    lost = true;
  if (lost) {
    P.lost_pass[i] = pass;
    P.lost_elem[i] = elem_index;
  }
}

cudaError_t launch_post_element_sweep(const DevParticles &P, int64_t n, const DevAperture *ap, int pass, int elem,
                                      cudaStream_t stream) {
  const int grid = (int)std::max<int64_t>(1, (n + 255) / 256);
  post_element_sweep_kernel<<<grid, 256, 0, stream>>>(P, n, ap, pass, elem);
  return cudaGetLastError();
}

/* exact drift of the particles of the bunches whose CSRDRIFT mode is `mode`
 * (every particle when the mode table is null) */
__global__ void edrift_kernel(DevParticles P, int64_t n, double L, CsrBunches B, int mode) {
  chain_enter();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n || P.lost_pass[i] >= 0)
    return;
  if (B.mode && B.mode[bunch_of(i, B)] != mode)
    return;
  double xp = P.xp[i], yp = P.yp[i];
  P.x[i] = P.x[i] + xp * L;
  P.y[i] = P.y[i] + yp * L;
  P.s[i] = P.s[i] + L * sqrt((1 + xp * xp) + yp * yp);
}

/* ------------------------------------------------------------------ host -- */

static int grid_for(int64_t n) { return (int)std::max<int64_t>(1, (n + 255) / 256); }

int csr_configure(CsrState &st, const b2e_element *el, int n, const CompiledLattice &lat, const b2e_run_options &opt,
                  std::string &err) {
  csr_release(st);
  st.elems.clear();
  st.p_central = opt.p_central;
  st.enabled = !lat.csr_elements.empty();
  if (!st.enabled)
    return B2E_OK;
  std::vector<double> sgw;
  std::vector<int> sgi;
  st.sg_offset.clear();
  for (int idx : lat.csr_elements) {
    const b2e_element &e = el[idx];
    const DevElem &d = lat.elems[idx];
    CsrElem ce;
    ce.index = idx;
    ce.kind = d.kind;
    if (d.kind == K_CSRCSBEND) {
      const double *p = e.p;
      ce.bins = (int)p[B2E_BEND_BINS];
      if (ce.bins < 2) {
        err = "Less than 2 bins for CSR!";
        return B2E_ERR_LATTICE;
      }
      if (ce.bins > B2E_CSR_MAX_BINS) {
        err = "CSRCSBEND BINS above the engine maximum (4096)";
        return B2E_ERR_LATTICE;
      }
      ce.nSlices = (int)d.c[CB_NSLICES];
      ce.nSub = (int)d.c[CB_NSUB];
      ce.sgHalf = (int)p[B2E_BEND_SG_HALFWIDTH];
      ce.sgOrder = (int)p[B2E_BEND_SG_ORDER];
      ce.sgdHalf = (int)p[B2E_BEND_SGDERIV_HALFWIDTH];
      ce.sgdOrder = (int)p[B2E_BEND_SGDERIV_ORDER];
      /* csbend.c:2042-2050 */
      if (ce.sgdHalf <= 0)
        ce.sgdHalf = ce.sgHalf;
      if (ce.sgdHalf <= 0)
        ce.sgdHalf = 1;
      if (ce.sgdOrder <= 0)
        ce.sgdOrder = ce.sgOrder;
      if (ce.sgdOrder <= 0)
        ce.sgdOrder = 1;
      if (2 * std::max(ce.sgHalf, ce.sgdHalf) + 1 > B2E_SG_MAX_WIDTH) {
        err = "Savitzky-Golay half-width too large";
        return B2E_ERR_LATTICE;
      }
      ce.trapz = p[B2E_BEND_TRAPAZOID_INTEGRATION] != 0;
      ce.steady = p[B2E_BEND_STEADY_STATE] != 0;
      ce.igf = p[B2E_BEND_IGF] != 0;
      if (ce.igf && !ce.steady) {
        err = "Must have STEADY_STATE=1 when IGF=1"; /* csbend.c:2598 */
        return B2E_ERR_LATTICE;
      }
      ce.csr = p[B2E_BEND_CSR] != 0;
      ce.lowCut0 = p[B2E_BEND_LOW_FREQUENCY_CUTOFF0];
      ce.lowCut1 = p[B2E_BEND_LOW_FREQUENCY_CUTOFF1];
      ce.highCut0 = p[B2E_BEND_HIGH_FREQUENCY_CUTOFF0];
      ce.highCut1 = p[B2E_BEND_HIGH_FREQUENCY_CUTOFF1];
      ce.lh = ce.highCut0 > 0 || ce.lowCut0 >= 0;
      ce.clip = p[B2E_BEND_CLIP_NEGATIVE_BINS] != 0;
      ce.angle = fabs(p[B2E_BEND_ANGLE]);
      ce.length = p[B2E_BEND_L];
      ce.rho0 = d.c[CB_RHO0];
      ce.binRangeFactor = p[B2E_BEND_BIN_RANGE_FACTOR] < 1.1 ? 1.1 : p[B2E_BEND_BIN_RANGE_FACTOR];
      ce.dzf = d.c[CB_DZF];
      memcpy(ce.bx.c, lat.rads[idx].c + RB_EXTRA0, sizeof(ce.bx.c));
      ce.z_end = d.z_end;
      /* SAME_BEND_PRECEDES of determine_bend_flags (bend_matrix.c:1342-1363):
       * MARKs in between are transparent */
      ce.same_bend_precedes = 0;
      for (int j = idx - 1; j >= 0; j--) {
        if (el[j].type == B2E_CSRCSBEND && strncmp(el[j].name, e.name, sizeof(e.name)) == 0) {
          ce.same_bend_precedes = 1;
          break;
        }
        if (el[j].type != B2E_MARK)
          break;
      }
      /* per-bin Savitzky-Golay weights for smoothing (order sgOrder, derivative 0)
       * and for the derivative (order sgdOrder, derivative 1) */
      st.sg_offset.push_back(sgw.size());
      for (int pass = 0; pass < 2; pass++) {
        int half = pass == 0 ? ce.sgHalf : ce.sgdHalf, order = pass == 0 ? ce.sgOrder : ce.sgdOrder;
        for (int b = 0; b < ce.bins; b++) {
          double w[B2E_SG_MAX_WIDTH] = {0};
          long width;
          long lo = b2e_sg_window(b, ce.bins, half, half, &width);
          long ord = order < width - 1 ? order : width - 1;
          if (pass == 0 && half <= 0) {
            width = 1;
            lo = b;
            w[0] = 1;
          } else if ((pass == 1 && 1 > ord) || b2e_sg_weights(w, width, lo - b, ord, pass)) {
            width = 0; /* derivative of a constant fit: zero */
          }
          for (int k = 0; k < B2E_SG_MAX_WIDTH; k++)
            sgw.push_back(w[k]);
          sgi.push_back((int)lo);
          sgi.push_back((int)width);
        }
      }
    } else {
      const double *p = e.p;
      ce.stupakov = p[B2E_CSRDRIFT_USE_STUPAKOV] != 0;
      ce.drift_length = p[B2E_CSRDRIFT_L];
      ce.drift_dz = p[B2E_CSRDRIFT_DZ];
      ce.drift_kicks = (int)p[B2E_CSRDRIFT_N_KICKS];
      ce.drift_csr = p[B2E_CSRDRIFT_CSR] != 0;
      ce.z_start = d.z_start;
      st.sg_offset.push_back(sgw.size());
    }
    st.elems.push_back(ce);
  }
  /* one CSRDRIFT mode behind each dipole (csbend.c:3259-3263 stops the run
   * otherwise); the line is read cyclically, as drifts ahead of the first
   * dipole follow the last one on the next pass */
  {
    const int ne = (int)st.elems.size();
    int mode = -1;
    for (int k = 0; k < 2 * ne; k++) {
      const CsrElem &c = st.elems[k % ne];
      if (c.kind == K_CSRCSBEND)
        mode = -1;
      else if (c.drift_csr) {
        if (mode >= 0 && mode != c.stupakov) {
          err = "CSRDRIFT mode changed between dipoles. Pick one mode following each dipole.";
          return B2E_ERR_LATTICE;
        }
        mode = c.stupakov;
      }
    }
  }
  st.revolution_length = lat.total_length;
  st.last_bend = -1;
  if (csr_set_bunches(st, 1, nullptr, err))
    return B2E_ERR_NOMEM;
  if (!sgw.empty()) {
    if (cudaMalloc(&st.d_sg, sizeof(double) * sgw.size()) != cudaSuccess ||
        cudaMalloc(&st.d_sg_idx, sizeof(int) * sgi.size()) != cudaSuccess) {
      err = "CSR weight allocation failed";
      return B2E_ERR_NOMEM;
    }
    cudaMemcpy(st.d_sg, sgw.data(), sizeof(double) * sgw.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(st.d_sg_idx, sgi.data(), sizeof(int) * sgi.size(), cudaMemcpyHostToDevice);
  }
  /* the index array runs parallel to the weights: 2 ints per bin row */
  return B2E_OK;
}

int csr_set_bunches(CsrState &st, int n_bunches, const int64_t *d_offsets, std::string &err) {
  if (n_bunches < 1 || (n_bunches > 1 && !d_offsets)) {
    err = "CSR: bad bunch layout";
    return B2E_ERR_ARG;
  }
  if (st.d_state)
    cudaFree(st.d_state);
  if (st.d_counts)
    cudaFree(st.d_counts);
  if (st.d_csr_const)
    cudaFree(st.d_csr_const);
  if (st.d_flags)
    cudaFree(st.d_flags);
  if (st.d_alive)
    cudaFree(st.d_alive);
  if (st.d_keys)
    cudaFree(st.d_keys);
  st.d_keys = nullptr;
  st.d_state = nullptr;
  st.d_counts = nullptr;
  st.d_csr_const = nullptr;
  st.d_flags = nullptr;
  st.d_alive = nullptr;
  st.n_bunches = n_bunches;
  st.d_offsets = d_offsets;
  st.wake_valid.assign(n_bunches, 0);
  st.macro_charge.assign(n_bunches, 0.0);
  if (cudaMalloc(&st.d_state, sizeof(CsrDevState) * n_bunches) != cudaSuccess ||
      cudaMalloc(&st.d_counts, sizeof(unsigned int) * B2E_CSR_MAX_BINS * n_bunches) != cudaSuccess ||
      cudaMalloc(&st.d_csr_const, 4 * sizeof(double) * n_bunches) != cudaSuccess ||
      cudaMalloc(&st.d_flags, 2 * n_bunches) != cudaSuccess ||
      cudaMalloc(&st.d_alive, sizeof(unsigned long long) * n_bunches) != cudaSuccess ||
      cudaMalloc(&st.d_keys, 2 * sizeof(unsigned long long) * n_bunches) != cudaSuccess) {
    err = "CSR state allocation failed";
    return B2E_ERR_NOMEM;
  }
  cudaMemset(st.d_state, 0, sizeof(CsrDevState) * n_bunches);
  cudaMemset(st.d_csr_const, 0, 4 * sizeof(double) * n_bunches);
  cudaMemset(st.d_flags, 0, 2 * n_bunches);
  csr_init_state_kernel<<<1, 256>>>((CsrDevState *)st.d_state, n_bunches);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    err = "CSR state initialisation failed";
    return B2E_ERR_CUDA;
  }
  return B2E_OK;
}

/* alive particles per bunch: blockIdx.y is the bunch */
__global__ void alive_per_bunch_kernel(const int32_t *lost_pass, int64_t n, const int64_t *offs, int nb,
                                       unsigned long long *alive) {
  const int b = blockIdx.y;
  const int64_t first = nb <= 1 ? 0 : offs[b], end = nb <= 1 ? n : offs[b + 1];
  unsigned long long c = 0;
  for (int64_t i = first + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < end;
       i += (int64_t)gridDim.x * blockDim.x)
    c += lost_pass[i] < 0;
  for (int off = 16; off > 0; off >>= 1)
    c += __shfl_down_sync(0xffffffffu, c, off);
  if ((threadIdx.x & 31) == 0 && c)
    atomicAdd(&alive[b], c);
}

int csr_count_alive(CsrState &st, const int32_t *lost_pass, int64_t n, std::vector<int64_t> &alive, cudaStream_t stream,
                    std::string &err) {
  const int nb = st.n_bunches;
  std::vector<unsigned long long> h(nb);
  if (cudaMemsetAsync(st.d_alive, 0, sizeof(unsigned long long) * nb, stream) != cudaSuccess) {
    err = "CSR: alive count failed";
    return B2E_ERR_CUDA;
  }
  const int gx = (int)std::min<int64_t>(std::max(1, 148 * 4 / nb), std::max<int64_t>(1, (n / nb + 255) / 256));
  alive_per_bunch_kernel<<<dim3(gx, nb), 256, 0, stream>>>(lost_pass, n, st.d_offsets, nb, st.d_alive);
  if (st.reducer && st.reducer(st.reducer_user, B2E_REDUCE_SUM_U64, st.d_alive, nb, stream)) {
    err = "CSR: the all-rank reduction of alive counts failed";
    return B2E_ERR_CUDA;
  }
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(h.data(), st.d_alive, sizeof(unsigned long long) * nb, cudaMemcpyDeviceToHost, stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess) {
    err = "CSR: alive count failed";
    return B2E_ERR_CUDA;
  }
  alive.assign(h.begin(), h.end());
  return B2E_OK;
}

int csr_reduce_counts(CsrState &st, std::vector<int64_t> &counts, cudaStream_t stream, std::string &err) {
  if (!st.reducer)
    return B2E_OK;
  const int nb = (int)counts.size();
  std::vector<unsigned long long> h(counts.begin(), counts.end());
  if (nb > st.n_bunches || cudaMemcpyAsync(st.d_alive, h.data(), sizeof(unsigned long long) * nb,
                                           cudaMemcpyHostToDevice, stream) != cudaSuccess ||
      st.reducer(st.reducer_user, B2E_REDUCE_SUM_U64, st.d_alive, nb, stream) ||
      cudaMemcpyAsync(h.data(), st.d_alive, sizeof(unsigned long long) * nb, cudaMemcpyDeviceToHost, stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess) {
    err = "CSR: the all-rank reduction of bunch sizes failed";
    return B2E_ERR_CUDA;
  }
  counts.assign(h.begin(), h.end());
  return B2E_OK;
}

/* all-rank min/max of every bunch's c*t keys (no-op without a reducer) */
static int reduce_keys(CsrState &st, const CsrBunches &B, cudaStream_t stream, std::string &err, int64_t *launches) {
  if (!st.reducer)
    return B2E_OK;
  csr_keys_gather_kernel<<<1, 32, 0, stream>>>(B, st.d_keys);
  if (st.reducer(st.reducer_user, B2E_REDUCE_MIN_U64, st.d_keys, B.n, stream) ||
      st.reducer(st.reducer_user, B2E_REDUCE_MAX_U64, st.d_keys + B.n, B.n, stream)) {
    err = "CSR: the all-rank reduction of the c*t range failed";
    return B2E_ERR_CUDA;
  }
  csr_keys_scatter_kernel<<<1, 32, 0, stream>>>(B, st.d_keys);
  (*launches) += 2;
  return cudaGetLastError() == cudaSuccess ? B2E_OK : B2E_ERR_CUDA;
}

void csr_reset(CsrState &st) {
  st.wakes_host.clear();
  st.wake_values = 0;
  st.page_values = 0;
  st.timed_kicks = st.timed_learned = 0;
  st.gate_values = 0;
  if (st.d_sur_counts)
    cudaMemset(st.d_sur_counts, 0, 2 * sizeof(unsigned long long));
  st.accumulated_angle = 0;
  st.wake_valid.assign(st.n_bunches, 0);
  st.last_bend = -1;
}

static int ensure_pagelog(CsrState &st, int64_t values) {
  if (values <= st.pagelog_cap)
    return B2E_OK;
  double *p = nullptr;
  if (cudaMalloc(&p, sizeof(double) * values) != cudaSuccess)
    return B2E_ERR_NOMEM;
  if (st.d_pagelog) {
    if (st.page_values)
      cudaMemcpy(p, st.d_pagelog, sizeof(double) * st.page_values, cudaMemcpyDeviceToDevice);
    cudaFree(st.d_pagelog);
  }
  st.d_pagelog = p;
  st.pagelog_cap = values;
  return B2E_OK;
}

static int ensure_wakelog(CsrState &st, int64_t values) {
  if (values <= st.wakelog_cap)
    return B2E_OK;
  double *p = nullptr;
  if (cudaMalloc(&p, sizeof(double) * values) != cudaSuccess)
    return B2E_ERR_NOMEM;
  if (st.d_wakelog) {
    if (st.wake_values)
      cudaMemcpy(p, st.d_wakelog, sizeof(double) * st.wake_values, cudaMemcpyDeviceToDevice);
    cudaFree(st.d_wakelog);
  }
  st.d_wakelog = p;
  st.wakelog_cap = values;
  return B2E_OK;
}

#define CSR_CUDA(call)                                                                                           \
  do {                                                                                                           \
    cudaError_t e_ = (call);                                                                                     \
    if (e_ != cudaSuccess) {                                                                                     \
      err = std::string(#call) + ": " + cudaGetErrorString(e_);                                                  \
      return B2E_ERR_CUDA;                                                                                       \
    }                                                                                                            \
  } while (0)

static int ensure_surrogate_buffers(CsrState &st, int64_t gate_values, std::string &err) {
  const int nb = st.n_bunches, L = wakenet_bins(st.net);
  if (st.sur_cap_bunches < nb) {
    cudaFree(st.d_sur_in);
    cudaFree(st.d_sur_out);
    cudaFree(st.d_sur_tab);
    cudaFree(st.d_sur_scal);
    st.d_sur_in = st.d_sur_out = nullptr;
    st.d_sur_tab = st.d_sur_scal = nullptr;
    st.sur_cap_bunches = 0;
    if (cudaMalloc(&st.d_sur_in, sizeof(float) * 4 * L * nb) != cudaSuccess ||
        cudaMalloc(&st.d_sur_out, sizeof(float) * L * nb) != cudaSuccess ||
        cudaMalloc(&st.d_sur_tab, sizeof(double) * 3 * B2E_CSR_MAX_BINS * nb) != cudaSuccess ||
        cudaMalloc(&st.d_sur_scal, sizeof(double) * 4 * nb) != cudaSuccess) {
      err = "CSR: wake network buffers";
      return B2E_ERR_NOMEM;
    }
    st.sur_cap_bunches = nb;
  }
  if (!st.d_sur_counts) {
    if (cudaMalloc(&st.d_sur_counts, 2 * sizeof(unsigned long long)) != cudaSuccess) {
      err = "CSR: wake network buffers";
      return B2E_ERR_NOMEM;
    }
    cudaMemset(st.d_sur_counts, 0, 2 * sizeof(unsigned long long));
  }
  if (st.gate_values + gate_values > st.gate_cap) {
    const int64_t cap = std::max<int64_t>(2 * st.gate_cap, st.gate_values + gate_values);
    double *p = nullptr;
    if (cudaMalloc(&p, sizeof(double) * cap) != cudaSuccess) {
      err = "CSR: gate log";
      return B2E_ERR_NOMEM;
    }
    if (st.d_gate_log) {
      if (st.gate_values)
        cudaMemcpy(p, st.d_gate_log, sizeof(double) * st.gate_values, cudaMemcpyDeviceToDevice);
      cudaFree(st.d_gate_log);
    }
    st.d_gate_log = p;
    st.gate_cap = cap;
  }
  return B2E_OK;
}

/* the filter arguments of applyLHPassFilters as the dipole passes them: the
 * low-frequency cutoffs are the high-pass ramp, the high-frequency cutoffs
 * the low-pass ramp (csbend.c:2559-2562) */
static void set_filter_args(WakeArgs &a, int lh, int clip, double lowCut0, double lowCut1, double highCut0,
                            double highCut1) {
  a.lh = lh;
  a.clip = clip;
  a.startHP = lowCut0;
  a.endHP = lowCut1;
  a.startLP = highCut0;
  a.endLP = highCut1;
}

/* CSRDRIFT with USE_STUPAKOV=1 (track_through_driftCSR_Stupakov,
 * csbend.c:3803-4159) for the bunches whose mode flag is set; the others have
 * had their exact drift.  Per kick: drift and c*t with the min/max keys, the
 * histogram of the last dipole's bin count and range factor, the wake (one
 * CTA per bunch), the kick; then the closing half drift. */
static int stupakov_drift(CsrState &st, const CsrElem &ce, const CsrBunches &B, const DevParticles &P, int64_t n,
                          double zStart, cudaStream_t stream, std::string &err, int64_t *launches) {
  if (st.last_bend < 0) {
    err = "CSRDRIFT: no dipole wake to follow";
    return B2E_ERR_STATE;
  }
  const CsrElem &bend = st.elems[st.last_bend];
  const int nb = bend.bins, nbunch = B.n, g = grid_for(n);
  const double Po = st.p_central, rho = st.last_rho, theta = st.last_theta;
  double length = ce.drift_length, dz_back = 0;
  if (zStart != st.zLast) {
    length += (dz_back = zStart - st.zLast);
    zStart = st.zLast;
  }
  long nKicks;
  if (ce.drift_dz > 0) {
    if ((nKicks = (long)(length / ce.drift_dz + 0.5)) < 1)
      nKicks = 1;
  } else
    nKicks = ce.drift_kicks;
  if (nKicks <= 0) {
    err = "nKicks=0 in CSR drift.";
    return B2E_ERR_LATTICE;
  }
  const double dz0 = length / nKicks;
  double dz = dz0 / 2, zTravel = zStart - st.z0;
  const double *sgw = st.d_sg + st.sg_offset[st.last_bend];
  const int *sgi = st.d_sg_idx + st.sg_offset[st.last_bend] / B2E_SG_MAX_WIDTH * 2;
  WakeArgs a = {};
  a.nBins = nb;
  a.sgHalf = bend.sgHalf;
  a.sgdHalf = bend.sgdHalf;
  a.trapz = bend.trapz;
  a.correct = bend.sgHalf > 0;
  a.sg_w = sgw;
  a.sgd_w = sgw + (size_t)nb * B2E_SG_MAX_WIDTH;
  a.sg_lo = sgi;
  a.sg_n = sgi + 1;
  a.sgd_lo = sgi + 2 * nb;
  a.sgd_n = sgi + 2 * nb + 1;
  set_filter_args(a, bend.lh, bend.clip, bend.lowCut0, bend.lowCut1, bend.highCut0, bend.highCut1);
  const size_t smem = sizeof(double) * (5 * nb + 8);
  CSR_CUDA(cudaFuncSetAttribute(stupakov_wake_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  CsrBunches H = B; /* the histogram bins the bunches in this mode */
  H.active = B.mode;
  for (long iKick = 0; iKick < nKicks; iKick++) {
    if (iKick == 1)
      dz = dz0;
    zTravel += dz;
    StupakovArgs sa;
    sa.x = zTravel / rho;
    sa.dsMax = rho / 24 * b2e_pow(theta, 3) * (theta + 4 * sa.x) / (theta + sa.x);
    sa.dsC = rho / 6 * (theta * theta) * (theta + 3 * sa.x);
    sa.theta = theta;
    sa.rho = rho;
    sa.dz0 = dz0;
    sa.trapz = bend.trapz;
    csr_reset_keys_kernel<<<1, 32, 0, stream>>>(B);
    CSR_CUDA(launch_chained(stupakov_drift_kernel, dim3(g), dim3(256), 0, stream, P, n, B, iKick == 0 ? dz_back : 0.0,
                            dz, Po));
    (*launches) += 2;
    CSR_CUDA(cudaGetLastError());
    int rrc = reduce_keys(st, B, stream, err, launches);
    if (rrc)
      return rrc;
    CSR_CUDA(cudaMemsetAsync(st.d_counts, 0, sizeof(unsigned int) * nb * nbunch, stream));
    const int64_t per = (n + nbunch - 1) / nbunch;
    const int hb = hist_blocks(per, nbunch);
    CSR_CUDA(launch_chained(csr_hist_kernel, dim3(hb, nbunch), dim3(1024), hist_smem(nb), stream, P, n, H,
                            st.d_counts, nb, bend.binRangeFactor));
    (*launches)++;
    CSR_CUDA(cudaGetLastError());
    if (st.reducer && st.reducer(st.reducer_user, B2E_REDUCE_SUM_U32, st.d_counts, (int64_t)nb * nbunch, stream)) {
      err = "CSR: the all-rank reduction of the histogram failed";
      return B2E_ERR_CUDA;
    }
    CSR_CUDA(launch_chained(stupakov_wake_kernel, dim3(nbunch), dim3(1024), smem, stream, B,
                            (const unsigned int *)st.d_counts, a, sa));
    CSR_CUDA(launch_chained(stupakov_kick_kernel, dim3(g), dim3(256), 0, stream, P, n, B, nb, Po));
    (*launches) += 2;
    CSR_CUDA(cudaGetLastError());
  }
  CSR_CUDA(launch_chained(edrift_kernel, dim3(g), dim3(256), 0, stream, P, n, dz0 / 2, B, 1));
  (*launches)++;
  CSR_CUDA(cudaGetLastError());
  st.zLast = zStart + length;
  return B2E_OK;
}

int csr_track_element(CsrState &st, const DevElem *d_elems, const DevElem &h_elem, const DevParticles &P, int64_t n,
                      const std::vector<int64_t> &alive, int elem, int pass, cudaStream_t stream, std::string &err,
                      int64_t *launches) {
  size_t k = 0;
  while (k < st.elems.size() && st.elems[k].index != elem)
    k++;
  if (k == st.elems.size()) {
    err = "CSR element not configured";
    return B2E_ERR_STATE;
  }
  if ((int)alive.size() != st.n_bunches) {
    err = "CSR: per-bunch alive counts do not match the bunch layout";
    return B2E_ERR_STATE;
  }
  const CsrElem &ce = st.elems[k];
  const int nbunch = st.n_bunches;
  CsrBunches B;
  B.offs = st.d_offsets;
  B.n = nbunch;
  B.st = (CsrDevState *)st.d_state;
  B.csr_const = st.d_csr_const;
  B.active = st.d_flags;
  B.mode = st.d_flags + nbunch;
  const double Po = st.p_central;
  const int g = grid_for(n);
  std::vector<unsigned char> flags(2 * nbunch, 0);
  if (ce.kind == K_CSRDRIFT) {
    /* track_through_driftCSR (csbend.c:3176-3533), mode 0: bunches with a
     * valid dipole wake and more than one particle get wake kicks, the others
     * an exact drift (csbend.c:3196-3212) */
    bool any = false;
    for (int b = 0; b < nbunch; b++) {
      flags[nbunch + b] = alive[b] > 1 && st.wake_valid[b] && ce.drift_csr;
      any = any || flags[nbunch + b];
    }
    if (!any) {
      CsrBunches all = B;
      all.mode = nullptr;
      edrift_kernel<<<g, 256, 0, stream>>>(P, n, ce.drift_length, all, 0);
      (*launches)++;
      CSR_CUDA(cudaGetLastError());
      return B2E_OK;
    }
    CSR_CUDA(cudaMemcpyAsync(st.d_flags, flags.data(), flags.size(), cudaMemcpyHostToDevice, stream));
    bool some_plain = false;
    for (int b = 0; b < nbunch; b++)
      some_plain = some_plain || !flags[nbunch + b];
    if (some_plain) {
      edrift_kernel<<<g, 256, 0, stream>>>(P, n, ce.drift_length, B, 0);
      (*launches)++;
      CSR_CUDA(cudaGetLastError());
    }
    double zStart = ce.z_start;
    /* a drift behind the previous pass's dipole (csbend.c:3251-3255) */
    for (int guard = 0; zStart + 1e-12 < st.zLast && st.revolution_length > 0 && guard < (1 << 20); guard++)
      zStart += st.revolution_length;
    if (ce.stupakov)
      return stupakov_drift(st, ce, B, P, n, zStart, stream, err, launches);
    int nKicks;
    if (ce.drift_dz > 0) {
      if ((nKicks = (int)(ce.drift_length / ce.drift_dz)) < 1)
        nKicks = 1;
    } else
      nKicks = ce.drift_kicks;
    if (nKicks <= 0) {
      err = "nKicks=0 in CSR drift.";
      return B2E_ERR_LATTICE;
    }
    double dz0 = ce.drift_length / nKicks, dz = dz0 / 2;
    double dzFirst = zStart - st.zLast;
    /* csrWake.bins: bins of the last CSRCSBEND tracked (on a later pass,
     * possibly one further down the line) */
    const int lastBins = st.last_bend >= 0 ? st.elems[st.last_bend].bins : 0;
    for (int iKick = 0; iKick < nKicks; iKick++) {
      if (iKick == 1)
        dz = dz0;
      double incr = dz + dzFirst;
      double factor = (dz0 + dzFirst) / st.ds0;
      CSR_CUDA(launch_chained(csr_drift_kick_kernel, dim3(g), dim3(256), 0, stream, P, n, B, dz, incr, factor, 1,
                              lastBins, Po));
      CSR_CUDA(launch_chained(csr_s0_add_kernel, dim3(1), dim3(32), 0, stream, B, incr));
      (*launches) += 2;
      CSR_CUDA(cudaGetLastError());
      dzFirst = 0;
    }
    dz = dz0 / 2;
    CSR_CUDA(launch_chained(edrift_kernel, dim3(g), dim3(256), 0, stream, P, n, dz, B, 1));
    CSR_CUDA(launch_chained(csr_s0_add_kernel, dim3(1), dim3(32), 0, stream, B, dz));
    (*launches) += 2;
    CSR_CUDA(cudaGetLastError());
    st.zLast = zStart + ce.drift_length;
    return B2E_OK;
  }

  /* ---- CSRCSBEND ---- */
  const DevElem *d_e = d_elems + elem;
  bool any_active = false;
  for (int b = 0; b < nbunch; b++) {
    flags[b] = alive[b] > 1; /* csbend.c:1987 */
    any_active = any_active || flags[b];
  }
  if (!ce.same_bend_precedes)
    st.accumulated_angle = 0;
  st.wake_valid.assign(nbunch, 0);
  if (st.beta0_cap < n) {
    if (st.d_beta0)
      cudaFree(st.d_beta0);
    if (cudaMalloc(&st.d_beta0, sizeof(double) * std::max<int64_t>(n, 1)) != cudaSuccess) {
      err = "CSR beta0 allocation failed";
      return B2E_ERR_NOMEM;
    }
    st.beta0_cap = n;
  }
  if (ensure_wakelog(st, st.wake_values + (int64_t)ce.nSlices * ce.bins * nbunch)) {
    err = "CSR wake log allocation failed";
    return B2E_ERR_NOMEM;
  }
  const int64_t page_stride = B2E_CSR_PAGE_HEADER + 4 * (int64_t)ce.bins;
  if (st.record_pages && ensure_pagelog(st, st.page_values + (int64_t)ce.nSlices * nbunch * page_stride)) {
    err = "CSR page record allocation failed";
    return B2E_ERR_NOMEM;
  }
  st.ds0 = ce.length / ce.nSlices;
  st.zLast = st.z0 = ce.z_end;
  /* CSRConstant (csbend.c:2378-2381), per bunch */
  const double eps0 = 1 / ((4 * kPI * 1e-7) * kC * kC);
  std::vector<double> csr_constant(4 * nbunch, 0.0);
  for (int b = 0; b < nbunch; b++) {
    if (ce.csr && flags[b])
      csr_constant[b] = 2 * st.macro_charge[b] * kE / b2e_pow(3 * ce.rho0 * ce.rho0, 1. / 3.) /
                        (4 * kPI * eps0 * kME * (kC * kC));
    /* the IGF wake's factor (csbend.c:2678-2679) */
    csr_constant[nbunch + b] = -st.macro_charge[b] / (kME * (kC * kC)) * ce.length / ce.nSlices;
    /* GSConstant for a Stupakov CSRDRIFT (csbend.c:2999) */
    csr_constant[2 * nbunch + b] = csr_constant[b] * b2e_pow(3 * ce.rho0 * ce.rho0, 1. / 3.) / 2;
    /* the macro-particle charge, for the page record */
    csr_constant[3 * nbunch + b] = st.macro_charge[b];
  }
  CSR_CUDA(cudaMemcpyAsync(st.d_csr_const, csr_constant.data(), 4 * sizeof(double) * nbunch, cudaMemcpyHostToDevice,
                           stream));
  CSR_CUDA(cudaMemcpyAsync(st.d_flags, flags.data(), flags.size(), cudaMemcpyHostToDevice, stream));
  const double *sgw = st.d_sg + st.sg_offset[k];
  const int *sgi = st.d_sg_idx + st.sg_offset[k] / B2E_SG_MAX_WIDTH * 2;
  const size_t wake_smem = sizeof(double) * (4 * ce.bins + 8);
  CSR_CUDA(cudaFuncSetAttribute(csr_wake_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wake_smem));
  /* learned wake: trained on the transient integral with trapezoid rule (the
   * CSRCSBEND defaults); other settings, or a bunch train larger than the
   * network's batch, use the plain integral */
  const bool use_net = st.net && any_active && !ce.steady && ce.trapz && !ce.lh && ce.bins <= wakenet_bins(st.net) &&
                       nbunch <= wakenet_max_batch(st.net);
  const size_t sur_smem = sizeof(double) * (3 * ce.bins + 1024);
  if (use_net) {
    int rc = ensure_surrogate_buffers(st, (int64_t)ce.nSlices * nbunch, err);
    if (rc)
      return rc;
    CSR_CUDA(cudaFuncSetAttribute(csr_sur_filter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)std::max(sur_smem, sizeof(double) * (4 * ce.bins + 1024))));
    CSR_CUDA(cudaFuncSetAttribute(csr_sur_combine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sur_smem));
  }

  CSR_CUDA(launch_chained(csr_entry_kernel, dim3(g), dim3(256), 0, stream, P, n, st.d_beta0, d_e, ce.bx, Po));
  (*launches)++;
  CSR_CUDA(cudaGetLastError());
  double phiBend = st.accumulated_angle;
  /* on the plain-integral path the wake kernel empties the range keys and the
   * counts for the next kick; otherwise both are reset before every kick */
  const bool recycle = any_active && !use_net;
  if (recycle)
    CSR_CUDA(cudaMemsetAsync(st.d_counts, 0, sizeof(unsigned int) * ce.bins * nbunch, stream));
  for (int kick = 0; kick < ce.nSlices; kick++) {
    if (!recycle || kick == 0) {
      csr_reset_keys_kernel<<<1, 32, 0, stream>>>(B);
      (*launches)++;
    }
    CSR_CUDA(launch_chained(csr_slice_kernel, dim3(g), dim3(256), 0, stream, P, n, (const double *)st.d_beta0, d_e,
                            (const DevAperture *)nullptr, B, (int)(kick > 0), ce.bins, Po, pass, elem));
    (*launches)++;
    CSR_CUDA(cudaGetLastError());
    if (!any_active)
      continue;
    int rrc = reduce_keys(st, B, stream, err, launches);
    if (rrc)
      return rrc;
    if (!recycle)
      CSR_CUDA(cudaMemsetAsync(st.d_counts, 0, sizeof(unsigned int) * ce.bins * nbunch, stream));
    int64_t per = (n + nbunch - 1) / nbunch;
    int hb = hist_blocks(per, nbunch);
    CSR_CUDA(launch_chained(csr_hist_kernel, dim3(hb, nbunch), dim3(1024), hist_smem(ce.bins), stream, P,
                            n, B, st.d_counts, ce.bins, ce.binRangeFactor));
    (*launches)++;
    CSR_CUDA(cudaGetLastError());
    if (st.reducer && st.reducer(st.reducer_user, B2E_REDUCE_SUM_U32, st.d_counts, (int64_t)ce.bins * nbunch, stream)) {
      err = "CSR: the all-rank reduction of the histogram failed";
      return B2E_ERR_CUDA;
    }
    phiBend += ce.angle / ce.nSlices;
    double slippage = fabs(ce.rho0 * (phiBend * phiBend * phiBend) / 24.0);
    WakeArgs a = {};
    a.nBins = ce.bins;
    a.sgHalf = ce.sgHalf;
    a.sgdHalf = ce.sgdHalf;
    a.trapz = ce.trapz;
    a.steady = ce.steady;
    a.correct = ce.sgHalf > 0;
    a.sg_w = sgw;
    a.sgd_w = sgw + (size_t)ce.bins * B2E_SG_MAX_WIDTH;
    a.sg_lo = sgi;
    a.sg_n = sgi + 1;
    a.sgd_lo = sgi + 2 * ce.bins;
    a.sgd_n = sgi + 2 * ce.bins + 1;
    a.slippage = slippage;
    a.slippage13 = b2e_pow(slippage, 1. / 3.);
    a.length = ce.length;
    a.nSlices = ce.nSlices;
    a.c1 = a.c2 = a.csr_constant = 0; /* per bunch in the kernel */
    a.wakelog = st.d_wakelog + st.wake_values;
    /* pages of the plain-integral kicks only (the learned wake writes none) */
    a.pagelog = st.record_pages && !use_net ? st.d_pagelog + st.page_values : nullptr;
    a.page_element = elem;
    a.page_kick = kick;
    a.page_angle = phiBend;
    a.page_ds_kick = ce.length / ce.nSlices;
    a.page_p_central = Po;
    a.page_range_factor = ce.binRangeFactor;
    a.igf = ce.igf;
    set_filter_args(a, ce.lh, ce.clip, ce.lowCut0, ce.lowCut1, ce.highCut0, ce.highCut1);
    {
      /* gamma^2, gamma^3 and the IGF constants as the reference forms them
       * (csbend.c:1981-1982, :2604, :2617) */
      const double gamma2 = Po * Po + 1;
      a.gamma2 = gamma2;
      a.gamma3 = b2e_pow(gamma2, 3. / 2);
      a.rho0 = ce.rho0;
      a.const1 = 6.0 - b2e_log(27.0 / 4.0);
      a.q4pe = kE / (4 * kPI * eps0);
      a.igf_factor = 0;
    }
    cudaEvent_t ev_end = nullptr;
    if (st.time_wake) {
      while ((int64_t)st.wake_events.size() < 2 * (st.timed_kicks + 1)) {
        cudaEvent_t e;
        CSR_CUDA(cudaEventCreate(&e));
        st.wake_events.push_back(e);
      }
      CSR_CUDA(cudaEventRecord(st.wake_events[2 * st.timed_kicks], stream));
      ev_end = st.wake_events[2 * st.timed_kicks + 1];
    }
    if (use_net) {
      const int L = wakenet_bins(st.net);
      csr_sur_filter_kernel<<<nbunch, 1024, std::max(sur_smem, sizeof(double) * 4 * ce.bins), stream>>>(B, st.d_counts, a, L, st.sc_dens, st.sc_deriv,
                                                                st.d_sur_tab, st.d_sur_scal, st.d_sur_in);
      CSR_CUDA(cudaGetLastError());
      int rc = wakenet_infer(st.net, st.d_sur_in, nbunch, st.d_sur_out, stream);
      if (rc) {
        err = "CSR: wake network inference failed";
        return rc;
      }
      csr_sur_combine_kernel<<<nbunch, 1024, sur_smem, stream>>>(B, a, st.d_sur_tab, st.d_sur_scal, st.d_sur_out, L,
                                                                 st.sc_target, st.gate_tol, st.gate_stride,
                                                                 kick % st.gate_stride, st.d_gate_log + st.gate_values,
                                                                 st.d_sur_counts);
      CSR_CUDA(cudaGetLastError());
      st.gate_values += nbunch;
      (*launches) += 3 + 7; /* filter, pack + 6 convolutions, combine */
    } else {
      CSR_CUDA(launch_chained(csr_wake_kernel, dim3(nbunch), dim3(1024), wake_smem, stream, B, st.d_counts, a,
                              recycle ? 1 : 0));
      (*launches)++;
      CSR_CUDA(cudaGetLastError());
    }
    if (ev_end) {
      CSR_CUDA(cudaEventRecord(ev_end, stream));
      st.timed_kicks++;
      st.timed_learned += use_net;
    }
    st.wake_values += (int64_t)ce.bins * nbunch;
    if (a.pagelog)
      st.page_values += nbunch * page_stride;
  }
  if (!recycle || ce.nSlices <= 0) {
    csr_reset_keys_kernel<<<1, 32, 0, stream>>>(B);
    (*launches)++;
  }
  CSR_CUDA(launch_chained(csr_last_kick_kernel, dim3(g), dim3(256), 0, stream, P, n, B, ce.bins, Po, ce.rho0));
  CSR_CUDA(cudaGetLastError());
  if (any_active) {
    int rrc = reduce_keys(st, B, stream, err, launches);
    if (rrc)
      return rrc;
  }
  CSR_CUDA(launch_chained(csr_exit_kernel, dim3(g), dim3(256), 0, stream, P, n, d_e, ce.bx, B, ce.binRangeFactor, Po, pass,
                          elem));
  (*launches) += 2;
  CSR_CUDA(cudaGetLastError());
  for (int b = 0; b < nbunch; b++)
    st.wake_valid[b] = flags[b];
  /* csrWake.rho, csrWake.bendingAngle (csbend.c:2992-2993) */
  st.last_bend = (int)k;
  st.last_rho = h_elem.c[CB_RHO_ACTUAL];
  st.last_theta = ce.same_bend_precedes ? fabs(phiBend) : ce.angle;
  st.accumulated_angle += ce.angle;
  if (use_net && wakenet_take_status(st.net, stream)) {
    err = "CSR: a bounded wait in the wake network gave up";
    return B2E_ERR_TIMEOUT;
  }
  return B2E_OK;
}

int csr_wake_timing(CsrState &st, double *ms, int64_t *kicks, int64_t *learned, std::string &err) {
  double total = 0;
  for (int64_t k = 0; k < st.timed_kicks; k++) {
    float t = 0;
    cudaError_t e = cudaEventSynchronize(st.wake_events[2 * k + 1]);
    if (e == cudaSuccess)
      e = cudaEventElapsedTime(&t, st.wake_events[2 * k], st.wake_events[2 * k + 1]);
    if (e != cudaSuccess) {
      err = cudaGetErrorString(e);
      return B2E_ERR_CUDA;
    }
    total += t;
  }
  *ms = total;
  *kicks = st.timed_kicks;
  *learned = st.timed_learned;
  return B2E_OK;
}

int csr_copy_pages(CsrState &st, double *pages, int64_t capacity, int64_t *written, std::string &err) {
  int64_t n = std::min<int64_t>(st.page_values, capacity);
  if (n > 0 && pages) {
    cudaError_t e = cudaMemcpy(pages, st.d_pagelog, sizeof(double) * n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      err = cudaGetErrorString(e);
      return B2E_ERR_CUDA;
    }
  }
  *written = pages ? n : st.page_values;
  return B2E_OK;
}

int csr_copy_wakes(CsrState &st, double *wakes, int64_t capacity, int64_t *written, std::string &err) {
  int64_t n = std::min<int64_t>(st.wake_values, capacity);
  if (n > 0 && wakes) {
    cudaError_t e = cudaMemcpy(wakes, st.d_wakelog, sizeof(double) * n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      err = cudaGetErrorString(e);
      return B2E_ERR_CUDA;
    }
  }
  *written = wakes ? n : st.wake_values;
  return B2E_OK;
}

void csr_release(CsrState &st) {
  if (st.d_beta0)
    cudaFree(st.d_beta0);
  if (st.d_state)
    cudaFree(st.d_state);
  if (st.d_counts)
    cudaFree(st.d_counts);
  if (st.d_csr_const)
    cudaFree(st.d_csr_const);
  if (st.d_flags)
    cudaFree(st.d_flags);
  if (st.d_alive)
    cudaFree(st.d_alive);
  if (st.d_keys)
    cudaFree(st.d_keys);
  st.d_keys = nullptr;
  st.d_csr_const = nullptr;
  st.d_flags = nullptr;
  st.d_alive = nullptr;
  void *sur[] = {st.d_sur_in, st.d_sur_out, st.d_sur_tab, st.d_sur_scal, st.d_gate_log, st.d_sur_counts};
  for (void *q : sur)
    if (q)
      cudaFree(q);
  st.d_sur_in = st.d_sur_out = nullptr;
  st.d_sur_tab = st.d_sur_scal = st.d_gate_log = nullptr;
  st.d_sur_counts = nullptr;
  st.sur_cap_bunches = st.gate_cap = st.gate_values = 0;
  if (st.d_sg)
    cudaFree(st.d_sg);
  if (st.d_sg_idx)
    cudaFree(st.d_sg_idx);
  if (st.d_wakelog)
    cudaFree(st.d_wakelog);
  if (st.d_pagelog)
    cudaFree(st.d_pagelog);
  for (cudaEvent_t e : st.wake_events)
    cudaEventDestroy(e);
  st.wake_events.clear();
  st.timed_kicks = st.timed_learned = 0;
  st.d_pagelog = nullptr;
  st.pagelog_cap = 0;
  st.page_values = 0;
  st.d_beta0 = nullptr;
  st.d_state = nullptr;
  st.d_counts = nullptr;
  st.d_sg = nullptr;
  st.d_sg_idx = nullptr;
  st.d_wakelog = nullptr;
  st.beta0_cap = 0;
  st.wakelog_cap = 0;
  st.wake_values = 0;
}

} // namespace b2e

/* ==========================================================================
 * Allocation-free CSR dipole: b2e_csr_bend_static (include/elegant_b200.h).
 *
 * Some callers cannot allocate device memory at the moment they need this
 * computation: a host program that has handed the whole card to its own
 * memory pool, code that runs where cudaMalloc is not permitted, or an
 * embedding that must never fail for lack of memory halfway through a run.
 * For them, this path keeps all of its working memory in one file-scope
 * device array that is part of the loaded library image, so a call needs only
 * the caller's own particle and output buffers.
 *
 * The array holds per-particle entrance velocities (up to
 * B2E_STATIC_MAX_PARTICLES), the CSR binning/wake state, the histogram, the
 * Savitzky-Golay weight tables (up to B2E_STATIC_MAX_BINS bins) and the
 * element record: about 10.2 MB.  Under lazy module loading (CUDA's default)
 * a device gives it memory when this module is first used there -- the
 * set-up in static_scratch() -- and keeps it until the process exits.  The
 * call only enqueues work: the alive count that decides whether CSR is
 * computed becomes the bunch's flags on the device, so the host never waits
 * for the GPU.  All calls share the array and it keeps the previous
 * call's contents; everything that must start at zero is cleared by each
 * call.  Two calls whose work overlaps on the GPU (different streams, or
 * different host threads) race on this memory: callers must serialise them.
 * ======================================================================== */

/* B2E_STATIC_MAX_PARTICLES and B2E_STATIC_MAX_BINS come from elegant_b200.h */
namespace b2e {

struct StaticCsrScratch {
  double beta0[B2E_STATIC_MAX_PARTICLES];
  CsrDevState state;
  unsigned int counts[B2E_STATIC_MAX_BINS];
  double sg_w[2 * B2E_STATIC_MAX_BINS * B2E_SG_MAX_WIDTH];
  int sg_idx[2 * B2E_STATIC_MAX_BINS * 2];
  DevElem elem;
  unsigned long long counters[2];
  double csr_const[2];    /* the one bunch's CSRConstant and IGF wake factor */
  unsigned char flags[2]; /* active, CSRDRIFT mode */
};

static __device__ __align__(256) unsigned char g_static_csr_scratch[sizeof(StaticCsrScratch)];

/* Device addresses of g_static_csr_scratch, one per device, looked up by the
 * first call made with that device current (the set-up step).  That lookup is
 * also what makes CUDA load this module on the device under lazy module
 * loading (the default), so the array and the kernels' code take their device
 * memory at that first call, not when the library is loaded.  The cached
 * address belongs to the device's primary context: the library must not be
 * used on a device after cudaDeviceReset. */
#define B2E_STATIC_MAX_DEVICES 64
static void *g_static_addr[B2E_STATIC_MAX_DEVICES];
static std::mutex g_static_mutex;

static StaticCsrScratch *static_scratch(char *err, int64_t errlen) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= B2E_STATIC_MAX_DEVICES) {
    snprintf(err, errlen, "b2e_csr_bend_static: no usable current device (%s)", cudaGetErrorString(e));
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_static_mutex);
  if (!g_static_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_csr_scratch);
    if (e != cudaSuccess || !p) {
      snprintf(err, errlen, "b2e_csr_bend_static: cudaGetSymbolAddress failed on device %d (%s)", dev,
               cudaGetErrorString(e));
      return nullptr;
    }
    g_static_addr[dev] = p;
  }
  return (StaticCsrScratch *)g_static_addr[dev];
}

__global__ void static_set_elem_kernel(DevElem e, DevElem *dst) { *dst = e; }

/* Savitzky-Golay weight tables for one element, on the device, with the same
 * helpers and layout as csr_configure (rows of B2E_SG_MAX_WIDTH weights;
 * interleaved (start, width) index pairs; smoothing rows then derivative rows). */
/* The bunch's flags from the entrance count (S->counters[1] = particles alive
 * at the entrance; CSR only for more than one, csbend.c:1987), formed on the
 * device so that the host never waits for the count. */
__global__ void static_set_bunch_kernel(StaticCsrScratch *S, double csr_constant, double igf_factor) {
  const int more_than_one = S->counters[1] > 1;
  S->csr_const[0] = more_than_one ? csr_constant : 0.0;
  S->csr_const[1] = igf_factor;
  S->flags[0] = (unsigned char)more_than_one;
  S->flags[1] = 0;
}

__global__ void static_sg_weights_kernel(int bins, int sgHalf, int sgOrder, int sgdHalf, int sgdOrder, double *w,
                                         int *idx) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= 2 * bins)
    return;
  const int pass = row >= bins, b = row - pass * bins;
  const int half = pass == 0 ? sgHalf : sgdHalf, order = pass == 0 ? sgOrder : sgdOrder;
  double ww[B2E_SG_MAX_WIDTH];
  for (int k = 0; k < B2E_SG_MAX_WIDTH; k++)
    ww[k] = 0;
  long width;
  long lo = b2e_sg_window(b, bins, half, half, &width);
  long ord = order < width - 1 ? order : width - 1;
  if (pass == 0 && half <= 0) {
    width = 1;
    lo = b;
    ww[0] = 1;
  } else if ((pass == 1 && 1 > ord) || b2e_sg_weights(ww, width, lo - b, ord, pass)) {
    width = 0;
  }
  for (int k = 0; k < B2E_SG_MAX_WIDTH; k++)
    w[(size_t)row * B2E_SG_MAX_WIDTH + k] = ww[k];
  idx[2 * row] = (int)lo;
  idx[2 * row + 1] = (int)width;
}

#define STATIC_TRY(call)                                                                                          \
  do {                                                                                                            \
    cudaError_t e_ = (call);                                                                                      \
    if (e_ != cudaSuccess) {                                                                                      \
      snprintf(err, errlen, "b2e_csr_bend_static: %s: %s", #call, cudaGetErrorString(e_));                       \
      return B2E_ERR_CUDA;                                                                                        \
    }                                                                                                             \
  } while (0)

} // namespace b2e

extern "C" int b2e_csr_bend_static(double *const dev_columns[6], int32_t *dev_lost_pass, int32_t *dev_lost_element,
                                   int64_t n, const b2e_element *bend, double p_central, double macro_particle_charge,
                                   double *dev_wakes, int64_t wake_capacity, void *stream, char *errbuf,
                                   int64_t errlen) {
  using namespace b2e;
  char local_err[256];
  char *err = errbuf && errlen > 0 ? errbuf : local_err;
  if (!(errbuf && errlen > 0))
    errlen = sizeof(local_err);
  err[0] = 0;
  /* n = 0 (the set-up call) touches no particle buffer: they may be NULL */
  if (!bend || n < 0 || p_central <= 0 || (n > 0 && (!dev_columns || !dev_lost_pass || !dev_lost_element))) {
    snprintf(err, errlen, "b2e_csr_bend_static: null pointer, negative count or nonpositive p_central");
    return B2E_ERR_ARG;
  }
  for (int c = 0; c < 6 && n > 0; c++)
    if (!dev_columns[c]) {
      snprintf(err, errlen, "b2e_csr_bend_static: column %d is null", c);
      return B2E_ERR_ARG;
    }
  if (n > B2E_STATIC_MAX_PARTICLES) {
    snprintf(err, errlen, "b2e_csr_bend_static: %lld particles exceed the static limit of %d", (long long)n,
             B2E_STATIC_MAX_PARTICLES);
    return B2E_ERR_ARG;
  }
  DevElem d;
  BendExtra bx;
  const char *msg = compile_single_csr_bend(*bend, d, bx);
  if (msg) {
    snprintf(err, errlen, "b2e_csr_bend_static: %s", msg);
    return B2E_ERR_LATTICE;
  }
  const double *p = bend->p;
  const int bins = (int)p[B2E_BEND_BINS], nSlices = (int)d.c[CB_NSLICES];
  if (bins < 2 || bins > B2E_STATIC_MAX_BINS) {
    snprintf(err, errlen, "b2e_csr_bend_static: BINS=%d outside [2, %d]", bins, B2E_STATIC_MAX_BINS);
    return B2E_ERR_ARG;
  }
  int sgHalf = (int)p[B2E_BEND_SG_HALFWIDTH], sgOrder = (int)p[B2E_BEND_SG_ORDER];
  int sgdHalf = (int)p[B2E_BEND_SGDERIV_HALFWIDTH], sgdOrder = (int)p[B2E_BEND_SGDERIV_ORDER];
  if (sgdHalf <= 0)
    sgdHalf = sgHalf;
  if (sgdHalf <= 0)
    sgdHalf = 1;
  if (sgdOrder <= 0)
    sgdOrder = sgOrder;
  if (sgdOrder <= 0)
    sgdOrder = 1;
  if (2 * (sgHalf > sgdHalf ? sgHalf : sgdHalf) + 1 > B2E_SG_MAX_WIDTH) {
    snprintf(err, errlen, "b2e_csr_bend_static: Savitzky-Golay half-width too large");
    return B2E_ERR_ARG;
  }
  if (p[B2E_BEND_IGF] != 0 && p[B2E_BEND_STEADY_STATE] == 0) {
    snprintf(err, errlen, "b2e_csr_bend_static: Must have STEADY_STATE=1 when IGF=1");
    return B2E_ERR_LATTICE;
  }
  if (dev_wakes && wake_capacity < (int64_t)nSlices * bins) {
    snprintf(err, errlen, "b2e_csr_bend_static: wake buffer holds %lld values, %lld needed",
             (long long)wake_capacity, (long long)nSlices * bins);
    return B2E_ERR_ARG;
  }
  StaticCsrScratch *S = static_scratch(err, errlen);
  if (!S)
    return B2E_ERR_CUDA;
  cudaStream_t s = (cudaStream_t)stream;
  DevParticles P;
  P.x = n > 0 ? dev_columns[0] : nullptr;
  P.xp = n > 0 ? dev_columns[1] : nullptr;
  P.y = n > 0 ? dev_columns[2] : nullptr;
  P.yp = n > 0 ? dev_columns[3] : nullptr;
  P.s = n > 0 ? dev_columns[4] : nullptr;
  P.dp = n > 0 ? dev_columns[5] : nullptr;
  P.lost_pass = dev_lost_pass;
  P.lost_elem = dev_lost_element;

  static_set_elem_kernel<<<1, 1, 0, s>>>(d, &S->elem);
  static_sg_weights_kernel<<<(2 * bins + 127) / 128, 128, 0, s>>>(bins, sgHalf, sgOrder, sgdHalf, sgdOrder, S->sg_w,
                                                                  S->sg_idx);
  STATIC_TRY(cudaGetLastError());
  /* particles alive at the entrance decide whether CSR is computed
   * (csbend.c:1987): counted and turned into the bunch's flags on the device;
   * the histogram and wake kernels do nothing for an inactive bunch */
  STATIC_TRY(cudaMemsetAsync(S->counters, 0, sizeof(S->counters), s));
  STATIC_TRY(launch_effort(dev_lost_pass, n, 0, 0, &S->counters[0], &S->counters[1], s));

  const double Po = p_central;
  const double angle = fabs(p[B2E_BEND_ANGLE]), length = p[B2E_BEND_L], rho0 = d.c[CB_RHO0];
  const double brf = p[B2E_BEND_BIN_RANGE_FACTOR] < 1.1 ? 1.1 : p[B2E_BEND_BIN_RANGE_FACTOR];
  const double eps0 = 1 / ((4 * kPI * 1e-7) * kC * kC);
  double csr_constant = 0;
  if (p[B2E_BEND_CSR] != 0)
    csr_constant = 2 * macro_particle_charge * kE / b2e_pow(3 * rho0 * rho0, 1. / 3.) / (4 * kPI * eps0 * kME * (kC * kC));
  const int g = (int)std::max<int64_t>(1, (n + 255) / 256);
  CsrDevState *dst = &S->state;
  static_set_bunch_kernel<<<1, 1, 0, s>>>(S, csr_constant,
                                          -macro_particle_charge / (kME * (kC * kC)) * length / nSlices);
  CsrBunches B;
  B.offs = nullptr;
  B.n = 1;
  B.st = dst;
  B.csr_const = S->csr_const;
  B.active = &S->flags[0];
  B.mode = &S->flags[1];

  /* the wake kernel's shared-memory limit is a per-function setting that the
   * context path also changes: set it for this call's bin count */
  const size_t wake_smem = sizeof(double) * (4 * bins + 8);
  STATIC_TRY(cudaFuncSetAttribute(csr_wake_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wake_smem));
  csr_entry_kernel<<<g, 256, 0, s>>>(P, n, S->beta0, &S->elem, bx, Po);
  STATIC_TRY(cudaGetLastError());
  double phiBend = 0;
  for (int kick = 0; kick < nSlices; kick++) {
    csr_reset_keys_kernel<<<1, 32, 0, s>>>(B);
    csr_slice_kernel<<<g, 256, 0, s>>>(P, n, S->beta0, &S->elem, nullptr, B, kick > 0, bins, Po, 0, 0);
    STATIC_TRY(cudaGetLastError());
    STATIC_TRY(cudaMemsetAsync(S->counts, 0, sizeof(unsigned int) * bins, s));
    int hb = hist_blocks(n, 1);
    csr_hist_kernel<<<dim3(hb, 1), 1024, sizeof(unsigned int) * bins, s>>>(P, n, B, S->counts, bins, brf);
    STATIC_TRY(cudaGetLastError());
    phiBend += angle / nSlices;
    double slippage = fabs(rho0 * (phiBend * phiBend * phiBend) / 24.0);
    WakeArgs a = {};
    a.nBins = bins;
    a.sgHalf = sgHalf;
    a.sgdHalf = sgdHalf;
    a.trapz = p[B2E_BEND_TRAPAZOID_INTEGRATION] != 0;
    a.steady = p[B2E_BEND_STEADY_STATE] != 0;
    a.correct = sgHalf > 0;
    a.sg_w = S->sg_w;
    a.sgd_w = S->sg_w + (size_t)bins * B2E_SG_MAX_WIDTH;
    a.sg_lo = S->sg_idx;
    a.sg_n = S->sg_idx + 1;
    a.sgd_lo = S->sg_idx + 2 * bins;
    a.sgd_n = S->sg_idx + 2 * bins + 1;
    a.slippage = slippage;
    a.slippage13 = b2e_pow(slippage, 1. / 3.);
    a.length = length;
    a.nSlices = nSlices;
    a.c1 = a.c2 = a.csr_constant = 0; /* formed in the kernel from B.csr_const */
    a.wakelog = dev_wakes ? dev_wakes + (size_t)kick * bins : nullptr;
    a.igf = p[B2E_BEND_IGF] != 0;
    set_filter_args(a, p[B2E_BEND_HIGH_FREQUENCY_CUTOFF0] > 0 || p[B2E_BEND_LOW_FREQUENCY_CUTOFF0] >= 0,
                    p[B2E_BEND_CLIP_NEGATIVE_BINS] != 0, p[B2E_BEND_LOW_FREQUENCY_CUTOFF0],
                    p[B2E_BEND_LOW_FREQUENCY_CUTOFF1], p[B2E_BEND_HIGH_FREQUENCY_CUTOFF0],
                    p[B2E_BEND_HIGH_FREQUENCY_CUTOFF1]);
    a.gamma2 = Po * Po + 1;
    a.gamma3 = b2e_pow(a.gamma2, 3. / 2);
    a.rho0 = rho0;
    a.const1 = 6.0 - b2e_log(27.0 / 4.0);
    a.q4pe = kE / (4 * kPI * eps0);
    a.igf_factor = 0;
    csr_wake_kernel<<<1, 1024, wake_smem, s>>>(B, S->counts, a, 0);
    STATIC_TRY(cudaGetLastError());
  }
  csr_reset_keys_kernel<<<1, 32, 0, s>>>(B);
  csr_last_kick_kernel<<<g, 256, 0, s>>>(P, n, B, bins, Po, rho0);
  csr_exit_kernel<<<g, 256, 0, s>>>(P, n, &S->elem, bx, B, brf, Po, 0, 0);
  STATIC_TRY(cudaGetLastError());
  STATIC_TRY(launch_post_element_sweep(P, n, nullptr, 0, 0, s));
  return B2E_OK;
}

/* Network inputs of batched profiles (b2e_wake_features), one CTA per
 * profile: the tracking path's feature step (csr_sur_filter_kernel) on
 * bin-unit density and derivative. */
namespace b2e {
__global__ void wake_features_kernel(const double *dens, const double *deriv, const double *slip, int nb,
                                     double sc_dens, double sc_deriv, int shift, float *inputs, double *scales) {
  __shared__ double red[1024];
  const int p = blockIdx.x;
  const double *h = dens + (size_t)p * nb, *d = deriv + (size_t)p * nb;
  float *in = inputs + (size_t)p * 4 * nb;
  double part = 0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x)
    part += h[i];
  double total = block_sum(part, red);
  total = total > 1e-300 ? total : 1e-300;
  part = 0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    const double g = d[i] / total;
    part += g * g;
  }
  const double ms = block_sum(part, red) / nb;
  double k = sqrt(ms);
  k = 1.0 / (k > 1e-300 ? k : 1e-300);
  const double sv = slip[p];
  long long dis = (long long)floor(sv);
  dis = dis < 1 ? 1 : (dis > nb ? nb : dis);
  const float code = (float)(log2((double)dis) / log2((double)nb));
  const double fd = k / total * sc_dens, fg = k / total * sc_deriv;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    in[i] = (float)(h[i] * fd);
    in[nb + i] = (float)(d[i] * fg);
    in[2 * nb + i] = code;
    in[3 * nb + i] = shift && i + dis < nb ? (float)(h[i + dis] * fd) : 0.f;
  }
  if (threadIdx.x == 0) {
    scales[2 * p] = total;
    scales[2 * p + 1] = k;
  }
}

__global__ void wake_t1_kernel(const float *y, const double *scales, const double *slip, int nb, double sc_target,
                               double *t1) {
  const int p = blockIdx.x;
  const double total = scales[2 * p], k = scales[2 * p + 1];
  const bool empty = slip[p] < 1; /* diS = 0: the integral is empty */
  for (int i = threadIdx.x; i < nb; i += blockDim.x)
    t1[(size_t)p * nb + i] = empty ? 0.0 : (double)y[(size_t)p * nb + i] / sc_target / k * total;
}
} // namespace b2e

extern "C" int b2e_wake_features(const double *dev_density, const double *dev_derivative,
                                 const double *dev_slippage_bins, int32_t n_profiles, int32_t bins,
                                 double density_scale, double derivative_scale, int32_t shift, float *dev_inputs,
                                 double *dev_scales, void *stream) {
  if (!dev_density || !dev_derivative || !dev_slippage_bins || !dev_inputs || !dev_scales || n_profiles < 0 ||
      bins < 2)
    return B2E_ERR_ARG;
  if (n_profiles == 0)
    return B2E_OK;
  b2e::wake_features_kernel<<<n_profiles, 1024, 0, (cudaStream_t)stream>>>(
      dev_density, dev_derivative, dev_slippage_bins, bins, density_scale, derivative_scale, shift, dev_inputs,
      dev_scales);
  return cudaGetLastError() == cudaSuccess ? B2E_OK : B2E_ERR_CUDA;
}

extern "C" int b2e_wake_t1_from_output(const float *dev_y, const double *dev_scales, const double *dev_slippage_bins,
                                       int32_t n_profiles, int32_t bins, double target_scale, double *dev_t1,
                                       void *stream) {
  if (!dev_y || !dev_scales || !dev_slippage_bins || !dev_t1 || n_profiles < 0 || bins < 2)
    return B2E_ERR_ARG;
  if (n_profiles == 0)
    return B2E_OK;
  b2e::wake_t1_kernel<<<n_profiles, 256, 0, (cudaStream_t)stream>>>(dev_y, dev_scales, dev_slippage_bins, bins,
                                                                   target_scale, dev_t1);
  return cudaGetLastError() == cudaSuccess ? B2E_OK : B2E_ERR_CUDA;
}

/* Batched wake integral for the wake-network data set: n_profiles histograms
 * of `bins` real-valued counts, each with its own slippage in bins. */
using b2e::WakeArgs;
using b2e::static_sg_weights_kernel;
using b2e::wake_batch_kernel;
extern "C" int b2e_csr_wake_batch(const double *dev_counts, const double *dev_slippage_bins, int32_t n_profiles,
                                  int32_t bins, int32_t sg_halfwidth, int32_t sg_order, int32_t sgd_halfwidth,
                                  int32_t sgd_order, int32_t trapezoid, int32_t steady, double *dev_t1,
                                  double *dev_density, double *dev_derivative, void *stream) {
  if (!dev_counts || !dev_slippage_bins || !dev_t1 || !dev_density || !dev_derivative || n_profiles < 0 ||
      bins < 2 || bins > B2E_CSR_MAX_BINS)
    return B2E_ERR_ARG;
  if (sgd_halfwidth <= 0)
    sgd_halfwidth = sg_halfwidth;
  if (sgd_halfwidth <= 0)
    sgd_halfwidth = 1;
  if (sgd_order <= 0)
    sgd_order = sg_order;
  if (sgd_order <= 0)
    sgd_order = 1;
  if (2 * std::max(sg_halfwidth, sgd_halfwidth) + 1 > B2E_SG_MAX_WIDTH)
    return B2E_ERR_ARG;
  if (n_profiles == 0)
    return B2E_OK;
  cudaStream_t s = (cudaStream_t)stream;
  double *w = nullptr;
  int *idx = nullptr;
  if (cudaMallocAsync((void **)&w, sizeof(double) * 2 * bins * B2E_SG_MAX_WIDTH, s) != cudaSuccess)
    return B2E_ERR_NOMEM;
  if (cudaMallocAsync((void **)&idx, sizeof(int) * 4 * bins, s) != cudaSuccess) {
    cudaFreeAsync(w, s);
    return B2E_ERR_NOMEM;
  }
  static_sg_weights_kernel<<<(2 * bins + 127) / 128, 128, 0, s>>>(bins, sg_halfwidth, sg_order, sgd_halfwidth,
                                                                  sgd_order, w, idx);
  WakeArgs a = {};
  a.nBins = bins;
  a.sgHalf = sg_halfwidth;
  a.sgdHalf = sgd_halfwidth;
  a.trapz = trapezoid != 0;
  a.steady = steady != 0;
  a.correct = sg_halfwidth > 0;
  a.sg_w = w;
  a.sgd_w = w + (size_t)bins * B2E_SG_MAX_WIDTH;
  a.sg_lo = idx;
  a.sg_n = idx + 1;
  a.sgd_lo = idx + 2 * bins;
  a.sgd_n = idx + 2 * bins + 1;
  a.slippage = 0;
  a.slippage13 = 1;
  a.c1 = 1;
  a.c2 = 0;
  a.csr_constant = 1;
  a.wakelog = nullptr;
  a.length = a.nSlices = 1;
  a.igf = 0;
  a.gamma2 = a.gamma3 = a.rho0 = a.const1 = a.q4pe = a.igf_factor = 0;
  const size_t smem = sizeof(double) * 4 * bins;
  cudaError_t e = cudaFuncSetAttribute(wake_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    wake_batch_kernel<<<n_profiles, 512, smem, s>>>(dev_counts, dev_slippage_bins, a, dev_t1, dev_density,
                                                    dev_derivative);
    e = cudaGetLastError();
  }
  cudaFreeAsync(w, s);
  cudaFreeAsync(idx, s);
  return e == cudaSuccess ? B2E_OK : B2E_ERR_CUDA;
}
