/*
 * Fused multi-pass tracking kernel for the non-collective element subset
 * (DRIF, EDRIFT, KQUAD, KSEXT, CSBEND, RFCA, MAXAMP, MARK, CHARGE).
 *
 * One thread owns one particle for the whole launch: the six coordinates stay
 * in registers across every element of every pass in the launch, so HBM
 * traffic is one 48-byte load and one 48-byte store per particle per launch
 * and the kernel is bound by the FP64 pipe.  This is the B200 replacement for
 * gpuElegant's one-launch-per-element functor kernels
 * (gpu_particle_template_function.hcu:64-86), which re-read and re-write every
 * particle for every element.
 *
 * A thread block tracks one tile (a contiguous run of particles of a single
 * lattice instance), so batched ensembles with uneven particle counts share
 * one launch without mixing instances inside a block.  The instance's
 * compiled elements and apertures are staged in shared memory at block start.
 *
 * Losses: a lost particle records (pass, element) in its loss columns and
 * stops; it keeps its slot (elegant instead swaps lost rows to the tail of the
 * array, do_tracking.c:4584 -- the order of rows is not part of the result,
 * IDs are).
 */
#include <cuda_runtime.h>
#include "b2e_elements.cuh"
#include "b2e_kernels.h"

namespace b2e {



/* Per-pass beam moments of one tile, for the ensemble history: count, means
 * of x, xp, y, yp, then sums of squared deviations (x, xp, xx', y, yp, yy')
 * about the tile means -- two reductions over the tile's four warps in a
 * fixed order, so the result does not depend on scheduling.  Every thread of
 * the block calls it; the 128-thread group g of the block reduces its own
 * tile and writes it to out (when out is not null). */
__device__ __forceinline__ void tile_moments(const Part &p, bool alive, double *out) {
  __shared__ double red_all[8][4][12];
  const int lane = threadIdx.x & 31, warp = (threadIdx.x >> 5) & 3;
  double(*red)[12] = red_all[threadIdx.x >> 7];
  double v[5] = {alive ? 1.0 : 0.0, alive ? p.x : 0.0, alive ? p.xp : 0.0, alive ? p.y : 0.0, alive ? p.yp : 0.0};
  for (int k = 0; k < 5; k++)
    for (int off = 16; off > 0; off >>= 1)
      v[k] += __shfl_down_sync(0xffffffffu, v[k], off);
  if (lane == 0)
    for (int k = 0; k < 5; k++)
      red[warp][k] = v[k];
  __syncthreads();
  double tot[5];
  for (int k = 0; k < 5; k++)
    tot[k] = ((red[0][k] + red[1][k]) + red[2][k]) + red[3][k];
  const double n = tot[0];
  double m[4];
  for (int k = 0; k < 4; k++)
    m[k] = n > 0 ? tot[k + 1] / n : 0.0;
  const double dx = p.x - m[0], dxp = p.xp - m[1], dy = p.y - m[2], dyp = p.yp - m[3];
  double q[6] = {alive ? dx * dx : 0.0,  alive ? dxp * dxp : 0.0, alive ? dx * dxp : 0.0,
                 alive ? dy * dy : 0.0,  alive ? dyp * dyp : 0.0, alive ? dy * dyp : 0.0};
  for (int k = 0; k < 6; k++)
    for (int off = 16; off > 0; off >>= 1)
      q[k] += __shfl_down_sync(0xffffffffu, q[k], off);
  if (lane == 0)
    for (int k = 0; k < 6; k++)
      red[warp][5 + k] = q[k];
  __syncthreads();
  if ((threadIdx.x & 127) == 0 && out) {
    out[0] = n;
    for (int k = 0; k < 4; k++)
      out[1 + k] = m[k];
    for (int k = 0; k < 6; k++)
      out[5 + k] = ((red[0][5 + k] + red[1][5 + k]) + red[2][5 + k]) + red[3][5 + k];
  }
  __syncthreads();
}

/* MINB is the occupancy target (blocks of 128 threads per SM) handed to the
 * register allocator: 4 keeps every value in registers (~118 registers),
 * 5/6/8 trade a few spills to L1 for more resident warps to hide FP64
 * latency.  SYNC sets how often the four warps of a block are brought back
 * in step: 0 never, 1 after every pass, 2 after every element; warps that
 * stay on the same element share its instruction stream and its shared-
 * memory record.  The arithmetic is identical in every variant.  HIST records
 * the per-pass tile moments (it needs SYNC >= 1); when SYNC >= 1 every thread
 * stays in the pass loop until the whole tile is lost. */
template <bool STAGED, int MINB, int SYNC, bool HIST, int TPB, bool RAD = false>
__global__ void __launch_bounds__(128 * TPB, MINB) ring_kernel(RingLaunch L) {
  static_assert(!HIST || SYNC >= 1, "history needs the per-pass barrier");
  static_assert(TPB == 1 || ((TPB == 2 || TPB == 4 || TPB == 8) && SYNC >= 1), "tiles of a block run in step");
  extern __shared__ __align__(16) unsigned char smem[];
  /* TPB tiles per block, 128 threads each; a missing second tile (odd tile
   * count) leaves its threads idle but inside the barriers */
  const int group = TPB == 1 ? 0 : (int)(threadIdx.x >> 7), lt = threadIdx.x & 127;
  (void)group;
  const int tidx = blockIdx.x * TPB + group;
  DevTile tile = {0, 0, 0};
  if (tidx < L.n_tiles)
    tile = L.tiles[tidx];
  const DevElem *elems = L.elems + (size_t)tile.inst * L.n_elems;
  const DevAperture *aps = L.aps + (size_t)tile.inst * L.n_aps;
  const DevRfState *rf = L.rf + (size_t)tile.inst * L.n_rf;

  if (STAGED) {
    /* stage this tile's instance's element and aperture records in shared memory */
    const size_t stage = sizeof(DevElem) * L.n_elems + sizeof(DevAperture) * L.n_aps;
    DevElem *se = reinterpret_cast<DevElem *>(smem + group * stage);
    DevAperture *sa = reinterpret_cast<DevAperture *>(smem + group * stage + sizeof(DevElem) * L.n_elems);
    const int nw_e = (int)(sizeof(DevElem) * L.n_elems / 8), nw_a = (int)(sizeof(DevAperture) * L.n_aps / 8);
    const double *src_e = reinterpret_cast<const double *>(elems);
    const double *src_a = reinterpret_cast<const double *>(aps);
    double *dst_e = reinterpret_cast<double *>(se), *dst_a = reinterpret_cast<double *>(sa);
    for (int i = lt; i < nw_e; i += 128)
      dst_e[i] = src_e[i];
    for (int i = lt; i < nw_a; i += 128)
      dst_a[i] = src_a[i];
    __syncthreads();
    elems = se;
    aps = sa;
  }

  const int64_t ip = tile.start + lt;
  const bool tracked = lt < tile.count && L.P.lost_pass[ip] < 0;
  if (SYNC == 0 && !tracked)
    return;

  Part p = {0, 0, 0, 0, 0, 0};
  if (tracked) {
    p.x = L.P.x[ip];
    p.xp = L.P.xp[ip];
    p.y = L.P.y[ip];
    p.yp = L.P.yp[ip];
    p.s = L.P.s[ip];
    p.dp = L.P.dp[ip];
  }

  int lost = LOSS_NONE, lost_pass = -1, lost_elem = -1;
  bool active = tracked;
  RadSite rs = {0, 0, 0, 0, 0, nullptr};
  const DevRad *rads = RAD ? L.rads + (size_t)tile.inst * L.n_elems : nullptr;
  if (RAD) {
    rs.id = tracked ? (L.ids ? L.ids[ip] : ip + 1) : 0;
    rs.seed = L.isr_seed;
    rs.limit = L.sr_limit;
  }
  for (int pass = L.pass_begin; pass <= L.pass_end; pass++) {
    if (SYNC == 0) {
      if (!active)
        break;
    } else if (!__syncthreads_or(active)) {
      break; /* the whole tile is lost (history slots stay zero: no survivors) */
    }
    const int e0 = pass == L.pass_begin ? L.elem_begin : 0;
    const int e1 = pass == L.pass_end ? L.elem_end : L.n_elems;
    for (int ie = e0; ie < e1; ie++) {
      if (SYNC == 2)
        __syncthreads();
      if (!active) {
        if (SYNC == 2)
          continue;
        break;
      }
      const DevElem &e = elems[ie];
      const int iap = pass == 0 ? e.ap_pass0 : e.ap_later;
      const DevAperture *ap = iap >= 0 ? &aps[iap] : nullptr;
      switch (e.kind) {
      case K_DRIF_O2:
        drif_o2(p, e);
        break;
      case K_DRIF_O1:
        drif_o1(p, e);
        break;
      case K_EDRIFT:
        edrift(p, e.c[DR_L]);
        break;
      case K_KMULT:
        if (RAD) {
          rs.pass = pass;
          rs.elem = ie;
          rs.rc = rads[ie].c;
        }
        lost = kmult<RAD>(p, e, ap, L.g, rs);
        break;
      case K_CSBEND:
        if (RAD) {
          rs.pass = pass;
          rs.elem = ie;
          rs.rc = rads[ie].c;
        }
        lost = csbend<RAD>(p, e, ap, L.g, rs);
        break;
      case K_MALIGN: {
        const double *mc = e.c;
        const int on_pass = (int)mc[MA_ON_PASS];
        if (on_pass == -1 || on_pass == pass) {
          bool hit = true;
          if (mc[MA_START_PID] >= 0) {
            const double id = (double)(L.ids ? L.ids[ip] : ip + 1);
            hit = !(id < mc[MA_START_PID] || id > mc[MA_END_PID]);
          }
          if (hit)
            malign(p, mc, L.g.p_central);
        }
        break;
      }
      case K_RFCA: {
        const DevRfState rs = rf[(int)e.c[RF_SLOT]];
        if (!rs.set) {
          /* the host runs the fiducial pass before any launch that needs it */
          atomicOr(L.error_flag, 1u);
          lost = LOSS_ENERGY;
        } else
          lost = rfca(p, e, rs, L.g);
        break;
      }
      default: /* MARK, CHARGE, WATCH (recorded between launches) */
        break;
      }
      if (!lost && !(e.flags & EF_NO_APERTURE) && ap && !maxamp_ok(p, *ap))
        lost = LOSS_APERTURE;
      if (!lost && !finite_xy(p))
        lost = LOSS_NAN;
      if (lost) {
        lost_pass = pass;
        lost_elem = ie;
        active = false;
      }
    }
    if (L.tbt && active && e1 == L.n_elems) {
      const int r = pass - L.tbt_pass0 + 1;
      if (r >= 1 && r < L.tbt_records) {
        double *o = L.tbt + (size_t)r * 4 * L.tbt_rows + ip;
        o[0] = p.x;
        o[L.tbt_rows] = p.xp;
        o[2 * L.tbt_rows] = p.y;
        o[3 * L.tbt_rows] = p.yp;
      }
    }
    if (HIST && e1 == L.n_elems && pass >= L.hist_pass0)
      tile_moments(p, active,
                   tidx < L.n_tiles ? L.hist + ((size_t)tidx * L.hist_passes + (pass - L.hist_pass0)) * 11 : nullptr);
  }

  if (!tracked)
    return;
  L.P.x[ip] = p.x;
  L.P.xp[ip] = p.xp;
  L.P.y[ip] = p.y;
  L.P.yp[ip] = p.yp;
  L.P.s[ip] = p.s;
  L.P.dp[ip] = p.dp;
  if (lost) {
    L.P.lost_pass[ip] = lost_pass;
    L.P.lost_elem[ip] = lost_elem;
  }
}

/* Ensemble history: merge the tiles of each instance, pass by pass, in tile
 * order with the pairwise update of Chan, Golub & LeVeque (1979) for means
 * and co-moments; rms emittance as rms_emittance (final_props.c:844-880):
 * sqrt(Sxx Sx'x' - Sxx'^2)/n.  out[inst][pass][5] = survivors, <x>, <y>,
 * emittance x, emittance y. */
__global__ void history_merge_kernel(const double *partials, int hist_passes, const int *tile_first, int n_inst,
                                     double *out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n_inst * hist_passes)
    return;
  const int inst = idx / hist_passes, j = idx - inst * hist_passes;
  double n = 0, m[4] = {0, 0, 0, 0}, S[6] = {0, 0, 0, 0, 0, 0};
  for (int t = tile_first[inst]; t < tile_first[inst + 1]; t++) {
    const double *b = partials + ((size_t)t * hist_passes + j) * 11;
    const double nb = b[0];
    if (nb == 0)
      continue;
    if (n == 0) {
      n = nb;
      for (int k = 0; k < 4; k++)
        m[k] = b[1 + k];
      for (int k = 0; k < 6; k++)
        S[k] = b[5 + k];
      continue;
    }
    const double N = n + nb, w = n * nb / N;
    double d[4];
    for (int k = 0; k < 4; k++)
      d[k] = b[1 + k] - m[k];
    S[0] += b[5] + d[0] * d[0] * w;
    S[1] += b[6] + d[1] * d[1] * w;
    S[2] += b[7] + d[0] * d[1] * w;
    S[3] += b[8] + d[2] * d[2] * w;
    S[4] += b[9] + d[3] * d[3] * w;
    S[5] += b[10] + d[2] * d[3] * w;
    for (int k = 0; k < 4; k++)
      m[k] += d[k] * nb / N;
    n = N;
  }
  double *o = out + (size_t)idx * 5;
  o[0] = n;
  o[1] = m[0];
  o[2] = m[2];
  double ex = S[0] * S[1] - S[2] * S[2], ey = S[3] * S[4] - S[5] * S[5];
  o[3] = n > 0 ? (ex > 0 ? sqrt(ex) : 0) / n : 0;
  o[4] = n > 0 ? (ey > 0 ? sqrt(ey) : 0) / n : 0;
}

cudaError_t launch_history_merge(const double *partials, int hist_passes, const int *tile_first, int n_inst,
                                 double *out, cudaStream_t stream) {
  const int total = n_inst * hist_passes;
  if (total <= 0)
    return cudaSuccess;
  history_merge_kernel<<<(total + 127) / 128, 128, 0, stream>>>(partials, hist_passes, tile_first, n_inst, out);
  return cudaGetLastError();
}

/* RFCA fiducial time (findFiducialTime, simple_rfca.c:62-257).  TMEAN:
 * Kahan-compensated mean of (s + sOffset)/(c*beta) over the particles that
 * reach the cavity on the first pass, summed in particle order.  One thread
 * per instance walks its particles sequentially so the sum is the
 * reference's serial Kahan sum, bit for bit, when no particle was lost
 * upstream on that pass (elegant's swap-to-tail would otherwise reorder the
 * survivors).  LIGHT: (zEnd - L + sOffset)/c (:97-100).  PMAXIMUM (:126-147):
 * the arrival time of the particle with the highest delta, found as the
 * reference's loop does: the first particle's delta is the starting best and
 * only a later, strictly higher one is taken, so a beam whose first particle
 * is highest has no fiducial particle (the reference stops there; here bit 2
 * of the error flag is set and the cavity stays unset). */
__global__ void rf_fiducial_kernel(DevParticles P, const int64_t *inst_offsets, int n_inst, const DevElem *elems,
                                   int n_elems, int elem_index, DevRfState *rf, int n_rf, double p_central,
                                   int64_t max_rows, unsigned int *error_flag) {
  const int inst = blockIdx.x * blockDim.x + threadIdx.x;
  if (inst >= n_inst)
    return;
  const DevElem &e = elems[(size_t)inst * n_elems + elem_index];
  const double sOffset = e.c[RF_SOFFSET];
  const int slot = (int)e.c[RF_SLOT];
  DevRfState &rs = rf[(size_t)inst * n_rf + slot];
  const int leader = (int)e.c[RF_LEADER];
  if (leader >= 0) {
    /* a later cavity of a PHASE_REFERENCE group: the group's phase
     * (REF_PHASE_RETURNED, simple_rfca.c:419-421) plus its own PHASE */
    const DevRfState &ls = rf[(size_t)inst * n_rf + leader];
    rs.phase_fiducial = ls.phase_fiducial;
    rs.phase = ls.phase_fiducial + e.c[RF_PHASE_DEG_RAD];
    rs.set = ls.set;
    return;
  }
  double tsum = 0, error = 0;
  int64_t nsum = 0;
  const int64_t first = inst_offsets[inst], end = inst_offsets[inst + 1];
  const int mode = (int)e.c[RF_FID_MODE];
  if (mode == B2E_FIDUCIAL_LIGHT) {
    tsum = ((e.z_end - e.c[RF_L_TOTAL]) + sOffset) / B2E_C_MKS;
    nsum = 1;
  } else if (mode == B2E_FIDUCIAL_PMAXIMUM) {
    double best = 0;
    int64_t ibest = -1;
    bool seen = false;
    for (int64_t ip = first; ip < end && (max_rows <= 0 || ip - first < max_rows); ip++) {
      if (P.lost_pass[ip] >= 0)
        continue;
      if (!seen) {
        best = P.dp[ip];
        seen = true;
      } else if (best < P.dp[ip]) {
        best = P.dp[ip];
        ibest = ip;
      }
    }
    if (ibest >= 0) {
      double pp = p_central * (1 + P.dp[ibest]);
      double beta = pp / sqrt(pp * pp + 1);
      tsum = (P.s[ibest] + sOffset) / (B2E_C_MKS * beta);
      nsum = 1;
    } else if (seen && e.c[RF_T_REFERENCE] == -1) {
      atomicOr(error_flag, 2u);
    }
  } else {
    for (int64_t ip = first; ip < end && (max_rows <= 0 || ip - first < max_rows); ip++) {
      if (P.lost_pass[ip] >= 0)
        continue;
      double pp = p_central * (1 + P.dp[ip]);
      double beta = pp / sqrt(pp * pp + 1); /* beta_from_delta, do_tracking.c:95 */
      double b = (P.s[ip] + sOffset) / (B2E_C_MKS * beta);
      /* KahanPlus (kahan.c:28-35) */
      double Y = b + error;
      double sum = tsum + Y;
      error = Y - (sum - tsum);
      tsum = sum;
      nsum++;
    }
  }
  if (e.c[RF_T_REFERENCE] != -1) {
    /* explicit T_REFERENCE replaces the fiducial search */
    tsum = e.c[RF_T_REFERENCE];
    nsum = 1;
  }
  if (nsum > 0) {
    const double omega = e.c[RF_OMEGA];
    double t0 = tsum / nsum;
    double phase_fiducial = -omega * t0;
    rs.phase_fiducial = phase_fiducial;
    rs.phase = phase_fiducial + e.c[RF_PHASE_DEG_RAD];
    rs.set = 1;
  } else {
    rs.set = 0;
  }
}

/* Effort (particle-passes) and survivor count from the loss columns. */
__global__ void effort_kernel(const int32_t *lost_pass, int64_t n, int pass_begin, int pass_end, unsigned long long *effort,
                              unsigned long long *survivors) {
  unsigned long long e = 0, s = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int lp = lost_pass[i];
    int alive = lp < 0 ? pass_end - pass_begin : lp - pass_begin;
    e += (unsigned long long)(alive < 0 ? 0 : (alive > pass_end - pass_begin ? pass_end - pass_begin : alive));
    s += lp < 0;
  }
  for (int off = 16; off > 0; off >>= 1) {
    e += __shfl_down_sync(0xffffffffu, e, off);
    s += __shfl_down_sync(0xffffffffu, s, off);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(effort, e);
    atomicAdd(survivors, s);
  }
}

template <int MINB, int SYNC, bool HIST, int TPB, bool RAD = false>
static cudaError_t launch_ring_v(const RingLaunch &L, int n_tiles, bool staged, size_t smem_bytes,
                                 cudaStream_t stream) {
  const int grid = (n_tiles + TPB - 1) / TPB;
  if (staged && smem_bytes * TPB > 200 * 1024)
    staged = false; /* two instances' records do not fit: read them from global memory */
  if (staged) {
    const size_t bytes = smem_bytes * TPB;
    cudaError_t err = cudaFuncSetAttribute(ring_kernel<true, MINB, SYNC, HIST, TPB, RAD>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (err != cudaSuccess)
      return err;
    ring_kernel<true, MINB, SYNC, HIST, TPB, RAD><<<grid, 128 * TPB, bytes, stream>>>(L);
  } else {
    ring_kernel<false, MINB, SYNC, HIST, TPB, RAD><<<grid, 128 * TPB, 0, stream>>>(L);
  }
  return cudaGetLastError();
}

template <int SYNC, bool HIST>
static cudaError_t launch_ring_s(const RingLaunch &L, int n_tiles, bool staged, size_t smem_bytes,
                                 cudaStream_t stream, int minb_index) {
  switch (minb_index) {
  case 1:
    return launch_ring_v<5, SYNC, HIST, 1>(L, n_tiles, staged, smem_bytes, stream);
  case 2:
    return launch_ring_v<6, SYNC, HIST, 1>(L, n_tiles, staged, smem_bytes, stream);
  case 3:
    return launch_ring_v<8, SYNC, HIST, 1>(L, n_tiles, staged, smem_bytes, stream);
  default:
    return launch_ring_v<4, SYNC, HIST, 1>(L, n_tiles, staged, smem_bytes, stream);
  }
}

template <bool HIST>
static cudaError_t launch_ring_group(const RingLaunch &L, int n_tiles, bool staged, size_t smem_bytes,
                                     cudaStream_t stream, int index) {
  switch (index) {
  case 1:
    return launch_ring_v<3, 2, HIST, 2>(L, n_tiles, staged, smem_bytes, stream);
  case 2:
    return launch_ring_v<4, 2, HIST, 2>(L, n_tiles, staged, smem_bytes, stream);
  case 3:
    return launch_ring_v<2, 2, HIST, 4>(L, n_tiles, staged, smem_bytes, stream);
  case 4:
    return launch_ring_v<1, 2, HIST, 8>(L, n_tiles, staged, smem_bytes, stream);
  default:
    return launch_ring_v<2, 2, HIST, 2>(L, n_tiles, staged, smem_bytes, stream);
  }
}

/* variant 1..12: one 128-particle tile per block, occupancy target MINB =
 * {4, 5, 6, 8}[(variant-1) % 4] blocks per SM, barrier level SYNC =
 * (variant-1) / 4 (with history at least 1).  Variants 13..17 keep several
 * tiles of a block in step with a barrier after every element: two tiles per
 * 256-thread block at {2, 3, 4} blocks per SM, four tiles per 512-thread
 * block at 2, eight tiles per 1024-thread block at 1. */
cudaError_t launch_ring(const RingLaunch &L, int n_tiles, bool staged, size_t smem_bytes, cudaStream_t stream,
                        int variant) {
  if (n_tiles <= 0)
    return cudaSuccess;
  if (L.rad) /* radiating lattices: one configuration (two tiles per block, a barrier per element) */
    return L.hist ? launch_ring_v<2, 2, true, 2, true>(L, n_tiles, staged, smem_bytes, stream)
                  : launch_ring_v<2, 2, false, 2, true>(L, n_tiles, staged, smem_bytes, stream);
  if (variant < 1 || variant > B2E_RING_VARIANTS)
    variant = 1;
  if (variant > 12)
    return L.hist ? launch_ring_group<true>(L, n_tiles, staged, smem_bytes, stream, variant - 13)
                  : launch_ring_group<false>(L, n_tiles, staged, smem_bytes, stream, variant - 13);
  const int minb_index = (variant - 1) % 4, sync = (variant - 1) / 4;
  if (L.hist)
    return sync == 2 ? launch_ring_s<2, true>(L, n_tiles, staged, smem_bytes, stream, minb_index)
                     : launch_ring_s<1, true>(L, n_tiles, staged, smem_bytes, stream, minb_index);
  switch (sync) {
  case 1:
    return launch_ring_s<1, false>(L, n_tiles, staged, smem_bytes, stream, minb_index);
  case 2:
    return launch_ring_s<2, false>(L, n_tiles, staged, smem_bytes, stream, minb_index);
  default:
    return launch_ring_s<0, false>(L, n_tiles, staged, smem_bytes, stream, minb_index);
  }
}

/* Stable partition of every instance's particles: survivors first, in their
 * order, lost particles after them (last to first).  One block per instance
 * walks its range in chunks of blockDim particles; a warp ballot gives each
 * particle its rank among its warp's survivors (or losses) and a scan over
 * the block's warp totals the chunk offsets (lost-particle compaction with
 * warp ballots and prefix sums). */
__global__ void compact_kernel(DevParticles src, const int64_t *ids_src, DevParticles dst, int64_t *ids_dst,
                               const int64_t *offs, int *alive_out) {
  __shared__ int warp_alive[32], warp_dead[32];
  __shared__ int base_alive, base_dead;
  const int inst = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int64_t first = offs[inst], end = offs[inst + 1];
  if (threadIdx.x == 0) {
    base_alive = 0;
    base_dead = 0;
  }
  __syncthreads();
  const unsigned below = (1u << lane) - 1u;
  for (int64_t c = first; c < end; c += blockDim.x) {
    const int64_t i = c + threadIdx.x;
    const bool valid = i < end;
    const bool alive = valid && src.lost_pass[i] < 0;
    const unsigned ba = __ballot_sync(0xffffffffu, alive), bd = __ballot_sync(0xffffffffu, valid && !alive);
    if (lane == 0) {
      warp_alive[warp] = __popc(ba);
      warp_dead[warp] = __popc(bd);
    }
    __syncthreads();
    int pa = 0, pd = 0, ta = 0, td = 0;
    for (int w = 0; w < nw; w++) {
      if (w < warp) {
        pa += warp_alive[w];
        pd += warp_dead[w];
      }
      ta += warp_alive[w];
      td += warp_dead[w];
    }
    if (valid) {
      const int64_t d = alive ? first + base_alive + pa + __popc(ba & below)
                              : end - 1 - (base_dead + pd + __popc(bd & below));
      dst.x[d] = src.x[i];
      dst.xp[d] = src.xp[i];
      dst.y[d] = src.y[i];
      dst.yp[d] = src.yp[i];
      dst.s[d] = src.s[i];
      dst.dp[d] = src.dp[i];
      dst.lost_pass[d] = src.lost_pass[i];
      dst.lost_elem[d] = src.lost_elem[i];
      ids_dst[d] = ids_src[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      base_alive += ta;
      base_dead += td;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    alive_out[inst] = base_alive;
}

cudaError_t launch_compact(DevParticles src, const int64_t *ids_src, DevParticles dst, int64_t *ids_dst,
                           const int64_t *offs, int n_inst, int *alive_out, cudaStream_t stream) {
  if (n_inst <= 0)
    return cudaSuccess;
  compact_kernel<<<n_inst, 1024, 0, stream>>>(src, ids_src, dst, ids_dst, offs, alive_out);
  return cudaGetLastError();
}

cudaError_t launch_fiducial(DevParticles P, const int64_t *inst_offsets, int n_inst, const DevElem *elems,
                            int n_elems, int elem_index, DevRfState *rf, int n_rf, double p_central,
                            int64_t max_rows, unsigned int *error_flag, cudaStream_t stream) {
  int tpb = 64, nb = (n_inst + tpb - 1) / tpb;
  rf_fiducial_kernel<<<nb, tpb, 0, stream>>>(P, inst_offsets, n_inst, elems, n_elems, elem_index, rf, n_rf,
                                             p_central, max_rows, error_flag);
  return cudaGetLastError();
}

__global__ void tbt_start_kernel(DevParticles P, int64_t n, double *tbt) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const bool live = P.lost_pass[i] < 0;
  tbt[i] = live ? P.x[i] : NAN;
  tbt[n + i] = live ? P.xp[i] : NAN;
  tbt[2 * n + i] = live ? P.y[i] : NAN;
  tbt[3 * n + i] = live ? P.yp[i] : NAN;
}

/* WATCH record of the particles alive at a WATCH element (the ring launches
 * stop there on its passes): x..delta and the ID as a double, NaN (left from
 * the fill) in the rows of lost particles. */
__global__ void watch_copy_kernel(DevParticles P, const int64_t *ids, int64_t n, double *out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n || P.lost_pass[i] >= 0)
    return;
  out[i] = P.x[i];
  out[n + i] = P.xp[i];
  out[2 * n + i] = P.y[i];
  out[3 * n + i] = P.yp[i];
  out[4 * n + i] = P.s[i];
  out[5 * n + i] = P.dp[i];
  out[6 * n + i] = (double)(ids ? ids[i] : i + 1);
}

cudaError_t launch_watch_copy(DevParticles P, const int64_t *ids, int64_t n, double *out, cudaStream_t stream) {
  if (n <= 0)
    return cudaSuccess;
  watch_copy_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(P, ids, n, out);
  return cudaGetLastError();
}

cudaError_t launch_tbt_start(DevParticles P, int64_t n, double *tbt, cudaStream_t stream) {
  if (n > 0)
    tbt_start_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(P, n, tbt);
  return cudaGetLastError();
}

cudaError_t launch_effort(const int32_t *lost_pass, int64_t n, int pass_begin, int pass_end, unsigned long long *effort,
                          unsigned long long *survivors, cudaStream_t stream) {
  int nb = (int)((n + 255) / 256);
  if (nb > 148 * 8)
    nb = 148 * 8;
  if (nb < 1)
    nb = 1;
  effort_kernel<<<nb, 256, 0, stream>>>(lost_pass, n, pass_begin, pass_end, effort, survivors);
  return cudaGetLastError();
}

} // namespace b2e

/* ---- division self-test (b2e_selftest_division) ------------------------- */
namespace b2e {

__global__ void division_selftest_kernel(const double *b, int nb, int64_t samples, uint64_t seed,
                                         unsigned long long *mismatches) {
  const int ib = blockIdx.y;
  const double bv = b[ib], y = 1 / bv;
  unsigned long long bad = 0;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < samples; k += (int64_t)gridDim.x * blockDim.x) {
    /* SplitMix64 of (seed, divisor, sample) -> sign, exponent, mantissa */
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (uint64_t)(k * nb + ib + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const int ex = (int)((z >> 52) % 81) - 40;
    const double m = 1.0 + (double)(z & ((1ull << 52) - 1)) * 0x1p-52;
    const double a = ldexp((z >> 63) ? -m : m, ex);
    const double q1 = a / bv, q2 = div_rn_recip(a, bv, y);
    bad += __double_as_longlong(q1) != __double_as_longlong(q2);
  }
  for (int off = 16; off > 0; off >>= 1)
    bad += __shfl_down_sync(0xffffffffu, bad, off);
  if ((threadIdx.x & 31) == 0 && bad)
    atomicAdd(mismatches, bad);
}

} // namespace b2e

extern "C" int b2e_selftest_division(const double *host_b, int32_t n_b, int64_t samples, uint64_t seed,
                                     int64_t *mismatches) {
  using namespace b2e;
  if (!host_b || n_b < 1 || n_b > 65535 || samples < 1 || !mismatches)
    return B2E_ERR_ARG;
  double *db = nullptr;
  unsigned long long *dm = nullptr, hm = 0;
  if (cudaMalloc(&db, sizeof(double) * n_b) != cudaSuccess)
    return B2E_ERR_NOMEM;
  if (cudaMalloc(&dm, sizeof(unsigned long long)) != cudaSuccess) {
    cudaFree(db);
    return B2E_ERR_NOMEM;
  }
  cudaMemcpy(db, host_b, sizeof(double) * n_b, cudaMemcpyHostToDevice);
  cudaMemset(dm, 0, sizeof(unsigned long long));
  division_selftest_kernel<<<dim3(148 * 4, n_b), 256>>>(db, n_b, samples, seed, dm);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpy(&hm, dm, sizeof(hm), cudaMemcpyDeviceToHost);
  cudaFree(db);
  cudaFree(dm);
  if (e != cudaSuccess)
    return B2E_ERR_CUDA;
  *mismatches = (int64_t)hm;
  return B2E_OK;
}
