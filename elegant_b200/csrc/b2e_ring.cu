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



/* MINB is the occupancy target (blocks of 128 threads per SM) handed to the
 * register allocator: 4 keeps every value in registers (~116 registers),
 * 5/6/8 trade a few spills to L1 for more resident warps to hide FP64
 * latency.  The arithmetic is identical in every variant. */
template <bool STAGED, int MINB>
__global__ void __launch_bounds__(128, MINB) ring_kernel(RingLaunch L) {
  extern __shared__ __align__(16) unsigned char smem[];
  const DevTile tile = L.tiles[blockIdx.x];
  const DevElem *elems = L.elems + (size_t)tile.inst * L.n_elems;
  const DevAperture *aps = L.aps + (size_t)tile.inst * L.n_aps;
  const DevRfState *rf = L.rf + (size_t)tile.inst * L.n_rf;

  if (STAGED) {
    /* stage this instance's element and aperture records in shared memory */
    DevElem *se = reinterpret_cast<DevElem *>(smem);
    DevAperture *sa = reinterpret_cast<DevAperture *>(smem + sizeof(DevElem) * L.n_elems);
    const int nw_e = (int)(sizeof(DevElem) * L.n_elems / 8), nw_a = (int)(sizeof(DevAperture) * L.n_aps / 8);
    const double *src_e = reinterpret_cast<const double *>(elems);
    const double *src_a = reinterpret_cast<const double *>(aps);
    double *dst_e = reinterpret_cast<double *>(se), *dst_a = reinterpret_cast<double *>(sa);
    for (int i = threadIdx.x; i < nw_e; i += blockDim.x)
      dst_e[i] = src_e[i];
    for (int i = threadIdx.x; i < nw_a; i += blockDim.x)
      dst_a[i] = src_a[i];
    __syncthreads();
    elems = se;
    aps = sa;
  }

  if ((int)threadIdx.x >= tile.count)
    return;
  const int64_t ip = tile.start + threadIdx.x;
  if (L.P.lost_pass[ip] >= 0)
    return;

  Part p;
  p.x = L.P.x[ip];
  p.xp = L.P.xp[ip];
  p.y = L.P.y[ip];
  p.yp = L.P.yp[ip];
  p.s = L.P.s[ip];
  p.dp = L.P.dp[ip];

  int lost = LOSS_NONE, lost_pass = -1, lost_elem = -1;
  for (int pass = L.pass_begin; pass <= L.pass_end && !lost; pass++) {
    const int e0 = pass == L.pass_begin ? L.elem_begin : 0;
    const int e1 = pass == L.pass_end ? L.elem_end : L.n_elems;
    for (int ie = e0; ie < e1; ie++) {
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
        lost = kmult(p, e, ap, L.g);
        break;
      case K_CSBEND:
        lost = csbend(p, e, ap, L.g);
        break;
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
      default:
        break;
      }
      if (!lost && !(e.flags & EF_NO_APERTURE) && ap && !maxamp_ok(p, *ap))
        lost = LOSS_APERTURE;
      if (!lost && !finite_xy(p))
        lost = LOSS_NAN;
      if (lost) {
        lost_pass = pass;
        lost_elem = ie;
        break;
      }
    }
  }

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

/* RFCA fiducial time, TMEAN mode (findFiducialTime, simple_rfca.c:177-230):
 * Kahan-compensated mean of (s + sOffset)/(c*beta) over the particles that
 * reach the cavity on the first pass, summed in particle order.  One thread
 * per instance walks its particles sequentially so the sum is the
 * reference's serial Kahan sum, bit for bit, when no particle was lost
 * upstream on that pass (elegant's swap-to-tail would otherwise reorder the
 * survivors). */
__global__ void rf_fiducial_kernel(DevParticles P, const int64_t *inst_offsets, int n_inst, const DevElem *elems,
                                   int n_elems, int elem_index, DevRfState *rf, int n_rf, double p_central) {
  const int inst = blockIdx.x * blockDim.x + threadIdx.x;
  if (inst >= n_inst)
    return;
  const DevElem &e = elems[(size_t)inst * n_elems + elem_index];
  const double sOffset = e.c[RF_SOFFSET];
  const int slot = (int)e.c[RF_SLOT];
  DevRfState &rs = rf[(size_t)inst * n_rf + slot];
  double tsum = 0, error = 0;
  int64_t nsum = 0;
  for (int64_t ip = inst_offsets[inst]; ip < inst_offsets[inst + 1]; ip++) {
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
  if (e.c[RF_T_REFERENCE] != -1) {
    /* explicit T_REFERENCE replaces the fiducial search */
    tsum = e.c[RF_T_REFERENCE];
    nsum = 1;
  }
  if (nsum > 0) {
    const double omega = e.c[RF_OMEGA];
    double t0 = tsum / nsum;
    double phase_fiducial = -omega * t0;
    rs.t0 = -phase_fiducial / omega;
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

template <int MINB>
static cudaError_t launch_ring_v(const RingLaunch &L, int n_tiles, bool staged, size_t smem_bytes,
                                 cudaStream_t stream) {
  if (staged) {
    cudaError_t err = cudaFuncSetAttribute(ring_kernel<true, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem_bytes);
    if (err != cudaSuccess)
      return err;
    ring_kernel<true, MINB><<<n_tiles, 128, smem_bytes, stream>>>(L);
  } else {
    ring_kernel<false, MINB><<<n_tiles, 128, 0, stream>>>(L);
  }
  return cudaGetLastError();
}

cudaError_t launch_ring(const RingLaunch &L, int n_tiles, bool staged, size_t smem_bytes, cudaStream_t stream,
                        int variant) {
  if (n_tiles <= 0)
    return cudaSuccess;
  switch (variant) {
  case 2:
    return launch_ring_v<5>(L, n_tiles, staged, smem_bytes, stream);
  case 3:
    return launch_ring_v<6>(L, n_tiles, staged, smem_bytes, stream);
  case 4:
    return launch_ring_v<8>(L, n_tiles, staged, smem_bytes, stream);
  default:
    return launch_ring_v<4>(L, n_tiles, staged, smem_bytes, stream);
  }
}

cudaError_t launch_fiducial(DevParticles P, const int64_t *inst_offsets, int n_inst, const DevElem *elems,
                            int n_elems, int elem_index, DevRfState *rf, int n_rf, double p_central,
                            cudaStream_t stream) {
  int tpb = 64, nb = (n_inst + tpb - 1) / tpb;
  rf_fiducial_kernel<<<nb, tpb, 0, stream>>>(P, inst_offsets, n_inst, elems, n_elems, elem_index, rf, n_rf,
                                             p_central);
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
