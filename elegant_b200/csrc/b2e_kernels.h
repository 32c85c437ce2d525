/*
 * Launch interfaces of the tracking kernels (b2e_ring.cu) used by the host
 * orchestration (b2e_capi.cu).
 */
#ifndef B2E_KERNELS_H
#define B2E_KERNELS_H
#include <cuda_runtime.h>
#include "b2e_engine.h"

namespace b2e {

struct RingLaunch {
  DevParticles P;
  const DevTile *tiles;
  const DevElem *elems;     /* [n_inst][n_elems] */
  const DevAperture *aps;   /* [n_inst][n_aps] */
  const DevRfState *rf;     /* [n_inst][n_rf] */
  int n_elems, n_aps, n_rf;
  int n_tiles;
  int pass_begin, elem_begin; /* first (pass, element) tracked */
  int pass_end, elem_end;     /* last pass tracked, and one past its last element */
  DevGlobals g;
  unsigned int *error_flag;
  double *hist;    /* per (tile, pass) moments [n_tiles][hist_passes][11], or null */
  int hist_pass0;  /* absolute pass of hist's first slot */
  int hist_passes;
  /* radiation (SYNCH_RAD / ISR elements present): the kernel with the
   * radiation code; ISR deviates are addressed by particle ID (ids, or the
   * row number + 1 without IDs), pass, element, slice and step */
  int rad;
  const DevRad *rads;       /* [n_inst][n_elems] */
  const int64_t *ids;
  uint64_t isr_seed;
  double sr_limit;
  /* turn-by-turn record [records][4][tbt_rows]: after each full pass p,
   * record p - tbt_pass0 + 1 < tbt_records gets x, x', y, y' of live rows */
  double *tbt;
  int tbt_pass0, tbt_records;
  int64_t tbt_rows;
};

/* variant 1..B2E_RING_VARIANTS selects the occupancy target and the barrier
 * level of the ring kernel (see launch_ring in b2e_ring.cu). */
cudaError_t launch_ring(const RingLaunch &L, int n_tiles, bool staged, size_t smem_bytes, cudaStream_t stream,
                        int variant);
/* survivors of every instance moved to the front of its range (src -> dst);
 * alive_out[inst] = survivors */
cudaError_t launch_compact(DevParticles src, const int64_t *ids_src, DevParticles dst, int64_t *ids_dst,
                           const int64_t *offs, int n_inst, int *alive_out, cudaStream_t stream);
cudaError_t launch_fiducial(DevParticles P, const int64_t *inst_offsets, int n_inst, const DevElem *elems,
                            int n_elems, int elem_index, DevRfState *rf, int n_rf, double p_central,
                            int64_t max_rows, unsigned int *error_flag, cudaStream_t stream);
/* one WATCH record [7][n]: x..delta and ID (double) of the live rows */
cudaError_t launch_watch_copy(DevParticles P, const int64_t *ids, int64_t n, double *out, cudaStream_t stream);
/* turn-by-turn record 0: x, x', y, y' of every row */
cudaError_t launch_tbt_start(DevParticles P, int64_t n, double *tbt, cudaStream_t stream);
/* NAFF (b2e_naff.cu): signals [n_signals][N] -> frequency, amplitude, phase */
cudaError_t launch_naff(const double *sig, int64_t n_signals, int N, double *freq, double *amp, double *phase,
                        cudaStream_t stream);
/* tunes of records [first, first + N) of turn-by-turn data [records][4][rows]:
 * scratch [4][3][rows], bad [rows] (zeroed by the caller), nu [4][rows] =
 * nux, nuy, ax, ay */
cudaError_t launch_tbt_tunes(const double *tbt, int64_t rows, int first, int N, double *scratch, int *bad,
                             double *nu, cudaStream_t stream);
cudaError_t launch_history_merge(const double *partials, int hist_passes, const int *tile_first, int n_inst,
                                 double *out, cudaStream_t stream);
cudaError_t launch_effort(const int32_t *lost_pass, int64_t n, int pass_begin, int pass_end, unsigned long long *effort,
                          unsigned long long *survivors, cudaStream_t stream);

} // namespace b2e
#endif
