/*
 * Collective CSR step (CSRCSBEND / CSRDRIFT) driver interface.
 *
 * Per CSRCSBEND kick the device runs, with no host round trip:
 *   slice   -- (previous kick's wake kick) + one integrator slice per particle
 *              + block min/max of c*t, folded into global order-preserving
 *              integer atomics (exact, order independent);
 *   bin     -- warp-aggregated shared-memory histogram of c*t (integer counts,
 *              exact) reduced into global counts;
 *   wake    -- one CTA: Savitzky-Golay smoothing, distribution correction,
 *              derivative, transient/steady T1/T2 integrals -> dGamma.
 * gpuElegant instead copies every histogram to the host and the wake back
 * (gpu_csbend.cu:3080-3140, :2689-2691).
 */
#ifndef B2E_CSR_H
#define B2E_CSR_H
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "b2e_engine.h"
#include "b2e_lattice.h"

namespace b2e {

#define B2E_CSR_MAX_BINS 4096

/* Host description of one CSR element. */
struct CsrElem {
  int index = -1;   /* lattice index */
  int kind = 0;     /* K_CSRCSBEND / K_CSRDRIFT */
  /* CSRCSBEND */
  int bins = 0, nSlices = 0, nSub = 0, sgHalf = 0, sgOrder = 1, sgdHalf = 1, sgdOrder = 1;
  int trapz = 1, steady = 0, csr = 1, same_bend_precedes = 0, bin_once = 0, igf = 0;
  double angle = 0, length = 0, rho0 = 0, binRangeFactor = 1.2, dzf = 0, z_end = 0;
  BendExtra bx = {};  /* ETILT offsets and second-order edge constants */
  /* histogram filters (applyLHPassFilters), csbend.c:2557-2562 */
  int lh = 0, clip = 1;
  double lowCut0 = -1, lowCut1 = -1, highCut0 = -1, highCut1 = -1;
  std::vector<int> sg_lo, sg_w_n, sgd_lo, sgd_w_n;   /* per bin window start and width */
  std::vector<double> sg_w, sgd_w;                    /* per bin weights, B2E_SG_MAX_WIDTH each */
  /* CSRDRIFT */
  double drift_length = 0, drift_dz = 0, z_start = 0;
  int drift_kicks = 1, drift_csr = 1, stupakov = 0;
};

struct CsrState {
  bool enabled = false;
  std::vector<CsrElem> elems;
  std::vector<double> wakes_host; /* filled on demand from the device log */
  int64_t wake_values = 0;        /* values written to the device log in this run */
  std::vector<double> macro_charge; /* per bunch: CHARGE TOTAL / its particles at pass start */
  double p_central = 0;
  double accumulated_angle = 0;
  /* bunches: contiguous particle ranges, each with its own CSR state */
  int n_bunches = 1;
  const int64_t *d_offsets = nullptr; /* [n_bunches + 1], owned by the caller */
  std::vector<unsigned char> wake_valid; /* per bunch: csrWake.valid */
  /* device buffers */
  double *d_beta0 = nullptr;
  int64_t beta0_cap = 0;
  void *d_state = nullptr;        /* CsrDevState[n_bunches] */
  unsigned int *d_counts = nullptr; /* [n_bunches][B2E_CSR_MAX_BINS] */
  double *d_csr_const = nullptr;  /* [4][n_bunches]: CSRConstant, IGF wake factor, GSConstant, macro charge */
  unsigned char *d_flags = nullptr; /* [2][n_bunches]: active, CSRDRIFT mode */
  unsigned long long *d_alive = nullptr; /* [n_bunches] */
  /* optional all-rank reduction (a bunch spread over several GPUs) */
  b2e_reduce_fn reducer = nullptr;
  void *reducer_user = nullptr;
  unsigned long long *d_keys = nullptr; /* [2][n_bunches]: gathered min, max keys */
  double *d_sg = nullptr;         /* weights of all elements, uploaded once */
  int *d_sg_idx = nullptr;
  std::vector<size_t> sg_offset;  /* per element: offset into d_sg / d_sg_idx */
  double *d_wakelog = nullptr;
  int64_t wakelog_cap = 0;
  /* optional page record of every plain-integral kick, for CSRCSBEND's
   * OUTPUT_FILE: per (kick, bunch) B2E_CSR_PAGE_HEADER values then the
   * density, its derivative, T1 and T2 over the bins */
  bool record_pages = false;
  double *d_pagelog = nullptr;
  int64_t pagelog_cap = 0, page_values = 0;
  /* optional timing of the wake stage of every CSRCSBEND kick (the plain
   * wake kernel, or the learned wake's filter + network + combine): a pair
   * of events per kick on the context's stream */
  bool time_wake = false;
  std::vector<cudaEvent_t> wake_events;
  int64_t timed_kicks = 0, timed_learned = 0;
  double ds0 = 0, zLast = 0, z0 = 0;
  double revolution_length = 0;   /* added to a CSRDRIFT's start behind the last dipole */
  /* what the last CSRCSBEND leaves for a Stupakov CSRDRIFT (csbend.c:2991-3003):
   * its entry in elems (bins, SG tables, range factor, trapezoid rule), the
   * actual bending radius and the bending angle; GSConstant is per bunch in
   * d_csr_const[2][b] */
  int last_bend = -1;
  double last_rho = 0, last_theta = 0;
  /* learned wake integral (optional): a trained wake network replaces the T1
   * integral of CSRCSBEND kicks, checked on every kick against the plain
   * integral at every gate_stride-th bin; above gate_tol relative rms error
   * of the wake the kick falls back to the plain wake */
  b2e_wakenet *net = nullptr;
  float sc_dens = 1, sc_deriv = 1, sc_target = 1;
  double gate_tol = 0.01;
  int gate_stride = 16;
  float *d_sur_in = nullptr, *d_sur_out = nullptr; /* [n_bunches][4][L], [n_bunches][L] */
  double *d_sur_tab = nullptr;                     /* [n_bunches][3][B2E_CSR_MAX_BINS] */
  double *d_sur_scal = nullptr;                    /* [n_bunches][4] */
  int64_t sur_cap_bunches = 0;
  double *d_gate_log = nullptr;                    /* one relative error per (kick, bunch) */
  int64_t gate_cap = 0, gate_values = 0;
  unsigned long long *d_sur_counts = nullptr;      /* evaluations, fallbacks */
};

int csr_configure(CsrState &st, const b2e_element *el, int n, const CompiledLattice &lat, const b2e_run_options &opt,
                  std::string &err);
void csr_reset(CsrState &st);
/* Bunch layout for the CSR step (n_bunches contiguous ranges; offsets on the
 * device, owned by the caller); allocates the per-bunch state. */
int csr_set_bunches(CsrState &st, int n_bunches, const int64_t *d_offsets, std::string &err);
/* all-rank sums of per-bunch counts (identity without a reducer) */
int csr_reduce_counts(CsrState &st, std::vector<int64_t> &counts, cudaStream_t stream, std::string &err);
/* particles alive (lost_pass < 0), per bunch */
int csr_count_alive(CsrState &st, const int32_t *lost_pass, int64_t n, std::vector<int64_t> &alive, cudaStream_t stream,
                    std::string &err);
/* alive: particles alive at the element entrance, per bunch */
int csr_track_element(CsrState &st, const DevElem *d_elems, const DevElem &h_elem, const DevParticles &P, int64_t n,
                      const std::vector<int64_t> &alive, int elem, int pass, cudaStream_t stream, std::string &err,
                      int64_t *launches);
int csr_copy_wakes(CsrState &st, double *wakes, int64_t capacity, int64_t *written, std::string &err);
int csr_copy_pages(CsrState &st, double *pages, int64_t capacity, int64_t *written, std::string &err);
/* total device time of the timed wake stages of the last run, and the kicks
 * (all, and those that took the learned wake) */
int csr_wake_timing(CsrState &st, double *ms, int64_t *kicks, int64_t *learned, std::string &err);
cudaError_t launch_post_element_sweep(const DevParticles &P, int64_t n, const DevAperture *ap, int pass, int elem,
                                      cudaStream_t stream);
void csr_release(CsrState &st);

} // namespace b2e
#endif
