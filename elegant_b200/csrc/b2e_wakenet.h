/*
 * Wake network: kernel launch interfaces (b2e_wakenet.cu) used by the C-ABI
 * context in the same file.
 */
#ifndef B2E_WAKENET_H
#define B2E_WAKENET_H
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "elegant_b200.h"

namespace b2e {

constexpr int WN_LAYERS = 6;
constexpr int WN_CH = 64;
constexpr int WN_TAPS = 5;
constexpr int WN_IN = 4; /* density, derivative, slippage code, density shifted by the slippage */
constexpr int WN_WSIZE = WN_TAPS * WN_CH * WN_CH;          /* weights of one layer */
constexpr int WN_NPARAM = WN_LAYERS * (WN_WSIZE + WN_CH);  /* weights then biases */
constexpr int WN_STAGES = 4;                               /* operand stages of the conv kernel */

enum ConvEpilogue { EPI_HIDDEN = 0, EPI_OUTPUT = 1, EPI_BWD = 2 };

struct ConvArgs {
  int L;        /* bins per profile, a multiple of 128 */
  int n_prof;   /* profiles in the batch */
  int dilation;
  int sign;     /* +1: tap t reads bin i + (t-2) d; -1: bin i - (t-2) d (transposed conv) */
  const float *bias;             /* EPI_HIDDEN / EPI_OUTPUT: [64] */
  __nv_bfloat16 *z_out;          /* EPI_HIDDEN: pre-activation (may be null) */
  __nv_bfloat16 *a_out;          /* EPI_HIDDEN: GELU(z); EPI_BWD: gradient of the previous pre-activation */
  const __nv_bfloat16 *z_prev;   /* EPI_BWD: pre-activation of the previous layer */
  float *y_out;                  /* EPI_OUTPUT: channel 0, [n_prof * L] */
  unsigned int *status;
};

struct WgradArgs {
  int L, n_prof, dilation;
  float *partial; /* [gridDim.x][5][64 ci][64 co] */
  unsigned int *status;
};

/* Inference on device buffers without a host synchronisation (the status
 * word is read by wakenet_take_status).  B2E_ERR_ARG if the batch or the bin
 * count does not fit the network. */
int wakenet_infer(b2e_wakenet *net, const float *dev_inputs, int n_prof, float *dev_out, cudaStream_t s);
int wakenet_bins(const b2e_wakenet *net);
int wakenet_max_batch(const b2e_wakenet *net);
/* status word of the network's kernels (nonzero: a bounded wait gave up), then cleared */
unsigned int wakenet_take_status(b2e_wakenet *net, cudaStream_t s);

cudaError_t launch_conv(int epi, const CUtensorMap &t_in, const CUtensorMap &t_w, const ConvArgs &a, int grid,
                        cudaStream_t s);
cudaError_t launch_wgrad(const CUtensorMap &t_in, const CUtensorMap &t_dz, const WgradArgs &a, int grid,
                         cudaStream_t s);

} // namespace b2e
#endif
