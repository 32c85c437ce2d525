/*
 * Collective CSR step (CSRCSBEND / CSRDRIFT) driver interface.
 */
#ifndef B2E_CSR_H
#define B2E_CSR_H
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "b2e_engine.h"
#include "b2e_lattice.h"

namespace b2e {

struct CsrState {
  bool enabled = false;
  std::vector<int> elements;
  std::vector<double> wakes_host;
  void *impl = nullptr; /* device buffers, owned by b2e_csr.cu */
};

int csr_configure(CsrState &st, const b2e_element *el, int n, const CompiledLattice &lat, const b2e_run_options &opt,
                  std::string &err);
void csr_reset(CsrState &st);
int csr_track_element(CsrState &st, const DevParticles &P, int64_t n, int elem, int pass, cudaStream_t stream,
                      std::string &err);
int csr_copy_wakes(CsrState &st, double *wakes, int64_t capacity, int64_t *written, std::string &err);
void csr_release(CsrState &st);

} // namespace b2e
#endif
