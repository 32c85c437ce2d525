/*
 * CSR driver: placeholder until the collective kernels land; lattices with
 * CSR elements are rejected at load time.
 */
#include "b2e_csr.h"

namespace b2e {

int csr_configure(CsrState &st, const b2e_element *el, int n, const CompiledLattice &lat, const b2e_run_options &opt,
                  std::string &err) {
  (void)el;
  (void)n;
  (void)opt;
  st.elements = lat.csr_elements;
  st.enabled = !lat.csr_elements.empty();
  if (st.enabled) {
    err = "CSRCSBEND/CSRDRIFT are not available in this build";
    return B2E_ERR_LATTICE;
  }
  return B2E_OK;
}

void csr_reset(CsrState &st) { st.wakes_host.clear(); }

int csr_track_element(CsrState &st, const DevParticles &P, int64_t n, int elem, int pass, cudaStream_t stream,
                      std::string &err) {
  (void)st;
  (void)P;
  (void)n;
  (void)elem;
  (void)pass;
  (void)stream;
  err = "CSR elements are not available in this build";
  return B2E_ERR_LATTICE;
}

int csr_copy_wakes(CsrState &st, double *wakes, int64_t capacity, int64_t *written, std::string &err) {
  (void)err;
  int64_t k = 0;
  for (; k < (int64_t)st.wakes_host.size() && k < capacity; k++)
    wakes[k] = st.wakes_host[k];
  *written = k;
  return B2E_OK;
}

void csr_release(CsrState &st) { st.wakes_host.clear(); }

} // namespace b2e
