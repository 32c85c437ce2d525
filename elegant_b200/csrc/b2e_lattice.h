/*
 * Host-side lattice compilation: b2e_element (elegant parameter names and
 * defaults) -> DevElem records with every per-element constant precomputed,
 * evaluated with the same expressions as the reference's per-call setup:
 *   KQUAD/KSEXT  multipole_tracking2      multipole.c:759-1017
 *   CSBEND       track_through_csbend     csbend.c:865-1138
 *   RFCA         trackRfCavityWithWakes   simple_rfca.c:384-508
 *   MAXAMP       do_tracking.c:1848-1858, setupMultApertureData multipole.c:1725
 *   DRIF         drift_matrix             compute_matrices.c:391-412
 * Elementary functions (sin, cos, tan) go through b2e_math.h so host
 * constants and device arithmetic agree with the oracle built the same way.
 */
#ifndef B2E_LATTICE_H
#define B2E_LATTICE_H
#include <string>
#include <vector>
#include "b2e_engine.h"

namespace b2e {

/* Defaults of elegant's parameter tables for the supported types. */
void element_defaults(int type, double *p);

struct CompiledLattice {
  std::vector<DevElem> elems;
  std::vector<DevRad> rads;        /* radiation constants, parallel to elems */
  std::vector<DevAperture> aps;
  std::vector<int> rf_elements;    /* element indices of RFCA, in lattice order */
  std::vector<int> csr_elements;   /* CSRCSBEND / CSRDRIFT indices */
  std::vector<int> watch_elements; /* recording WATCH indices, in lattice order (WA_ORDINAL) */
  int n_rf = 0;
  double total_length = 0;
};

/* One standalone CSRCSBEND -> DevElem; nullptr on success, else a message. */
const char *compile_single_csr_bend(const b2e_element &el, DevElem &d, BendExtra &bx);

/* Returns an empty string on success, else a description of the problem. */
std::string compile_lattice(const b2e_element *elements, int n, const b2e_run_options &opt, CompiledLattice &out);

} // namespace b2e

#endif
