/*
 * Symbols referenced by the compiled elegant sources but reachable only from
 * features outside the supported hot-path subset (SDDS file output, wakes,
 * matter, apertures from files, matrix concatenation, RPN, optimisation).
 * Each one reports a fatal error through the driver's trap.  They are defined
 * without prototypes on purpose: none of them is ever expected to return.
 * Globals that elegant.c defines for the MPI build are given their serial
 * values.  Test infrastructure only.
 */
#include <stdio.h>
#include <string.h>

extern char b2e_ref_errmsg[512];
void b2e_ref_offpath(const char *name);

long isMaster = 1, isSlave = 1, notSinglePart = 0;

#define OFFPATH(name) \
  void name() { b2e_ref_offpath(#name); }

OFFPATH(INTERPOLATE)
OFFPATH(SDDS_CheckColumn)
OFFPATH(SDDS_CheckParameter)
OFFPATH(SDDS_GetColumnInDoubles)
OFFPATH(SDDS_GetColumnInLong)
OFFPATH(SDDS_GetParameterAsDouble)
OFFPATH(SDDS_GetParameterAsLong)
OFFPATH(SDDS_InitializeInputFromSearchPath)
OFFPATH(SDDS_PrintErrors)
OFFPATH(SDDS_ReadPage)
OFFPATH(SDDS_RowCount)
OFFPATH(SDDS_SetError)
OFFPATH(SDDS_SetRowValues)
OFFPATH(SDDS_Terminate)
OFFPATH(SDDS_UpdatePage)
OFFPATH(addLSCKick)
OFFPATH(bend_matrix)
OFFPATH(binaryArraySearch)
OFFPATH(concat_matrices)
OFFPATH(convertLocalCoordinatesToGlobal)
OFFPATH(copy_matrices1)
OFFPATH(do_match_energy)
OFFPATH(double_cmpasc)
OFFPATH(edge_matrix)
OFFPATH(factor)
OFFPATH(get_double)
OFFPATH(initializeApContour)
OFFPATH(interpretScraperDirection)
OFFPATH(log_and)
OFFPATH(log_or)
OFFPATH(m_add)
OFFPATH(m_alloc)
OFFPATH(m_copy)
OFFPATH(m_invert)
OFFPATH(m_mult)
OFFPATH(m_scmul)
OFFPATH(m_subtract)
OFFPATH(m_trans)
OFFPATH(m_zero)
OFFPATH(performSliceAnalysisOutput)
OFFPATH(pointIsInsideContour)
OFFPATH(pop_log)
OFFPATH(push_log)
OFFPATH(rpn)
OFFPATH(rpn_clear)
OFFPATH(simplexMin)
OFFPATH(track_through_matter)
OFFPATH(track_through_trwake)
OFFPATH(track_through_wake)

/* CSR support routines: restated in ref_csr_support.c when that file is
 * linked; these weak fallbacks keep the ring-only build linkable. */
#define OFFPATH_WEAK(name) \
  __attribute__((weak)) void name() { b2e_ref_offpath(#name); }
OFFPATH_WEAK(SavitzyGolaySmooth)
OFFPATH_WEAK(approximateBeamWidth)
OFFPATH_WEAK(compute_percentiles)
OFFPATH_WEAK(fill_double_array)
OFFPATH_WEAK(index_min_max)
OFFPATH_WEAK(interp)
OFFPATH_WEAK(rms_emittance)
OFFPATH_WEAK(zeroInterp)
OFFPATH_WEAK(zeroNewton)
