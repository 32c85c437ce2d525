/*
 * Host helpers that build TMA tensor maps for BF16 row tensors with 64
 * values (128 bytes) per row and the 128-byte swizzle.  The driver entry
 * point is fetched through the runtime, so the library does not link libcuda.
 */
#ifndef B2E_TMAP_H
#define B2E_TMAP_H
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace b2e {

/* rows of 64 BF16 values; dims: [n_outer][n_rows][64]; box: [box_rows][64].
 * Out-of-range rows of a box read as zero. */
cudaError_t make_tmap_rows64(CUtensorMap *map, const void *base, int64_t n_rows, int64_t n_outer, int box_rows);

} // namespace b2e
#endif
