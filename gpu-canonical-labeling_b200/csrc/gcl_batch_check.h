// gcl_batch_check.h -- host checks of a batch in the ragged arena layout of
// include/gcl.h (voff, eoff, local rowptrs back to back, col; output offsets
// ooff / roff), made before anything of it reaches the device.  Host code
// only; the batched entry points share it.
#pragma once
#include <algorithm>
#include <cstddef>
#include <cstdint>

#include "../../include/gcl.h"

namespace gcl {

constexpr int kBatchSmallN = 64;  // graphs up to this size take the warp kernel

struct BatchShape {
  int max_n = 0;          // largest vertex count
  int64_t max_m2 = 0;     // largest CSR size of a graph above kBatchSmallN vertices
  size_t nv = 0, ne = 0;  // vertices and CSR entries of the whole batch
  size_t nrp = 0;         // rowptr entries (nv + count)
  size_t dense_bytes = 0, rows_words = 0;  // output sizes (ooff[count], roff[count])
};

// GCL_OK with the batch's shape, or the status its batched call returns: a
// vertex count above GCL_MAX_N gives GCL_ERR_TOO_LARGE, a graph whose local
// rowptr does not run from 0 to its CSR size GCL_ERR_BAD_INPUT, every other
// inconsistency GCL_ERR_ARG; the first failing graph decides.  ooff / roff
// are checked when given (the dense and the packed-row outputs).
inline int check_batch(int count, const int64_t* voff, const int64_t* eoff,
                       const int32_t* rowptr, const int32_t* col, const int64_t* ooff,
                       const int64_t* roff, BatchShape* out) {
  BatchShape B;
  if (count <= 0) {
    *out = B;
    return count == 0 ? GCL_OK : GCL_ERR_ARG;
  }
  if (voff[0] != 0 || eoff[0] != 0) return GCL_ERR_ARG;
  // output offsets start at 0: the kernels write at out + off[g]
  if ((ooff && ooff[0] != 0) || (roff && roff[0] != 0)) return GCL_ERR_ARG;
  for (int g = 0; g < count; ++g) {
    const int64_t n = voff[g + 1] - voff[g], m = eoff[g + 1] - eoff[g];
    if (n > kBatchSmallN) B.max_m2 = std::max(B.max_m2, m);
    if (n < 0 || m < 0 || n > GCL_MAX_N) return n > GCL_MAX_N ? GCL_ERR_TOO_LARGE : GCL_ERR_ARG;
    if (rowptr[voff[g] + g] != 0 || rowptr[voff[g + 1] + g] != m) return GCL_ERR_BAD_INPUT;
    if (ooff && ooff[g + 1] - ooff[g] != n * n) return GCL_ERR_ARG;
    if (roff && roff[g + 1] - roff[g] != n * ((n + 63) / 64)) return GCL_ERR_ARG;
    B.max_n = std::max<int>(B.max_n, (int)n);
  }
  if (eoff[count] > 0 && !col) return GCL_ERR_ARG;
  B.nv = (size_t)voff[count];
  B.ne = (size_t)eoff[count];
  B.nrp = B.nv + (size_t)count;
  B.dense_bytes = ooff ? (size_t)ooff[count] : 0;
  B.rows_words = roff ? (size_t)roff[count] : 0;
  *out = B;
  return GCL_OK;
}

}  // namespace gcl
