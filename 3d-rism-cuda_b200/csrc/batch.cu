// Batched small solutes (rism3d_solve_batch).
#include "rism3d_impl.h"

extern "C" int rism3d_solve_batch(rism3d_ctx *, int, const int *, const int *, const double *,
                                  const double *, const double *, const double *, const double *,
                                  rism3d_result *) {
  return RISM3D_BAD_STATE;
}
