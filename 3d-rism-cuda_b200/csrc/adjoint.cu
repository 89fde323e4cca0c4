// Adjoint gradients of mu_ex (see compute_adjoint).
#include "rism3d_impl.h"

namespace rism3d {

int compute_adjoint(Context &c, double *, double *, double *, double *) {
  c.err = "adjoint gradients are not built yet";
  return RISM3D_BAD_STATE;
}

}  // namespace rism3d
