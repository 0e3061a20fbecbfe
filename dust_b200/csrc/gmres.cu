// gmres.cu -- learned-preconditioned GMRES for the moving-body system.
// (Filled in by the learned-preconditioner component; until a trained
// network is attached to the handle the solve reports "not converged" and
// the caller falls back to plain LU.)
#include "linsys_internal.h"

int linsys_gmres_nn(dust_linsys *L, const double *Af, double *x, dust_solve_report *rep) {
  (void)L;
  (void)Af;
  (void)x;
  if (rep) rep->iterations = 0;
  return DUST_ERR_NOT_CONVERGED;
}
