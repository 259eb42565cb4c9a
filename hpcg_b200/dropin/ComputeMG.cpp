// ComputeMG.cpp (drop-in) -- replaces src/ComputeMG.cpp
// (interface src/ComputeMG.hpp:20): the whole V-cycle of src/ComputeMG_ref.cpp
// runs on the GPU with restriction and prolongation fused into the smoother
// sweeps.  Only the finest level is an entry point, as in the driver.
#include "ComputeMG.hpp"

#include "hpcgx_dropin.hpp"

int ComputeMG(const SparseMatrix &A, const Vector &r, Vector &x) {
  hpcgx_dropin::LevelState *s = hpcgx_dropin::state(A);
  if (!s || s->level != 0) return HPCGX_ESTATE;
  int rc = hpcgx_dropin::sync_diagonals(A);
  if (rc != HPCGX_OK) return rc;
  return hpcgx_dropin::report(hpcgx_mg_host(s->problem, r.values, x.values), "ComputeMG");
}
