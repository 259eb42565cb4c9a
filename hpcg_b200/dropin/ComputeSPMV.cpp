// ComputeSPMV.cpp (drop-in) -- replaces src/ComputeSPMV.cpp
// (interface src/ComputeSPMV.hpp:20): y = A x on the GPU, host vectors in/out.
#include "ComputeSPMV.hpp"

#include "hpcgx_dropin.hpp"

int ComputeSPMV(const SparseMatrix &A, Vector &x, Vector &y) {
  hpcgx_dropin::LevelState *s = hpcgx_dropin::state(A);
  if (!s) return HPCGX_ESTATE;
  int rc = hpcgx_dropin::sync_diagonals(A);
  if (rc != HPCGX_OK) return rc;
  return hpcgx_dropin::report(hpcgx_spmv_host(s->problem, s->level, x.values, y.values),
                              "ComputeSPMV");
}
