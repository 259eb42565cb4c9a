// ComputeSYMGS.cpp (drop-in) -- replaces src/ComputeSYMGS.cpp
// (interface src/ComputeSYMGS.hpp:20): one symmetric Gauss-Seidel sweep in
// 8-colour order (forward colours 0..7, backward 7..0) on the GPU.
#include "ComputeSYMGS.hpp"

#include "hpcgx_dropin.hpp"

int ComputeSYMGS(const SparseMatrix &A, const Vector &r, Vector &x) {
  hpcgx_dropin::LevelState *s = hpcgx_dropin::state(A);
  if (!s) return HPCGX_ESTATE;
  int rc = hpcgx_dropin::sync_diagonals(A);
  if (rc != HPCGX_OK) return rc;
  return hpcgx_dropin::report(hpcgx_symgs_host(s->problem, s->level, r.values, x.values),
                              "ComputeSYMGS");
}
