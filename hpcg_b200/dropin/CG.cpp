// CG.cpp (drop-in) -- the PCG driver on the GPU.
//
// Replaces src/CG.cpp (interface src/CG.hpp:22-24).  The whole solve runs in
// libhpcgx (hpcgx_cg_host): b and x are copied to the device at entry, x back
// at exit; alpha, beta and the residual norms stay on the GPU and each
// iteration is one CUDA graph.  times[0] (total), times[2] (vector ops with
// their fused dot products), times[3] (SpMV with fused p.Ap) and times[5]
// (preconditioner) are accumulated as src/CG.cpp:133-141 does; the dot
// products are fused into their producers, so times[1] gets no separate share.
#include "CG.hpp"

#include "hpcgx_dropin.hpp"

int CG(const SparseMatrix &A, CGData &data, const Vector &b, Vector &x, const int max_iter,
       const double tolerance, int &niters, double &normr, double &normr0, double *times,
       bool doPreconditioning) {
  (void)data;
  hpcgx_dropin::LevelState *s = hpcgx_dropin::state(A);
  if (!s || s->level != 0) return HPCGX_ESTATE;
  int rc = hpcgx_dropin::sync_diagonals(A);
  if (rc != HPCGX_OK) return rc;
  rc = hpcgx_cg_host(s->problem, doPreconditioning ? HPCGX_CG_MG : HPCGX_CG_PLAIN, b.values,
                     x.values, max_iter, tolerance, &niters, &normr, &normr0, times);
  return hpcgx_dropin::report(rc, "CG");
}
