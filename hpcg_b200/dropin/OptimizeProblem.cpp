// OptimizeProblem.cpp (drop-in) -- builds the device layout of every level.
//
// Replaces src/OptimizeProblem.cpp (interface src/OptimizeProblem.hpp:22,28).
// Each level's rows (nonzerosInRow / mtxIndL / matrixValues) are uploaded into
// libhpcgx's colour-sorted sliced-ELL layout; the multicolouring is the
// 8-colour (ix, iy, iz parity) colouring that the reference's greedy
// colouring (src/OptimizeProblem.cpp:43-96) produces on this stencil.  The
// injection operators are checked against the geometric injection the
// kernels use.  The time spent here is charged by the driver to times[7].
#include "OptimizeProblem.hpp"

#include <cstdlib>
#include <fstream>

#include "hpcg.hpp"
#include "hpcgx_dropin.hpp"

namespace {

void release_at_exit() {
  hpcgx_problem *p = hpcgx_dropin::current();
  if (p) hpcgx_destroy(p);
  hpcgx_dropin::set_current(nullptr);
}

}  // namespace

int OptimizeProblem(SparseMatrix &A, CGData &data, Vector &b, Vector &x, Vector &xexact) {
  (void)data;
  (void)b;
  (void)x;
  (void)xexact;
  if (A.geom->size != 1) {
    HPCG_fout << "OptimizeProblem: the hpcgx drop-in runs one process per problem" << std::endl;
    return HPCGX_EINVAL;
  }
  int levels = 1;
  for (const SparseMatrix *m = &A; m->mgData; m = m->Ac) ++levels;
  const char *dev = std::getenv("HPCGX_DEVICE");
  hpcgx_problem *p = nullptr;
  int rc = hpcgx_create(dev ? std::atoi(dev) : 0, A.geom->nx, A.geom->ny, A.geom->nz, levels, &p);
  if (rc != HPCGX_OK) return hpcgx_dropin::report(rc, "OptimizeProblem: hpcgx_create");
  int level = 0;
  for (SparseMatrix *m = &A; m; m = m->Ac, ++level) {
    rc = hpcgx_load_level_rows(p, level, m->nonzerosInRow, m->mtxIndL, m->matrixValues);
    if (rc != HPCGX_OK) return hpcgx_dropin::report(rc, "OptimizeProblem: hpcgx_load_level_rows");
    if (m->mgData) {
      rc = hpcgx_check_f2c(p, level, m->mgData->f2cOperator, m->mgData->rc->localLength);
      if (rc != HPCGX_OK) return hpcgx_dropin::report(rc, "OptimizeProblem: hpcgx_check_f2c");
    }
    hpcgx_dropin::LevelState *s = new hpcgx_dropin::LevelState;
    s->problem = p;
    s->level = level;
    s->diagonal.resize(m->localNumberOfRows);
    for (local_int_t i = 0; i < m->localNumberOfRows; ++i) s->diagonal[i] = *m->matrixDiagonal[i];
    m->optimizationData = s;
  }
  if (!hpcgx_dropin::current()) std::atexit(release_at_exit);
  else hpcgx_destroy(hpcgx_dropin::current());
  hpcgx_dropin::set_current(p);
  return 0;
}

double OptimizeProblemMemoryUse(const SparseMatrix &A) {
  hpcgx_dropin::LevelState *s = hpcgx_dropin::state(A);
  double bytes = 0.0;
  if (s) hpcgx_memory_bytes(s->problem, &bytes);
  return bytes;
}
