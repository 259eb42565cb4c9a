// GenerateProblem.cpp (drop-in) -- replaces src/GenerateProblem.cpp.
//
// Builds exactly the data structures GenerateProblem_ref builds
// (src/GenerateProblem_ref.cpp:50-219; CheckProblem verifies them), but fills
// the rows in parallel without a critical section per row: the reference
// serialises every row on `omp critical` for its global-to-local map and its
// nonzero counter (:141-143, :174-176) and allocates row arrays in serial
// loops, which made problem set-up (times[9], charged per CG set by the rating
// at src/ReportResults.cpp:353) cost far more than the solves.  Here the
// counter is an OpenMP reduction, row arrays are allocated inside the
// parallel loop (or as one block each under HPCG_CONTIGUOUS_ARRAYS), and the
// global-to-local map is filled afterwards in one reserved pass.
#ifndef HPCG_NO_MPI
#include <mpi.h>
#endif
#ifndef HPCG_NO_OPENMP
#include <omp.h>
#endif

#include <cassert>

#include "GenerateProblem.hpp"
#include "hpcgx_dropin.hpp"

void GenerateProblem(SparseMatrix &A, Vector *b, Vector *x, Vector *xexact) {
  // the CUDA context is made on another thread while the host builds the rows
  hpcgx_dropin::start_device_init();
  const global_int_t nx = A.geom->nx, ny = A.geom->ny, nz = A.geom->nz;
  const global_int_t gnx = A.geom->gnx, gny = A.geom->gny, gnz = A.geom->gnz;
  const global_int_t gix0 = A.geom->gix0, giy0 = A.geom->giy0, giz0 = A.geom->giz0;
  const local_int_t n = nx * ny * nz;
  assert(n > 0);
  const int perRow = 27;
  const global_int_t totalNumberOfRows = gnx * gny * gnz;
  assert(totalNumberOfRows > 0);

  char *nonzerosInRow = new char[n];
  global_int_t **mtxIndG = new global_int_t *[n];
  local_int_t **mtxIndL = new local_int_t *[n];
  double **matrixValues = new double *[n];
  double **matrixDiagonal = new double *[n];
  if (b) InitializeVector(*b, n);
  if (x) InitializeVector(*x, n);
  if (xexact) InitializeVector(*xexact, n);
  double *bv = b ? b->values : 0;
  double *xv = x ? x->values : 0;
  double *xexactv = xexact ? xexact->values : 0;
  A.localToGlobalMap.resize(n);

#ifdef HPCG_CONTIGUOUS_ARRAYS
  local_int_t *blockL = new local_int_t[(size_t)n * perRow];
  double *blockV = new double[(size_t)n * perRow];
  global_int_t *blockG = new global_int_t[(size_t)n * perRow];
#endif

  long long nnzTotal = 0;
#ifndef HPCG_NO_OPENMP
#pragma omp parallel for reduction(+ : nnzTotal) schedule(static)
#endif
  for (local_int_t iz = 0; iz < nz; iz++) {
    const global_int_t giz = giz0 + iz;
    for (local_int_t iy = 0; iy < ny; iy++) {
      const global_int_t giy = giy0 + iy;
      for (local_int_t ix = 0; ix < nx; ix++) {
        const global_int_t gix = gix0 + ix;
        const local_int_t row = iz * nx * ny + iy * nx + ix;
        const global_int_t grow = giz * gnx * gny + giy * gnx + gix;
#ifdef HPCG_CONTIGUOUS_ARRAYS
        mtxIndL[row] = blockL + (size_t)row * perRow;
        matrixValues[row] = blockV + (size_t)row * perRow;
        mtxIndG[row] = blockG + (size_t)row * perRow;
#else
        mtxIndL[row] = new local_int_t[perRow];
        matrixValues[row] = new double[perRow];
        mtxIndG[row] = new global_int_t[perRow];
#endif
        A.localToGlobalMap[row] = grow;
        char k = 0;
        double *v = matrixValues[row];
        global_int_t *g = mtxIndG[row];
        for (int sz = -1; sz <= 1; sz++) {
          if (giz + sz < 0 || giz + sz >= gnz) continue;
          for (int sy = -1; sy <= 1; sy++) {
            if (giy + sy < 0 || giy + sy >= gny) continue;
            for (int sx = -1; sx <= 1; sx++) {
              if (gix + sx < 0 || gix + sx >= gnx) continue;
              const global_int_t col = grow + sz * gnx * gny + sy * gnx + sx;
              if (col == grow) {
                matrixDiagonal[row] = v;
                *v++ = 26.0;
              } else {
                *v++ = -1.0;
              }
              *g++ = col;
              k++;
            }
          }
        }
        nonzerosInRow[row] = k;
        nnzTotal += k;
        if (bv) bv[row] = 26.0 - ((double)(k - 1));
        if (xv) xv[row] = 0.0;
        if (xexactv) xexactv[row] = 1.0;
      }
    }
  }
  A.globalToLocalMap.reserve(n);
  for (local_int_t row = 0; row < n; row++) A.globalToLocalMap[A.localToGlobalMap[row]] = row;

  global_int_t totalNumberOfNonzeros = 0;
#ifndef HPCG_NO_MPI
  long long lnnz = nnzTotal, gnnz = 0;
  MPI_Allreduce(&lnnz, &gnnz, 1, MPI_LONG_LONG_INT, MPI_SUM, MPI_COMM_WORLD);
  totalNumberOfNonzeros = gnnz;
#else
  totalNumberOfNonzeros = nnzTotal;
#endif
  assert(totalNumberOfNonzeros > 0);

  A.title = 0;
  A.totalNumberOfRows = totalNumberOfRows;
  A.totalNumberOfNonzeros = totalNumberOfNonzeros;
  A.localNumberOfRows = n;
  A.localNumberOfColumns = n;
  A.localNumberOfNonzeros = (local_int_t)nnzTotal;
  A.nonzerosInRow = nonzerosInRow;
  A.mtxIndG = mtxIndG;
  A.mtxIndL = mtxIndL;
  A.matrixValues = matrixValues;
  A.matrixDiagonal = matrixDiagonal;
}
