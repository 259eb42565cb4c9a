// general.cuh -- the reference operators on a general sparse matrix.
//
// The stencil layout of common.cuh serves HPCG's own 27-point matrix.  The
// reference's rules ask more of an implementation: "any code must work for
// general unstructured sparse matrices" (src/GenerateProblem.cpp:47-49,
// src/SetupHalo.cpp:45).  A general problem holds each multigrid level as it
// is given -- any pattern, any number of entries per row, any injection
// operator f2c -- and runs the reference's operators on it:
//   * OptimizeProblem's greedy multicolouring computed from the matrix graph
//     (src/OptimizeProblem.cpp:50-79), rows stored colour-major (natural
//     order inside a colour);
//   * sliced ELL over the stored rows: 32-row slices, each as wide as its
//     longest row, entries kept in the row's own order with stored int32
//     columns, so every row sum rounds as the reference's;
//   * SpMV (src/ComputeSPMV_ref.cpp:58-71), SYMGS in colour order -- one
//     launch per colour and direction (src/ComputeSYMGS_ref.cpp:67-100 on
//     the colour-permuted matrix) --, ComputeMG_ref's V-cycle
//     (src/ComputeMG_ref.cpp:39-63) with restriction and prolongation through
//     the given f2c, and CG (src/CG.cpp:76-130) as one CUDA graph per
//     iteration.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hpcgx {

struct GeneralProblem;

// nlev levels on the current device, work on stream s.
GeneralProblem *general_create(int nlev, cudaStream_t s);
void general_destroy(GeneralProblem *g);
void general_set_stream(GeneralProblem *g, cudaStream_t s);
// Loads level `level` from host rows (nnz[i] entries of row i in cols[i] /
// vals[i]) and, for every level but the last, the injection to the next
// level (f2c[i] = fine row of coarse row i, nc coarse rows).  Returns an
// HPCGX_* status; *msg explains a rejected matrix.
int general_load_level(GeneralProblem *g, int level, int64_t n, const char *nnz,
                       const int32_t *const *cols, const double *const *vals, const int32_t *f2c,
                       int64_t nc, const char **msg);
int64_t general_rows(const GeneralProblem *g, int level);
int general_colours(const GeneralProblem *g, int level);
bool general_ready(const GeneralProblem *g);
double general_bytes(const GeneralProblem *g);
int64_t general_launches(const GeneralProblem *g);
// Device vectors in natural row order.
int general_spmv(GeneralProblem *g, int level, const double *x, double *y);
int general_symgs(GeneralProblem *g, int level, const double *r, double *x);
int general_mg(GeneralProblem *g, const double *r, double *x);
// CG on device vectors b, x (x: initial guess in, solution out); times as
// hpcgx_cg.  Returns HPCGX_ENONFINITE when a residual norm is not finite.
int general_cg(GeneralProblem *g, const double *b, double *x, int max_iter, double tol,
               int precond, int *niters, double *normr, double *normr0, double *times);
// Diagonal of a level in natural row order, host memory.
int general_set_diagonal(GeneralProblem *g, int level, const double *diag);
int general_get_diagonal(GeneralProblem *g, int level, double *diag);

}  // namespace hpcgx
