// ref_shim.cpp -- C entry points over the reference's own HPCG code.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile together with the
// reference's sources (read in place, never copied) into oracle/_ref/.  It
// lets tests/ pin the C restatement in hpcg_oracle.c against the real
// reference functions, generate golden vectors, and time the reference's CPU
// path (CG_ref) for bench.py's CPU baseline.  Nothing in the product links it.
//
// Problem set-up follows the reference driver (src/main.cpp:116-159):
// GenerateGeometry, GenerateProblem, SetupHalo, three GenerateCoarseProblem
// calls and CheckProblem on every level.
#include <cstdint>
#include <cstring>
#include <fstream>
#include <vector>

#include "CG_ref.hpp"
#include "CGData.hpp"
#include "CheckProblem.hpp"
#include "ComputeDotProduct_ref.hpp"
#include "ComputeMG_ref.hpp"
#include "ComputeProlongation_ref.hpp"
#include "ComputeResidual.hpp"
#include "ComputeRestriction_ref.hpp"
#include "ComputeSPMV_ref.hpp"
#include "ComputeSYMGS_ref.hpp"
#include "ComputeWAXPBY_ref.hpp"
#include "GenerateCoarseProblem.hpp"
#include "GenerateGeometry.hpp"
#include "GenerateProblem.hpp"
#include "SetupHalo.hpp"
#include "SparseMatrix.hpp"
#include "Vector.hpp"
#include "hpcg.hpp"
#include "mytimer.hpp"

// The reference declares this log stream in hpcg.hpp and defines it in
// init.cpp, which the shim does not link; it stays closed (writes are dropped).
std::ofstream HPCG_fout;

namespace {

const int kLevels = 4;  // src/main.cpp:139

struct RefProblem {
  int nlev = kLevels;     // levels built (fewer for grids that do not coarsen 3 times)
  Geometry *geom = nullptr;
  SparseMatrix A;
  Vector b, x, xexact;
  CGData data;
  SparseMatrix *level[kLevels] = {};
  // colour-permuted copy of the hierarchy (built on demand)
  std::vector<SparseMatrix *> perm;
  std::vector<std::vector<local_int_t>> pos;  // natural row -> permuted row
};

Vector view(double *p, local_int_t n) {
  Vector v;
  v.localLength = n;
  v.values = p;
  v.optimizationData = nullptr;
  return v;
}

// Builds P A P^T for one level: row pos[i] of the copy is row i of A with its
// entries kept in order and their columns renumbered; the diagonal pointer
// follows its entry.
SparseMatrix *permuted_copy(const SparseMatrix &A, const std::vector<local_int_t> &pos) {
  const local_int_t n = A.localNumberOfRows;
  SparseMatrix *P = new SparseMatrix;
  InitializeSparseMatrix(*P, A.geom);
  P->totalNumberOfRows = A.totalNumberOfRows;
  P->totalNumberOfNonzeros = A.totalNumberOfNonzeros;
  P->localNumberOfRows = n;
  P->localNumberOfColumns = A.localNumberOfColumns;
  P->localNumberOfNonzeros = A.localNumberOfNonzeros;
  P->nonzerosInRow = new char[n];
  P->mtxIndL = new local_int_t *[n];
  P->mtxIndG = new global_int_t *[n];
  P->matrixValues = new double *[n];
  P->matrixDiagonal = new double *[n];
  for (local_int_t i = 0; i < n; i++) {
    local_int_t k = pos[i];
    int nz = A.nonzerosInRow[i];
    P->nonzerosInRow[k] = (char)nz;
    P->mtxIndL[k] = new local_int_t[27];
    P->mtxIndG[k] = new global_int_t[27];
    P->matrixValues[k] = new double[27];
    for (int j = 0; j < nz; j++) {
      P->mtxIndL[k][j] = pos[A.mtxIndL[i][j]];
      P->mtxIndG[k][j] = pos[A.mtxIndL[i][j]];
      P->matrixValues[k][j] = A.matrixValues[i][j];
      if (&A.matrixValues[i][j] == A.matrixDiagonal[i]) P->matrixDiagonal[k] = &P->matrixValues[k][j];
    }
  }
  return P;
}

void free_permuted(SparseMatrix *P) {
  for (local_int_t i = 0; i < P->localNumberOfRows; i++) {
    delete[] P->mtxIndL[i];
    delete[] P->mtxIndG[i];
    delete[] P->matrixValues[i];
  }
  delete[] P->nonzerosInRow;
  delete[] P->mtxIndL;
  delete[] P->mtxIndG;
  delete[] P->matrixValues;
  delete[] P->matrixDiagonal;
  if (P->mgData) {
    delete[] P->mgData->f2cOperator;
    DeleteVector(*P->mgData->rc);
    DeleteVector(*P->mgData->xc);
    DeleteVector(*P->mgData->Axf);
    delete P->mgData->rc;
    delete P->mgData->xc;
    delete P->mgData->Axf;
    delete P->mgData;
  }
  delete P;
}

}  // namespace

extern "C" {

// The reference's set-up with `levels` multigrid levels (1..4): every level but
// the last must have even dimensions (GenerateCoarseProblem asserts it).
void *ref_create_levels(int nx, int ny, int nz, int levels) {
  if (levels < 1 || levels > kLevels) return nullptr;
  RefProblem *p = new RefProblem;
  p->nlev = levels;
  p->geom = new Geometry;
  GenerateGeometry(1, 0, 1, 0, 0, 0, nx, ny, nz, 1, 1, 1, p->geom);
  InitializeSparseMatrix(p->A, p->geom);
  GenerateProblem(p->A, &p->b, &p->x, &p->xexact);
  SetupHalo(p->A);
  SparseMatrix *cur = &p->A;
  for (int l = 1; l < p->nlev; ++l) {
    GenerateCoarseProblem(*cur);
    cur = cur->Ac;
  }
  cur = &p->A;
  for (int l = 0; l < p->nlev; ++l) {
    p->level[l] = cur;
    CheckProblem(*cur, l == 0 ? &p->b : nullptr, l == 0 ? &p->x : nullptr,
                 l == 0 ? &p->xexact : nullptr);
    cur = cur->Ac;
  }
  InitializeSparseCGData(p->A, p->data);
  return p;
}

void *ref_create(int nx, int ny, int nz) { return ref_create_levels(nx, ny, nz, kLevels); }

void ref_destroy(void *h) {
  RefProblem *p = static_cast<RefProblem *>(h);
  for (SparseMatrix *P : p->perm) free_permuted(P);
  DeleteMatrix(p->A);  // also deletes the geometry and the coarse levels
  DeleteCGData(p->data);
  DeleteVector(p->b);
  DeleteVector(p->x);
  DeleteVector(p->xexact);
  delete p;
}

int64_t ref_level_rows(void *h, int level) {
  return static_cast<RefProblem *>(h)->level[level]->localNumberOfRows;
}

int64_t ref_level_nnz(void *h, int level) {
  return static_cast<RefProblem *>(h)->level[level]->totalNumberOfNonzeros;
}

// Copies one level into the contiguous 27-slot layout (unused slots: col=row, val=0).
void ref_export_level(void *h, int level, uint8_t *nnz, int32_t *cols, double *vals,
                      int32_t *diag, int32_t *f2c) {
  const SparseMatrix &A = *static_cast<RefProblem *>(h)->level[level];
  for (local_int_t i = 0; i < A.localNumberOfRows; i++) {
    int nz = A.nonzerosInRow[i];
    nnz[i] = (uint8_t)nz;
    for (int j = 0; j < 27; j++) {
      cols[(int64_t)i * 27 + j] = j < nz ? A.mtxIndL[i][j] : i;
      vals[(int64_t)i * 27 + j] = j < nz ? A.matrixValues[i][j] : 0.0;
      if (j < nz && &A.matrixValues[i][j] == A.matrixDiagonal[i]) diag[i] = j;
    }
  }
  if (f2c && A.mgData)
    std::memcpy(f2c, A.mgData->f2cOperator, sizeof(int32_t) * A.mgData->rc->localLength);
}

void ref_get_vectors(void *h, double *b, double *x, double *xexact) {
  RefProblem *p = static_cast<RefProblem *>(h);
  local_int_t n = p->A.localNumberOfRows;
  if (b) std::memcpy(b, p->b.values, sizeof(double) * n);
  if (x) std::memcpy(x, p->x.values, sizeof(double) * n);
  if (xexact) std::memcpy(xexact, p->xexact.values, sizeof(double) * n);
}

// Overwrites the values of one level (contiguous 27-slot layout, entries in
// the reference's order); the pattern and the diagonal pointers stay.
void ref_set_level_values(void *h, int level, const double *vals) {
  SparseMatrix &A = *static_cast<RefProblem *>(h)->level[level];
  for (local_int_t i = 0; i < A.localNumberOfRows; i++)
    for (int j = 0; j < A.nonzerosInRow[i]; j++) A.matrixValues[i][j] = vals[(int64_t)i * 27 + j];
}

// ReplaceMatrixDiagonal (src/SparseMatrix.hpp:139-145) on one level.
void ref_replace_diagonal(void *h, int level, const double *d) {
  SparseMatrix &A = *static_cast<RefProblem *>(h)->level[level];
  Vector v = view(const_cast<double *>(d), A.localNumberOfRows);
  ReplaceMatrixDiagonal(A, v);
}

int ref_spmv(void *h, int level, const double *x, double *y) {
  SparseMatrix &A = *static_cast<RefProblem *>(h)->level[level];
  Vector xv = view(const_cast<double *>(x), A.localNumberOfColumns);
  Vector yv = view(y, A.localNumberOfRows);
  return ComputeSPMV_ref(A, xv, yv);
}

int ref_symgs(void *h, int level, const double *r, double *x) {
  SparseMatrix &A = *static_cast<RefProblem *>(h)->level[level];
  Vector rv = view(const_cast<double *>(r), A.localNumberOfRows);
  Vector xv = view(x, A.localNumberOfColumns);
  return ComputeSYMGS_ref(A, rv, xv);
}

int ref_mg(void *h, const double *r, double *x) {
  SparseMatrix &A = static_cast<RefProblem *>(h)->A;
  Vector rv = view(const_cast<double *>(r), A.localNumberOfRows);
  Vector xv = view(x, A.localNumberOfColumns);
  return ComputeMG_ref(A, rv, xv);
}

// ComputeRestriction_ref on `level` with a caller-supplied fine residual
// product Axf; writes the coarse residual rc.
int ref_restriction(void *h, int level, const double *rf, const double *Axf, double *rc) {
  SparseMatrix &A = *static_cast<RefProblem *>(h)->level[level];
  std::memcpy(A.mgData->Axf->values, Axf, sizeof(double) * A.localNumberOfRows);
  Vector rfv = view(const_cast<double *>(rf), A.localNumberOfRows);
  int ierr = ComputeRestriction_ref(A, rfv);
  std::memcpy(rc, A.mgData->rc->values, sizeof(double) * A.mgData->rc->localLength);
  return ierr;
}

int ref_prolongation(void *h, int level, const double *xc, double *xf) {
  SparseMatrix &A = *static_cast<RefProblem *>(h)->level[level];
  std::memcpy(A.mgData->xc->values, xc, sizeof(double) * A.mgData->xc->localLength);
  Vector xfv = view(xf, A.localNumberOfColumns);
  return ComputeProlongation_ref(A, xfv);
}

double ref_dot(int64_t n, const double *x, const double *y) {
  Vector xv = view(const_cast<double *>(x), (local_int_t)n);
  Vector yv = view(const_cast<double *>(y), (local_int_t)n);
  double r = 0.0, t = 0.0;
  ComputeDotProduct_ref((local_int_t)n, xv, x == y ? xv : yv, r, t);
  return r;
}

int ref_waxpby(int64_t n, double alpha, const double *x, double beta, const double *y,
               double *w) {
  Vector xv = view(const_cast<double *>(x), (local_int_t)n);
  Vector yv = view(const_cast<double *>(y), (local_int_t)n);
  Vector wv = view(w, (local_int_t)n);
  return ComputeWAXPBY_ref((local_int_t)n, alpha, xv, beta, yv, wv);
}

double ref_residual(int64_t n, const double *v1, const double *v2) {
  Vector a = view(const_cast<double *>(v1), (local_int_t)n);
  Vector b = view(const_cast<double *>(v2), (local_int_t)n);
  double r = 0.0;
  ComputeResidual((local_int_t)n, a, b, r);
  return r;
}

// CG_ref (src/CG_ref.cpp:58) on the problem's own CGData; times[0..5] as there.
int ref_cg(void *h, const double *b, double *x, int max_iter, double tol, int precond,
           int *niters, double *normr, double *normr0, double *times) {
  RefProblem *p = static_cast<RefProblem *>(h);
  Vector bv = view(const_cast<double *>(b), p->A.localNumberOfRows);
  Vector xv = view(x, p->A.localNumberOfColumns);
  return CG_ref(p->A, p->data, bv, xv, max_iter, tol, *niters, *normr, *normr0, times,
                precond != 0);
}

// Builds (once) the colour-permuted hierarchy: positions[l][i] is the new
// index of row i on level l (the permutation OptimizeProblem's greedy
// colouring produces, src/OptimizeProblem.cpp:81-96).  f2c is renumbered on
// both sides so that injection picks the same points.
int ref_build_permuted(void *h, const int64_t *const *positions) {
  RefProblem *p = static_cast<RefProblem *>(h);
  if (!p->perm.empty()) return 0;
  p->pos.resize(p->nlev);
  for (int l = 0; l < p->nlev; l++) {
    local_int_t n = p->level[l]->localNumberOfRows;
    p->pos[l].resize(n);
    for (local_int_t i = 0; i < n; i++) p->pos[l][i] = (local_int_t)positions[l][i];
    p->perm.push_back(permuted_copy(*p->level[l], p->pos[l]));
  }
  for (int l = 0; l + 1 < p->nlev; l++) {
    const SparseMatrix &A = *p->level[l];
    local_int_t nc = A.mgData->rc->localLength;
    local_int_t *f2c = new local_int_t[A.localNumberOfRows];
    for (local_int_t ic = 0; ic < nc; ic++)
      f2c[p->pos[l + 1][ic]] = p->pos[l][A.mgData->f2cOperator[ic]];
    Vector *rc = new Vector, *xc = new Vector, *Axf = new Vector;
    InitializeVector(*rc, nc);
    InitializeVector(*xc, nc);
    InitializeVector(*Axf, A.localNumberOfColumns);
    MGData *mg = new MGData;
    InitializeMGData(f2c, rc, xc, Axf, *mg);
    p->perm[l]->mgData = mg;
    p->perm[l]->Ac = p->perm[l + 1];
  }
  return 0;
}

// ComputeSYMGS_ref / ComputeMG_ref on the permuted hierarchy, with r and x
// given (and returned) in natural order.
int ref_symgs_permuted(void *h, int level, const double *r, double *x) {
  RefProblem *p = static_cast<RefProblem *>(h);
  if (p->perm.empty()) return -1;
  local_int_t n = p->level[level]->localNumberOfRows;
  std::vector<double> rp(n), xp(n);
  for (local_int_t i = 0; i < n; i++) { rp[p->pos[level][i]] = r[i]; xp[p->pos[level][i]] = x[i]; }
  Vector rv = view(rp.data(), n), xv = view(xp.data(), n);
  int ierr = ComputeSYMGS_ref(*p->perm[level], rv, xv);
  for (local_int_t i = 0; i < n; i++) x[i] = xp[p->pos[level][i]];
  return ierr;
}

int ref_mg_permuted(void *h, const double *r, double *x) {
  RefProblem *p = static_cast<RefProblem *>(h);
  if (p->perm.empty()) return -1;
  local_int_t n = p->A.localNumberOfRows;
  std::vector<double> rp(n), xp(n);
  for (local_int_t i = 0; i < n; i++) rp[p->pos[0][i]] = r[i];
  Vector rv = view(rp.data(), n), xv = view(xp.data(), n);
  // A permuted hierarchy shares the coarse pointers set up above.
  int ierr = ComputeMG_ref(*p->perm[0], rv, xv);
  for (local_int_t i = 0; i < n; i++) x[i] = xp[p->pos[0][i]];
  return ierr;
}

// CG_ref on the permuted hierarchy, b and x in natural order.
int ref_cg_permuted(void *h, const double *b, double *x, int max_iter, double tol, int precond,
                    int *niters, double *normr, double *normr0) {
  RefProblem *p = static_cast<RefProblem *>(h);
  if (p->perm.empty()) return -1;
  local_int_t n = p->A.localNumberOfRows;
  std::vector<double> bp(n), xp(n);
  for (local_int_t i = 0; i < n; i++) { bp[p->pos[0][i]] = b[i]; xp[p->pos[0][i]] = x[i]; }
  Vector bv = view(bp.data(), n), xv = view(xp.data(), n);
  std::vector<double> times(10, 0.0);
  int ierr = CG_ref(*p->perm[0], p->data, bv, xv, max_iter, tol, *niters, *normr, *normr0,
                    times.data(), precond != 0);
  for (local_int_t i = 0; i < n; i++) x[i] = xp[p->pos[0][i]];
  return ierr;
}

double ref_wtime(void) { return mytimer(); }

}  // extern "C"
