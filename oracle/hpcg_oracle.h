/*
 * hpcg_oracle.h -- CPU restatement of HPCG 3.1's reference ("_ref") PCG path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA product
 * in hpcg_b200/: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it.  The product never links, calls or falls back to it.
 *
 * Matrices use the reference's contiguous row layout (HPCG_CONTIGUOUS_ARRAYS,
 * src/GenerateProblem_ref.cpp:113-124): row i owns slots [27*i, 27*i+27) of
 * `cols` / `vals`, the first nnz[i] of them used, in the order the reference
 * generator emits them (sz, sy, sx ascending, src/GenerateProblem_ref.cpp:152-172).
 * `diag[i]` is the slot of the diagonal inside row i (the reference keeps a
 * pointer, src/SparseMatrix.hpp:50).
 *
 * Every function cites the reference file:line it restates.  Functions marked
 * "no reference counterpart" restate this project's additions (mixed precision
 * V-cycle, flexible CG, variable-coefficient generator, adjoint gradient).
 */
#ifndef HPCG_ORACLE_H
#define HPCG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_STENCIL 27

/* One level of the multigrid hierarchy (FP64). */
typedef struct or_level {
  int64_t nrow;
  const uint8_t *nnz;     /* nonzerosInRow                          */
  const int32_t *cols;    /* 27*nrow column indices (mtxIndL)       */
  const double *vals;     /* 27*nrow values (matrixValues)          */
  const int32_t *diag;    /* slot of the diagonal in each row       */
  const int64_t *order;   /* SYMGS visiting order, NULL = natural   */
  const int32_t *f2c;     /* injection to next level, NULL=coarsest */
  int64_t nc;             /* rows of the next level                 */
  double *Axf;            /* work: nrow                             */
  double *rc;             /* work: nc                               */
  double *xc;             /* work: nc                               */
  int64_t slab_rows;      /* z-slab decomposition: rows per rank (0: one rank) */
} or_level;

/* One level of the mixed-precision hierarchy: BF16 values, FP32 vectors. */
typedef struct or_level32 {
  int64_t nrow;
  const uint8_t *nnz;
  const int32_t *cols;
  const uint16_t *vals;   /* BF16 bit patterns, 27*nrow             */
  const int32_t *diag;
  const int64_t *order;
  const int32_t *f2c;
  int64_t nc;
  float *Axf;
  float *rc;
  float *xc;
  int64_t slab_rows;
} or_level32;

/* --- problem generation ------------------------------------------------ */
int64_t or_generate_problem(int nx, int ny, int nz, uint8_t *nnz, int32_t *cols,
                            double *vals, int32_t *diag, double *b, double *x,
                            double *xexact);
void or_f2c(int nxf, int nyf, int nzf, int32_t *f2c);
int or_check_problem(int nx, int ny, int nz, const uint8_t *nnz, const int32_t *cols,
                     const double *vals, const int32_t *diag, const double *b,
                     const double *x, const double *xexact);

/* --- kernels ------------------------------------------------------------ */
void or_spmv(int64_t nrow, const uint8_t *nnz, const int32_t *cols, const double *vals,
             const double *x, double *y);
void or_symgs(int64_t nrow, const uint8_t *nnz, const int32_t *cols, const double *vals,
              const int32_t *diag, const int64_t *order, const double *r, double *x);
void or_restriction(int64_t nc, const int32_t *f2c, const double *rf, const double *Axf,
                    double *rc);
void or_prolongation(int64_t nc, const int32_t *f2c, const double *xc, double *xf);
double or_dot(int64_t n, const double *x, const double *y);
/* z-slab decomposition (slab_rows rows per rank, 0: one rank) */
void or_symgs_slab(int64_t nrow, const uint8_t *nnz, const int32_t *cols, const double *vals,
                   const int32_t *diag, const int64_t *order, int64_t slab_rows, const double *r,
                   double *x);
double or_dot_slab(int64_t n, const double *x, const double *y, int64_t slab_rows);
void or_waxpby(int64_t n, double alpha, const double *x, double beta, const double *y,
               double *w);
double or_residual(int64_t n, const double *v1, const double *v2);
int or_mg(const or_level *L, int nlev, const double *r, double *x);
int or_cg(const or_level *L, int nlev, const double *b, double *x, int max_iter,
          double tolerance, int precond, int *niters, double *normr, double *normr0,
          double *work);

/* --- colouring (OptimizeProblem hook) ---------------------------------- */
int or_greedy_colour(int64_t nrow, const uint8_t *nnz, const int32_t *cols,
                     int32_t *colors, int64_t *position);

/* --- mixed precision (no reference counterpart) ------------------------ */
uint16_t or_bf16_from_double(double v);
float or_float_from_bf16(uint16_t h);
void or_vals_to_bf16(int64_t n, const double *v, uint16_t *h);
void or_spmv32(int64_t nrow, const uint8_t *nnz, const int32_t *cols, const uint16_t *vals,
               const float *x, float *y);
void or_symgs32(int64_t nrow, const uint8_t *nnz, const int32_t *cols,
                const uint16_t *vals, const int32_t *diag, const int64_t *order,
                const double *r64, const float *r32, float *x);
void or_symgs32_slab(int64_t nrow, const uint8_t *nnz, const int32_t *cols,
                     const uint16_t *vals, const int32_t *diag, const int64_t *order,
                     int64_t slab_rows, const double *r64, const float *r32, float *x);
int or_mg32(const or_level32 *L, int nlev, const double *r64, const float *r32, float *x);
int or_fcg(const or_level *L64, const or_level32 *L32, int nlev, const double *b,
           double *x, int max_iter, double tolerance, int *niters, double *normr,
           double *normr0, double *work, float *z32);

/* --- seeded inputs (no reference counterpart) -------------------------- */
uint64_t or_splitmix64(uint64_t x);
double or_uniform(uint64_t seed, uint64_t i);
double or_normal(uint64_t seed, uint64_t i);
void or_fill_uniform(uint64_t seed, int64_t n, double lo, double hi, double *v);
void or_fill_normal(uint64_t seed, int64_t n, double *v);
int64_t or_generate_varcoef(int nx, int ny, int nz, int level, uint64_t seed, double sigma,
                            uint8_t *nnz, int32_t *cols, double *vals, int32_t *diag);
void or_adjoint_grad(int64_t nrow, const uint8_t *nnz, const int32_t *cols,
                     const double *lambda, const double *x, double *grad);

/* matrix-free restatements on the reference problem (benchmark-size grids) */
void or_stencil_spmv(int nx, int ny, int nz, const double *x, double *y);
void or_stencil_symgs(int nx, int ny, int nz, const double *r, double *x);
void or_stencil_symgs32(int nx, int ny, int nz, const double *r64, float *x);

#ifdef __cplusplus
}
#endif
#endif
