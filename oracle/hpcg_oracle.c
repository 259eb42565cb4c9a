/*
 * hpcg_oracle.c -- CPU restatement of HPCG 3.1's reference PCG path.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker for the CUDA product, never
 * part of it.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.
 *
 * Build flags matter: the recipe in oracle/Makefile compiles with
 * -O2 -fno-fast-math -ffp-contract=off so that every multiply and add is
 * rounded separately, exactly as the reference's own -O3 x86-64 build does.
 * The oracle is pinned against the reference itself (oracle/_ref, compiled
 * from the reference sources) and against the committed golden vectors in
 * tests/golden/ by tests/test_oracle_pin.py.
 */
#include "hpcg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Problem generation                                                       */
/* ------------------------------------------------------------------------ */

/* Restates GenerateProblem_ref (src/GenerateProblem_ref.cpp:130-181) for one
 * rank (gix0 = giy0 = giz0 = 0, gn* = n*): the 27-point stencil with 26 on the
 * diagonal and -1 elsewhere, entries in (sz, sy, sx) order, b = 27 - nnz
 * (:178), x = 0 (:179), xexact = 1 (:180).  Returns the number of nonzeros. */
int64_t or_generate_problem(int nx, int ny, int nz, uint8_t *nnz, int32_t *cols,
                            double *vals, int32_t *diag, double *b, double *x,
                            double *xexact) {
  int64_t total = 0;
  for (int64_t iz = 0; iz < nz; iz++)
    for (int64_t iy = 0; iy < ny; iy++)
      for (int64_t ix = 0; ix < nx; ix++) {
        int64_t row = iz * nx * ny + iy * nx + ix;
        int k = 0;
        for (int sz = -1; sz <= 1; sz++) {
          if (iz + sz < 0 || iz + sz >= nz) continue;
          for (int sy = -1; sy <= 1; sy++) {
            if (iy + sy < 0 || iy + sy >= ny) continue;
            for (int sx = -1; sx <= 1; sx++) {
              if (ix + sx < 0 || ix + sx >= nx) continue;
              int64_t col = row + sz * (int64_t)nx * ny + sy * (int64_t)nx + sx;
              if (col == row) {
                diag[row] = k;
                vals[row * OR_STENCIL + k] = 26.0;
              } else {
                vals[row * OR_STENCIL + k] = -1.0;
              }
              cols[row * OR_STENCIL + k] = (int32_t)col;
              k++;
            }
          }
        }
        for (int j = k; j < OR_STENCIL; j++) {   /* unused slots: defined, never read */
          cols[row * OR_STENCIL + j] = (int32_t)row;
          vals[row * OR_STENCIL + j] = 0.0;
        }
        nnz[row] = (uint8_t)k;
        total += k;
        if (b) b[row] = 26.0 - ((double)(k - 1));
        if (x) x[row] = 0.0;
        if (xexact) xexact[row] = 1.0;
      }
  return total;
}

/* Restates the injection operator of GenerateCoarseProblem
 * (src/GenerateCoarseProblem.cpp:71-82): coarse row (ixc, iyc, izc) takes the
 * fine row (2ixc, 2iyc, 2izc). */
void or_f2c(int nxf, int nyf, int nzf, int32_t *f2c) {
  int64_t nxc = nxf / 2, nyc = nyf / 2, nzc = nzf / 2;
  for (int64_t izc = 0; izc < nzc; izc++)
    for (int64_t iyc = 0; iyc < nyc; iyc++)
      for (int64_t ixc = 0; ixc < nxc; ixc++) {
        int64_t c = izc * nxc * nyc + iyc * nxc + ixc;
        f2c[c] = (int32_t)((2 * izc) * (int64_t)nxf * nyf + (2 * iyc) * (int64_t)nxf + 2 * ixc);
      }
}

/* Restates the structural assertions of CheckProblem
 * (src/CheckProblem.cpp:87-122).  Returns 0 when every value, column,
 * diagonal position, row count and vector entry matches. */
int or_check_problem(int nx, int ny, int nz, const uint8_t *nnz, const int32_t *cols,
                     const double *vals, const int32_t *diag, const double *b,
                     const double *x, const double *xexact) {
  for (int64_t iz = 0; iz < nz; iz++)
    for (int64_t iy = 0; iy < ny; iy++)
      for (int64_t ix = 0; ix < nx; ix++) {
        int64_t row = iz * nx * ny + iy * nx + ix;
        int k = 0;
        for (int sz = -1; sz <= 1; sz++) {
          if (iz + sz < 0 || iz + sz >= nz) continue;
          for (int sy = -1; sy <= 1; sy++) {
            if (iy + sy < 0 || iy + sy >= ny) continue;
            for (int sx = -1; sx <= 1; sx++) {
              if (ix + sx < 0 || ix + sx >= nx) continue;
              int64_t col = row + sz * (int64_t)nx * ny + sy * (int64_t)nx + sx;
              double v = vals[row * OR_STENCIL + k];
              if (col == row) {
                if (diag[row] != k || v != 26.0) return 1;
              } else if (v != -1.0) {
                return 2;
              }
              if (cols[row * OR_STENCIL + k] != col) return 3;
              k++;
            }
          }
        }
        if (nnz[row] != k) return 4;
        if (b && b[row] != 26.0 - ((double)(k - 1))) return 5;
        if (x && x[row] != 0.0) return 6;
        if (xexact && xexact[row] != 1.0) return 7;
      }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* FP64 kernels                                                             */
/* ------------------------------------------------------------------------ */

/* Restates ComputeSPMV_ref (src/ComputeSPMV_ref.cpp:58-71): per row, a
 * left-to-right sum of value*x over the row's entries, starting from 0. */
void or_spmv(int64_t nrow, const uint8_t *nnz, const int32_t *cols, const double *vals,
             const double *x, double *y) {
  for (int64_t i = 0; i < nrow; i++) {
    double sum = 0.0;
    const int32_t *c = cols + i * OR_STENCIL;
    const double *v = vals + i * OR_STENCIL;
    for (int j = 0; j < nnz[i]; j++) sum += v[j] * x[c[j]];
    y[i] = sum;
  }
}

/* One Gauss-Seidel row update exactly as src/ComputeSYMGS_ref.cpp:72-80:
 * sum = r_i - sum_j a_ij x_j (diagonal included), then add back x_i*a_ii and
 * divide by a_ii. */
static inline void gs_row(int64_t i, const uint8_t *nnz, const int32_t *cols,
                          const double *vals, const int32_t *diag, const double *r,
                          double *x) {
  const int32_t *c = cols + i * OR_STENCIL;
  const double *v = vals + i * OR_STENCIL;
  const double d = v[diag[i]];
  double sum = r[i];
  for (int j = 0; j < nnz[i]; j++) sum -= v[j] * x[c[j]];
  sum += x[i] * d;
  x[i] = sum / d;
}

/* Restates ComputeSYMGS_ref (src/ComputeSYMGS_ref.cpp:54-103): a forward sweep
 * over the rows then a backward sweep.  With `order` non-NULL the rows are
 * visited in that order (forward) and its reverse (backward); this is
 * ComputeSYMGS_ref applied to the symmetrically permuted matrix P A P^T whose
 * row k is row order[k] (entries kept in their order), with r and x permuted
 * the same way, and the result permuted back. */
void or_symgs(int64_t nrow, const uint8_t *nnz, const int32_t *cols, const double *vals,
              const int32_t *diag, const int64_t *order, const double *r, double *x) {
  for (int64_t k = 0; k < nrow; k++)
    gs_row(order ? order[k] : k, nnz, cols, vals, diag, r, x);
  for (int64_t k = nrow - 1; k >= 0; k--)
    gs_row(order ? order[k] : k, nnz, cols, vals, diag, r, x);
}

/* The SYMGS of a z-slab decomposition (slab_rows rows per rank): every rank
 * runs ComputeSYMGS_ref (src/ComputeSYMGS_ref.cpp:53-100) on its own rows
 * after ExchangeHalo (:56), so a row reads its own slab's current values and
 * every other slab's values as they were when the sweep began -- for the
 * forward and the backward sweep alike (block Jacobi across ranks).  With
 * slab_rows == 0 this is or_symgs. */
void or_symgs_slab(int64_t nrow, const uint8_t *nnz, const int32_t *cols, const double *vals,
                   const int32_t *diag, const int64_t *order, int64_t slab_rows, const double *r,
                   double *x) {
  if (slab_rows <= 0 || slab_rows >= nrow) {
    or_symgs(nrow, nnz, cols, vals, diag, order, r, x);
    return;
  }
  double *x0 = (double *)malloc(sizeof(double) * (size_t)nrow);
  memcpy(x0, x, sizeof(double) * (size_t)nrow);
  for (int pass = 0; pass < 2; pass++) {
    for (int64_t k = 0; k < nrow; k++) {
      const int64_t kk = pass == 0 ? k : nrow - 1 - k;
      const int64_t i = order ? order[kk] : kk;
      const int64_t si = i / slab_rows;
      const int32_t *c = cols + i * OR_STENCIL;
      const double *v = vals + i * OR_STENCIL;
      const double d = v[diag[i]];
      double sum = r[i];
      for (int j = 0; j < nnz[i]; j++) sum -= v[j] * (c[j] / slab_rows == si ? x[c[j]] : x0[c[j]]);
      sum += x[i] * d;
      x[i] = sum / d;
    }
  }
  free(x0);
}

/* A dot product of the z-slab decomposition: every rank sums its rows in
 * order (ComputeDotProduct_ref, src/ComputeDotProduct_ref.cpp:53-64), then
 * the rank totals are summed in rank order (the MPI_Allreduce of :66-77). */
double or_dot_slab(int64_t n, const double *x, const double *y, int64_t slab_rows) {
  if (slab_rows <= 0 || slab_rows >= n) return or_dot(n, x, y);
  double s = 0.0;
  for (int64_t b = 0; b < n; b += slab_rows) s += or_dot(slab_rows, x + b, y + b);
  return s;
}

/* Restates ComputeRestriction_ref (src/ComputeRestriction_ref.cpp:51). */
void or_restriction(int64_t nc, const int32_t *f2c, const double *rf, const double *Axf,
                    double *rc) {
  for (int64_t i = 0; i < nc; i++) rc[i] = rf[f2c[i]] - Axf[f2c[i]];
}

/* Restates ComputeProlongation_ref (src/ComputeProlongation_ref.cpp:49). */
void or_prolongation(int64_t nc, const int32_t *f2c, const double *xc, double *xf) {
  for (int64_t i = 0; i < nc; i++) xf[f2c[i]] += xc[i];
}

/* Restates ComputeDotProduct_ref (src/ComputeDotProduct_ref.cpp:53-64) in
 * sequential order (the reference's OpenMP reduction order varies with the
 * thread count; parity on dot products is therefore a relative tolerance). */
double or_dot(int64_t n, const double *x, const double *y) {
  double s = 0.0;
  if (x == y)
    for (int64_t i = 0; i < n; i++) s += x[i] * x[i];
  else
    for (int64_t i = 0; i < n; i++) s += x[i] * y[i];
  return s;
}

/* Restates ComputeWAXPBY_ref (src/ComputeWAXPBY_ref.cpp:52-67) including its
 * alpha == 1 and beta == 1 branches, which round differently from the general
 * form when alpha or beta is 1. */
void or_waxpby(int64_t n, double alpha, const double *x, double beta, const double *y,
               double *w) {
  if (alpha == 1.0)
    for (int64_t i = 0; i < n; i++) w[i] = x[i] + beta * y[i];
  else if (beta == 1.0)
    for (int64_t i = 0; i < n; i++) w[i] = alpha * x[i] + y[i];
  else
    for (int64_t i = 0; i < n; i++) w[i] = alpha * x[i] + beta * y[i];
}

/* Restates ComputeResidual (src/ComputeResidual.cpp:71-77): max |v1 - v2|. */
double or_residual(int64_t n, const double *v1, const double *v2) {
  double m = 0.0;
  for (int64_t i = 0; i < n; i++) {
    double d = fabs(v1[i] - v2[i]);
    if (d > m) m = d;
  }
  return m;
}

/* Restates ComputeMG_ref (src/ComputeMG_ref.cpp:39-63): zero x, one
 * pre-smoothing SYMGS, fine residual product, injection restriction,
 * recursion, prolongation, one post-smoothing SYMGS; one SYMGS on the
 * coarsest level.  The smoothing counts are fixed at 1/1 as in
 * src/MGData.hpp:51-52. */
int or_mg(const or_level *L, int nlev, const double *r, double *x) {
  const or_level *A = &L[0];
  memset(x, 0, sizeof(double) * (size_t)A->nrow);
  if (nlev > 1 && A->f2c) {
    or_symgs_slab(A->nrow, A->nnz, A->cols, A->vals, A->diag, A->order, A->slab_rows, r, x);
    or_spmv(A->nrow, A->nnz, A->cols, A->vals, x, A->Axf);
    or_restriction(A->nc, A->f2c, r, A->Axf, A->rc);
    int ierr = or_mg(L + 1, nlev - 1, A->rc, A->xc);
    if (ierr) return ierr;
    or_prolongation(A->nc, A->f2c, A->xc, x);
    or_symgs_slab(A->nrow, A->nnz, A->cols, A->vals, A->diag, A->order, A->slab_rows, r, x);
  } else {
    or_symgs_slab(A->nrow, A->nnz, A->cols, A->vals, A->diag, A->order, A->slab_rows, r, x);
  }
  return 0;
}

/* Restates CG_ref (src/CG_ref.cpp:58-144) without timers.  work holds
 * 4*nrow doubles: r, z, p, Ap (src/CGData.hpp:41-49).  The unpreconditioned
 * branch copies r to z with WAXPBY(1, r, 0, r) as CG_ref does (:51). */
int or_cg(const or_level *L, int nlev, const double *b, double *x, int max_iter,
          double tolerance, int precond, int *niters, double *normr, double *normr0,
          double *work) {
  const or_level *A = &L[0];
  const int64_t n = A->nrow;
  double *r = work, *z = work + n, *p = work + 2 * n, *Ap = work + 3 * n;
  double rtz = 0.0, oldrtz = 0.0, alpha = 0.0, beta = 0.0, pAp = 0.0;
  *normr = 0.0;
  *niters = 0;
  memcpy(p, x, sizeof(double) * (size_t)n);
  or_spmv(n, A->nnz, A->cols, A->vals, p, Ap);
  or_waxpby(n, 1.0, b, -1.0, Ap, r);
  *normr = sqrt(or_dot_slab(n, r, r, A->slab_rows));
  *normr0 = *normr;
  for (int k = 1; k <= max_iter && *normr / *normr0 > tolerance; k++) {
    if (precond) {
      int ierr = or_mg(L, nlev, r, z);
      if (ierr) return ierr;
    } else {
      or_waxpby(n, 1.0, r, 0.0, r, z);
    }
    if (k == 1) {
      memcpy(p, z, sizeof(double) * (size_t)n);
      rtz = or_dot_slab(n, r, z, A->slab_rows);
    } else {
      oldrtz = rtz;
      rtz = or_dot_slab(n, r, z, A->slab_rows);
      beta = rtz / oldrtz;
      or_waxpby(n, 1.0, z, beta, p, p);
    }
    or_spmv(n, A->nnz, A->cols, A->vals, p, Ap);
    pAp = or_dot_slab(n, p, Ap, A->slab_rows);
    alpha = rtz / pAp;
    or_waxpby(n, 1.0, x, alpha, p, x);
    or_waxpby(n, 1.0, r, -alpha, Ap, r);
    *normr = sqrt(or_dot_slab(n, r, r, A->slab_rows));
    *niters = k;
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Colouring                                                                */
/* ------------------------------------------------------------------------ */

/* Restates the greedy multicolouring of OptimizeProblem
 * (src/OptimizeProblem.cpp:43-96, compiled there only under
 * HPCG_USE_MULTICOLORING): rows in natural order take the lowest colour not
 * used by an already-coloured neighbour; a prefix scan over colour counts then
 * turns colours into positions in colour-major, natural-within-colour order.
 * Returns the number of colours. */
int or_greedy_colour(int64_t nrow, const uint8_t *nnz, const int32_t *cols,
                     int32_t *colors, int64_t *position) {
  int total = 1;
  for (int64_t i = 0; i < nrow; i++) colors[i] = -1;
  colors[0] = 0;
  for (int64_t i = 1; i < nrow; i++) {
    int used[OR_STENCIL + 1];
    memset(used, 0, sizeof(used));
    for (int j = 0; j < nnz[i]; j++) {
      int32_t c = cols[i * OR_STENCIL + j];
      if (c < i) used[colors[c]] = 1;
    }
    int pick = -1;
    for (int k = 0; k < total; k++)
      if (!used[k]) { pick = k; break; }
    if (pick < 0) pick = total++;
    colors[i] = pick;
  }
  int64_t counters[OR_STENCIL + 1];
  memset(counters, 0, sizeof(counters));
  for (int64_t i = 0; i < nrow; i++) counters[colors[i]]++;
  int64_t run = 0;
  for (int k = 0; k < total; k++) { int64_t t = counters[k]; counters[k] = run; run += t; }
  for (int64_t i = 0; i < nrow; i++) position[i] = counters[colors[i]]++;
  return total;
}

/* ------------------------------------------------------------------------ */
/* Mixed precision V-cycle: BF16 values, FP32 vectors (no reference         */
/* counterpart; same control flow as ComputeMG_ref and ComputeSYMGS_ref).   */
/* ------------------------------------------------------------------------ */

/* FP64 -> BF16 conversion used everywhere in this project: round to FP32
 * (nearest-even), then round the FP32 bit pattern to BF16 (nearest-even).
 * NaN is kept quiet. */
uint16_t or_bf16_from_double(double v) {
  float f = (float)v;
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u && (u & 0x007fffffu)) return (uint16_t)((u >> 16) | 0x40);
  uint32_t lsb = (u >> 16) & 1u;
  u += 0x7fffu + lsb;
  return (uint16_t)(u >> 16);
}

float or_float_from_bf16(uint16_t h) {
  uint32_t u = ((uint32_t)h) << 16;
  float f;
  memcpy(&f, &u, 4);
  return f;
}

void or_vals_to_bf16(int64_t n, const double *v, uint16_t *h) {
  for (int64_t i = 0; i < n; i++) h[i] = or_bf16_from_double(v[i]);
}

/* The mixed V-cycle's FP32 arithmetic accumulates with fused multiply-adds
 * (C's fmaf, correctly rounded): sum + v x and sum - v x in one rounding each,
 * in the row's entry order. */
void or_spmv32(int64_t nrow, const uint8_t *nnz, const int32_t *cols, const uint16_t *vals,
               const float *x, float *y) {
  for (int64_t i = 0; i < nrow; i++) {
    float sum = 0.0f;
    const int32_t *c = cols + i * OR_STENCIL;
    const uint16_t *v = vals + i * OR_STENCIL;
    for (int j = 0; j < nnz[i]; j++) sum = fmaf(or_float_from_bf16(v[j]), x[c[j]], sum);
    y[i] = sum;
  }
}

static inline void gs_row32(int64_t i, const uint8_t *nnz, const int32_t *cols,
                            const uint16_t *vals, const int32_t *diag, const double *r64,
                            const float *r32, float *x) {
  const int32_t *c = cols + i * OR_STENCIL;
  const uint16_t *v = vals + i * OR_STENCIL;
  const float d = or_float_from_bf16(v[diag[i]]);
  float sum = r64 ? (float)r64[i] : r32[i];
  for (int j = 0; j < nnz[i]; j++) sum = fmaf(-or_float_from_bf16(v[j]), x[c[j]], sum);
  sum = fmaf(x[i], d, sum);
  x[i] = sum / d;
}

/* FP32 symmetric Gauss-Seidel with BF16 values; the right-hand side is either
 * FP64 (finest level: rounded to FP32 where it is read) or FP32. */
void or_symgs32(int64_t nrow, const uint8_t *nnz, const int32_t *cols,
                const uint16_t *vals, const int32_t *diag, const int64_t *order,
                const double *r64, const float *r32, float *x) {
  for (int64_t k = 0; k < nrow; k++)
    gs_row32(order ? order[k] : k, nnz, cols, vals, diag, r64, r32, x);
  for (int64_t k = nrow - 1; k >= 0; k--)
    gs_row32(order ? order[k] : k, nnz, cols, vals, diag, r64, r32, x);
}

/* or_symgs_slab in FP32 with BF16 values. */
void or_symgs32_slab(int64_t nrow, const uint8_t *nnz, const int32_t *cols,
                     const uint16_t *vals, const int32_t *diag, const int64_t *order,
                     int64_t slab_rows, const double *r64, const float *r32, float *x) {
  if (slab_rows <= 0 || slab_rows >= nrow) {
    or_symgs32(nrow, nnz, cols, vals, diag, order, r64, r32, x);
    return;
  }
  float *x0 = (float *)malloc(sizeof(float) * (size_t)nrow);
  memcpy(x0, x, sizeof(float) * (size_t)nrow);
  for (int pass = 0; pass < 2; pass++) {
    for (int64_t k = 0; k < nrow; k++) {
      const int64_t kk = pass == 0 ? k : nrow - 1 - k;
      const int64_t i = order ? order[kk] : kk;
      const int64_t si = i / slab_rows;
      const int32_t *c = cols + i * OR_STENCIL;
      const uint16_t *v = vals + i * OR_STENCIL;
      const float d = or_float_from_bf16(v[diag[i]]);
      float sum = r64 ? (float)r64[i] : r32[i];
      for (int j = 0; j < nnz[i]; j++)
        sum = fmaf(-or_float_from_bf16(v[j]), c[j] / slab_rows == si ? x[c[j]] : x0[c[j]], sum);
      sum = fmaf(x[i], d, sum);
      x[i] = sum / d;
    }
  }
  free(x0);
}

/* The mixed-precision V-cycle: ComputeMG_ref's flow in FP32. */
int or_mg32(const or_level32 *L, int nlev, const double *r64, const float *r32, float *x) {
  const or_level32 *A = &L[0];
  memset(x, 0, sizeof(float) * (size_t)A->nrow);
  or_symgs32_slab(A->nrow, A->nnz, A->cols, A->vals, A->diag, A->order, A->slab_rows, r64, r32,
                  x);
  if (nlev > 1 && A->f2c) {
    or_spmv32(A->nrow, A->nnz, A->cols, A->vals, x, A->Axf);
    for (int64_t i = 0; i < A->nc; i++) {
      int64_t f = A->f2c[i];
      float rf = r64 ? (float)r64[f] : r32[f];
      A->rc[i] = rf - A->Axf[f];
    }
    int ierr = or_mg32(L + 1, nlev - 1, NULL, A->rc, A->xc);
    if (ierr) return ierr;
    for (int64_t i = 0; i < A->nc; i++) x[A->f2c[i]] += A->xc[i];
    or_symgs32_slab(A->nrow, A->nnz, A->cols, A->vals, A->diag, A->order, A->slab_rows, r64, r32,
                    x);
  }
  return 0;
}

/* Flexible PCG with the FP32/BF16 V-cycle as preconditioner (no reference
 * counterpart).  The outer loop is CG_ref's (src/CG_ref.cpp:58-144) in FP64
 * with the Polak-Ribiere beta
 *     beta_k = (r_k.z_k - r_{k-1}.z_k) / (r_{k-1}.z_{k-1}),
 * evaluated through the residual recurrence r_k = r_{k-1} - alpha Ap_{k-1} as
 *     beta_k = -(z_k.Ap_{k-1}) / (p_{k-1}.Ap_{k-1}),
 * which needs no stored r_{k-1}.  work holds 4*nrow doubles (r, z, p, Ap);
 * z32 holds nrow floats (the V-cycle output). */
int or_fcg(const or_level *L64, const or_level32 *L32, int nlev, const double *b,
           double *x, int max_iter, double tolerance, int *niters, double *normr,
           double *normr0, double *work, float *z32) {
  const or_level *A = &L64[0];
  const int64_t n = A->nrow;
  double *r = work, *z = work + n, *p = work + 2 * n, *Ap = work + 3 * n;
  double rtz = 0.0, alpha = 0.0, beta = 0.0, pAp = 0.0;
  *niters = 0;
  memcpy(p, x, sizeof(double) * (size_t)n);
  or_spmv(n, A->nnz, A->cols, A->vals, p, Ap);
  or_waxpby(n, 1.0, b, -1.0, Ap, r);
  *normr = sqrt(or_dot_slab(n, r, r, A->slab_rows));
  *normr0 = *normr;
  for (int k = 1; k <= max_iter && *normr / *normr0 > tolerance; k++) {
    int ierr = or_mg32(L32, nlev, r, NULL, z32);
    if (ierr) return ierr;
    for (int64_t i = 0; i < n; i++) z[i] = (double)z32[i];
    rtz = or_dot_slab(n, r, z, A->slab_rows);
    if (k == 1) {
      memcpy(p, z, sizeof(double) * (size_t)n);
    } else {
      double zAp = or_dot_slab(n, z, Ap, A->slab_rows);
      beta = -zAp / pAp;
      or_waxpby(n, 1.0, z, beta, p, p);
    }
    or_spmv(n, A->nnz, A->cols, A->vals, p, Ap);
    pAp = or_dot_slab(n, p, Ap, A->slab_rows);
    alpha = rtz / pAp;
    or_waxpby(n, 1.0, x, alpha, p, x);
    or_waxpby(n, 1.0, r, -alpha, Ap, r);
    *normr = sqrt(or_dot_slab(n, r, r, A->slab_rows));
    *niters = k;
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Seeded inputs (no reference counterpart).                                */
/* ------------------------------------------------------------------------ */

/* SplitMix64 (Steele, Lea, Flood 2014; constants as published by Vigna). */
uint64_t or_splitmix64(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* Counter-based uniform in [0, 1): 53 high bits of splitmix64(splitmix64(seed) + i). */
double or_uniform(uint64_t seed, uint64_t i) {
  uint64_t h = or_splitmix64(or_splitmix64(seed) + i);
  return (double)(h >> 11) * 0x1.0p-53;
}

/* Standard normal by the Box-Muller transform on uniforms 2i and 2i+1. */
double or_normal(uint64_t seed, uint64_t i) {
  double u1 = 1.0 - or_uniform(seed, 2 * i);  /* (0, 1] */
  double u2 = or_uniform(seed, 2 * i + 1);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

void or_fill_uniform(uint64_t seed, int64_t n, double lo, double hi, double *v) {
  for (int64_t i = 0; i < n; i++) v[i] = lo + (hi - lo) * or_uniform(seed, (uint64_t)i);
}

void or_fill_normal(uint64_t seed, int64_t n, double *v) {
  for (int64_t i = 0; i < n; i++) v[i] = or_normal(seed, (uint64_t)i);
}

/* Variable-coefficient SPD 27-point matrix on the same pattern and entry order
 * as or_generate_problem.  Each undirected edge {i, j} gets one draw
 * z ~ N(0,1) and a_ij = a_ji = -exp(sigma * z); the diagonal is
 * sum_j |a_ij| + 2 (summed in entry order), so A is symmetric and strictly
 * diagonally dominant.  The edge id is lo_f*13 + (s - 14) where lo = min(i, j),
 * lo_f is the finest-level index of lo's point (coordinates times 2^level on
 * the grid (nx << level, ny << level)) and s in [14, 27) is the stencil slot
 * (dz+1)*9 + (dy+1)*3 + (dx+1) of the other endpoint as seen from lo.  A coarse
 * level therefore takes, for each edge, the finest-level value of the edge
 * leaving its injected point in the same direction. */
int64_t or_generate_varcoef(int nx, int ny, int nz, int level, uint64_t seed, double sigma,
                            uint8_t *nnz, int32_t *cols, double *vals, int32_t *diag) {
  const int64_t nx0 = (int64_t)nx << level, ny0 = (int64_t)ny << level;
  int64_t total = 0;
  for (int64_t iz = 0; iz < nz; iz++)
    for (int64_t iy = 0; iy < ny; iy++)
      for (int64_t ix = 0; ix < nx; ix++) {
        int64_t row = iz * nx * ny + iy * nx + ix;
        int k = 0;
        double dsum = 0.0;
        for (int sz = -1; sz <= 1; sz++) {
          if (iz + sz < 0 || iz + sz >= nz) continue;
          for (int sy = -1; sy <= 1; sy++) {
            if (iy + sy < 0 || iy + sy >= ny) continue;
            for (int sx = -1; sx <= 1; sx++) {
              if (ix + sx < 0 || ix + sx >= nx) continue;
              int64_t col = row + sz * (int64_t)nx * ny + sy * (int64_t)nx + sx;
              cols[row * OR_STENCIL + k] = (int32_t)col;
              if (col == row) {
                diag[row] = k;
              } else {
                int s = (sz + 1) * 9 + (sy + 1) * 3 + (sx + 1);
                int64_t lx = ix, ly = iy, lz = iz;
                if (s < 13) { lx += sx; ly += sy; lz += sz; s = 26 - s; }
                int64_t lo_f = ((lz << level) * ny0 + (ly << level)) * nx0 + (lx << level);
                uint64_t edge = (uint64_t)lo_f * 13u + (uint64_t)(s - 14);
                double a = -exp(sigma * or_normal(seed, edge));
                vals[row * OR_STENCIL + k] = a;
                dsum += fabs(a);
              }
              k++;
            }
          }
        }
        vals[row * OR_STENCIL + diag[row]] = dsum + 2.0;
        for (int j = k; j < OR_STENCIL; j++) {
          cols[row * OR_STENCIL + j] = (int32_t)row;
          vals[row * OR_STENCIL + j] = 0.0;
        }
        nnz[row] = (uint8_t)k;
        total += k;
      }
  return total;
}

/* Gradient of L with respect to every stored matrix value for x = A^{-1} b:
 * dL/da_ij = -lambda_i * x_j where A lambda = dL/dx (A symmetric). */
void or_adjoint_grad(int64_t nrow, const uint8_t *nnz, const int32_t *cols,
                     const double *lambda, const double *x, double *grad) {
  for (int64_t i = 0; i < nrow; i++) {
    for (int j = 0; j < OR_STENCIL; j++)
      grad[i * OR_STENCIL + j] = j < nnz[i] ? -(lambda[i] * x[cols[i * OR_STENCIL + j]]) : 0.0;
  }
}

/* ------------------------------------------------------------------------ */
/* Matrix-free restatements for benchmark-size grids                         */
/* ------------------------------------------------------------------------ */
/* At 256^3 and 512^3 the stored-matrix restatements above need 6 to 50 GB of
 * host memory.  These functions apply the same reference operators to the
 * reference problem of src/GenerateProblem_ref.cpp:152-172 with every row
 * generated where it is used: present neighbours in (sz, sy, sx) order, 26 on
 * the diagonal and -1 elsewhere.  The arithmetic per row is exactly that of
 * or_spmv / gs_row / gs_row32 (same terms, same order), so the results are
 * bit-identical to the stored-matrix functions (checked on small grids by
 * tests/test_oracle_pin.py).  Rows of one colour are independent (no two are
 * neighbours), so the loops over a colour's rows run in parallel (OpenMP)
 * without changing a bit. */

/* Neighbour columns of row (ix, iy, iz) in entry order; returns the count and
 * the entry index of the diagonal in *diag. */
static inline int stencil_row(int nx, int ny, int nz, int64_t ix, int64_t iy, int64_t iz,
                              int64_t *col, int *diag) {
  const int64_t row = (iz * ny + iy) * nx + ix;
  int k = 0;
  for (int sz = -1; sz <= 1; sz++) {
    if (iz + sz < 0 || iz + sz >= nz) continue;
    for (int sy = -1; sy <= 1; sy++) {
      if (iy + sy < 0 || iy + sy >= ny) continue;
      for (int sx = -1; sx <= 1; sx++) {
        if (ix + sx < 0 || ix + sx >= nx) continue;
        const int64_t c = row + sz * (int64_t)nx * ny + sy * (int64_t)nx + sx;
        if (c == row) *diag = k;
        col[k++] = c;
      }
    }
  }
  return k;
}

/* ComputeSPMV_ref (src/ComputeSPMV_ref.cpp:58-71) on the reference problem. */
void or_stencil_spmv(int nx, int ny, int nz, const double *x, double *y) {
  const int64_t n = (int64_t)nx * ny * nz;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    const int64_t ix = i % nx, iy = (i / nx) % ny, iz = i / ((int64_t)nx * ny);
    int64_t col[OR_STENCIL];
    int dg = 0;
    const int k = stencil_row(nx, ny, nz, ix, iy, iz, col, &dg);
    double sum = 0.0;
    for (int j = 0; j < k; j++) sum += (j == dg ? 26.0 : -1.0) * x[col[j]];
    y[i] = sum;
  }
}

/* One colour's rows, natural order: colour (ix&1) + 2(iy&1) + 4(iz&1). */
#define OR_FOR_COLOUR(c, body)                                                       \
  do {                                                                               \
    const int px_ = (c) & 1, py_ = ((c) >> 1) & 1, pz_ = ((c) >> 2) & 1;             \
    const int64_t cz_ = (nz - pz_ + 1) / 2, cy_ = (ny - py_ + 1) / 2,                \
                  cx_ = (nx - px_ + 1) / 2;                                          \
    _Pragma("omp parallel for schedule(static)")                                     \
    for (int64_t t_ = 0; t_ < cz_ * cy_ * cx_; t_++) {                               \
      const int64_t ix = px_ + 2 * (t_ % cx_), iy = py_ + 2 * ((t_ / cx_) % cy_),    \
                    iz = pz_ + 2 * (t_ / (cx_ * cy_));                               \
      body                                                                           \
    }                                                                                \
  } while (0)

/* ComputeSYMGS_ref (src/ComputeSYMGS_ref.cpp:54-103) on the reference problem
 * in colour order (forward colours 0..7, backward 7..0): or_symgs with the
 * order of Oracle.colour_order. */
void or_stencil_symgs(int nx, int ny, int nz, const double *r, double *x) {
  for (int pass = 0; pass < 2; pass++)
    for (int cc = 0; cc < 8; cc++) {
      const int c = pass == 0 ? cc : 7 - cc;
      OR_FOR_COLOUR(c, {
        const int64_t i = (iz * ny + iy) * nx + ix;
        int64_t col[OR_STENCIL];
        int dg = 0;
        const int k = stencil_row(nx, ny, nz, ix, iy, iz, col, &dg);
        double sum = r[i];
        for (int j = 0; j < k; j++) sum -= (j == dg ? 26.0 : -1.0) * x[col[j]];
        sum += x[i] * 26.0;
        x[i] = sum / 26.0;
      });
    }
}

/* or_symgs32 (BF16 values -- 26 and -1 are exact -- FP32 vectors, fused
 * multiply-adds) on the reference problem in colour order; r64 is the FP64
 * right-hand side of the finest level, rounded to FP32 where it is read. */
void or_stencil_symgs32(int nx, int ny, int nz, const double *r64, float *x) {
  for (int pass = 0; pass < 2; pass++)
    for (int cc = 0; cc < 8; cc++) {
      const int c = pass == 0 ? cc : 7 - cc;
      OR_FOR_COLOUR(c, {
        const int64_t i = (iz * ny + iy) * nx + ix;
        int64_t col[OR_STENCIL];
        int dg = 0;
        const int k = stencil_row(nx, ny, nz, ix, iy, iz, col, &dg);
        float sum = (float)r64[i];
        for (int j = 0; j < k; j++) sum = fmaf(-(j == dg ? 26.0f : -1.0f), x[col[j]], sum);
        sum = fmaf(x[i], 26.0f, sum);
        x[i] = sum / 26.0f;
      });
    }
}
