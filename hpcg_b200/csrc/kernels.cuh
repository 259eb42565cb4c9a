// kernels.cuh -- host-side view of the device kernels of libhpcgx.
#pragma once
#include "common.cuh"

#include <vector>

namespace hpcgx {

// One multigrid level on the device.
struct LevelDev {
  int nx = 0, ny = 0, nz = 0;
  int64_t n = 0;              // rows
  int64_t storage_rows = 0;   // rows incl. the padding that aligns colours to 32
  int64_t cstart[8] = {}, ccount[8] = {};
  ClassInfo cls[4] = {};
  int lines_per_block[4] = {}, blocks[4] = {}, threads[4] = {};
  int spmv_blocks = 0;        // all four classes in one launch (one line group per block)
  // FP64 operators derive their columns from the stencil offsets instead of
  // reading the int32 column arrays (hpcgx_set_stencil_columns)
  bool stencil_cols = false;
  // z-slab of a sharded problem: a neighbouring rank owns the plane below
  // (zlo) / above (zhi); vectors read by SpMV and Gauss-Seidel then hold one
  // halo plane on each side (indices -nx*ny..-1 and n..n+nx*ny-1)
  int zlo = 0, zhi = 0;
  double *vals = nullptr;     // storage_rows*27, FP64
  int32_t *cols = nullptr;    // storage_rows*27
  uint16_t *vals16 = nullptr; // storage_rows*27, BF16 (mixed precision)
  // multigrid work vectors of this level (levels >= 1: right-hand side and
  // correction; level 0 uses the caller's vectors)
  double *r64 = nullptr, *x64 = nullptr;
  float *r32 = nullptr, *x32 = nullptr;
};

// Device-side state of a CG solve (scalars never leave the GPU except the
// residual norm read once per host check).
struct CgState {
  double normr, normr0, rtz, oldrtz, pAp, alpha, beta, zAp, tol;
  int k;         // iteration about to run (1-based)
  int max_iter;
  int done;      // 1 once the loop condition of CG (src/CG.cpp:100) is false
  int niters;
  int flexible;  // Polak-Ribiere beta for a variable (mixed) preconditioner
  int nonfinite; // a non-finite residual norm stopped the loop
};

// Scratch of the deterministic grid reductions: per-block partial sums and a
// completion counter (reset to zero by the last block).
struct Reduce {
  double *partials = nullptr;   // NV per block, then NV per group of 1024 blocks
  unsigned int *counter = nullptr;   // [0]: blocks or groups done; [1 + g]: group g
  int64_t capacity = 0;       // doubles in partials
  // Sharded solve: the last block stores this rank's totals here instead of
  // applying the scalar step, which launch_finish applies after the totals
  // were summed over the ranks.
  double *defer = nullptr;
};

// Which scalar a finished reduction updates.
enum Finish : int {
  FIN_STORE = 0,     // out[0..] = totals
  FIN_CG_INIT = 1,   // normr = normr0 = sqrt(total), k = 1, done test
  FIN_CG_RZ = 2,     // rtz (and zAp) -> beta
  FIN_CG_PAP = 3,    // pAp -> alpha
  FIN_CG_RR = 4,     // normr, k++, done test
  FIN_MAX = 5,       // out[0] = max (infinity-norm reductions)
};

// GS_SYM3: class 3's forward half sweep fused with the backward half sweep that
// follows it (one launch; combines with GS_ZERO_GUESS for the first sweep).
enum GsMode : int {
  GS_PLAIN = 0,
  GS_ZERO_GUESS = 1,
  GS_RESTRICT = 2,
  GS_PROLONG = 4,
  GS_SYM3 = 8,
  // internal to the kernels: the FP64 sweeps derive their columns from the
  // stencil offsets (LevelDev::stencil_cols)
  GS_STENCIL = 32
};

// Layout / set-up ---------------------------------------------------------
void plan_level(LevelDev &L, int nx, int ny, int nz);
int64_t storage_row_host(const LevelDev &L, int64_t row);
int launch_generate_hpcg(const LevelDev &L, cudaStream_t s);
int launch_generate_varcoef(const LevelDev &L, int level, int nx0, int ny0, uint64_t seed,
                             double sigma, cudaStream_t s);
int launch_coarsen_varcoef(const LevelDev &F, const LevelDev &Cc, cudaStream_t s);
int launch_to_bf16(const LevelDev &L, cudaStream_t s);
int launch_set_values(const LevelDev &L, const double *vals27, cudaStream_t s);
int launch_get_values(const LevelDev &L, double *vals27, int32_t *cols27, cudaStream_t s);
int launch_set_diagonal(const LevelDev &L, const double *diag, cudaStream_t s);
int launch_get_diagonal(const LevelDev &L, double *diag, cudaStream_t s);

// Operators ---------------------------------------------------------------
// implicit_cols: columns from the stencil offsets (no int32 column reads).
int launch_spmv(const LevelDev &L, const double *x, double *y, const Reduce *dot, int fin,
                 void *fin_target, const int *done, cudaStream_t s, bool implicit_cols = false);
int launch_spmv32(const LevelDev &L, const float *x, float *y, cudaStream_t s);
// One class launch of a Gauss-Seidel half sweep over lines [jbeg, jend) of
// the class (default: all).  T = double (FP64 values and vectors) or float
// (BF16 values, FP32 vectors); RT is the right-hand side type.
template <class T, class RT>
int launch_gs_class(const LevelDev &L, int q, int backward, int mode, const RT *r, T *x,
                     const T *xc, T *rc, const int *done, cudaStream_t s, int jbeg = 0,
                     int jend = -1);


// Vectors -----------------------------------------------------------------
int launch_waxpby(int64_t n, double alpha, const double *x, double beta, const double *y,
                   double *w, const int *done, cudaStream_t s);
int launch_dot(int64_t n, const double *x, const double *y, const Reduce &red, double *out,
                cudaStream_t s);
// x.y followed by the CG scalar step `fin` (skipped once st->done is set).
int launch_dot_finish(int64_t n, const double *x, const double *y, const Reduce &red, int fin,
                      CgState *st, cudaStream_t s);
int launch_absmax_diff(int64_t n, const double *a, const double *b, const Reduce &red,
                        double *out, cudaStream_t s);
int launch_restriction(int64_t nc, const LevelDev &F, const double *rf, const double *Axf,
                        double *rc, cudaStream_t s);
int launch_prolongation(int64_t nc, const LevelDev &F, const double *xc, double *xf,
                         cudaStream_t s);
int launch_copy(int64_t n, const double *x, double *y, const int *done, cudaStream_t s);
int launch_fill_uniform(int64_t n, uint64_t seed, uint64_t offset, double lo, double hi,
                         double *v, cudaStream_t s);
int launch_fill_normal(int64_t n, uint64_t seed, uint64_t offset, double *v, cudaStream_t s);

// CG pieces ---------------------------------------------------------------
// r32 (may be null): also the FP32 copy of r.
int launch_cg_init(int64_t n, const double *b, const double *Ap, double *r, float *r32,
                   const Reduce &red, CgState *st, cudaStream_t s);
// Index-check record of a -DHPCGX_CHECKED build (0 = clean; else site << 56 |
// index of the first bad index), cleared by reading; always 0 otherwise.
// Returns a cudaError_t value.
int read_check_record(unsigned long long *record);
// The scalar step `fin` on nv totals (a deferred reduction, summed over ranks).
int launch_finish(int fin, int nv, const double *tot, CgState *st, cudaStream_t s);
// bufs: device array of nranks pointers to `count` doubles each; every buffer
// receives the sum over the ranks, taken in rank order.
int launch_rank_sum(int nranks, double *const *bufs, int count, cudaStream_t s);
// Standalone restriction of the residual at the injected points,
// rc = rf - (A x) there (src/ComputeSPMV_ref.cpp + src/ComputeRestriction_ref.cpp:51),
// and prolongation xf += xc at the injected points, over the first nc coarse
// points (coarse row order); used where a halo exchange separates them from
// the sweeps.
template <class T, class RT>
int launch_restrict_residual(const LevelDev &F, int64_t nc, const RT *rf, const T *xf, T *rc,
                             const int *done, cudaStream_t s);
template <class T>
int launch_prolong(const LevelDev &F, int64_t nc, const T *xc, T *xf, const int *done,
                   cudaStream_t s);
template <class ZT>
int launch_cg_rz(int64_t n, const double *r, const ZT *z, const double *Ap, const Reduce &red,
                  CgState *st, cudaStream_t s);
template <class ZT>
int launch_cg_p(int64_t n, const ZT *z, double *p, CgState *st, cudaStream_t s,
                double *x = nullptr);
int launch_cg_xflush(int64_t n, const double *p, double *x, const CgState *st, cudaStream_t s);
int launch_cg_xr(int64_t n, const double *p, const double *Ap, double *x, double *r, float *r32,
                 const Reduce &red, CgState *st, cudaStream_t s);
int launch_copy_z(int64_t n, const double *r, double *z, const CgState *st, cudaStream_t s);

// Differentiable solve ----------------------------------------------------
int launch_adjoint_grad(const LevelDev &L, const double *lambda, const double *x, double *grad,
                         cudaStream_t s);

// Reduction helpers -------------------------------------------------------
int vector_blocks(int64_t n);

}  // namespace hpcgx
