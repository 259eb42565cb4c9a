/*
 * hpcgx.h -- C ABI of libhpcgx, the B200 (sm_100a) implementation of HPCG 3.1's
 * multigrid-preconditioned CG iteration.
 *
 * Every function returns an int status: HPCGX_OK (0) on success, non-zero on
 * error, which is the convention of the reference's operator API (callers
 * count errors and carry on, src/main.cpp:190-192).  hpcgx_last_error() gives
 * the message of the last failure on the calling thread.
 *
 * Pointers named *_host are host memory; every other vector pointer is device
 * memory of the problem's GPU.  Vectors are in the reference's natural row
 * order (row = iz*nx*ny + iy*nx + ix).  Calls are synchronous with respect to
 * the host unless stated otherwise.
 *
 * The C++ drop-in files in hpcg_b200/dropin/ implement the reference's
 * replaceable operator files on top of this ABI; each entry below names the
 * reference interface it serves.
 */
#ifndef HPCGX_H
#define HPCGX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HPCGX_OK 0
#define HPCGX_EINVAL 1     /* bad argument or size                       */
#define HPCGX_ECUDA 2      /* a CUDA call failed                          */
#define HPCGX_ESTATE 3     /* call out of order (e.g. no matrix loaded)   */
#define HPCGX_ENONFINITE 4 /* CG met a non-finite residual norm           */
#define HPCGX_ELAYOUT 5    /* matrix is not a 27-point stencil matrix     */
#define HPCGX_ENOMEM 6     /* device allocation failed                    */
#define HPCGX_ECOMM 7      /* a halo exchange or reduction across ranks failed */
#define HPCGX_ETIMEOUT 8   /* sharded work did not finish within HPCGX_WAIT_TIMEOUT_S */
#define HPCGX_ECHECK 9     /* index-checked build: a kernel met an out-of-range index */

#define HPCGX_GEN_HPCG 0    /* the reference problem: 26 / -1 stencil     */
#define HPCGX_GEN_VARCOEF 1 /* variable-coefficient SPD stencil           */

typedef struct hpcgx_problem hpcgx_problem;
typedef struct hpcgx_group hpcgx_group;

const char *hpcgx_last_error(void);
int hpcgx_version(void);
/* Makes `device` the calling thread's device and creates its CUDA context
 * (the process's first CUDA call, about a second), so that a later
 * hpcgx_create finds it ready.  Any thread may call it: the context is
 * shared by the process.  No counterpart in the reference; the drop-in
 * starts it on a thread of its own while the host builds the problem. */
int hpcgx_init_device(int device);

/* ---- problem set-up: OptimizeProblem (src/OptimizeProblem.hpp:22) ------ */

/* Creates the device structures of an nx*ny*nz grid with `levels` multigrid
 * levels (the reference uses 4, src/main.cpp:139; every level but the last
 * needs even dimensions, src/GenerateCoarseProblem.cpp:52).  Allocates the
 * matrix storage and work vectors; no values yet. */
int hpcgx_create(int device, int nx, int ny, int nz, int levels, hpcgx_problem **out);
int hpcgx_destroy(hpcgx_problem *p);

/* Loads one level from a host matrix in the reference's contiguous row
 * layout (src/GenerateProblem_ref.cpp:113-124): row i owns entries
 * [27 i, 27 i + nnz[i]) of cols / vals.  Entries must be stencil neighbours of
 * row i in the level's geometry, in increasing stencil order as the reference
 * generator emits them.  Replaces the data movement of OptimizeProblem. */
int hpcgx_load_level(hpcgx_problem *p, int level, const uint8_t *nnz_host,
                     const int32_t *cols_host, const double *vals_host);
/* Same from the row-pointer arrays a SparseMatrix holds
 * (nonzerosInRow, mtxIndL, matrixValues; src/SparseMatrix.hpp:47-50). */
int hpcgx_load_level_rows(hpcgx_problem *p, int level, const char *nnz_host,
                          const int32_t *const *cols_host, const double *const *vals_host);
/* General-pattern problems.  The reference requires that an implementation
 * work for general unstructured sparse matrices (src/GenerateProblem.cpp:47-49,
 * src/SetupHalo.cpp:45); the loaders above accept only the 27-point stencil
 * matrix whose structure the fast layout uses.  hpcgx_create_general makes a
 * problem that takes each level as given: rows of any pattern (each with a
 * diagonal entry), the injection f2c to the next level (f2c[i] = fine row of
 * coarse row i, nc coarse rows; NULL on the last level), the multicolouring
 * computed from the matrix graph by OptimizeProblem's greedy rule
 * (src/OptimizeProblem.cpp:50-79).  hpcgx_spmv, hpcgx_symgs (colour order),
 * hpcgx_mg, hpcgx_cg (plain and MG), their *_host forms, the diagonal
 * accessors and the vector operators work on it; the mixed solver, the
 * generators, stencil-only operators and sharding return HPCGX_ESTATE.
 * Rows are the SparseMatrix arrays (nonzerosInRow, mtxIndL, matrixValues;
 * src/SparseMatrix.hpp:47-50); a malformed row returns HPCGX_ELAYOUT. */
int hpcgx_create_general(int device, int levels, hpcgx_problem **out);
int hpcgx_load_level_general(hpcgx_problem *p, int level, int64_t nrows, const char *nnz_host,
                             const int32_t *const *cols_host, const double *const *vals_host,
                             const int32_t *f2c_host, int64_t nc);
/* Colours of a level's multicolouring (8 for the stencil layout). */
int hpcgx_colours(hpcgx_problem *p, int level);
/* Checks that a level's injection operator (MGData::f2cOperator,
 * src/MGData.hpp:31) is the geometric injection the kernels use. */
int hpcgx_check_f2c(hpcgx_problem *p, int level, const int32_t *f2c_host, int64_t nc);
/* Writes the matrix of every level on the device: HPCGX_GEN_HPCG is
 * GenerateProblem_ref's matrix (src/GenerateProblem_ref.cpp:152-172) on each
 * level as GenerateCoarseProblem builds it; HPCGX_GEN_VARCOEF draws
 * a_ij = -exp(sigma z), z ~ N(0,1) per edge, diagonal sum|a_ij| + 2 (no
 * reference counterpart). */
int hpcgx_generate(hpcgx_problem *p, int kind, uint64_t seed, double sigma);
/* Builds (or refreshes) the BF16 value copies used by the mixed solver. */
int hpcgx_build_mixed(hpcgx_problem *p);
/* on != 0: the FP64 operators (SpMV, SYMGS, MG, CG) derive every column from
 * the level's stencil offsets instead of reading the int32 column arrays, as
 * the mixed solver always does (no reference counterpart; loaded levels are
 * 27-point stencil matrices, so the results are the same bits).  This is the
 * FP64 solve to compare the mixed one with when only the precision differs.
 * Default off. */
int hpcgx_set_stencil_columns(hpcgx_problem *p, int on);
/* Coherence with ReplaceMatrixDiagonal (src/SparseMatrix.hpp:139-145):
 * writes level `level`'s diagonal from host memory. */
int hpcgx_set_diagonal_host(hpcgx_problem *p, int level, const double *diag_host);
int hpcgx_get_diagonal_host(hpcgx_problem *p, int level, double *diag_host);
/* Level values in natural row order, 27 stencil slots per row
 * (slot (dz+1)*9+(dy+1)*3+(dx+1)); device pointers.  set_values ignores
 * slots without a neighbour; with recoarsen != 0 the coarse levels are
 * rebuilt from the new finest values (variable-coefficient rule). */
int hpcgx_set_values(hpcgx_problem *p, int level, const double *vals27, int recoarsen);
int hpcgx_get_values(hpcgx_problem *p, int level, double *vals27, int32_t *cols27);
/* Device memory held by the problem (OptimizeProblemMemoryUse,
 * src/OptimizeProblem.hpp:28). */
int hpcgx_memory_bytes(hpcgx_problem *p, double *bytes);
int64_t hpcgx_rows(hpcgx_problem *p, int level);

/* ---- operators (device vectors) ---------------------------------------- */

/* ComputeSPMV (src/ComputeSPMV.hpp:20): y = A_level x. */
int hpcgx_spmv(hpcgx_problem *p, int level, const double *x, double *y);
/* y = A_level x in FP64 with every column derived from the stencil offsets
 * (row + offset) instead of read from the int32 column arrays: the outer SpMV
 * of the mixed solver (no reference counterpart).  Loaded matrices are
 * 27-point stencil matrices, so the sums are those of hpcgx_spmv. */
int hpcgx_spmv_stencil(hpcgx_problem *p, int level, const double *x, double *y);
/* ComputeSYMGS (src/ComputeSYMGS.hpp:20): one symmetric Gauss-Seidel sweep in
 * colour order (forward colours 0..7, backward 7..0), x updated in place. */
int hpcgx_symgs(hpcgx_problem *p, int level, const double *r, double *x);
/* ComputeMG (src/ComputeMG.hpp:20): one V-cycle from the finest level,
 * x = M^{-1} r (x is overwritten, not read). */
int hpcgx_mg(hpcgx_problem *p, const double *r, double *x);
/* ComputeRestriction_ref / ComputeProlongation_ref
 * (src/ComputeRestriction_ref.hpp, src/ComputeProlongation_ref.hpp) of
 * level -> level+1. */
int hpcgx_restriction(hpcgx_problem *p, int level, const double *rf, const double *Axf,
                      double *rc);
int hpcgx_prolongation(hpcgx_problem *p, int level, const double *xc, double *xf);
/* ComputeDotProduct (src/ComputeDotProduct.hpp:18); result to host. */
int hpcgx_dot(hpcgx_problem *p, int64_t n, const double *x, const double *y,
              double *result_host);
/* ComputeWAXPBY (src/ComputeWAXPBY.hpp:18): w = alpha x + beta y. */
int hpcgx_waxpby(hpcgx_problem *p, int64_t n, double alpha, const double *x, double beta,
                 const double *y, double *w);
/* ComputeResidual (src/ComputeResidual.hpp:18): max_i |v1_i - v2_i|. */
int hpcgx_residual(hpcgx_problem *p, int64_t n, const double *v1, const double *v2,
                   double *result_host);

/* Host-buffer forms of the operators above, for callers that hold host
 * vectors (the reference's Vector::values): the inputs are copied to device
 * staging buffers of the problem, the operator runs, and the outputs are
 * copied back.  These serve the drop-in operator files in hpcg_b200/dropin. */
int hpcgx_spmv_host(hpcgx_problem *p, int level, const double *x_host, double *y_host);
int hpcgx_symgs_host(hpcgx_problem *p, int level, const double *r_host, double *x_host);
int hpcgx_mg_host(hpcgx_problem *p, const double *r_host, double *x_host);
int hpcgx_dot_host(hpcgx_problem *p, int64_t n, const double *x_host, const double *y_host,
                   double *result_host);
int hpcgx_waxpby_host(hpcgx_problem *p, int64_t n, double alpha, const double *x_host,
                      double beta, const double *y_host, double *w_host);

/* Mixed-precision operators (BF16 values, FP32 vectors; no reference
 * counterpart): y = A x, one symmetric sweep with an FP64 (r64) or FP32 (r32)
 * right-hand side, and the FP32 V-cycle of an FP64 residual. */
int hpcgx_spmv_mixed(hpcgx_problem *p, int level, const float *x, float *y);
int hpcgx_symgs_mixed(hpcgx_problem *p, int level, const double *r64, const float *r32,
                      float *x);
int hpcgx_mg_mixed(hpcgx_problem *p, const double *r, float *x);

/* Dot product that allocates nothing (no counterpart in the reference).  For
 * callers that may not allocate device memory -- code living inside another
 * framework's memory pool, or latency-critical loops in which cudaMalloc /
 * cudaFree would stall or synchronise the device.  It needs no problem
 * handle: the per-block partial sums live in a fixed 256 KiB array inside the
 * library (present on every GPU that loads the library, until exit).
 *   - n must not exceed HPCGX_DOT_NOALLOC_MAX_N (67,108,864 elements);
 *     larger n returns HPCGX_EINVAL (use hpcgx_dot);
 *   - x, y: device vectors of the current device; result: one device double;
 *   - runs asynchronously on `stream` (NULL: the legacy default stream);
 *   - the first call on a device (and the first after the device's context
 *     was torn down and created again, e.g. by cudaDeviceReset) looks up the
 *     array's device address; make that call before any stream capture on
 *     that device;
 *   - every call shares the one array, so calls that overlap on the GPU (on
 *     different streams, or from several host threads) race and must not be
 *     issued concurrently. */
#define HPCGX_DOT_NOALLOC_MAX_N 67108864LL
int hpcgx_dot_noalloc(int64_t n, const double *x, const double *y, double *result,
                      void *stream);

/* ---- solvers ------------------------------------------------------------ */

/* CG (src/CG.hpp:22-24) on device vectors: b read, x initial guess in and
 * solution out; stops when normr/normr0 <= tolerance or after max_iter
 * iterations.  times[0] += wall time, times[2] += vector ops, times[3] +=
 * SpMV, times[5] += preconditioner (CUDA events); NULL is allowed.
 * Returns HPCGX_ENONFINITE if a residual norm became NaN/Inf. */
int hpcgx_cg(hpcgx_problem *p, const double *b, double *x, int max_iter, double tolerance,
             int precond, int *niters, double *normr, double *normr0, double *times);
/* Flexible CG in FP64 with the FP32/BF16 V-cycle as preconditioner and the
 * Polak-Ribiere beta (no reference counterpart). */
int hpcgx_cg_mixed(hpcgx_problem *p, const double *b, double *x, int max_iter,
                   double tolerance, int *niters, double *normr, double *normr0,
                   double *times);
/* The same solves from host buffers (pinned memory gives full copy speed):
 * b_host and x_host are copied to the device, solved, and x copied back.
 * mode: HPCGX_CG_PLAIN (unpreconditioned), HPCGX_CG_MG (FP64 MG-PCG, the
 * reference's CG), HPCGX_CG_MIXED (flexible CG, FP32/BF16 V-cycle). */
#define HPCGX_CG_PLAIN 0
#define HPCGX_CG_MG 1
#define HPCGX_CG_MIXED 2
int hpcgx_cg_host(hpcgx_problem *p, int mode, const double *b_host, double *x_host,
                  int max_iter, double tolerance, int *niters, double *normr,
                  double *normr0, double *times);

/* ---- differentiable solve (no reference counterpart) ------------------- */

/* grad[27 i + s] = -lambda_i x_{col(i,s)} for the finest level, natural row
 * order and stencil slots (0 where the slot has no neighbour): the gradient
 * of L with respect to the stored values when A lambda = dL/dx. */
int hpcgx_adjoint_grad(hpcgx_problem *p, const double *lambda, const double *x, double *grad);

/* ---- seeded inputs ------------------------------------------------------ */

/* v_i = lo + (hi - lo) u(seed, i), u = 53-bit SplitMix64 counter draw. */
int hpcgx_fill_uniform(hpcgx_problem *p, int64_t n, uint64_t seed, double lo, double hi,
                       double *v);
/* v_i = Box-Muller normal of draws 2(offset+i), 2(offset+i)+1. */
int hpcgx_fill_normal(hpcgx_problem *p, int64_t n, uint64_t seed, uint64_t offset, double *v);

/* ---- measurement -------------------------------------------------------- */

#define HPCGX_PROBE_NONE 0
#define HPCGX_PROBE_GS_FINE 1       /* every finest-level Gauss-Seidel class launch     */
#define HPCGX_PROBE_SPMV_FINE 2     /* the CG SpMV (with fused p.Ap)                    */
#define HPCGX_PROBE_GS_FINE_BWD 4   /* finest-level plain backward class launches only  */
/* Brackets the selected launches (a bit mask of the kinds above) inside the
 * solvers' CUDA graphs with CUDA events; hpcgx_probe_read returns, for one
 * kind, their summed device time, launch count and algorithmic bytes
 * (compulsory traffic: real nonzeros, no padding) since the last reset.
 * Events are read at every host check of the solver, so solvers run with one
 * iteration between checks while a probe is set. */
int hpcgx_set_probe(hpcgx_problem *p, int probe_mask);
int hpcgx_probe_read(hpcgx_problem *p, int kind, double *ms, int64_t *launches, double *bytes,
                     int reset);
/* Kernel launches issued by the library on this problem since creation. */
int64_t hpcgx_launch_count(hpcgx_problem *p);
/* Algorithmic bytes of one CG iteration of `mode` (HPCGX_CG_PLAIN / _MG /
 * _MIXED) as this implementation moves them: every launch of the iteration's
 * CUDA graph with the probes' byte model (real nonzeros, each vector element
 * once per launch that reads or writes it).  Available after a solve of that
 * mode on the one-GPU solver; HPCGX_ESTATE before. */
int hpcgx_iteration_bytes(hpcgx_problem *p, int mode, double *bytes);
/* Waits for all work of the problem's stream. */
int hpcgx_synchronize(hpcgx_problem *p);
/* Index-checked build (libhpcgx_checked.so, compiled with -DHPCGX_CHECKED):
 * HPCGX_ECHECK if a kernel has met an out-of-range storage row, vector row
 * or column since the last call (the first one is named in the message; the
 * access itself was redirected into the buffers), else HPCGX_OK.  Synchronises
 * the device.  Always HPCGX_OK in the regular build, which has no checks. */
int hpcgx_check_status(void);

/* ---- sharding over ranks (z-slabs) --------------------------------------
 * The reference's MPI decomposition with a process grid of 1 x 1 x nranks
 * (src/GenerateGeometry.cpp:49-169): rank r owns the planes r*nz .. r*nz+nz-1
 * of an nx x ny x (nz*nranks) grid; every level coarsens its own slab
 * (src/GenerateCoarseProblem.cpp:52).  SpMV and Gauss-Seidel read one halo
 * plane from each neighbouring rank, exchanged where the reference calls
 * ExchangeHalo (src/ExchangeHalo.cpp:34-110: before each SpMV and each
 * SYMGS, src/ComputeSPMV_ref.cpp:55, src/ComputeSYMGS_ref.cpp:56), so the
 * smoother is block Jacobi across ranks as in the reference; every dot
 * product of CG is summed over the ranks (src/ComputeDotProduct_ref.cpp:66-77).
 * Sharded problems are generated on the device (hpcgx_generate, HPCGX_GEN_HPCG);
 * hpcgx_fill_uniform of a finest-level vector fills the rank's part of the
 * global vector. */

/* Creates slab `rank` of `nranks` (nz = planes per rank).  hpcgx_create is
 * hpcgx_create_slab(..., 1, 0, ...). */
int hpcgx_create_slab(int device, int nx, int ny, int nz, int levels, int nranks, int rank,
                      hpcgx_problem **out);
/* One process per GPU: rank 0 makes an NCCL unique id (bytes >= 128), every
 * rank receives it (e.g. through torch.distributed) and attaches.  After
 * that hpcgx_spmv, hpcgx_symgs, hpcgx_mg, hpcgx_cg, hpcgx_cg_mixed and
 * hpcgx_cg_host are collective: every rank calls them with its own vectors.
 * NCCL is loaded at run time (libnccl.so.2); HPCGX_ECOMM if it cannot be. */
int hpcgx_nccl_unique_id(void *id, int bytes);
int hpcgx_attach_nccl(hpcgx_problem *p, const void *id, int bytes);
/* A caller's own transport (MPI, a host channel, ...) instead of NCCL:
 *   halo(ctx, send_lo, recv_lo, send_hi, recv_hi, count, esize, stream)
 *     sends `count` elements of esize bytes at send_lo to the rank below and
 *     receives as many from it into recv_lo, and the same with the rank above
 *     through send_hi / recv_hi (both NULL where there is no such rank); the
 *     pointers are device memory, valid once the work queued on `stream` (a
 *     cudaStream_t) has run;
 *   sum(ctx, buf, count, stream) replaces the `count` device doubles at buf
 *     by their sum over the ranks, every rank receiving the same values.
 * Both return 0 on success; the library turns anything else into
 * HPCGX_ECOMM.  After the call the operators and CG are collective, as with
 * hpcgx_attach_nccl. */
typedef int (*hpcgx_halo_fn)(void *ctx, void *send_lo, void *recv_lo, void *send_hi,
                             void *recv_hi, int64_t count, int esize, void *stream);
typedef int (*hpcgx_sum_fn)(void *ctx, double *buf, int count, void *stream);
int hpcgx_attach_comm(hpcgx_problem *p, hpcgx_halo_fn halo, hpcgx_sum_fn sum, void *ctx);
/* Every rank in one process on one GPU (ranks[r] = slab r of nranks): the
 * ranks run step by step in lockstep on one stream, halo planes are device
 * copies and sums are taken in rank order.  Vector arguments are arrays of
 * one device pointer per rank.  While the group exists its ranks run on the
 * stream of rank 0; hpcgx_group_destroy gives every rank its stream back. */
int hpcgx_group_create(hpcgx_problem *const *ranks, int nranks, hpcgx_group **out);
int hpcgx_group_destroy(hpcgx_group *g);
int hpcgx_group_spmv(hpcgx_group *g, int level, const double *const *x, double *const *y);
int hpcgx_group_symgs(hpcgx_group *g, int level, const double *const *r, double *const *x);
int hpcgx_group_mg(hpcgx_group *g, const double *const *r, double *const *x);
/* mode: HPCGX_CG_PLAIN / HPCGX_CG_MG / HPCGX_CG_MIXED as for hpcgx_cg_host. */
int hpcgx_group_cg(hpcgx_group *g, int mode, const double *const *b, double *const *x,
                   int max_iter, double tolerance, int *niters, double *normr, double *normr0);
/* Makes the library launch on `stream` (a cudaStream_t of the problem's
 * device, not the legacy default stream, since solvers capture CUDA graphs);
 * NULL returns to the problem's own stream.  Lets a caller order library
 * work with its own kernels and time it with events on that stream. */
int hpcgx_set_stream(hpcgx_problem *p, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* HPCGX_H */
