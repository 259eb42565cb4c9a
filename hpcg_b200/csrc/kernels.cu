// kernels.cu -- the sm_100a kernels of libhpcgx.
//
// All kernels are HBM-bandwidth bound (no step of HPCG's PCG iteration is a
// dense contraction, so nothing here uses tensor cores).  The design points:
//   * stencil rows are walked by x-line classes (fixed iy&1, iz&1): a CTA owns
//     whole x-lines and treats the even-x rows, then the odd-x rows of those
//     lines, so the vector sectors a line touches are completed by one CTA
//     while they sit in L2;
//   * a Gauss-Seidel half sweep is ONE launch per class: the two colours of a
//     class only depend on each other along x inside a line, so a
//     __syncthreads between them replaces a second launch; the last class's
//     forward and backward half sweeps are one launch too (its last colour's
//     backward update follows its forward update from registers), so a
//     symmetric sweep is 7 launches instead of 16;
//   * restriction (src/ComputeRestriction_ref.cpp:51) is fused into the last
//     colour of the pre-smoother's backward sweep and prolongation
//     (src/ComputeProlongation_ref.cpp:49) into the first colour of the
//     post-smoother's forward sweep: the injected points are exactly colour 0;
//   * the first forward sweep of ComputeMG starts from x = 0
//     (src/ComputeMG_ref.cpp:42) and skips every term that multiplies a zero;
//   * reductions are deterministic: fixed per-block partials, then the last
//     block to finish sums them in index order and applies the CG scalar
//     update, so alpha/beta never leave the device.
#include "kernels.cuh"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <type_traits>

namespace hpcgx {

namespace {

constexpr int kThreads = 256;

// ---------------------------------------------------------------- reductions

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <bool MAX>
__device__ __forceinline__ double warp_red(double v) {
  return MAX ? warp_max(v) : warp_sum(v);
}

// Sums (or maxes) `count` partials p[0], p[stride], ... over the block in a
// fixed order (strided per thread, warp tree, warps in order); the result is
// valid in every thread.
template <int NV, bool MAX>
__device__ void block_sum_partials(const double *p, int64_t count, int64_t stride,
                                   double (&out)[NV], double (&sh)[NV][32]) {
  __shared__ double res[NV];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double t = 0.0;
    for (int64_t b = threadIdx.x; b < count; b += blockDim.x) {
      const double q = __ldcg(p + (int64_t)i * stride + b);
      t = MAX ? fmax(t, q) : t + q;
    }
    t = warp_red<MAX>(t);
    __syncthreads();
    if (lane == 0) sh[i][wid] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s = MAX ? fmax(s, sh[i][w]) : s + sh[i][w];
      res[i] = s;
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < NV; ++i) out[i] = res[i];
}

// Reduces NV values over the block and publishes one partial per block; the
// last block to arrive returns true with the totals in tot (valid in every
// thread of that block).  Up to kReduceGroup blocks the last block sums the
// partials in block order.  Larger grids (the SpMV's one block per line
// group) reduce in two levels so that no counter takes more than
// kReduceGroup atomics and no block reads more than that many partials: the
// last block of each group of kReduceGroup sums its group's partials in block
// order, and the last group sums the group totals in group order.
// Deterministic for a fixed grid size either way.
constexpr int kReduceGroup = 1024;
template <int NV, bool MAX = false>
__device__ bool grid_reduce(double (&v)[NV], const Reduce &red, double (&tot)[NV]) {
  __shared__ double sh[NV][32];
  __shared__ int amlast;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  const int64_t G = gridDim.x;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double t = warp_red<MAX>(v[i]);
    if (lane == 0) sh[i][wid] = t;
  }
  __syncthreads();
  const int64_t ngroups = (G + kReduceGroup - 1) / kReduceGroup;
  const int64_t group = blockIdx.x / kReduceGroup;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double t = 0.0;
      for (int w = 0; w < nw; ++w) t = MAX ? fmax(t, sh[i][w]) : t + sh[i][w];
      red.partials[(int64_t)i * G + blockIdx.x] = t;
    }
    __threadfence();
    const int64_t gsize = ngroups == 1 ? G : min((int64_t)kReduceGroup, G - group * kReduceGroup);
    unsigned int *ctr = ngroups == 1 ? red.counter : red.counter + 1 + group;
    const unsigned int prev = atomicAdd(ctr, 1u);
    amlast = (prev == gsize - 1);
  }
  __syncthreads();
  if (!amlast) return false;
  __threadfence();
  if (ngroups == 1) {
    block_sum_partials<NV, MAX>(red.partials, G, G, tot, sh);
    if (threadIdx.x == 0) *red.counter = 0u;
    return true;
  }
  // last block of its group: the group's total, then the group-level count
  const int64_t base = group * kReduceGroup;
  const int64_t gsize = min((int64_t)kReduceGroup, G - base);
  double gt[NV];
  block_sum_partials<NV, MAX>(red.partials + base, gsize, G, gt, sh);
  double *gp = red.partials + (int64_t)NV * G;   // group totals
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) gp[(int64_t)i * ngroups + group] = gt[i];
    red.counter[1 + group] = 0u;
    __threadfence();
    const unsigned int prev = atomicAdd(red.counter, 1u);
    amlast = (prev == ngroups - 1);
  }
  __syncthreads();
  if (!amlast) return false;
  __threadfence();
  block_sum_partials<NV, MAX>(gp, ngroups, ngroups, tot, sh);
  if (threadIdx.x == 0) *red.counter = 0u;
  return true;
}

// The scalar step that follows a reduction (done by one thread of the last
// block).  The formulas are CG's (src/CG.cpp:93-124).
template <int NV>
__device__ void finish(int fin, void *target, const double (&tot)[NV]) {
  if (fin == FIN_STORE || fin == FIN_MAX) {
    double *o = static_cast<double *>(target);
    for (int i = 0; i < NV; ++i) o[i] = tot[i];
    return;
  }
  CgState *st = static_cast<CgState *>(target);
  switch (fin) {
    case FIN_CG_INIT:
      st->normr = sqrt(tot[0]);
      st->normr0 = st->normr;
      st->k = 1;
      st->niters = 0;
      st->nonfinite = !isfinite(st->normr);
      st->done = !(st->normr / st->normr0 > st->tol) || st->max_iter < 1 || st->nonfinite;
      break;
    case FIN_CG_RZ:
      if (st->k == 1) {
        st->rtz = tot[0];
      } else {
        st->oldrtz = st->rtz;
        st->rtz = tot[0];
        if (st->flexible) {
          st->zAp = tot[NV > 1 ? 1 : 0];
          st->beta = -st->zAp / st->pAp;
        } else {
          st->beta = st->rtz / st->oldrtz;
        }
      }
      break;
    case FIN_CG_PAP:
      st->pAp = tot[0];
      st->alpha = st->rtz / st->pAp;
      break;
    case FIN_CG_RR:
      st->normr = sqrt(tot[0]);
      st->niters = st->k;
      st->k += 1;
      st->nonfinite = !isfinite(st->normr);
      st->done = !(st->normr / st->normr0 > st->tol) || st->k > st->max_iter || st->nonfinite;
      break;
    default:
      break;
  }
}

// Applies the scalar step, or (sharded solve) stores this rank's totals for
// the sum over the ranks that precedes it.
template <int NV>
__device__ void finish_or_defer(const Reduce &red, int fin, void *target, const double (&tot)[NV]) {
  if (red.defer) {
    for (int i = 0; i < NV; ++i) red.defer[i] = tot[i];
    return;
  }
  finish<NV>(fin, target, tot);
}

template <int NV>
__global__ void k_finish(int fin, const double *__restrict__ tot, CgState *st) {
  double t[NV];
  for (int i = 0; i < NV; ++i) t[i] = tot[i];
  finish<NV>(fin, st, t);
}

// Sum over the ranks of an in-process group, in rank order, written back to
// every rank's buffer.
__global__ void k_rank_sum(int nranks, double *const *bufs, int count) {
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    double s = 0.0;
    for (int r = 0; r < nranks; ++r) s += bufs[r][i];
    for (int r = 0; r < nranks; ++r) bufs[r][i] = s;
  }
}

// ---------------------------------------------------------------- index checks

// Built with -DHPCGX_CHECKED (libhpcgx_checked.so), the row kernels verify
// every storage row, vector row and gathered column before using it; a bad
// one is recorded (the first, as site << 56 | index) and replaced by index 0,
// which is always inside the buffers, so nothing outside them is touched.
// hpcgx_check_status() reports and clears the record.  The stand-in for a
// memory checker; without the macro the checks compile to nothing.
#ifdef HPCGX_CHECKED
__device__ unsigned long long g_check_record = 0ull;
__device__ __noinline__ void check_fail(int site, int64_t index) {
  atomicCAS(&g_check_record, 0ull,
            ((unsigned long long)site << 56) | ((unsigned long long)index & ((1ull << 56) - 1)));
}
#endif

struct RowId;
template <class VT>
__device__ __forceinline__ void check_row(const LevelMat<VT> &A, RowId &id, int site);
template <class VT, class NEED>
__device__ __forceinline__ void check_cols(const LevelMat<VT> &A, int32_t *col, NEED need,
                                           int site);
__device__ __forceinline__ int64_t check_index(int64_t i, int64_t n, int site) {
#ifdef HPCGX_CHECKED
  if (i < 0 || i >= n) {
    check_fail(site, i);
    return 0;
  }
#endif
  return i;
}

// ---------------------------------------------------------------- geometry

struct ClassSet {
  ClassInfo c[4];
  int lpb[4];      // lines per block
  int nblk[4];     // blocks of each class
  int common;      // min over the classes of nblk
  int total;       // sum of nblk: the grid
};

// Block g of a launch over all four classes -> (class, block inside the
// class).  The classes are interleaved round-robin (block b of class q is
// launch block 4 b + q) so that the four classes walk up the z-planes
// together and a plane of x is still in L2 when the next class reads it;
// blocks beyond the smallest class's count follow class by class.
__device__ __forceinline__ void class_block(const ClassSet &cs, int g, int &q, int &b) {
  if (g < 4 * cs.common) {
    q = g & 3;
    b = g >> 2;
    return;
  }
  g -= 4 * cs.common;
  q = 0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const int extra = cs.nblk[q] - cs.common;
    if (g < extra) break;
    g -= extra;
    ++q;
  }
  b = cs.common + g;
}

// Row handled by thread-slot t of half px in a block that owns lines [j0, ...).
struct RowId {
  int64_t row;   // natural index
  int64_t k;     // storage row
  int ix, iy, iz;
};

template <class VT>
__device__ __forceinline__ void check_row(const LevelMat<VT> &A, RowId &id, int site) {
#ifdef HPCGX_CHECKED
  if (id.row < 0 || id.row >= A.n) {
    check_fail(site, id.row);
    id.row = 0;
  }
  if (id.k < 0 || id.k >= A.srows) {
    check_fail(site, id.k);
    id.k = 0;
  }
#endif
}

template <class VT, class NEED>
__device__ __forceinline__ void check_cols(const LevelMat<VT> &A, int32_t *col, NEED need,
                                           int site) {
#ifdef HPCGX_CHECKED
#pragma unroll
  for (int s = 0; s < HPCGX_STENCIL; ++s)
    if (need(s) && (uint32_t)(col[s] - A.lo) >= (uint32_t)A.span) {
      check_fail(site, col[s]);
      col[s] = 0;
    }
#endif
}

__device__ __forceinline__ RowId row_of(const ClassInfo &C, int nx, int ny, int px, int j0,
                                        int t) {
  const int Lp = C.len[px];
  const int jl = (int)fdiv((uint32_t)t, C.dlen[px]);
  const int pos = t - jl * Lp;
  const int j = j0 + jl;
  const int jz = (int)fdiv((uint32_t)j, C.dnyq);
  RowId r;
  r.iy = C.py + 2 * (j - jz * C.nyq);
  r.iz = C.pz + 2 * jz;
  r.ix = px + 2 * pos;
  r.row = ((int64_t)r.iz * ny + r.iy) * nx + r.ix;
  r.k = C.start[px] + (int64_t)j * Lp + pos;
  return r;
}

// ---------------------------------------------------------------- row loads

// Vector loads of one stencil z-plane (9 slots) of storage row k; a group is
// loaded only if need(s) holds for one of its slots (need folds to a
// constant in every kernel, so skipped groups cost nothing).
template <class NEED>
__device__ __forceinline__ void load_plane(const double *__restrict__ vals, int64_t k, int p,
                                           NEED need, double *v) {
  const double *q = vals + (k >> 5) * kSliceElems + p * kPlaneElems;
  const int lane = (int)(k & 31);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (need(9 * p + 2 * j) || need(9 * p + 2 * j + 1)) {
      const double2 t = __ldg(reinterpret_cast<const double2 *>(q + j * 64 + lane * 2));
      v[2 * j] = t.x;
      v[2 * j + 1] = t.y;
    }
  }
  if (need(9 * p + 8)) v[8] = __ldg(q + 256 + lane);
}

template <class NEED>
__device__ __forceinline__ void load_plane(const uint16_t *__restrict__ vals, int64_t k, int p,
                                           NEED need, uint16_t *v) {
  const uint16_t *q = vals + (k >> 5) * kSliceElems + p * kPlaneElems;
  const int lane = (int)(k & 31);
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    if (need(9 * p + 4 * j) || need(9 * p + 4 * j + 1) || need(9 * p + 4 * j + 2) ||
        need(9 * p + 4 * j + 3)) {
      const uint2 t = __ldg(reinterpret_cast<const uint2 *>(q + j * 128 + lane * 4));
      v[4 * j] = (uint16_t)(t.x & 0xffffu);
      v[4 * j + 1] = (uint16_t)(t.x >> 16);
      v[4 * j + 2] = (uint16_t)(t.y & 0xffffu);
      v[4 * j + 3] = (uint16_t)(t.y >> 16);
    }
  }
  if (need(9 * p + 8)) v[8] = __ldg(q + 256 + lane);
}

template <class NEED>
__device__ __forceinline__ void load_plane(const int32_t *__restrict__ cols, int64_t k, int p,
                                           NEED need, int32_t *c) {
  const int32_t *q = cols + (k >> 5) * kSliceElems + p * kPlaneElems;
  const int lane = (int)(k & 31);
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    if (need(9 * p + 4 * j) || need(9 * p + 4 * j + 1) || need(9 * p + 4 * j + 2) ||
        need(9 * p + 4 * j + 3)) {
      const int4 t = __ldg(reinterpret_cast<const int4 *>(q + j * 128 + lane * 4));
      c[4 * j] = t.x;
      c[4 * j + 1] = t.y;
      c[4 * j + 2] = t.z;
      c[4 * j + 3] = t.w;
    }
  }
  if (need(9 * p + 8)) c[8] = __ldg(q + 256 + lane);
}

// BF16 values of one z-plane straight to FP32 (a BF16 pattern is the high
// half of the FP32 pattern of the same number).
template <class NEED>
__device__ __forceinline__ void load_plane_f32(const uint16_t *__restrict__ vals, int64_t k, int p,
                                               NEED need, float *v) {
  const uint16_t *q = vals + (k >> 5) * kSliceElems + p * kPlaneElems;
  const int lane = (int)(k & 31);
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    if (need(9 * p + 4 * j) || need(9 * p + 4 * j + 1) || need(9 * p + 4 * j + 2) ||
        need(9 * p + 4 * j + 3)) {
      const uint2 t = __ldg(reinterpret_cast<const uint2 *>(q + j * 128 + lane * 4));
      v[4 * j] = __uint_as_float(t.x << 16);
      v[4 * j + 1] = __uint_as_float(t.x & 0xffff0000u);
      v[4 * j + 2] = __uint_as_float(t.y << 16);
      v[4 * j + 3] = __uint_as_float(t.y & 0xffff0000u);
    }
  }
  if (need(9 * p + 8)) v[8] = __uint_as_float((uint32_t)__ldg(q + 256 + lane) << 16);
}
template <class NEED>
__device__ __forceinline__ void load_vals(const double *__restrict__ vals, int64_t k, int p,
                                          NEED need, double *v) {
  load_plane(vals, k, p, need, v);
}
template <class NEED>
__device__ __forceinline__ void load_vals(const uint16_t *__restrict__ vals, int64_t k, int p,
                                          NEED need, float *v) {
  load_plane_f32(vals, k, p, need, v);
}

struct NeedAll {
  __device__ constexpr bool operator()(int) const { return true; }
};

// ---------------------------------------------------------------- SpMV

// Columns of storage row id derived from the stencil offsets, row + off[s] in
// 32-bit arithmetic (vectors hold fewer than 2^31 rows).  Every level matrix
// is a 27-point stencil matrix (the loaders reject any other pattern) whose
// absent neighbours hold the value 0 and the row itself as column, so the
// stored int32 columns carry no information: an interior row reads exactly
// row + off[s].  A slot of a boundary row without a neighbour multiplies its
// x entry by 0.  EXACT takes the row itself for every such slot, as the
// stored columns do: the Gauss-Seidel sweeps need it, since another block of
// the same launch may write some rows for the first time (x there may hold
// anything, NaN included) while this row's own entry is written already, and
// it also keeps their gathers on lines the row reads anyway.  The SpMV reads
// a fully written x, where any entry serves: it keeps row + off[s] where that
// lies inside the vector and takes the row itself elsewhere (one compare per
// slot, fewer instructions than the exact test).
template <bool EXACT, class VT, class NEED>
__device__ __forceinline__ void stencil_cols(const LevelMat<VT> &A, const RowId &id, NEED need,
                                             int32_t *col) {
  const int r32 = (int)id.row;
  const bool xm = id.ix > 0, xp = id.ix + 1 < A.nx, ym = id.iy > 0, yp = id.iy + 1 < A.ny,
             zm = id.iz > 0 || A.zlo, zp = id.iz + 1 < A.nz || A.zhi;
  if (xm && xp && ym && yp && zm && zp) {
#pragma unroll
    for (int s = 0; s < HPCGX_STENCIL; ++s)
      if (need(s)) col[s] = r32 + A.off[s];
  } else if (EXACT) {
#pragma unroll
    for (int s = 0; s < HPCGX_STENCIL; ++s)
      if (need(s)) {
        const int dx = s % 3 - 1, dy = (s / 3) % 3 - 1, dz = s / 9 - 1;
        const bool nb = (dx < 0 ? xm : dx > 0 ? xp : true) && (dy < 0 ? ym : dy > 0 ? yp : true) &&
                        (dz < 0 ? zm : dz > 0 ? zp : true);
        col[s] = nb ? r32 + A.off[s] : r32;
      }
  } else {
#pragma unroll
    for (int s = 0; s < HPCGX_STENCIL; ++s)
      if (need(s)) {
        const int cc = r32 + A.off[s];
        col[s] = (uint32_t)(cc - A.lo) < (uint32_t)A.span ? cc : r32;
      }
  }
}

// y = A x, rows summed left to right over the slots as ComputeSPMV_ref does
// (src/ComputeSPMV_ref.cpp:64-70).  With DOT, also reduces sum_i x_i y_i (the
// p.Ap of CG, src/CG.cpp:119) and runs the finishing scalar step.  IMPL
// derives the columns from the stencil offsets instead of reading them.
// Occupancy: with stored columns a row keeps 54 loads in flight and two
// blocks per SM saturate HBM; without column loads the gathers issue at once
// and three blocks per SM (80 registers) hide their latency best (measured at
// 512^3: 4.60 ms against 5.06 ms at four blocks and 5.80 ms at five).
template <bool IMPL>
constexpr int spmv_min_blocks() { return IMPL ? 3 : 2; }

template <class VT, class T, bool DOT, bool IMPL>
__global__ void __launch_bounds__(kThreads, spmv_min_blocks<IMPL>())
k_spmv(LevelMat<VT> A, ClassSet cs, const T *__restrict__ x, T *__restrict__ y, Reduce red,
       int fin, void *fin_target, const int *__restrict__ done) {
  if (done && *done) return;
  int q, b;
  class_block(cs, (int)blockIdx.x, q, b);
  const ClassInfo &C = cs.c[q];
  const int j0 = b * cs.lpb[q];
  const int j1 = min(j0 + cs.lpb[q], C.lines);
  double acc = 0.0;
  for (int px = 0; px < 2; ++px) {
    const int cnt = (j1 - j0) * C.len[px];
    for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
      RowId id = row_of(C, A.nx, A.ny, px, j0, t);
      check_row(A, id, 1);
      int32_t col[HPCGX_STENCIL];
      VT val[HPCGX_STENCIL];
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        if (!IMPL) load_plane(A.cols, id.k, p, NeedAll(), col + 9 * p);
        load_plane(A.vals, id.k, p, NeedAll(), val + 9 * p);
      }
      if (IMPL) stencil_cols<false>(A, id, NeedAll(), col);
      check_cols(A, col, NeedAll(), 2);
      T xv[HPCGX_STENCIL];
#pragma unroll
      for (int s = 0; s < HPCGX_STENCIL; ++s) xv[s] = __ldg(x + col[s]);
      T sum = T(0);
#pragma unroll
      for (int s = 0; s < HPCGX_STENCIL; ++s) sum = mac_add(sum, to_arith(val[s], T()), xv[s]);
      const T xrow = xv[HPCGX_DIAG_SLOT];
      y[id.row] = sum;
      if (DOT) acc += (double)xrow * (double)sum;
    }
  }
  if (DOT) {
    double v[1] = {acc}, tot[1];
    if (grid_reduce<1>(v, red, tot) && threadIdx.x == 0)
      finish_or_defer<1>(red, fin, fin_target, tot);
  }
}

// ---------------------------------------------------------------- Gauss-Seidel

// One Gauss-Seidel row update, src/ComputeSYMGS_ref.cpp:72-80:
//   sum = r_i - sum_j a_ij x_j (diagonal included, slot order); sum += x_i a_ii;
//   x_i = sum / a_ii.
// The loads are issued in three stages (every column and value, then every
// neighbour of x, then the arithmetic) so that a thread keeps ~54 independent
// loads in flight instead of walking a chain of dependent ones.
// ZERO: x is known to be zero for every colour above c and for row i itself
//       (first forward sweep after ZeroVector); those terms, and the padding
//       slots (column = row), are skipped.  Skipping a product with a zero
//       changes nothing but possibly the sign of an exact zero.
// PRO:  x_i first receives the prolongated coarse correction (colour 0) --
//       except in the first plane of a slab with a halo below, whose
//       correction is added before the halo exchange (the slab below reads
//       that plane).
// RES:  after the update, the fine residual at this injected point is formed
//       and restricted: rc = r_i - (A x)_i with (A x)_i summed as in SpMV.
//       (A slab with a halo below forms its first plane's again once the
//       halo holds the slab below's smoothed values.)
// SYM:  forward update of a row of the last colour, immediately followed by
//       its backward update (the first step of the backward sweep): between
//       the two only x_i changes, so the backward value is recomputed from the
//       same registers and only that value is stored.
template <bool ZERO, bool PRO, bool RES, bool SYM = false, bool STN = false, class VT, class T,
          class RT>
__device__ __forceinline__ void gs_row(const LevelMat<VT> &A, const RowId &id0, int c,
                                       const RT *__restrict__ r, T *x, const T *__restrict__ xc,
                                       T *__restrict__ rc) {
  RowId id = id0;
  check_row(A, id, 3);
  int32_t col[HPCGX_STENCIL];
  T val[HPCGX_STENCIL];   // values converted to the arithmetic type as loaded
  // slots whose neighbour is read: all, or (zero guess) the lower colours
  auto need = [c](int s) { return !ZERO || s == HPCGX_DIAG_SLOT || ((c ^ slot_mask(s)) < c); };
  // The mixed V-cycle (BF16 values) derives its columns from the stencil
  // offsets; the FP64 path reads the stored int32 columns, or derives them
  // too (STN, the FP64 solve with stencil columns).
  constexpr bool IMPLICIT = STN || std::is_same<VT, uint16_t>::value;
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    load_vals(A.vals, id.k, p, need, val + 9 * p);
    if (!IMPLICIT) load_plane(A.cols, id.k, p, need, col + 9 * p);
  }
  if (IMPLICIT) stencil_cols<true>(A, id, need, col);
  check_cols(A, col, need, 4);
  const T rhs = vec_to(__ldg(r + id.row), T());
  int64_t crow = 0;
  if (PRO || RES) {
    const int nxc = A.nx >> 1, nyc = A.ny >> 1;
    crow = ((int64_t)(id.iz >> 1) * nyc + (id.iy >> 1)) * nxc + (id.ix >> 1);
    crow = check_index(crow, (int64_t)nxc * nyc * (A.nz >> 1), 5);
  }
  T xi = ZERO ? T(0) : x[id.row];
  if (PRO && !(A.zlo && id.iz == 0)) xi = rn_add(xi, __ldg(xc + crow));
  // A slot without a neighbour holds value 0 and the row itself as column; in
  // the zero-guess sweep x_i is unwritten, so that term -- a product with 0 --
  // is skipped below.  The gather itself does not wait for the value: every
  // column is in range.
  T xv[HPCGX_STENCIL];
#pragma unroll
  for (int s = 0; s < HPCGX_STENCIL; ++s) {
    if (s == HPCGX_DIAG_SLOT) continue;
    if (ZERO && ((c ^ slot_mask(s)) > c)) continue;
    xv[s] = x[col[s]];
  }
  T sum = rhs;
  const T d = val[HPCGX_DIAG_SLOT];
#pragma unroll
  for (int s = 0; s < HPCGX_STENCIL; ++s) {
    if (s == HPCGX_DIAG_SLOT) {
      if (!ZERO) sum = mac_sub(sum, d, xi);
      continue;
    }
    if (ZERO && (((c ^ slot_mask(s)) > c) || val[s] == T(0))) continue;
    sum = mac_sub(sum, val[s], xv[s]);
  }
  if (!ZERO) sum = mac_add(sum, xi, d);
  const T xn = rn_div(sum, d);
  if (SYM) {
    T sum2 = rhs;
#pragma unroll
    for (int s = 0; s < HPCGX_STENCIL; ++s) {
      if (s == HPCGX_DIAG_SLOT) {
        sum2 = mac_sub(sum2, d, xn);
        continue;
      }
      if (val[s] == T(0)) continue;   // a product with 0: no change
      sum2 = mac_sub(sum2, val[s], xv[s]);
    }
    sum2 = mac_add(sum2, xn, d);
    x[id.row] = rn_div(sum2, d);
    return;
  }
  x[id.row] = xn;
  if (RES) {
    T ax = T(0);
#pragma unroll
    for (int s = 0; s < HPCGX_STENCIL; ++s)
      ax = mac_add(ax, val[s], s == HPCGX_DIAG_SLOT ? xn : xv[s]);
    rc[crow] = rn_sub(rhs, ax);
  }
}

// One half sweep of class Q over the lines [j0, j1) of the class: colours
// 2Q then 2Q+1 (DIR = 0) or 2Q+1 then 2Q (DIR = 1).  A block owns whole lines,
// so the x-neighbours of a row (the other colour of the class) are its own.
// PRO / RES act on colour 0 only.
template <int MODE, int Q, int DIR, class VT, class T, class RT>
__device__ __forceinline__ void gs_lines(const LevelMat<VT> &A, const ClassInfo &C, int j0, int j1,
                                         const RT *__restrict__ r, T *x,
                                         const T *__restrict__ xc, T *__restrict__ rc) {
  constexpr bool ZERO = (MODE & GS_ZERO_GUESS) != 0, PRO = (MODE & GS_PROLONG) != 0,
                 RES = (MODE & GS_RESTRICT) != 0, STN = (MODE & GS_STENCIL) != 0;
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    const int px = DIR ? 1 - half : half;
    const int c = px + 2 * (Q >= 0 ? Q : C.q);
    const int cnt = (j1 - j0) * C.len[px];
    for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
      const RowId id = row_of(C, A.nx, A.ny, px, j0, t);
      if ((PRO || RES) && c == 0)
        gs_row<ZERO, PRO, RES, false, STN>(A, id, c, r, x, xc, rc);
      else
        gs_row<ZERO, false, false, false, STN>(A, id, c, r, x, xc, rc);
    }
    if (half == 0) __syncthreads();
  }
}

// The last class of a forward sweep fused with the first class of the
// following backward sweep, over the lines [j0, j1) of class 3: colour 6
// forward, colour 7 forward and backward (SYM), colour 6 backward.  Class 3's
// colours only depend on each other along x inside a line, so the block's own
// lines carry every dependency; the matrix rows of the class are read from
// DRAM once instead of twice (colour 6's rows come back from L2 in the last
// phase).
template <int MODE, class VT, class T, class RT>
__device__ __forceinline__ void gs_lines_sym3(const LevelMat<VT> &A, const ClassInfo &C, int j0,
                                              int j1, const RT *__restrict__ r, T *x) {
  constexpr bool ZERO = (MODE & GS_ZERO_GUESS) != 0, STN = (MODE & GS_STENCIL) != 0;
  const int cnt0 = (j1 - j0) * C.len[0], cnt1 = (j1 - j0) * C.len[1];
  for (int t = threadIdx.x; t < cnt0; t += blockDim.x)
    gs_row<ZERO, false, false, false, STN>(A, row_of(C, A.nx, A.ny, 0, j0, t), 6, r, x,
                                           (const T *)nullptr, (T *)nullptr);
  __syncthreads();
  for (int t = threadIdx.x; t < cnt1; t += blockDim.x)
    gs_row<ZERO, false, false, true, STN>(A, row_of(C, A.nx, A.ny, 1, j0, t), 7, r, x,
                                          (const T *)nullptr, (T *)nullptr);
  __syncthreads();
  // Colour 6 backward multiplies every slot; after a zero-guess forward part,
  // rows of colours 6 and 7 in other blocks may still be unwritten, which the
  // exact columns of slots without a neighbour never reach.
  for (int t = threadIdx.x; t < cnt0; t += blockDim.x)
    gs_row<false, false, false, false, STN>(A, row_of(C, A.nx, A.ny, 0, j0, t), 6, r, x,
                                            (const T *)nullptr, (T *)nullptr);
}

// A half sweep over one class, lpb lines per block.  MODE bits:
// GS_ZERO_GUESS for the whole launch; GS_PROLONG and GS_RESTRICT act on
// colour 0 only.  QS >= 0 fixes the class at compile time, which lets the
// zero-guess sweep drop the loads of the skipped slots statically.
// Occupancy: the FP64 sweeps stream 12 B per slot and saturate HBM with two
// 256-thread blocks per SM; the BF16 sweeps read 2 B per slot and are latency
// bound, so they are held to 64 registers for four blocks per SM (five,
// at 48 registers, spill and run slower).
template <class VT>
constexpr int gs_min_blocks() { return std::is_same<VT, uint16_t>::value ? 4 : 2; }

// Lines [jbeg, jend) of the class, lpb per block (a sharded sweep splits its
// first launch into the lines that read no halo plane and the rest).
template <int MODE, int DIR, int QS, class VT, class T, class RT>
__global__ void __launch_bounds__(kThreads, gs_min_blocks<VT>())
k_gs_class(LevelMat<VT> A, ClassInfo C, int lpb, int jbeg, int jend, const RT *__restrict__ r,
           T *x, const T *__restrict__ xc, T *__restrict__ rc, const int *__restrict__ done) {
  if (done && *done) return;
  const int j0 = jbeg + blockIdx.x * lpb;
  const int j1 = min(j0 + lpb, jend);
  gs_lines<MODE, QS, DIR>(A, C, j0, j1, r, x, xc, rc);
}

template <int MODE, class VT, class T, class RT>
__global__ void __launch_bounds__(kThreads, gs_min_blocks<VT>())
k_gs_class3_sym(LevelMat<VT> A, ClassInfo C, int lpb, const RT *__restrict__ r, T *x,
                const int *__restrict__ done) {
  if (done && *done) return;
  const int j0 = blockIdx.x * lpb;
  const int j1 = min(j0 + lpb, C.lines);
  gs_lines_sym3<MODE>(A, C, j0, j1, r, x);
}

// Residual restricted at the injected points (colour 0: even ix, iy, iz):
// rc = rf - (A x) there, (A x)_i summed over the slots from 0 in order as
// ComputeSPMV_ref does (src/ComputeSPMV_ref.cpp:64-70), then
// src/ComputeRestriction_ref.cpp:51.  The standalone form of GS_RESTRICT, for
// the sharded V-cycle, where the halo of x is exchanged between the sweep and
// the residual (src/ComputeMG_ref.cpp:49-51): launched over the first coarse
// plane only (nc = nxc * nyc), the one injected plane that reads the halo.
template <class VT, class T, class RT>
__global__ void __launch_bounds__(kThreads)
k_restrict_residual(LevelMat<VT> A, ClassInfo C0, int64_t nc, const RT *__restrict__ rf,
                    const T *__restrict__ x, T *__restrict__ rc, const int *__restrict__ done) {
  if (done && *done) return;
  constexpr bool IMPLICIT = std::is_same<VT, uint16_t>::value;
  const int nxc = A.nx >> 1, nyc = A.ny >> 1;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nc;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int ixc = (int)(i % nxc), iyc = (int)((i / nxc) % nyc);
    const int izc = (int)(i / ((int64_t)nxc * nyc));
    RowId id;
    id.ix = 2 * ixc;
    id.iy = 2 * iyc;
    id.iz = 2 * izc;
    id.row = ((int64_t)id.iz * A.ny + id.iy) * A.nx + id.ix;
    id.k = C0.start[0] + ((int64_t)izc * C0.nyq + iyc) * C0.len[0] + ixc;  // colour 0
    check_row(A, id, 6);
    int32_t col[HPCGX_STENCIL];
    T val[HPCGX_STENCIL];
#pragma unroll
    for (int p = 0; p < 3; ++p) {
      load_vals(A.vals, id.k, p, NeedAll(), val + 9 * p);
      if (!IMPLICIT) load_plane(A.cols, id.k, p, NeedAll(), col + 9 * p);
    }
    if (IMPLICIT) stencil_cols<true>(A, id, NeedAll(), col);
    check_cols(A, col, NeedAll(), 7);
    T ax = T(0);
#pragma unroll
    for (int s = 0; s < HPCGX_STENCIL; ++s) ax = mac_add(ax, val[s], x[col[s]]);
    rc[i] = rn_sub(vec_to(__ldg(rf + id.row), T()), ax);
  }
}

// xf += xc at the injected points (src/ComputeProlongation_ref.cpp:49), in the
// vector type of the V-cycle.  The sharded V-cycle launches it over the first
// coarse plane only, before the halo exchange; GS_PROLONG adds the rest.
template <class T>
__global__ void __launch_bounds__(kThreads)
k_prolong(int64_t nc, int nxf, int nyf, const T *__restrict__ xc, T *xf,
          const int *__restrict__ done) {
  if (done && *done) return;
  const int nxc = nxf >> 1, nyc = nyf >> 1;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nc;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t ixc = i % nxc, iyc = (i / nxc) % nyc, izc = i / ((int64_t)nxc * nyc);
    const int64_t f = ((2 * izc) * nyf + 2 * iyc) * nxf + 2 * ixc;
    xf[f] = rn_add(xf[f], xc[i]);
  }
}

// ---------------------------------------------------------------- vectors

__global__ void __launch_bounds__(kThreads)
k_waxpby(int64_t n, double alpha, const double *__restrict__ x, double beta,
         const double *__restrict__ y, double *w, const int *__restrict__ done) {
  if (done && *done) return;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  // The three branches of src/ComputeWAXPBY_ref.cpp:52-67 round differently.
  if (alpha == 1.0) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride)
      w[i] = rn_add(x[i], rn_mul(beta, y[i]));
  } else if (beta == 1.0) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride)
      w[i] = rn_add(rn_mul(alpha, x[i]), y[i]);
  } else {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride)
      w[i] = rn_add(rn_mul(alpha, x[i]), rn_mul(beta, y[i]));
  }
}

// x.y; the last block stores the total (FIN_STORE into target) or runs a CG
// scalar step on it (target: the CgState).
__global__ void __launch_bounds__(kThreads)
k_dot(int64_t n, const double *__restrict__ x, const double *__restrict__ y, Reduce red, int fin,
      void *target, const int *__restrict__ done) {
  if (done && *done) return;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride)
    acc += x[i] * y[i];
  double v[1] = {acc}, tot[1];
  if (grid_reduce<1>(v, red, tot) && threadIdx.x == 0) finish_or_defer<1>(red, fin, target, tot);
}

__global__ void __launch_bounds__(kThreads)
k_absmax_diff(int64_t n, const double *__restrict__ a, const double *__restrict__ b, Reduce red,
              double *out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  double m = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride)
    m = fmax(m, fabs(a[i] - b[i]));
  double v[1] = {m}, tot[1];
  if (grid_reduce<1, true>(v, red, tot) && threadIdx.x == 0) out[0] = tot[0];
}

__device__ __forceinline__ int64_t fine_of_coarse(int64_t ic, int nxf, int nyf) {
  const int nxc = nxf >> 1, nyc = nyf >> 1;
  const int64_t ixc = ic % nxc, iyc = (ic / nxc) % nyc, izc = ic / ((int64_t)nxc * nyc);
  return (2 * izc) * (int64_t)nxf * nyf + (2 * iyc) * (int64_t)nxf + 2 * ixc;
}

// src/ComputeRestriction_ref.cpp:51 with f2c of src/GenerateCoarseProblem.cpp:71-82.
__global__ void k_restriction(int64_t nc, int nxf, int nyf, const double *__restrict__ rf,
                              const double *__restrict__ Axf, double *rc) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nc;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t f = fine_of_coarse(i, nxf, nyf);
    rc[i] = rn_sub(rf[f], Axf[f]);
  }
}

// src/ComputeProlongation_ref.cpp:49.
__global__ void k_prolongation(int64_t nc, int nxf, int nyf, const double *__restrict__ xc,
                               double *xf) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nc;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t f = fine_of_coarse(i, nxf, nyf);
    xf[f] = rn_add(xf[f], xc[i]);
  }
}

__global__ void k_copy(int64_t n, const double *__restrict__ x, double *y,
                       const int *__restrict__ done) {
  if (done && *done) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = x[i];
}

__global__ void k_fill_uniform(int64_t n, uint64_t seed, uint64_t offset, double lo, double hi,
                               double *v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    v[i] = rn_add(lo, rn_mul(rn_sub(hi, lo), uniform01(seed, offset + (uint64_t)i)));
}

__device__ __forceinline__ double normal01(uint64_t seed, uint64_t i) {
  const double u1 = 1.0 - uniform01(seed, 2 * i);
  const double u2 = uniform01(seed, 2 * i + 1);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

__global__ void k_fill_normal(int64_t n, uint64_t seed, uint64_t offset, double *v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    v[i] = normal01(seed, offset + (uint64_t)i);
}

// ---------------------------------------------------------------- CG pieces

// r = b - Ap (WAXPBY(1, b, -1, Ap), src/CG.cpp:88) and |r|^2 -> normr0.
__global__ void __launch_bounds__(kThreads)
k_cg_init(int64_t n, const double *__restrict__ b, const double *__restrict__ Ap, double *r,
          float *r32, Reduce red, CgState *st) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    const double ri = rn_add(b[i], rn_mul(-1.0, Ap[i]));
    r[i] = ri;
    if (r32) r32[i] = (float)ri;
    acc += ri * ri;
  }
  double v[1] = {acc}, tot[1];
  if (grid_reduce<1>(v, red, tot) && threadIdx.x == 0)
    finish_or_defer<1>(red, FIN_CG_INIT, st, tot);
}

// rtz = r.z (src/CG.cpp:109/112); for the flexible solver also z.Ap_{k-1}.
template <class ZT, bool FLEX>
__global__ void __launch_bounds__(kThreads)
k_cg_rz(int64_t n, const double *__restrict__ r, const ZT *__restrict__ z,
        const double *__restrict__ Ap, Reduce red, CgState *st) {
  if (st->done) return;
  const bool two = FLEX && st->k > 1;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  double a0 = 0.0, a1 = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    const double zi = (double)z[i];
    a0 += r[i] * zi;
    if (two) a1 += zi * Ap[i];
  }
  if (FLEX) {
    double v[2] = {a0, a1}, tot[2];
    if (grid_reduce<2>(v, red, tot) && threadIdx.x == 0)
      finish_or_defer<2>(red, FIN_CG_RZ, st, tot);
  } else {
    double v[1] = {a0}, tot[1];
    if (grid_reduce<1>(v, red, tot) && threadIdx.x == 0)
      finish_or_defer<1>(red, FIN_CG_RZ, st, tot);
  }
}

// p = z (k == 1) or p = z + beta p (WAXPBY(1, z, beta, p), src/CG.cpp:115).
// With x given, the previous iteration's x += alpha p (src/CG.cpp:121) is
// applied here, while p_{k-1} is read anyway, instead of in k_cg_xr: the same
// operation on the same operands, one read of p fewer per iteration.
// k_cg_xflush applies the last iteration's update after the loop.
template <class ZT>
__global__ void __launch_bounds__(kThreads)
k_cg_p(int64_t n, const ZT *__restrict__ z, double *p, const CgState *__restrict__ st,
       double *x) {
  if (st->done) return;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const bool first = st->k == 1;
  const double beta = st->beta, alpha = st->alpha;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    const double zi = (double)z[i];
    if (first) {
      p[i] = zi;
    } else {
      const double pi = p[i];
      if (x) x[i] = rn_add(x[i], rn_mul(alpha, pi));
      p[i] = rn_add(zi, rn_mul(beta, pi));
    }
  }
}

// The deferred x += alpha p of the last iteration that ran.
__global__ void __launch_bounds__(kThreads)
k_cg_xflush(int64_t n, const double *__restrict__ p, double *x, const CgState *__restrict__ st) {
  if (st->niters < 1) return;
  const double alpha = st->alpha;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] = rn_add(x[i], rn_mul(alpha, p[i]));
}

// x += alpha p (unless deferred: x null); r -= alpha Ap; |r|^2
// (src/CG.cpp:121-124).  r32 (mixed solver): the FP32 copy of r that the
// V-cycle's finest level reads -- the value it would round r to itself.
__global__ void __launch_bounds__(kThreads)
k_cg_xr(int64_t n, const double *__restrict__ p, const double *__restrict__ Ap, double *x,
        double *r, float *r32, Reduce red, CgState *st) {
  if (st->done) return;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const double alpha = st->alpha, malpha = -st->alpha;
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    if (x) x[i] = rn_add(x[i], rn_mul(alpha, p[i]));
    const double ri = rn_add(r[i], rn_mul(malpha, Ap[i]));
    r[i] = ri;
    if (r32) r32[i] = (float)ri;
    acc += ri * ri;
  }
  double v[1] = {acc}, tot[1];
  if (grid_reduce<1>(v, red, tot) && threadIdx.x == 0)
    finish_or_defer<1>(red, FIN_CG_RR, st, tot);
}

__global__ void k_copy_z(int64_t n, const double *__restrict__ r, double *z,
                         const CgState *__restrict__ st) {
  if (st->done) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    z[i] = r[i];
}

// ---------------------------------------------------------------- set-up

struct Geo {
  int nx, ny, nz;
  int zlo, zhi;   // z-slab: the planes below / above belong to a neighbouring rank
  int64_t cstart[8], ccount[8];
  int len[2];
  int nyq[4];
};

__device__ __forceinline__ bool storage_to_natural(const Geo &g, int64_t k, int64_t &row, int &ix,
                                                   int &iy, int &iz) {
  int c = 0;
#pragma unroll
  for (int i = 1; i < 8; ++i)
    if (k >= g.cstart[i]) c = i;
  const int64_t rem = k - g.cstart[c];
  if (rem >= g.ccount[c]) return false;
  const int px = c & 1, q = c >> 1, py = q & 1, pz = q >> 1;
  const int Lp = g.len[px];
  const int64_t j = rem / Lp;
  const int pos = (int)(rem - j * Lp);
  iy = py + 2 * (int)(j % g.nyq[q]);
  iz = pz + 2 * (int)(j / g.nyq[q]);
  ix = px + 2 * pos;
  row = ((int64_t)iz * g.ny + iy) * g.nx + ix;
  return true;
}

__device__ __forceinline__ int64_t natural_to_storage(const Geo &g, int64_t row) {
  const int ix = (int)(row % g.nx);
  const int iy = (int)((row / g.nx) % g.ny);
  const int iz = (int)(row / ((int64_t)g.nx * g.ny));
  const int px = ix & 1, q = (iy & 1) + 2 * (iz & 1);
  const int c = px + 2 * q;
  const int64_t j = (int64_t)(iz >> 1) * g.nyq[q] + (iy >> 1);
  return g.cstart[c] + j * g.len[px] + (ix >> 1);
}

__device__ __forceinline__ bool neighbour(const Geo &g, int ix, int iy, int iz, int s,
                                          int64_t row, int64_t &col) {
  const int dx = s % 3 - 1, dy = (s / 3) % 3 - 1, dz = s / 9 - 1;
  const int jx = ix + dx, jy = iy + dy, jz = iz + dz;
  if (jx < 0 || jx >= g.nx || jy < 0 || jy >= g.ny) return false;
  if ((jz < 0 && !g.zlo) || (jz >= g.nz && !g.zhi)) return false;
  col = row + (int64_t)dz * g.nx * g.ny + (int64_t)dy * g.nx + dx;
  return true;
}

// The reference problem (src/GenerateProblem_ref.cpp:152-172) written
// straight into the device layout: 26 on the diagonal, -1 elsewhere.
__global__ void k_generate_hpcg(Geo g, int64_t storage_rows, double *vals, int32_t *cols) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < storage_rows;
       k += (int64_t)gridDim.x * blockDim.x) {
    int64_t row;
    int ix, iy, iz;
    const bool real = storage_to_natural(g, k, row, ix, iy, iz);
    for (int s = 0; s < HPCGX_STENCIL; ++s) {
      int64_t col = 0;
      double v = 0.0;
      if (real) {
        if (neighbour(g, ix, iy, iz, s, row, col))
          v = (s == HPCGX_DIAG_SLOT) ? 26.0 : -1.0;
        else
          col = row;
      }
      vals[vidx(k, s)] = v;
      cols[cidx(k, s)] = (int32_t)col;
    }
  }
}

// Variable-coefficient SPD matrix (the oracle's or_generate_varcoef): each
// undirected edge {lo, hi} draws z ~ N(0,1) keyed by the finest-level index of
// lo and the direction, a = -exp(sigma z); diagonal = sum |a| + 2.
__global__ void k_generate_varcoef(Geo g, int64_t storage_rows, int level, int nx0, int ny0,
                                   uint64_t seed, double sigma, double *vals, int32_t *cols) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < storage_rows;
       k += (int64_t)gridDim.x * blockDim.x) {
    int64_t row;
    int ix, iy, iz;
    const bool real = storage_to_natural(g, k, row, ix, iy, iz);
    double dsum = 0.0;
    for (int s = 0; s < HPCGX_STENCIL; ++s) {
      int64_t col = 0;
      double v = 0.0;
      if (real) {
        if (neighbour(g, ix, iy, iz, s, row, col)) {
          if (s != HPCGX_DIAG_SLOT) {
            int lx = ix, ly = iy, lz = iz, h = s - 14;
            if (s < HPCGX_DIAG_SLOT) {
              lx = ix + (s % 3 - 1);
              ly = iy + ((s / 3) % 3 - 1);
              lz = iz + (s / 9 - 1);
              h = 12 - s;
            }
            const int64_t lo = ((int64_t)(lz << level) * ny0 + (ly << level)) * nx0 + (lx << level);
            v = -exp(sigma * normal01(seed, (uint64_t)lo * 13u + (uint64_t)h));
            dsum += fabs(v);
          }
        } else {
          col = row;
        }
      }
      vals[vidx(k, s)] = v;
      cols[cidx(k, s)] = (int32_t)col;
    }
    if (real) vals[vidx(k, HPCGX_DIAG_SLOT)] = dsum + 2.0;
  }
}

// Coarse variable-coefficient operator from the fine one: the coarse edge
// {lo, lo+d} takes the fine value of the edge leaving the injected point of lo
// in direction d; the diagonal is again sum |a| + 2.
__global__ void k_coarsen_varcoef(Geo gf, Geo gc, int64_t storage_rows_c,
                                  const double *__restrict__ fvals, double *cvals) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < storage_rows_c;
       k += (int64_t)gridDim.x * blockDim.x) {
    int64_t row;
    int ix, iy, iz;
    if (!storage_to_natural(gc, k, row, ix, iy, iz)) continue;
    double dsum = 0.0;
    for (int s = 0; s < HPCGX_STENCIL; ++s) {
      if (s == HPCGX_DIAG_SLOT) continue;
      int64_t col;
      if (!neighbour(gc, ix, iy, iz, s, row, col)) continue;
      int lx = ix, ly = iy, lz = iz, sl = s;
      if (s < HPCGX_DIAG_SLOT) {
        lx = ix + (s % 3 - 1);
        ly = iy + ((s / 3) % 3 - 1);
        lz = iz + (s / 9 - 1);
        sl = 26 - s;
      }
      const int64_t frow = ((int64_t)(2 * lz) * gf.ny + 2 * ly) * gf.nx + 2 * lx;
      const int64_t fk = natural_to_storage(gf, frow);
      const double v = fvals[vidx(fk, sl)];
      cvals[vidx(k, s)] = v;
      dsum += fabs(v);
    }
    cvals[vidx(k, HPCGX_DIAG_SLOT)] = dsum + 2.0;
  }
}

// BF16 copy of the FP64 values (the two arrays group slots differently).
__global__ void k_to_bf16(int64_t m, const double *__restrict__ v, uint16_t *h) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = i / HPCGX_STENCIL;
    const int s = (int)(i - k * HPCGX_STENCIL);
    h[cidx(k, s)] = bf16_from_double(v[vidx(k, s)]);
  }
}

// Values in natural row order, 27 stencil slots per row -> device layout.
// Slots without a neighbour stay 0 whatever the input holds.
__global__ void k_set_values(Geo g, int64_t n, const double *__restrict__ in, double *vals) {
  for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < n;
       row += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = natural_to_storage(g, row);
    const int ix = (int)(row % g.nx), iy = (int)((row / g.nx) % g.ny),
              iz = (int)(row / ((int64_t)g.nx * g.ny));
    for (int s = 0; s < HPCGX_STENCIL; ++s) {
      int64_t col;
      const bool has = neighbour(g, ix, iy, iz, s, row, col);
      vals[vidx(k, s)] = has ? in[row * HPCGX_STENCIL + s] : 0.0;
    }
  }
}

__global__ void k_get_values(Geo g, int64_t n, const double *__restrict__ vals,
                             const int32_t *__restrict__ cols, double *out, int32_t *cout) {
  for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < n;
       row += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = natural_to_storage(g, row);
    for (int s = 0; s < HPCGX_STENCIL; ++s) {
      if (out) out[row * HPCGX_STENCIL + s] = vals[vidx(k, s)];
      if (cout) cout[row * HPCGX_STENCIL + s] = cols[cidx(k, s)];
    }
  }
}

__global__ void k_set_diagonal(Geo g, int64_t n, const double *__restrict__ d, double *vals) {
  for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < n;
       row += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = natural_to_storage(g, row);
    vals[vidx(k, HPCGX_DIAG_SLOT)] = d[row];
  }
}

__global__ void k_get_diagonal(Geo g, int64_t n, const double *__restrict__ vals, double *d) {
  for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < n;
       row += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = natural_to_storage(g, row);
    d[row] = vals[vidx(k, HPCGX_DIAG_SLOT)];
  }
}

// dL/da_ij = -lambda_i x_j for every stored slot, natural row order, 27 slots
// per row (zero where the stencil has no neighbour).
__global__ void k_adjoint_grad(Geo g, int64_t n, const int32_t *__restrict__ cols,
                               const double *__restrict__ lambda, const double *__restrict__ x,
                               double *grad) {
  for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < n;
       row += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = natural_to_storage(g, row);
    const int ix = (int)(row % g.nx), iy = (int)((row / g.nx) % g.ny),
              iz = (int)(row / ((int64_t)g.nx * g.ny));
    const double li = lambda[row];
    for (int s = 0; s < HPCGX_STENCIL; ++s) {
      int64_t col;
      const bool has = neighbour(g, ix, iy, iz, s, row, col);
      grad[row * HPCGX_STENCIL + s] = has ? -(li * x[__ldg(cols + cidx(k, s))]) : 0.0;
    }
  }
}

Geo geo_of(const LevelDev &L) {
  Geo g;
  g.nx = L.nx;
  g.ny = L.ny;
  g.nz = L.nz;
  g.zlo = L.zlo;
  g.zhi = L.zhi;
  for (int c = 0; c < 8; ++c) {
    g.cstart[c] = L.cstart[c];
    g.ccount[c] = L.ccount[c];
  }
  g.len[0] = L.cls[0].len[0];
  g.len[1] = L.cls[0].len[1];
  for (int q = 0; q < 4; ++q) g.nyq[q] = L.cls[q].nyq;
  return g;
}

int grid_for(int64_t n, int threads = kThreads) {
  int64_t b = (n + threads - 1) / threads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 16));
}

template <class VT>
LevelMat<VT> mat_of(const LevelDev &L, const VT *vals) {
  LevelMat<VT> A;
  A.vals = vals;
  A.cols = L.cols;
  for (int s = 0; s < HPCGX_STENCIL; ++s)
    A.off[s] = (s / 9 - 1) * L.nx * L.ny + ((s / 3) % 3 - 1) * L.nx + (s % 3 - 1);
  A.nx = L.nx;
  A.ny = L.ny;
  A.nz = L.nz;
  A.n = L.n;
  A.zlo = L.zlo;
  A.zhi = L.zhi;
  A.lo = L.zlo ? -L.nx * L.ny : 0;
  A.span = (int)L.n - A.lo + (L.zhi ? L.nx * L.ny : 0);
  A.srows = L.storage_rows;
  return A;
}

// The SpMV's blocks: `groups` Gauss-Seidel line groups per block (the SpMV has
// no colour order, so a block can take several and amortise its epilogue,
// the fused dot product's block reduction).
ClassSet classes_of(const LevelDev &L, int groups = 1) {
  ClassSet cs;
  cs.common = INT_MAX;
  cs.total = 0;
  for (int q = 0; q < 4; ++q) {
    const ClassInfo &C = L.cls[q];
    const int lpb = std::min(L.lines_per_block[q] * groups, std::max(C.lines, 1));
    cs.c[q] = C;
    cs.lpb[q] = lpb;
    cs.nblk[q] = C.lines > 0 ? (C.lines + lpb - 1) / lpb : 0;
    cs.common = std::min(cs.common, cs.nblk[q]);
    cs.total += cs.nblk[q];
  }
  return cs;
}

}  // namespace

// ======================================================================== host
// Every launch_* returns the number of kernels it launched (0 or 1).

int vector_blocks(int64_t n) {
  int64_t b = (n + kThreads * 4 - 1) / (kThreads * 4);
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 8));
}

void plan_level(LevelDev &L, int nx, int ny, int nz) {
  L.nx = nx;
  L.ny = ny;
  L.nz = nz;
  L.n = (int64_t)nx * ny * nz;
  int64_t start = 0;
  for (int c = 0; c < 8; ++c) {
    const int px = c & 1, py = (c >> 1) & 1, pz = (c >> 2) & 1;
    const int64_t cx = (nx - px + 1) / 2, cy = (ny - py + 1) / 2, cz = (nz - pz + 1) / 2;
    L.ccount[c] = cx * cy * cz;
    L.cstart[c] = start;
    start += (L.ccount[c] + 31) / 32 * 32;
  }
  L.storage_rows = start;
  L.spmv_blocks = 0;
  for (int q = 0; q < 4; ++q) {
    ClassInfo &C = L.cls[q];
    C.q = q;
    C.py = q & 1;
    C.pz = q >> 1;
    C.nyq = (ny - C.py + 1) / 2;
    const int nzq = (nz - C.pz + 1) / 2;
    C.lines = C.nyq * nzq;
    C.len[0] = (nx + 1) / 2;
    C.len[1] = nx / 2;
    C.start[0] = L.cstart[2 * q];
    C.start[1] = L.cstart[2 * q + 1];
    C.dlen[0] = make_fastdiv((uint32_t)C.len[0]);
    C.dlen[1] = make_fastdiv((uint32_t)C.len[1]);
    C.dnyq = make_fastdiv((uint32_t)C.nyq);
    const int len = std::max(C.len[0], 1);
    int lpb = std::max(1, kThreads / len);
    lpb = std::min(lpb, std::max(C.lines, 1));
    L.lines_per_block[q] = lpb;
    L.blocks[q] = C.lines > 0 ? (C.lines + lpb - 1) / lpb : 0;
    int th = std::min(kThreads, ((lpb * len) + 31) / 32 * 32);
    L.threads[q] = std::max(th, 32);
    L.spmv_blocks += L.blocks[q];
  }
}

int64_t storage_row_host(const LevelDev &L, int64_t row) {
  const int ix = (int)(row % L.nx), iy = (int)((row / L.nx) % L.ny),
            iz = (int)(row / ((int64_t)L.nx * L.ny));
  const int px = ix & 1, q = (iy & 1) + 2 * (iz & 1), c = px + 2 * q;
  const int64_t j = (int64_t)(iz >> 1) * L.cls[q].nyq + (iy >> 1);
  return L.cstart[c] + j * L.cls[q].len[px] + (ix >> 1);
}

int launch_generate_hpcg(const LevelDev &L, cudaStream_t s) {
  k_generate_hpcg<<<grid_for(L.storage_rows), kThreads, 0, s>>>(geo_of(L), L.storage_rows, L.vals,
                                                                L.cols);
  return 1;
}

int launch_generate_varcoef(const LevelDev &L, int level, int nx0, int ny0, uint64_t seed,
                            double sigma, cudaStream_t s) {
  k_generate_varcoef<<<grid_for(L.storage_rows), kThreads, 0, s>>>(
      geo_of(L), L.storage_rows, level, nx0, ny0, seed, sigma, L.vals, L.cols);
  return 1;
}

int launch_coarsen_varcoef(const LevelDev &F, const LevelDev &Cc, cudaStream_t s) {
  k_coarsen_varcoef<<<grid_for(Cc.storage_rows), kThreads, 0, s>>>(geo_of(F), geo_of(Cc),
                                                                    Cc.storage_rows, F.vals, Cc.vals);
  return 1;
}

int launch_to_bf16(const LevelDev &L, cudaStream_t s) {
  const int64_t m = L.storage_rows * HPCGX_STENCIL;
  k_to_bf16<<<grid_for(m), kThreads, 0, s>>>(m, L.vals, L.vals16);
  return 1;
}

int launch_set_values(const LevelDev &L, const double *vals27, cudaStream_t s) {
  k_set_values<<<grid_for(L.n), kThreads, 0, s>>>(geo_of(L), L.n, vals27, L.vals);
  return 1;
}

int launch_get_values(const LevelDev &L, double *vals27, int32_t *cols27, cudaStream_t s) {
  k_get_values<<<grid_for(L.n), kThreads, 0, s>>>(geo_of(L), L.n, L.vals, L.cols, vals27, cols27);
  return 1;
}

int launch_set_diagonal(const LevelDev &L, const double *diag, cudaStream_t s) {
  k_set_diagonal<<<grid_for(L.n), kThreads, 0, s>>>(geo_of(L), L.n, diag, L.vals);
  return 1;
}

int launch_get_diagonal(const LevelDev &L, double *diag, cudaStream_t s) {
  k_get_diagonal<<<grid_for(L.n), kThreads, 0, s>>>(geo_of(L), L.n, L.vals, diag);
  return 1;
}

int launch_spmv(const LevelDev &L, const double *x, double *y, const Reduce *dot, int fin,
                void *fin_target, const int *done, cudaStream_t s, bool implicit_cols) {
  if (L.spmv_blocks == 0) return 0;
  implicit_cols = implicit_cols || L.stencil_cols;
  // measured at 512^3: two line groups per block help the stencil-column
  // SpMV (4.77 against 5.11 ms with the fused dot product), not the other
  const ClassSet cs = classes_of(L, implicit_cols ? 2 : 1);
  const LevelMat<double> A = mat_of(L, L.vals);
  const Reduce red = dot ? *dot : Reduce();
  if (dot && implicit_cols)
    k_spmv<double, double, true, true><<<cs.total, kThreads, 0, s>>>(A, cs, x, y, red, fin,
                                                                     fin_target, done);
  else if (dot)
    k_spmv<double, double, true, false><<<cs.total, kThreads, 0, s>>>(A, cs, x, y, red, fin,
                                                                      fin_target, done);
  else if (implicit_cols)
    k_spmv<double, double, false, true><<<cs.total, kThreads, 0, s>>>(A, cs, x, y, red, 0,
                                                                      nullptr, done);
  else
    k_spmv<double, double, false, false><<<cs.total, kThreads, 0, s>>>(A, cs, x, y, red, 0,
                                                                       nullptr, done);
  return 1;
}

int launch_spmv32(const LevelDev &L, const float *x, float *y, cudaStream_t s) {
  if (L.spmv_blocks == 0) return 0;
  const ClassSet cs = classes_of(L, 2);
  k_spmv<uint16_t, float, false, true><<<cs.total, kThreads, 0, s>>>(
      mat_of(L, L.vals16), cs, x, y, Reduce(), 0, nullptr, nullptr);
  return 1;
}

template <class T>
struct ValsOf;
template <>
struct ValsOf<double> {
  using VT = double;
  static const double *get(const LevelDev &L) { return L.vals; }
};
template <>
struct ValsOf<float> {
  using VT = uint16_t;
  static const uint16_t *get(const LevelDev &L) { return L.vals16; }
};

// The class kernels.  EXTRA: GS_STENCIL (FP64: columns from the stencil
// offsets), added to every launch's mode.
template <int EXTRA, class T, class RT>
int launch_gs_rows(const LevelDev &L, int q, int backward, int mode, const RT *r, T *x,
                   const T *xc, T *rc, const int *done, cudaStream_t s, int jbeg, int jend) {
  using VT = typename ValsOf<T>::VT;
  const LevelMat<VT> A = mat_of(L, ValsOf<T>::get(L));
  const int lpb = L.lines_per_block[q];
  const dim3 g((unsigned)((jend - jbeg + lpb - 1) / lpb)), b(L.threads[q]);
  const ClassInfo &C = L.cls[q];
  if (mode & GS_SYM3) {
    if (q != 3) return 0;
    if (mode & GS_ZERO_GUESS)
      k_gs_class3_sym<GS_ZERO_GUESS | EXTRA><<<g, b, 0, s>>>(A, C, lpb, r, x, done);
    else
      k_gs_class3_sym<GS_PLAIN | EXTRA><<<g, b, 0, s>>>(A, C, lpb, r, x, done);
    return 1;
  }
  if (mode == GS_ZERO_GUESS && !backward) {
    switch (q) {
      case 0: k_gs_class<GS_ZERO_GUESS | EXTRA, 0, 0><<<g, b, 0, s>>>(A, C, lpb, jbeg, jend, r, x, xc, rc, done); break;
      case 1: k_gs_class<GS_ZERO_GUESS | EXTRA, 0, 1><<<g, b, 0, s>>>(A, C, lpb, jbeg, jend, r, x, xc, rc, done); break;
      case 2: k_gs_class<GS_ZERO_GUESS | EXTRA, 0, 2><<<g, b, 0, s>>>(A, C, lpb, jbeg, jend, r, x, xc, rc, done); break;
      default: k_gs_class<GS_ZERO_GUESS | EXTRA, 0, 3><<<g, b, 0, s>>>(A, C, lpb, jbeg, jend, r, x, xc, rc, done); break;
    }
    return 1;
  }
  if (mode == GS_RESTRICT && backward && q == 0) {
    k_gs_class<GS_RESTRICT | EXTRA, 1, 0><<<g, b, 0, s>>>(A, C, lpb, jbeg, jend, r, x, xc, rc, done);
    return 1;
  }
  if (mode == GS_PROLONG && !backward && q == 0) {
    k_gs_class<GS_PROLONG | EXTRA, 0, 0><<<g, b, 0, s>>>(A, C, lpb, jbeg, jend, r, x, xc, rc, done);
    return 1;
  }
  if (mode != GS_PLAIN) return 0;
  if (backward)
    k_gs_class<GS_PLAIN | EXTRA, 1, -1><<<g, b, 0, s>>>(A, C, lpb, jbeg, jend, r, x, xc, rc, done);
  else
    k_gs_class<GS_PLAIN | EXTRA, 0, -1><<<g, b, 0, s>>>(A, C, lpb, jbeg, jend, r, x, xc, rc, done);
  return 1;
}

template <class T, class RT>
int launch_gs_class(const LevelDev &L, int q, int backward, int mode, const RT *r, T *x,
                    const T *xc, T *rc, const int *done, cudaStream_t s, int jbeg, int jend) {
  if (jend < 0) jend = L.cls[q].lines;
  if (L.blocks[q] == 0 || jend <= jbeg) return 0;
  if ((mode & GS_SYM3) && (jbeg != 0 || jend != L.cls[q].lines)) return 0;   // whole class only
  if constexpr (std::is_same<T, double>::value) {
    if (L.stencil_cols)
      return launch_gs_rows<GS_STENCIL>(L, q, backward, mode, r, x, xc, rc, done, s, jbeg, jend);
  }
  return launch_gs_rows<0>(L, q, backward, mode, r, x, xc, rc, done, s, jbeg, jend);
}

template <class T, class RT>
int launch_restrict_residual(const LevelDev &F, int64_t nc, const RT *rf, const T *xf, T *rc,
                             const int *done, cudaStream_t s) {
  if (nc <= 0) return 0;
  nc = std::min(nc, (int64_t)(F.nx / 2) * (F.ny / 2) * (F.nz / 2));
  k_restrict_residual<<<grid_for(nc), kThreads, 0, s>>>(mat_of(F, ValsOf<T>::get(F)), F.cls[0],
                                                        nc, rf, xf, rc, done);
  return 1;
}
template int launch_restrict_residual<double, double>(const LevelDev &, int64_t, const double *,
                                                      const double *, double *, const int *,
                                                      cudaStream_t);
template int launch_restrict_residual<float, double>(const LevelDev &, int64_t, const double *,
                                                     const float *, float *, const int *,
                                                     cudaStream_t);
template int launch_restrict_residual<float, float>(const LevelDev &, int64_t, const float *,
                                                    const float *, float *, const int *,
                                                    cudaStream_t);

template <class T>
int launch_prolong(const LevelDev &F, int64_t nc, const T *xc, T *xf, const int *done,
                   cudaStream_t s) {
  if (nc <= 0) return 0;
  nc = std::min(nc, (int64_t)(F.nx / 2) * (F.ny / 2) * (F.nz / 2));
  k_prolong<T><<<grid_for(nc), kThreads, 0, s>>>(nc, F.nx, F.ny, xc, xf, done);
  return 1;
}
template int launch_prolong<double>(const LevelDev &, int64_t, const double *, double *,
                                    const int *, cudaStream_t);
template int launch_prolong<float>(const LevelDev &, int64_t, const float *, float *, const int *,
                                   cudaStream_t);

int read_check_record(unsigned long long *record) {
  *record = 0ull;
#ifdef HPCGX_CHECKED
  cudaError_t e = cudaMemcpyFromSymbol(record, g_check_record, sizeof(*record));
  if (e != cudaSuccess) return (int)e;
  const unsigned long long zero = 0ull;
  e = cudaMemcpyToSymbol(g_check_record, &zero, sizeof(zero));
  if (e != cudaSuccess) return (int)e;
#endif
  return 0;
}

int launch_finish(int fin, int nv, const double *tot, CgState *st, cudaStream_t s) {
  if (nv == 2)
    k_finish<2><<<1, 1, 0, s>>>(fin, tot, st);
  else
    k_finish<1><<<1, 1, 0, s>>>(fin, tot, st);
  return 1;
}

int launch_rank_sum(int nranks, double *const *bufs, int count, cudaStream_t s) {
  k_rank_sum<<<1, 32, 0, s>>>(nranks, bufs, count);
  return 1;
}

template int launch_gs_class<double, double>(const LevelDev &, int, int, int, const double *,
                                             double *, const double *, double *, const int *,
                                             cudaStream_t, int, int);
template int launch_gs_class<float, double>(const LevelDev &, int, int, int, const double *,
                                            float *, const float *, float *, const int *,
                                            cudaStream_t, int, int);
template int launch_gs_class<float, float>(const LevelDev &, int, int, int, const float *,
                                           float *, const float *, float *, const int *,
                                           cudaStream_t, int, int);

int launch_waxpby(int64_t n, double alpha, const double *x, double beta, const double *y,
                  double *w, const int *done, cudaStream_t s) {
  k_waxpby<<<vector_blocks(n), kThreads, 0, s>>>(n, alpha, x, beta, y, w, done);
  return 1;
}

int launch_dot(int64_t n, const double *x, const double *y, const Reduce &red, double *out,
               cudaStream_t s) {
  k_dot<<<vector_blocks(n), kThreads, 0, s>>>(n, x, y, red, FIN_STORE, out, nullptr);
  return 1;
}

int launch_dot_finish(int64_t n, const double *x, const double *y, const Reduce &red, int fin,
                      CgState *st, cudaStream_t s) {
  k_dot<<<vector_blocks(n), kThreads, 0, s>>>(n, x, y, red, fin, st, &st->done);
  return 1;
}

int launch_absmax_diff(int64_t n, const double *a, const double *b, const Reduce &red,
                       double *out, cudaStream_t s) {
  k_absmax_diff<<<vector_blocks(n), kThreads, 0, s>>>(n, a, b, red, out);
  return 1;
}

int launch_restriction(int64_t nc, const LevelDev &F, const double *rf, const double *Axf,
                       double *rc, cudaStream_t s) {
  k_restriction<<<grid_for(nc), kThreads, 0, s>>>(nc, F.nx, F.ny, rf, Axf, rc);
  return 1;
}

int launch_prolongation(int64_t nc, const LevelDev &F, const double *xc, double *xf,
                        cudaStream_t s) {
  k_prolongation<<<grid_for(nc), kThreads, 0, s>>>(nc, F.nx, F.ny, xc, xf);
  return 1;
}

int launch_copy(int64_t n, const double *x, double *y, const int *done, cudaStream_t s) {
  k_copy<<<vector_blocks(n), kThreads, 0, s>>>(n, x, y, done);
  return 1;
}

int launch_fill_uniform(int64_t n, uint64_t seed, uint64_t offset, double lo, double hi, double *v,
                        cudaStream_t s) {
  k_fill_uniform<<<grid_for(n), kThreads, 0, s>>>(n, seed, offset, lo, hi, v);
  return 1;
}

int launch_fill_normal(int64_t n, uint64_t seed, uint64_t offset, double *v, cudaStream_t s) {
  k_fill_normal<<<grid_for(n), kThreads, 0, s>>>(n, seed, offset, v);
  return 1;
}

int launch_cg_init(int64_t n, const double *b, const double *Ap, double *r, float *r32,
                   const Reduce &red, CgState *st, cudaStream_t s) {
  k_cg_init<<<vector_blocks(n), kThreads, 0, s>>>(n, b, Ap, r, r32, red, st);
  return 1;
}

template <class ZT>
int launch_cg_rz(int64_t n, const double *r, const ZT *z, const double *Ap, const Reduce &red,
                 CgState *st, cudaStream_t s) {
  if (Ap)
    k_cg_rz<ZT, true><<<vector_blocks(n), kThreads, 0, s>>>(n, r, z, Ap, red, st);
  else
    k_cg_rz<ZT, false><<<vector_blocks(n), kThreads, 0, s>>>(n, r, z, Ap, red, st);
  return 1;
}
template int launch_cg_rz<double>(int64_t, const double *, const double *, const double *,
                                  const Reduce &, CgState *, cudaStream_t);
template int launch_cg_rz<float>(int64_t, const double *, const float *, const double *,
                                 const Reduce &, CgState *, cudaStream_t);

template <class ZT>
int launch_cg_p(int64_t n, const ZT *z, double *p, CgState *st, cudaStream_t s, double *x) {
  k_cg_p<ZT><<<vector_blocks(n), kThreads, 0, s>>>(n, z, p, st, x);
  return 1;
}
template int launch_cg_p<double>(int64_t, const double *, double *, CgState *, cudaStream_t,
                                 double *);
template int launch_cg_p<float>(int64_t, const float *, double *, CgState *, cudaStream_t,
                                double *);

int launch_cg_xflush(int64_t n, const double *p, double *x, const CgState *st, cudaStream_t s) {
  k_cg_xflush<<<vector_blocks(n), kThreads, 0, s>>>(n, p, x, st);
  return 1;
}

int launch_cg_xr(int64_t n, const double *p, const double *Ap, double *x, double *r, float *r32,
                 const Reduce &red, CgState *st, cudaStream_t s) {
  k_cg_xr<<<vector_blocks(n), kThreads, 0, s>>>(n, p, Ap, x, r, r32, red, st);
  return 1;
}

int launch_copy_z(int64_t n, const double *r, double *z, const CgState *st, cudaStream_t s) {
  k_copy_z<<<vector_blocks(n), kThreads, 0, s>>>(n, r, z, st);
  return 1;
}

int launch_adjoint_grad(const LevelDev &L, const double *lambda, const double *x, double *grad,
                        cudaStream_t s) {
  k_adjoint_grad<<<grid_for(L.n), kThreads, 0, s>>>(geo_of(L), L.n, L.cols, lambda, x, grad);
  return 1;
}

}  // namespace hpcgx
