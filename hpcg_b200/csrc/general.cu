// general.cu -- the reference operators on a general sparse matrix (any
// pattern); see general.cuh for the layout and what each operator restates.
#include "general.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/hpcgx.h"
#include "kernels.cuh"

namespace hpcgx {

int set_error(int code, const char *msg);

namespace {

constexpr int kT = 256;

// ------------------------------------------------------------------ kernels

// Entry j of storage row k: slice k / 32, lane k % 32, entries of a slice
// interleaved across its 32 rows (a warp's loads of entry j are contiguous).
__device__ __forceinline__ int64_t gen_entry(const int64_t *__restrict__ slice_off, int64_t k,
                                             int j) {
  return slice_off[k >> 5] + (int64_t)j * 32 + (k & 31);
}

// y = A x over the storage rows (src/ComputeSPMV_ref.cpp:58-71: a sum from 0
// over the row's entries in order, each product and sum rounded on its own).
__global__ void __launch_bounds__(kT)
k_gen_spmv(int64_t n, const int64_t *__restrict__ slice_off, const uint8_t *__restrict__ nnz,
           const int32_t *__restrict__ perm, const int32_t *__restrict__ cols,
           const double *__restrict__ vals, const double *__restrict__ x, double *__restrict__ y,
           const int *__restrict__ done) {
  if (done && *done) return;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int m = nnz[k];
    double sum = 0.0;
    for (int j = 0; j < m; ++j) {
      const int64_t e = gen_entry(slice_off, k, j);
      sum = __dadd_rn(sum, __dmul_rn(__ldg(vals + e), __ldg(x + __ldg(cols + e))));
    }
    y[perm[k]] = sum;
  }
}

// The Gauss-Seidel update of storage rows [k0, k1), one colour
// (src/ComputeSYMGS_ref.cpp:72-80): sum = r_i - sum_j a_ij x_j over the row's
// entries (diagonal included), sum += x_i a_ii, x_i = sum / a_ii.  Rows of one
// colour share no entry, so they update in parallel.
__global__ void __launch_bounds__(kT)
k_gen_gs(int64_t k0, int64_t k1, const int64_t *__restrict__ slice_off,
         const uint8_t *__restrict__ nnz, const int32_t *__restrict__ perm,
         const int32_t *__restrict__ cols, const double *__restrict__ vals,
         const double *__restrict__ diag, const double *__restrict__ r, double *x,
         const int *__restrict__ done) {
  if (done && *done) return;
  for (int64_t k = k0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < k1;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int m = nnz[k];
    const int32_t i = perm[k];
    const double d = diag[k];
    double sum = r[i];
    for (int j = 0; j < m; ++j) {
      const int64_t e = gen_entry(slice_off, k, j);
      sum = __dsub_rn(sum, __dmul_rn(__ldg(vals + e), x[__ldg(cols + e)]));
    }
    sum = __dadd_rn(sum, __dmul_rn(x[i], d));
    x[i] = __ddiv_rn(sum, d);
  }
}

// src/ComputeRestriction_ref.cpp:51 and src/ComputeProlongation_ref.cpp:49
// through a given injection f2c.
__global__ void k_gen_restrict(int64_t nc, const int32_t *__restrict__ f2c,
                               const double *__restrict__ rf, const double *__restrict__ Axf,
                               double *__restrict__ rc, const int *__restrict__ done) {
  if (done && *done) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nc;
       i += (int64_t)gridDim.x * blockDim.x)
    rc[i] = __dsub_rn(rf[f2c[i]], Axf[f2c[i]]);
}

__global__ void k_gen_prolong(int64_t nc, const int32_t *__restrict__ f2c,
                              const double *__restrict__ xc, double *xf,
                              const int *__restrict__ done) {
  if (done && *done) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nc;
       i += (int64_t)gridDim.x * blockDim.x)
    xf[f2c[i]] = __dadd_rn(xf[f2c[i]], xc[i]);
}

__global__ void k_gen_zero(int64_t n, double *x, const int *__restrict__ done) {
  if (done && *done) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] = 0.0;
}

// Writes (set) or reads the diagonal of every row, natural order.
__global__ void k_gen_diag(int64_t n, const int64_t *__restrict__ slice_off,
                           const int32_t *__restrict__ perm, const uint8_t *__restrict__ dpos,
                           double *vals, double *diag, double *nat, int set) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = gen_entry(slice_off, k, dpos[k]);
    if (set) {
      vals[e] = nat[perm[k]];
      diag[k] = nat[perm[k]];
    } else {
      nat[perm[k]] = diag[k];
    }
  }
}

int grid(int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + kT - 1) / kT, 148 * 16));
}

template <class F>
void host_parallel(int64_t n, F f) {
  const unsigned hw = std::thread::hardware_concurrency();
  const int64_t nt = std::max<int64_t>(1, std::min<int64_t>(hw ? hw : 1, 64));
  if (n < 65536 || nt == 1) {
    f(0, n);
    return;
  }
  std::vector<std::thread> ts;
  const int64_t chunk = (n + nt - 1) / nt;
  for (int64_t t = 0; t < nt; ++t) {
    const int64_t a = t * chunk, b = std::min(n, a + chunk);
    if (a < b) ts.emplace_back(f, a, b);
  }
  for (auto &th : ts) th.join();
}

}  // namespace

// ------------------------------------------------------------------ host side

struct GLevel {
  int64_t n = 0, nc = 0, entries = 0;
  int ncolors = 0;
  std::vector<int64_t> cstart;     // storage row of the first row of each colour (+ end)
  int64_t *slice_off = nullptr;
  uint8_t *nnz = nullptr, *dpos = nullptr;
  int32_t *perm = nullptr, *cols = nullptr, *f2c = nullptr;
  double *vals = nullptr, *diag = nullptr;
  double *r = nullptr, *x = nullptr, *Axf = nullptr;   // V-cycle work vectors
  bool loaded = false;
};

struct GeneralProblem {
  int nlev = 0;
  cudaStream_t stream = nullptr;
  GLevel L[kMaxLevels];
  std::vector<void *> allocs;
  double bytes = 0.0;
  int64_t launches = 0;
  // CG
  double *r = nullptr, *z = nullptr, *p = nullptr, *Ap = nullptr;
  CgState *st = nullptr;
  Reduce red;
  cudaGraphExec_t graph[2] = {};
  const double *graph_x[2] = {};   // the solution vector a graph was captured for
  cudaEvent_t phase[2][5] = {};
  bool capturing = false;

  int alloc(void **ptr, size_t n) {
    cudaError_t e = cudaMalloc(ptr, std::max<size_t>(n, 8));
    if (e != cudaSuccess) {
      *ptr = nullptr;
      cudaGetLastError();
      return set_error(HPCGX_ENOMEM, ("cudaMalloc of " + std::to_string(n) + " bytes failed").c_str());
    }
    allocs.push_back(*ptr);
    bytes += (double)n;
    return HPCGX_OK;
  }
  ~GeneralProblem() {
    for (int k = 0; k < 2; ++k) {
      if (graph[k]) cudaGraphExecDestroy(graph[k]);
      for (cudaEvent_t &ev : phase[k])
        if (ev) cudaEventDestroy(ev);
    }
    for (void *ptr : allocs) cudaFree(ptr);
  }
  void note(int k) { launches += k; }

  // ---- operators (launches only; the caller synchronises)
  void spmv(int l, const double *x, double *y, const int *done) {
    const GLevel &A = L[l];
    k_gen_spmv<<<grid(A.n), kT, 0, stream>>>(A.n, A.slice_off, A.nnz, A.perm, A.cols, A.vals, x,
                                             y, done);
    note(1);
  }
  void symgs(int l, const double *r, double *x, const int *done) {
    const GLevel &A = L[l];
    auto colour = [&](int c) {
      const int64_t k0 = A.cstart[c], k1 = A.cstart[c + 1];
      if (k1 > k0) {
        k_gen_gs<<<grid(k1 - k0), kT, 0, stream>>>(k0, k1, A.slice_off, A.nnz, A.perm, A.cols,
                                                   A.vals, A.diag, r, x, done);
        note(1);
      }
    };
    for (int c = 0; c < A.ncolors; ++c) colour(c);
    for (int c = A.ncolors - 1; c >= 0; --c) colour(c);
  }
  // src/ComputeMG_ref.cpp:39-63, one pre- and one post-smoothing sweep
  // (src/MGData.hpp:51-52).
  void mg(int l, const double *r, double *x, const int *done) {
    const GLevel &A = L[l];
    k_gen_zero<<<grid(A.n), kT, 0, stream>>>(A.n, x, done);
    note(1);
    symgs(l, r, x, done);
    if (l + 1 < nlev) {
      GLevel &C = L[l + 1];
      spmv(l, x, A.Axf, done);
      k_gen_restrict<<<grid(A.nc), kT, 0, stream>>>(A.nc, A.f2c, r, A.Axf, C.r, done);
      mg(l + 1, C.r, C.x, done);
      k_gen_prolong<<<grid(A.nc), kT, 0, stream>>>(A.nc, A.f2c, C.x, x, done);
      note(2);
      symgs(l, r, x, done);
    }
  }
  // One CG iteration (src/CG.cpp:100-130) on the device scalars of st.
  void iteration(int precond, double *x) {
    const int64_t n = L[0].n;
    const int *done = &st->done;
    if (capturing) cudaEventRecordWithFlags(phase[precond][0], stream, cudaEventRecordExternal);
    if (precond)
      mg(0, r, z, done);
    else
      note(launch_copy_z(n, r, z, st, stream));
    if (capturing) cudaEventRecordWithFlags(phase[precond][1], stream, cudaEventRecordExternal);
    note(launch_cg_rz<double>(n, r, z, nullptr, red, st, stream));
    note(launch_cg_p<double>(n, z, p, st, stream));
    if (capturing) cudaEventRecordWithFlags(phase[precond][2], stream, cudaEventRecordExternal);
    spmv(0, p, Ap, done);
    note(launch_dot_finish(n, p, Ap, red, FIN_CG_PAP, st, stream));
    if (capturing) cudaEventRecordWithFlags(phase[precond][3], stream, cudaEventRecordExternal);
    note(launch_cg_xr(n, p, Ap, x, r, nullptr, red, st, stream));
    if (capturing) cudaEventRecordWithFlags(phase[precond][4], stream, cudaEventRecordExternal);
  }
};

#define GTRY(x)                     \
  do {                              \
    const int rc_ = (x);            \
    if (rc_ != HPCGX_OK) return rc_; \
  } while (0)
#define GCK(x)                                                           \
  do {                                                                   \
    const cudaError_t e_ = (x);                                          \
    if (e_ != cudaSuccess) {                                             \
      cudaGetLastError();                                                \
      return set_error(HPCGX_ECUDA, cudaGetErrorString(e_));             \
    }                                                                    \
  } while (0)

GeneralProblem *general_create(int nlev, cudaStream_t s) {
  GeneralProblem *g = new GeneralProblem;
  g->nlev = nlev;
  g->stream = s;
  return g;
}

void general_destroy(GeneralProblem *g) { delete g; }
void general_set_stream(GeneralProblem *g, cudaStream_t s) {
  g->stream = s;
  for (int k = 0; k < 2; ++k)
    if (g->graph[k]) {
      cudaGraphExecDestroy(g->graph[k]);
      g->graph[k] = nullptr;
    }
}

int64_t general_rows(const GeneralProblem *g, int level) {
  return (level >= 0 && level < g->nlev) ? g->L[level].n : -1;
}
int general_colours(const GeneralProblem *g, int level) {
  return (level >= 0 && level < g->nlev) ? g->L[level].ncolors : -1;
}
bool general_ready(const GeneralProblem *g) {
  for (int l = 0; l < g->nlev; ++l)
    if (!g->L[l].loaded) return false;
  return true;
}
double general_bytes(const GeneralProblem *g) { return g->bytes; }
int64_t general_launches(const GeneralProblem *g) { return g->launches; }

int general_load_level(GeneralProblem *g, int level, int64_t n, const char *nnz,
                       const int32_t *const *cols, const double *const *vals, const int32_t *f2c,
                       int64_t nc, const char **msg) {
  static thread_local std::string why;
  auto reject = [&](const std::string &m) {
    why = m;
    *msg = why.c_str();
    return HPCGX_ELAYOUT;
  };
  *msg = nullptr;
  if (level < 0 || level >= g->nlev) return set_error(HPCGX_EINVAL, "level out of range");
  if (g->L[level].loaded) return set_error(HPCGX_ESTATE, "level already loaded");
  if (n < 1 || n >= ((int64_t)1 << 31)) return set_error(HPCGX_EINVAL, "row count out of range");
  if (level > 0 && n != g->L[level - 1].nc)
    return set_error(HPCGX_EINVAL, "rows differ from the finer level's coarse row count");
  const bool coarse = level + 1 < g->nlev;
  if (coarse && (!f2c || nc < 1 || nc > n))
    return set_error(HPCGX_EINVAL, "every level but the last needs its injection f2c");
  GLevel &A = g->L[level];
  // ---- checks: entries in range, one diagonal entry per row (on the host's
  // cores; the failing row with the lowest index is reported)
  std::vector<uint8_t> dposn(n);
  auto check_row = [&](int64_t i, const char **why_row) {
    const int m = (unsigned char)nnz[i];
    if (m < 1) {
      *why_row = "no entries";
      return false;
    }
    int d = -1;
    for (int j = 0; j < m; ++j) {
      const int32_t c = cols[i][j];
      if (c < 0 || c >= n) {
        *why_row = "column out of range";
        return false;
      }
      if (c == i && d < 0) d = j;
    }
    if (d < 0) {
      *why_row = "no diagonal entry";
      return false;
    }
    dposn[i] = (uint8_t)d;
    return true;
  };
  std::atomic<int64_t> bad{n};
  host_parallel(n, [&](int64_t a, int64_t b) {
    const char *why_row = nullptr;
    for (int64_t i = a; i < b; ++i)
      if (!check_row(i, &why_row)) {
        int64_t seen = bad.load();
        while (i < seen && !bad.compare_exchange_weak(seen, i)) {
        }
        return;
      }
  });
  if (bad.load() < n) {
    const char *why_row = "";
    check_row(bad.load(), &why_row);
    return reject("row " + std::to_string(bad.load()) + ": " + why_row);
  }
  if (coarse)
    for (int64_t i = 0; i < nc; ++i)
      if (f2c[i] < 0 || f2c[i] >= n) return reject("f2c entry out of range");
  // ---- greedy multicolouring in natural row order, the algorithm of
  // src/OptimizeProblem.cpp:50-79: row i takes the lowest colour that no
  // already coloured neighbour (column < i) has.
  std::vector<int32_t> colour(n, -1);
  int total = 1;
  colour[0] = 0;
  std::vector<char> used;
  for (int64_t i = 1; i < n; ++i) {
    used.assign(total + 1, 0);
    const int m = (unsigned char)nnz[i];
    for (int j = 0; j < m; ++j) {
      const int32_t c = cols[i][j];
      if (c < i) used[colour[c]] = 1;
    }
    int pick = 0;
    while (pick < total && used[pick]) ++pick;
    if (pick == total) ++total;
    colour[i] = pick;
  }
  A.ncolors = total;
  // ---- storage order: colour-major, natural order inside a colour
  A.cstart.assign(total + 1, 0);
  for (int64_t i = 0; i < n; ++i) A.cstart[colour[i] + 1]++;
  for (int c = 0; c < total; ++c) A.cstart[c + 1] += A.cstart[c];
  std::vector<int32_t> perm(n);
  {
    std::vector<int64_t> next(A.cstart.begin(), A.cstart.end() - 1);
    for (int64_t i = 0; i < n; ++i) perm[next[colour[i]]++] = (int32_t)i;
  }
  // ---- sliced ELL: slice s (storage rows 32s .. 32s+31) is as wide as its
  // longest row; padding entries hold value 0 and column 0 and are never read
  const int64_t slices = (n + 31) / 32;
  std::vector<int64_t> off(slices + 1, 0);
  for (int64_t s = 0; s < slices; ++s) {
    int w = 0;
    for (int64_t k = 32 * s; k < std::min(n, 32 * s + 32); ++k)
      w = std::max(w, (int)(unsigned char)nnz[perm[k]]);
    off[s + 1] = off[s] + 32 * (int64_t)w;
  }
  const int64_t entries = off[slices];
  // staging written by the host's threads in one pass, padding included
  // (no serial zero-fill of the 12 B per entry first)
  std::unique_ptr<int32_t[]> hcp(new int32_t[entries]);
  std::unique_ptr<double[]> hvp(new double[entries]);
  int32_t *hc = hcp.get();
  double *hv = hvp.get();
  std::vector<uint8_t> hn(n), hd(n);
  std::vector<double> hdiag(n);
  host_parallel(n, [&](int64_t a, int64_t b) {
    for (int64_t k = a; k < b; ++k) {
      const int32_t i = perm[k];
      const int m = (unsigned char)nnz[i];
      hn[k] = (uint8_t)m;
      hd[k] = dposn[i];
      hdiag[k] = vals[i][dposn[i]];
      const int64_t sl = k >> 5, base = off[sl] + (k & 31);
      const int w = (int)((off[sl + 1] - off[sl]) / 32);
      for (int j = 0; j < m; ++j) {
        hc[base + 32 * j] = cols[i][j];
        hv[base + 32 * j] = vals[i][j];
      }
      for (int j = m; j < w; ++j) {
        hc[base + 32 * j] = 0;
        hv[base + 32 * j] = 0.0;
      }
    }
  });
  // lanes of the last slice past the last row
  for (int64_t k = n; k < 32 * slices; ++k) {
    const int64_t sl = k >> 5, base = off[sl] + (k & 31);
    for (int64_t j = 0; j < (off[sl + 1] - off[sl]) / 32; ++j) {
      hc[base + 32 * j] = 0;
      hv[base + 32 * j] = 0.0;
    }
  }
  // ---- device copies
  A.n = n;
  A.nc = coarse ? nc : 0;
  A.entries = entries;
  GTRY(g->alloc((void **)&A.slice_off, (slices + 1) * sizeof(int64_t)));
  GTRY(g->alloc((void **)&A.nnz, n));
  GTRY(g->alloc((void **)&A.dpos, n));
  GTRY(g->alloc((void **)&A.perm, n * sizeof(int32_t)));
  GTRY(g->alloc((void **)&A.cols, entries * sizeof(int32_t)));
  GTRY(g->alloc((void **)&A.vals, entries * sizeof(double)));
  GTRY(g->alloc((void **)&A.diag, n * sizeof(double)));
  GTRY(g->alloc((void **)&A.Axf, n * sizeof(double)));
  if (level > 0) {
    GTRY(g->alloc((void **)&A.r, n * sizeof(double)));
    GTRY(g->alloc((void **)&A.x, n * sizeof(double)));
  }
  if (coarse) GTRY(g->alloc((void **)&A.f2c, nc * sizeof(int32_t)));
  cudaStream_t s = g->stream;
  GCK(cudaMemcpyAsync(A.slice_off, off.data(), (slices + 1) * sizeof(int64_t),
                      cudaMemcpyHostToDevice, s));
  GCK(cudaMemcpyAsync(A.nnz, hn.data(), n, cudaMemcpyHostToDevice, s));
  GCK(cudaMemcpyAsync(A.dpos, hd.data(), n, cudaMemcpyHostToDevice, s));
  GCK(cudaMemcpyAsync(A.perm, perm.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  GCK(cudaMemcpyAsync(A.cols, hc, entries * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  GCK(cudaMemcpyAsync(A.vals, hv, entries * sizeof(double), cudaMemcpyHostToDevice, s));
  GCK(cudaMemcpyAsync(A.diag, hdiag.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
  if (coarse) GCK(cudaMemcpyAsync(A.f2c, f2c, nc * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  if (level == 0) {
    for (double **v : {&g->r, &g->z, &g->p, &g->Ap}) GTRY(g->alloc((void **)v, n * sizeof(double)));
    GTRY(g->alloc((void **)&g->st, sizeof(CgState)));
    const int64_t blocks = vector_blocks(n);
    const int64_t cap = 2 * blocks + 2 * ((blocks + 1023) / 1024);
    GTRY(g->alloc((void **)&g->red.partials, cap * sizeof(double)));
    const int64_t counters = 1 + (cap + 1023) / 1024;
    GTRY(g->alloc((void **)&g->red.counter, counters * sizeof(unsigned int)));
    g->red.capacity = cap;
    GCK(cudaMemsetAsync(g->red.counter, 0, counters * sizeof(unsigned int), s));
  }
  GCK(cudaStreamSynchronize(s));
  A.loaded = true;
  return HPCGX_OK;
}

int general_spmv(GeneralProblem *g, int level, const double *x, double *y) {
  g->spmv(level, x, y, nullptr);
  GCK(cudaStreamSynchronize(g->stream));
  GCK(cudaGetLastError());
  return HPCGX_OK;
}

int general_symgs(GeneralProblem *g, int level, const double *r, double *x) {
  g->symgs(level, r, x, nullptr);
  GCK(cudaStreamSynchronize(g->stream));
  GCK(cudaGetLastError());
  return HPCGX_OK;
}

int general_mg(GeneralProblem *g, const double *r, double *x) {
  g->mg(0, r, x, nullptr);
  GCK(cudaStreamSynchronize(g->stream));
  GCK(cudaGetLastError());
  return HPCGX_OK;
}

int general_cg(GeneralProblem *g, const double *b, double *x, int max_iter, double tol,
               int precond, int *niters, double *normr, double *normr0, double *times) {
  if (max_iter < 0) return set_error(HPCGX_EINVAL, "max_iter < 0");
  const auto t0 = std::chrono::steady_clock::now();
  const int64_t n = g->L[0].n;
  const int kind = precond ? 1 : 0;
  cudaStream_t s = g->stream;
  CgState h;
  std::memset(&h, 0, sizeof(h));
  h.tol = tol;
  h.max_iter = max_iter;
  GCK(cudaMemcpyAsync(g->st, &h, sizeof(h), cudaMemcpyHostToDevice, s));
  // p = x, Ap = A p, r = b - Ap, normr0 (src/CG.cpp:86-96)
  GCK(cudaMemcpyAsync(g->p, x, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  g->spmv(0, g->p, g->Ap, nullptr);
  g->note(launch_cg_init(n, b, g->Ap, g->r, nullptr, g->red, g->st, s));
  // one CUDA graph per iteration, captured on first use for this x
  if (!g->graph[kind] || g->graph_x[kind] != x) {
    if (g->graph[kind]) {
      GCK(cudaGraphExecDestroy(g->graph[kind]));
      g->graph[kind] = nullptr;
    }
    for (cudaEvent_t &ev : g->phase[kind])
      if (!ev) GCK(cudaEventCreate(&ev));
    cudaGraph_t gr = nullptr;
    GCK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    g->capturing = true;
    const int64_t before = g->launches;
    g->iteration(kind, x);
    g->capturing = false;
    g->launches = before;
    GCK(cudaStreamEndCapture(s, &gr));
    const cudaError_t e = cudaGraphInstantiate(&g->graph[kind], gr, 0);
    cudaGraphDestroy(gr);
    GCK(e);
    g->graph_x[kind] = x;
  }
  double t_mg = 0, t_vec = 0, t_spmv = 0;
  int launched = 0;
  while (launched < max_iter) {
    GCK(cudaGraphLaunch(g->graph[kind], s));
    ++launched;
    GCK(cudaMemcpyAsync(&h, g->st, sizeof(h), cudaMemcpyDeviceToHost, s));
    GCK(cudaStreamSynchronize(s));
    if (h.niters == launched) {
      float a = 0, b2 = 0, c = 0, d = 0;
      GCK(cudaEventElapsedTime(&a, g->phase[kind][0], g->phase[kind][1]));
      GCK(cudaEventElapsedTime(&b2, g->phase[kind][1], g->phase[kind][2]));
      GCK(cudaEventElapsedTime(&c, g->phase[kind][2], g->phase[kind][3]));
      GCK(cudaEventElapsedTime(&d, g->phase[kind][3], g->phase[kind][4]));
      t_mg += a * 1e-3;
      t_vec += (b2 + d) * 1e-3;
      t_spmv += c * 1e-3;
    }
    if (h.done) break;
  }
  if (launched == 0) {
    GCK(cudaMemcpyAsync(&h, g->st, sizeof(h), cudaMemcpyDeviceToHost, s));
    GCK(cudaStreamSynchronize(s));
  }
  if (niters) *niters = h.niters;
  if (normr) *normr = h.normr;
  if (normr0) *normr0 = h.normr0;
  if (times) {
    times[0] += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    times[2] += t_vec;
    times[3] += t_spmv;
    times[5] += t_mg;
  }
  if (h.nonfinite) return set_error(HPCGX_ENONFINITE, "CG: residual norm is not finite");
  return HPCGX_OK;
}

// The level's Axf work vector stages the natural-order diagonal.
int general_set_diagonal(GeneralProblem *g, int level, const double *diag) {
  GLevel &A = g->L[level];
  GCK(cudaMemcpyAsync(A.Axf, diag, A.n * sizeof(double), cudaMemcpyHostToDevice, g->stream));
  k_gen_diag<<<grid(A.n), kT, 0, g->stream>>>(A.n, A.slice_off, A.perm, A.dpos, A.vals, A.diag,
                                              A.Axf, 1);
  GCK(cudaGetLastError());
  GCK(cudaStreamSynchronize(g->stream));
  return HPCGX_OK;
}

int general_get_diagonal(GeneralProblem *g, int level, double *diag) {
  GLevel &A = g->L[level];
  k_gen_diag<<<grid(A.n), kT, 0, g->stream>>>(A.n, A.slice_off, A.perm, A.dpos, A.vals, A.diag,
                                              A.Axf, 0);
  GCK(cudaGetLastError());
  GCK(cudaMemcpyAsync(diag, A.Axf, A.n * sizeof(double), cudaMemcpyDeviceToHost, g->stream));
  GCK(cudaStreamSynchronize(g->stream));
  return HPCGX_OK;
}

}  // namespace hpcgx
