// problem.cu -- problem set-up, multigrid / CG drivers and the C ABI of libhpcgx.
//
// A problem owns one CUDA stream.  Matrix levels live in the colour-sorted
// sliced-ELL layout described in common.cuh; CG keeps every scalar on the
// device and runs each iteration as one CUDA graph (the V-cycle's 49 class
// launches -- 7 per symmetric sweep, two sweeps on each of three levels and
// one on the coarsest -- plus the 4 fused vector/SpMV kernels), so the host
// only reads the residual norm when it has to test convergence.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <memory>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <type_traits>
#include <functional>
#include <mutex>
#include <vector>

#include "../../include/hpcgx.h"
#include "general.cuh"
#include "kernels.cuh"

using namespace hpcgx;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

// The status of a failed CUDA call, its error taken off the thread's
// last-error slot as CK does.
int cuda_fail(cudaError_t e) {
  cudaGetLastError();
  return fail(e == cudaErrorMemoryAllocation ? HPCGX_ENOMEM : HPCGX_ECUDA, cudaGetErrorString(e));
}

// A failed CUDA call becomes the returned status; its error is also taken
// off the thread's last-error slot, so that a later call does not report it
// a second time (errors that break the context persist regardless).
#define CK(call)                                                                  \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess) {                                                      \
      cudaGetLastError();                                                         \
      return fail(e_ == cudaErrorMemoryAllocation ? HPCGX_ENOMEM : HPCGX_ECUDA,   \
                  std::string(#call) + ": " + cudaGetErrorString(e_));            \
    }                                                                             \
  } while (0)

#define TRY(expr)               \
  do {                          \
    int rc_ = (expr);           \
    if (rc_ != HPCGX_OK) return rc_; \
  } while (0)

// A named range around each library call for timeline tools (NVTX; costs a
// pointer test when no tool is attached).
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Count of the rows of colour c whose slot s has a neighbour (algorithmic
// byte model: real nonzeros only).
int64_t axis_count(int n, int p, int d) {
  int64_t c = 0;
  for (int i = p; i < n; i += 2)
    if (i + d >= 0 && i + d < n) ++c;
  return c;
}

// Multigrid work vectors of a level by arithmetic type.
inline double *lvl_x(LevelDev &A, double *) { return A.x64; }
inline float *lvl_x(LevelDev &A, float *) { return A.x32; }
inline double *lvl_r(LevelDev &A, double *) { return A.r64; }
inline float *lvl_r(LevelDev &A, float *) { return A.r32; }

enum GraphKind { G_FP64_PREC = 0, G_FP64_NOPREC = 1, G_MIXED = 2, G_COUNT = 3 };

// One step of a sharded operation (see hpcgx_problem::add*).
enum StepKind { STEP_LAUNCH = 0, STEP_HALO = 1, STEP_SUM = 2 };
struct Step {
  int kind = STEP_LAUNCH;
  std::function<int()> launch;   // STEP_LAUNCH: enqueue on the problem's stream
  int level = 0;                 // STEP_HALO: level vector vec of esize-byte elements
  void *vec = nullptr;
  int esize = 0;
  // STEP_HALO: work that reads no halo plane and writes none of the planes
  // sent, run after the exchange was issued -- beside it where the backend
  // exchanges on the GPU (NCCL), after it otherwise
  std::function<int()> interior;
  int fin = -1, nv = 0;          // STEP_SUM: nv totals in gsum, then scalar step fin
};
using Plan = std::vector<Step>;

struct Probe {
  cudaEvent_t a, b;
  double bytes;
  int kind;   // one HPCGX_PROBE_* bit
};

int probe_slot(int kind) { return kind == HPCGX_PROBE_GS_FINE ? 0 : kind == HPCGX_PROBE_SPMV_FINE ? 1 : 2; }

}  // namespace

namespace hpcgx {
// Records an error message for hpcgx_last_error() from other translation units.
int set_error(int code, const char *msg) { return fail(code, msg); }
}  // namespace hpcgx

// 32-row slices per chunk of the host loaders' pinned staging (2 chunks of
// 4096 x 864 values and columns: 2 x 42 MB)
constexpr int64_t kPinnedSlices = 4096;

static int env_int(const char *name, int dflt) {
  const char *e = std::getenv(name);
  return e && *e ? std::atoi(e) : dflt;
}

struct hpcgx_problem {
  int device = 0;
  int nlev = 0;
  // a general-pattern problem (hpcgx_create_general): the operators run on
  // this instead of the stencil levels below, which stay empty
  GeneralProblem *gen = nullptr;
  LevelDev L[kMaxLevels];
  cudaStream_t stream = nullptr;      // stream in use
  cudaStream_t own_stream = nullptr;  // stream created with the problem
  bool loaded[kMaxLevels] = {};
  bool mixed_ready = false;
  bool mixed_stale = true;
  // CG work vectors (finest level)
  double *b = nullptr, *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *Ap = nullptr;
  float *z32 = nullptr;
  // FP32 copy of r, written by the CG update for the mixed V-cycle's finest
  // level (which reads r on every one of its 14 launches: 4 B a row instead
  // of 8); HPCGX_R32=0 makes the V-cycle read the FP64 r instead
  float *r32 = nullptr;
  bool fine_r32 = env_int("HPCGX_R32", 1) != 0;
  double *tmp = nullptr;      // staging for host diagonals
  double *stage[3] = {};      // staging of the host-buffer operators (allocated on first use)
  double *result = nullptr;   // device scalars of standalone reductions
  CgState *st = nullptr;
  Reduce red;
  // graphs of one CG iteration
  cudaGraphExec_t graph[G_COUNT] = {};
  int graph_kernels[G_COUNT] = {};
  int graph_probe[G_COUNT] = {};
  // algorithmic bytes of one iteration of each graph (this implementation's
  // byte model, summed over its launches while the graph is captured)
  double graph_bytes[G_COUNT] = {};
  cudaEvent_t phase[G_COUNT][5] = {};
  // capture bookkeeping
  bool capturing = false;
  int capture_kind = 0;
  int64_t launches = 0;
  // probe
  int probe = HPCGX_PROBE_NONE;
  std::vector<Probe> probes[G_COUNT];
  std::vector<Probe> event_pool;  // created outside stream capture
  size_t pool_next = 0;
  double probe_ms[3] = {}, probe_bytes[3] = {};
  int64_t probe_launches[3] = {};
  size_t bytes = 0;
  // vectors that SpMV / Gauss-Seidel read as x carry one halo plane below and
  // above (zero unless a neighbouring rank fills them); their allocations
  std::vector<void *> halo_bases;
  // ---- sharding: this problem is z-slab `rank` of `nranks`; the global grid
  // is nx x ny x (nz nranks) (src/GenerateGeometry.cpp with npx = npy = 1)
  int nranks = 1, rank = 0;
  struct NcclLink *nccl = nullptr;   // exchange backend, one process per GPU
  hpcgx_halo_fn comm_halo = nullptr; // caller-provided exchange backend
  hpcgx_sum_fn comm_sum = nullptr;
  void *comm_ctx = nullptr;
  double *gsum = nullptr;            // this rank's deferred reduction totals
  double *hstage[kMaxLevels] = {};   // haloed FP64 staging of operator inputs
  bool sharded() const { return nranks > 1 || nccl != nullptr || comm_halo != nullptr; }
  // side stream and events of the NCCL halo exchanges that run beside
  // interior work (created on first use)
  cudaStream_t comm_stream = nullptr;
  cudaEvent_t ev_ready = nullptr, ev_halo = nullptr;
  int overlap_streams() {
    if (comm_stream) return HPCGX_OK;
    // the highest priority: the exchange's kernels take SM slots as the
    // interior launch's blocks retire
    int lo = 0, hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    CK(cudaStreamCreateWithPriority(&comm_stream, cudaStreamNonBlocking, hi));
    CK(cudaEventCreateWithFlags(&ev_ready, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev_halo, cudaEventDisableTiming));
    return HPCGX_OK;
  }
  // ---- pinned host staging of the host loaders: two chunks of kPinnedSlices
  // 32-row slices (values and columns), allocated on the first load
  double *pin_vals[2] = {};
  int32_t *pin_cols[2] = {};
  cudaEvent_t pin_copied[2] = {};
  int pinned_staging() {
    if (pin_vals[0]) return HPCGX_OK;
    const size_t e = (size_t)kPinnedSlices * kSliceElems;
    for (int h = 0; h < 2; ++h) {
      CK(cudaHostAlloc((void **)&pin_vals[h], e * sizeof(double), cudaHostAllocDefault));
      CK(cudaHostAlloc((void **)&pin_cols[h], e * sizeof(int32_t), cudaHostAllocDefault));
      CK(cudaEventCreateWithFlags(&pin_copied[h], cudaEventDisableTiming));
    }
    return HPCGX_OK;
  }

  ~hpcgx_problem();
  int alloc(void **ptr, size_t n) {
    cudaError_t e = cudaMalloc(ptr, n);
    if (e != cudaSuccess) {
      *ptr = nullptr;
      cudaGetLastError();   // reported through the status; do not leave it for a later call
      return fail(HPCGX_ENOMEM, "cudaMalloc of " + std::to_string(n) + " bytes failed: " +
                                    cudaGetErrorString(e));
    }
    bytes += n;
    return HPCGX_OK;
  }
  // n elements of esize bytes with one zeroed halo plane (plane elements) on
  // each side; *ptr points at element 0.
  int alloc_halo(void **ptr, int64_t n, size_t esize, int64_t plane) {
    void *base = nullptr;
    TRY(alloc(&base, (size_t)(n + 2 * plane) * esize));
    halo_bases.push_back(base);
    // zeroed on the problem's stream, ahead of any use there (a plain
    // cudaMemset runs on the legacy stream, which the problem's non-blocking
    // stream does not wait for)
    CK(cudaMemsetAsync(base, 0, (size_t)(n + 2 * plane) * esize, stream));
    *ptr = static_cast<char *>(base) + plane * esize;
    return HPCGX_OK;
  }
  void note(int launched) { launches += launched; }

  // ---- byte model of one class launch (for probes)
  double gs_bytes(int l, int q, int mode, bool mixed, double rb0 = 8.0) const {
    const LevelDev &A = L[l];
    // mixed: BF16 value per slot, columns derived from the stencil offsets
    // (FP64 with stencil columns: no column reads either)
    const double vb = mixed ? 2.0 : 8.0, cb = (mixed || A.stencil_cols) ? 0.0 : 4.0;
    const double xb = mixed ? 4.0 : 8.0;
    const double rb = l > 0 ? (mixed ? 4.0 : 8.0) : rb0;
    double total = 0.0;
    for (int px = 0; px < 2; ++px) {
      const int c = px + 2 * q, py = q & 1, pz = q >> 1;
      int64_t rows = A.ccount[c];
      double nnzb = 0.0;
      for (int s = 0; s < HPCGX_STENCIL; ++s) {
        const int dx = s % 3 - 1, dy = (s / 3) % 3 - 1, dz = s / 9 - 1;
        const int64_t cnt = axis_count(A.nx, px, dx) * axis_count(A.ny, py, dy) *
                            axis_count(A.nz, pz, dz);
        const bool skipped = (mode == GS_ZERO_GUESS) && s != HPCGX_DIAG_SLOT &&
                             ((c ^ slot_mask(s)) > c);
        nnzb += (double)cnt * (skipped ? vb : vb + cb);
      }
      double vec = rows * (rb + xb + ((mode & GS_ZERO_GUESS) ? 0.0 : xb));
      // (GS_SYM3: the class's matrix, right-hand side and x once; the second
      //  pass over colour 6 is served by L2)
      if ((mode & GS_RESTRICT) && c == 0) vec += rows * xb;
      if ((mode & GS_PROLONG) && c == 0) vec += rows * xb;
      total += nnzb + vec;
    }
    return total;
  }

  // ---- probed launch helpers (events only while capturing a graph)
  // kinds: the probe bits this launch belongs to; it is bracketed by events
  // (once) if one of them is armed and a graph is being captured.
  template <class F>
  int probed(int kinds, double bytes_model, F &&launch) {
    if (capturing) graph_bytes[capture_kind] += bytes_model;
    const int armed = capturing ? (kinds & probe) : 0;
    if (armed) {
      if (pool_next >= event_pool.size()) return fail(HPCGX_ESTATE, "probe event pool exhausted");
      Probe pr = event_pool[pool_next++];
      pr.bytes = bytes_model;
      CK(cudaEventRecordWithFlags(pr.a, stream, cudaEventRecordExternal));
      int k = launch();
      CK(cudaEventRecordWithFlags(pr.b, stream, cudaEventRecordExternal));
      for (int bit = 1; bit <= 4; bit <<= 1)
        if (k && (armed & bit)) {
          pr.kind = bit;
          probes[capture_kind].push_back(pr);
        }
      note(k);
    } else {
      note(launch());
    }
    return HPCGX_OK;
  }

  // ---- multigrid
  template <class T, class RT0>
  int gs_launch(int l, int q, int backward, int mode, const void *r, T *x, const T *xc, T *rc,
                const int *done) {
    const bool mixed = std::is_same<T, float>::value;
    const int sweep = mode;
    int kinds = 0;
    if (l == 0) {
      kinds |= HPCGX_PROBE_GS_FINE;
      if (sweep == GS_PLAIN && backward) kinds |= HPCGX_PROBE_GS_FINE_BWD;
    }
    double bytes = 0.0;
    if ((kinds & probe) || capturing) {
      bytes = gs_bytes(l, q, sweep, mixed, (double)sizeof(RT0));
    }
    return probed(kinds, bytes, [&]() {
      if (l == 0)
        return launch_gs_class<T, RT0>(L[l], q, backward, mode, static_cast<const RT0 *>(r), x,
                                       xc, rc, done, stream);
      return launch_gs_class<T, T>(L[l], q, backward, mode, static_cast<const T *>(r), x, xc,
                                   rc, done, stream);
    });
  }

  // One V-cycle (src/ComputeMG_ref.cpp:39-63) with all levels fused as
  // described in kernels.cu.  r0 / x0 are the finest level's vectors.
  template <class T, class RT0>
  int vcycle(const RT0 *r0, T *x0, const int *done) {
    const void *rl[kMaxLevels];
    T *xl[kMaxLevels];
    for (int l = 0; l < nlev; ++l) {
      rl[l] = l == 0 ? static_cast<const void *>(r0) : static_cast<const void *>(lvl_r(L[l], (T *)nullptr));
      xl[l] = l == 0 ? x0 : lvl_x(L[l], (T *)nullptr);
    }
    // Each symmetric sweep: forward classes 0..2, class 3 forward+backward in
    // one launch (GS_SYM3), backward classes 2..0 -- 7 launches.
    // descend: pre-smooth (zero initial guess) and restrict
    for (int l = 0; l + 1 < nlev; ++l) {
      for (int q = 0; q < 3; ++q)
        TRY((gs_launch<T, RT0>(l, q, 0, GS_ZERO_GUESS, rl[l], xl[l], nullptr, nullptr, done)));
      TRY((gs_launch<T, RT0>(l, 3, 0, GS_SYM3 | GS_ZERO_GUESS, rl[l], xl[l], nullptr, nullptr,
                             done)));
      for (int q = 2; q >= 0; --q)
        TRY((gs_launch<T, RT0>(l, q, 1, q == 0 ? GS_RESTRICT : GS_PLAIN, rl[l], xl[l], nullptr,
                               lvl_r(L[l + 1], (T *)nullptr), done)));
    }
    // coarsest level: one symmetric sweep from zero
    const int c = nlev - 1;
    for (int q = 0; q < 3; ++q)
      TRY((gs_launch<T, RT0>(c, q, 0, GS_ZERO_GUESS, rl[c], xl[c], nullptr, nullptr, done)));
    TRY((gs_launch<T, RT0>(c, 3, 0, GS_SYM3 | GS_ZERO_GUESS, rl[c], xl[c], nullptr, nullptr,
                           done)));
    for (int q = 2; q >= 0; --q)
      TRY((gs_launch<T, RT0>(c, q, 1, GS_PLAIN, rl[c], xl[c], nullptr, nullptr, done)));
    // ascend: prolongate and post-smooth
    for (int l = nlev - 2; l >= 0; --l) {
      for (int q = 0; q < 3; ++q)
        TRY((gs_launch<T, RT0>(l, q, 0, q == 0 ? GS_PROLONG : GS_PLAIN, rl[l], xl[l],
                               lvl_x(L[l + 1], (T *)nullptr), nullptr, done)));
      TRY((gs_launch<T, RT0>(l, 3, 0, GS_SYM3, rl[l], xl[l], nullptr, nullptr, done)));
      for (int q = 2; q >= 0; --q)
        TRY((gs_launch<T, RT0>(l, q, 1, GS_PLAIN, rl[l], xl[l], nullptr, nullptr, done)));
    }
    return HPCGX_OK;
  }

  template <class T, class RT>
  int symgs(int l, const RT *r, T *x) {
    for (int q = 0; q < 3; ++q)
      note(launch_gs_class<T, RT>(L[l], q, 0, GS_PLAIN, r, x, nullptr, nullptr, nullptr, stream));
    note(launch_gs_class<T, RT>(L[l], 3, 0, GS_SYM3, r, x, nullptr, nullptr, nullptr, stream));
    for (int q = 2; q >= 0; --q)
      note(launch_gs_class<T, RT>(L[l], q, 1, GS_PLAIN, r, x, nullptr, nullptr, nullptr, stream));
    return HPCGX_OK;
  }

  int staging() {
    for (double *&ptr : stage)
      if (!ptr) TRY(alloc((void **)&ptr, L[0].n * sizeof(double)));
    return HPCGX_OK;
  }
  int up(double *dst, const double *src, int64_t n) {
    CK(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyHostToDevice, stream));
    return HPCGX_OK;
  }
  int down(double *dst, const double *src, int64_t n) {
    CK(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    return HPCGX_OK;
  }

  int check_ready(bool mixed) {
    for (int l = 0; l < nlev; ++l)
      if (!loaded[l]) return fail(HPCGX_ESTATE, "matrix level " + std::to_string(l) + " not loaded");
    if (mixed && (!mixed_ready || mixed_stale)) {
      for (int l = 0; l < nlev; ++l) {
        LevelDev &A = L[l];
        if (!A.vals16) TRY(alloc((void **)&A.vals16, A.storage_rows * HPCGX_STENCIL * 2));
        note(launch_to_bf16(A, stream));
      }
      mixed_ready = true;
      mixed_stale = false;
    }
    return HPCGX_OK;
  }

  // ---- CG
  int iteration(int kind) {
    const int64_t n = L[0].n;
    const int *done = &st->done;
    if (kind == G_FP64_NOPREC) {
      note(launch_copy_z(n, r, z, st, stream));
    } else if (kind == G_FP64_PREC) {
      TRY((vcycle<double, double>(r, z, done)));
    } else if (fine_r32) {
      TRY((vcycle<float, float>(r32, z32, done)));
    } else {
      TRY((vcycle<float, double>(r, z32, done)));
    }
    if (capturing) CK(cudaEventRecordWithFlags(phase[kind][1], stream, cudaEventRecordExternal));
    // vector kernels, bytes per row: r.z reads r, z (and Ap); p = z + beta p
    // reads z and p and writes p, and applies the previous iteration's
    // x += alpha p (reads and writes x); r -= alpha Ap reads Ap and reads and
    // writes r
    auto vec_bytes = [&](double per_row) {
      if (capturing) graph_bytes[kind] += per_row * (double)n;
    };
    if (kind == G_FP64_NOPREC) vec_bytes(16.0);
    if (kind == G_MIXED) {
      // r.z and z.Ap_{k-1} (src/CG.cpp:109-112)
      note(launch_cg_rz<float>(n, r, z32, Ap, red, st, stream));
      vec_bytes(20.0);
      note(launch_cg_p<float>(n, z32, p, st, stream, x));
      vec_bytes(20.0 + 16.0);
    } else {
      note(launch_cg_rz<double>(n, r, z, nullptr, red, st, stream));
      note(launch_cg_p<double>(n, z, p, st, stream, x));
      vec_bytes(16.0 + 24.0 + 16.0);
    }
    if (capturing) CK(cudaEventRecordWithFlags(phase[kind][2], stream, cudaEventRecordExternal));
    // The mixed solver's FP64 SpMV derives its columns from the stencil
    // offsets; the plain FP64 solver reads the int32 column arrays.
    const bool implicit_cols = kind == G_MIXED || L[0].stencil_cols;
    double spmv_bytes = 0.0;
    if ((probe & HPCGX_PROBE_SPMV_FINE) || capturing) {
      // 12 B (8 B without column reads) per real nonzero, x and y once; the
      // fused p.Ap reads nothing extra
      int64_t nnz = 0;
      for (int s = 0; s < HPCGX_STENCIL; ++s) {
        const int dx = s % 3 - 1, dy = (s / 3) % 3 - 1, dz = s / 9 - 1;
        int64_t cx = 0, cy = 0, cz = 0;
        for (int i = 0; i < L[0].nx; ++i) cx += (i + dx >= 0 && i + dx < L[0].nx);
        for (int i = 0; i < L[0].ny; ++i) cy += (i + dy >= 0 && i + dy < L[0].ny);
        for (int i = 0; i < L[0].nz; ++i) cz += (i + dz >= 0 && i + dz < L[0].nz);
        nnz += cx * cy * cz;
      }
      spmv_bytes = (implicit_cols ? 8.0 : 12.0) * nnz + 16.0 * n;
    }
    TRY(probed(HPCGX_PROBE_SPMV_FINE, spmv_bytes, [&]() {
      return launch_spmv(L[0], p, Ap, &red, FIN_CG_PAP, st, done, stream, implicit_cols);
    }));
    if (capturing) CK(cudaEventRecordWithFlags(phase[kind][3], stream, cudaEventRecordExternal));
    float *r32_out = (kind == G_MIXED && fine_r32) ? r32 : nullptr;
    note(launch_cg_xr(n, p, Ap, nullptr, r, r32_out, red, st, stream));
    vec_bytes(r32_out ? 28.0 : 24.0);
    if (capturing) CK(cudaEventRecordWithFlags(phase[kind][4], stream, cudaEventRecordExternal));
    return HPCGX_OK;
  }

  int build_graph(int kind) {
    if (graph[kind] && graph_probe[kind] == probe) return HPCGX_OK;
    if (graph[kind]) {
      cudaGraphExecDestroy(graph[kind]);
      graph[kind] = nullptr;
      probes[kind].clear();
    }
    for (int i = 0; i < 5; ++i)
      if (!phase[kind][i]) CK(cudaEventCreate(&phase[kind][i]));
    // every launch a probe can bracket in one iteration: 14 class launches
    // per level (two symmetric sweeps of 7), plus the SpMV, with room to spare
    const size_t need = 16 * kMaxLevels + 1;
    if (probe != HPCGX_PROBE_NONE) {
      // events of earlier graphs may still be referenced: keep them, add new
      while (event_pool.size() - pool_next < need) {
        Probe pr;
        CK(cudaEventCreate(&pr.a));
        CK(cudaEventCreate(&pr.b));
        pr.bytes = 0.0;
        event_pool.push_back(pr);
      }
    }
    cudaGraph_t g = nullptr;
    const int64_t before = launches;
    graph_bytes[kind] = 0.0;
    CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    capturing = true;
    capture_kind = kind;
    cudaEventRecordWithFlags(phase[kind][0], stream, cudaEventRecordExternal);
    int rc = iteration(kind);
    capturing = false;
    cudaError_t e = cudaStreamEndCapture(stream, &g);
    graph_kernels[kind] = (int)(launches - before);
    launches = before;
    if (rc != HPCGX_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    CK(e);
    e = cudaGraphInstantiate(&graph[kind], g, 0);
    cudaGraphDestroy(g);
    CK(e);
    graph_probe[kind] = probe;
    return HPCGX_OK;
  }

  int read_probes(int kind) {
    for (auto &pr : probes[kind]) {
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, pr.a, pr.b));
      const int slot = probe_slot(pr.kind);
      probe_ms[slot] += ms;
      probe_bytes[slot] += pr.bytes;
      probe_launches[slot] += 1;
    }
    return HPCGX_OK;
  }

  int cg(int kind, const double *bu, double *xu, int max_iter, double tol, int *niters,
         double *normr, double *normr0, double *times) {
    TRY(check_ready(kind == G_MIXED));
    if (max_iter < 0) return fail(HPCGX_EINVAL, "max_iter < 0");
    const double t0 = now_s();
    const int64_t n = L[0].n;
    CgState h;
    std::memset(&h, 0, sizeof(h));
    h.tol = tol;
    h.max_iter = max_iter;
    h.flexible = kind == G_MIXED;
    CK(cudaMemcpyAsync(st, &h, sizeof(h), cudaMemcpyHostToDevice, stream));
    // p = x (CopyVector, src/CG.cpp:86); x lives in the problem's own buffer so
    // that the iteration graph never changes
    if (xu != x) CK(cudaMemcpyAsync(x, xu, n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    CK(cudaMemcpyAsync(p, x, n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    note(launch_spmv(L[0], p, Ap, nullptr, 0, nullptr, nullptr, stream, kind == G_MIXED));
    note(launch_cg_init(n, bu, Ap, r, (kind == G_MIXED && fine_r32) ? r32 : nullptr, red, st,
                        stream));
    TRY(build_graph(kind));
    const bool per_iter = tol > 0.0 || probe != HPCGX_PROBE_NONE || times != nullptr;
    double t_mg = 0, t_vec = 0, t_spmv = 0;
    int launched = 0;
    while (launched < max_iter) {
      const int batch = per_iter ? 1 : max_iter - launched;
      for (int i = 0; i < batch; ++i) {
        CK(cudaGraphLaunch(graph[kind], stream));
        launches += graph_kernels[kind];
      }
      launched += batch;
      CK(cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
      if (per_iter && h.niters == launched) {
        float a = 0, b2 = 0, c = 0;
        CK(cudaEventElapsedTime(&a, phase[kind][0], phase[kind][1]));
        CK(cudaEventElapsedTime(&b2, phase[kind][1], phase[kind][2]));
        CK(cudaEventElapsedTime(&c, phase[kind][2], phase[kind][3]));
        float d = 0;
        CK(cudaEventElapsedTime(&d, phase[kind][3], phase[kind][4]));
        t_mg += a * 1e-3;
        t_vec += (b2 + d) * 1e-3;
        t_spmv += c * 1e-3;
        TRY(read_probes(kind));
      }
      if (h.done) break;
    }
    if (launched == 0) {
      // max_iter == 0: no iteration ran, but the initial residual norm is
      // still a result (src/CG.cpp:89-96 sets normr and normr0 before the loop)
      CK(cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, stream));
    }
    // the last iteration's x += alpha p, deferred by k_cg_p
    note(launch_cg_xflush(n, p, x, st, stream));
    if (xu != x) CK(cudaMemcpyAsync(xu, x, n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    CK(cudaStreamSynchronize(stream));
    if (niters) *niters = h.niters;
    if (normr) *normr = h.normr;
    if (normr0) *normr0 = h.normr0;
    if (times) {
      times[0] += now_s() - t0;
      times[2] += t_vec;
      times[3] += t_spmv;
      times[5] += t_mg;
    }
    if (h.nonfinite) return fail(HPCGX_ENONFINITE, "CG: residual norm is not finite");
    return HPCGX_OK;
  }

  // ---- sharded operations as step lists
  // The steps of one operation on this rank: kernel launches, halo exchanges
  // of a level vector (src/ExchangeHalo.cpp:34-110) and sums over the ranks of
  // the deferred reduction totals followed by their scalar step (the
  // MPI_Allreduce of src/ComputeDotProduct_ref.cpp:66-77).  Every rank plans
  // the same sequence; a runner executes it over NCCL or in-process.
  Reduce deferred() const {
    Reduce d = red;
    d.defer = gsum;
    return d;
  }
  void add(Plan &pl, std::function<int()> f) {
    Step s;
    s.kind = STEP_LAUNCH;
    s.launch = std::move(f);
    pl.push_back(std::move(s));
  }
  void add_halo(Plan &pl, int l, void *v, int esize, std::function<int()> interior = {}) {
    Step s;
    s.kind = STEP_HALO;
    s.level = l;
    s.vec = v;
    s.esize = esize;
    s.interior = std::move(interior);
    pl.push_back(std::move(s));
  }
  void add_sum(Plan &pl, int fin, int nv) {
    Step s;
    s.kind = STEP_SUM;
    s.fin = fin;
    s.nv = nv;
    pl.push_back(std::move(s));
  }
  // The halo planes of x read as zero (the first sweep after ZeroVector:
  // ExchangeHalo of a zero vector, src/ComputeMG_ref.cpp:42 + src/ComputeSYMGS_ref.cpp:56).
  template <class T>
  int zero_halo(int l, T *x) {
    const LevelDev &A = L[l];
    const int64_t plane = (int64_t)A.nx * A.ny;
    if (A.zlo) CK(cudaMemsetAsync(x - plane, 0, plane * sizeof(T), stream));
    if (A.zhi) CK(cudaMemsetAsync(x + A.n, 0, plane * sizeof(T), stream));
    return HPCGX_OK;
  }
  // One symmetric sweep of level l (7 class launches).  xc: the first
  // forward class adds the prolongated correction (GS_PROLONG); rc: the last
  // backward class forms the restricted residual (GS_RESTRICT).  halo: the
  // sweep starts with the halo exchange of x (src/ComputeSYMGS_ref.cpp:56),
  // and the first launch -- class 0 forward, the planes iz = 0, 2, ... --
  // runs its lines above plane 0 (which read no halo plane, and write none of
  // the planes sent) beside the exchange, then the lines of plane 0.  The
  // halo above is read first by class 2, launches later.
  template <class T, class RT>
  void plan_sweeps(Plan &pl, int l, const RT *r, T *x, bool zero, const int *done,
                   const T *xc = nullptr, T *rc = nullptr, bool halo = false) {
    const int m0 = zero ? GS_ZERO_GUESS : GS_PLAIN;
    for (int q = 0; q < 3; ++q) {
      const int m = (q == 0 && xc) ? GS_PROLONG : m0;
      if (q == 0 && halo) {
        const int nyq = L[l].cls[0].nyq;
        add_halo(pl, l, x, sizeof(T), [=]() {
          note(launch_gs_class<T, RT>(L[l], 0, 0, m, r, x, xc, nullptr, done, stream, nyq, -1));
          return HPCGX_OK;
        });
        add(pl, [=]() {
          note(launch_gs_class<T, RT>(L[l], 0, 0, m, r, x, xc, nullptr, done, stream, 0, nyq));
          return HPCGX_OK;
        });
        continue;
      }
      add(pl, [=]() {
        note(launch_gs_class<T, RT>(L[l], q, 0, m, r, x, xc, nullptr, done, stream));
        return HPCGX_OK;
      });
    }
    add(pl, [=]() {
      note(launch_gs_class<T, RT>(L[l], 3, 0, GS_SYM3 | m0, r, x, nullptr, nullptr, done, stream));
      return HPCGX_OK;
    });
    for (int q = 2; q >= 0; --q) {
      const int m = (q == 0 && rc) ? GS_RESTRICT : GS_PLAIN;
      add(pl, [=]() {
        note(launch_gs_class<T, RT>(L[l], q, 1, m, r, x, nullptr, rc, done, stream));
        return HPCGX_OK;
      });
    }
  }
  // The V-cycle of src/ComputeMG_ref.cpp:39-63 on a z-slab.  The reference
  // exchanges the halo of x between the pre-smoother and the residual and
  // between the prolongation and the post-smoother.  Only the first plane of
  // a slab (even z, injected) reads the halo below, and no injected point
  // reads the halo above (the local z-extent is even), so restriction and
  // prolongation stay fused into the sweeps and two one-plane launches
  // restore the reference's order there: after the exchange that follows the
  // pre-smoother, the first plane's residual is formed again; before the
  // exchange that precedes the post-smoother, the first plane receives its
  // correction (which the fused prolongation then skips).  x0 must be a
  // haloed vector.
  template <class T, class RT0>
  void plan_vcycle(Plan &pl, const RT0 *r0, T *x0, const int *done) {
    T *xl[kMaxLevels];
    for (int l = 0; l < nlev; ++l) xl[l] = l == 0 ? x0 : lvl_x(L[l], (T *)nullptr);
    auto rl = [&](int l) { return lvl_r(L[l], (T *)nullptr); };
    for (int l = 0; l + 1 < nlev; ++l) {
      T *x = xl[l];
      T *rc = rl(l + 1);
      add(pl, [=]() { return zero_halo<T>(l, x); });
      if (l == 0)
        plan_sweeps<T, RT0>(pl, 0, r0, x, true, done, nullptr, rc);
      else
        plan_sweeps<T, T>(pl, l, rl(l), x, true, done, nullptr, rc);
      add_halo(pl, l, x, sizeof(T));
      // (every rank plans the same steps; the one-plane launches are empty
      //  on a slab without a halo below)
      const int64_t plane_c = L[l].zlo ? (int64_t)L[l + 1].nx * L[l + 1].ny : 0;
      if (l == 0)
        add(pl, [=]() {
          note(launch_restrict_residual<T, RT0>(L[0], plane_c, r0, x, rc, done, stream));
          return HPCGX_OK;
        });
      else {
        const T *rf = rl(l);
        add(pl, [=]() {
          note(launch_restrict_residual<T, T>(L[l], plane_c, rf, x, rc, done, stream));
          return HPCGX_OK;
        });
      }
    }
    const int c = nlev - 1;
    {
      T *x = xl[c];
      add(pl, [=]() { return zero_halo<T>(c, x); });
      if (c == 0)
        plan_sweeps<T, RT0>(pl, 0, r0, x, true, done);
      else
        plan_sweeps<T, T>(pl, c, rl(c), x, true, done);
    }
    for (int l = nlev - 2; l >= 0; --l) {
      T *x = xl[l];
      const T *xc = xl[l + 1];
      const int64_t plane_c = L[l].zlo ? (int64_t)L[l + 1].nx * L[l + 1].ny : 0;
      add(pl, [=]() {
        note(launch_prolong<T>(L[l], plane_c, xc, x, done, stream));
        return HPCGX_OK;
      });
      if (l == 0)
        plan_sweeps<T, RT0>(pl, 0, r0, x, false, done, xc, nullptr, true);
      else
        plan_sweeps<T, T>(pl, l, rl(l), x, false, done, xc, nullptr, true);
    }
  }
  // The haloed staging vector of level l (operator inputs arrive without halo).
  int staging_halo(int l, double **out) {
    if (!hstage[l]) {
      const int64_t plane = (int64_t)L[l].nx * L[l].ny;
      TRY(alloc_halo((void **)&hstage[l], L[l].n, sizeof(double), plane));
    }
    *out = hstage[l];
    return HPCGX_OK;
  }
  void plan_copy(Plan &pl, const double *from, double *to, int64_t n) {
    add(pl, [=]() {
      CK(cudaMemcpyAsync(to, from, n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
      return HPCGX_OK;
    });
  }
  int plan_spmv(Plan &pl, int l, const double *x, double *y) {
    double *xs = nullptr;
    TRY(staging_halo(l, &xs));
    plan_copy(pl, x, xs, L[l].n);
    add_halo(pl, l, xs, sizeof(double));
    add(pl, [=]() {
      note(launch_spmv(L[l], xs, y, nullptr, 0, nullptr, nullptr, stream));
      return HPCGX_OK;
    });
    return HPCGX_OK;
  }
  int plan_symgs(Plan &pl, int l, const double *r, double *x) {
    double *xs = nullptr;
    TRY(staging_halo(l, &xs));
    plan_copy(pl, x, xs, L[l].n);
    // the halo exchange of src/ComputeSYMGS_ref.cpp:56 opens the sweep
    plan_sweeps<double, double>(pl, l, r, xs, false, nullptr, nullptr, nullptr, true);
    plan_copy(pl, xs, x, L[l].n);
    return HPCGX_OK;
  }
  int plan_mg(Plan &pl, const double *r, double *x) {
    double *xs = nullptr;
    TRY(staging_halo(0, &xs));
    plan_vcycle<double, double>(pl, r, xs, nullptr);
    plan_copy(pl, xs, x, L[0].n);
    return HPCGX_OK;
  }
  // CG set-up (src/CG.cpp:86-92): p = x, Ap = A p, r = b - Ap, normr0.
  void plan_cg_init(Plan &pl, int kind, const double *bu) {
    const int64_t n = L[0].n;
    add(pl, [=]() {
      CK(cudaMemcpyAsync(p, x, n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
      return HPCGX_OK;
    });
    add_halo(pl, 0, p, sizeof(double));
    add(pl, [=]() {
      note(launch_spmv(L[0], p, Ap, nullptr, 0, nullptr, nullptr, stream, kind == G_MIXED));
      return HPCGX_OK;
    });
    add(pl, [=]() {
      note(launch_cg_init(n, bu, Ap, r, nullptr, deferred(), st, stream));
      return HPCGX_OK;
    });
    add_sum(pl, FIN_CG_INIT, 1);
  }
  // One CG iteration (src/CG.cpp:100-130): the fused kernels of the one-GPU
  // iteration with every reduction summed over the ranks before its scalar step.
  void plan_cg_iteration(Plan &pl, int kind) {
    const int64_t n = L[0].n;
    const int *done = &st->done;
    if (kind == G_FP64_NOPREC)
      add(pl, [=]() {
        note(launch_copy_z(n, r, z, st, stream));
        return HPCGX_OK;
      });
    else if (kind == G_FP64_PREC)
      plan_vcycle<double, double>(pl, r, z, done);
    const bool mixed = kind == G_MIXED;
    if (mixed) plan_vcycle<float, double>(pl, r, z32, done);
    add(pl, [=]() {
      if (mixed) {
        note(launch_cg_rz<float>(n, r, z32, Ap, deferred(), st, stream));
      } else {
        note(launch_cg_rz<double>(n, r, z, nullptr, deferred(), st, stream));
      }
      return HPCGX_OK;
    });
    add_sum(pl, FIN_CG_RZ, mixed ? 2 : 1);
    add(pl, [=]() {
      if (mixed)
        note(launch_cg_p<float>(n, z32, p, st, stream, x));
      else
        note(launch_cg_p<double>(n, z, p, st, stream, x));
      return HPCGX_OK;
    });
    add_halo(pl, 0, p, sizeof(double));
    add(pl, [=]() {
      const Reduce d = deferred();
      note(launch_spmv(L[0], p, Ap, &d, FIN_CG_PAP, st, done, stream, mixed));
      return HPCGX_OK;
    });
    add_sum(pl, FIN_CG_PAP, 1);
    add(pl, [=]() {
      note(launch_cg_xr(n, p, Ap, nullptr, r, nullptr, deferred(), st, stream));
      return HPCGX_OK;
    });
    add_sum(pl, FIN_CG_RR, 1);
  }
};

void nccl_release(NcclLink *link);

hpcgx_problem::~hpcgx_problem() {
  cudaSetDevice(device);
  if (comm_stream) cudaStreamSynchronize(comm_stream);
  if (nccl) nccl_release(nccl);
  if (stream) cudaStreamSynchronize(stream);
  if (ev_ready) cudaEventDestroy(ev_ready);
  if (ev_halo) cudaEventDestroy(ev_halo);
  if (comm_stream) cudaStreamDestroy(comm_stream);
  for (auto &pr : event_pool) {
    cudaEventDestroy(pr.a);
    cudaEventDestroy(pr.b);
  }
  for (int k = 0; k < G_COUNT; ++k) {
    if (graph[k]) cudaGraphExecDestroy(graph[k]);
    for (int i = 0; i < 5; ++i)
      if (phase[k][i]) cudaEventDestroy(phase[k][i]);
  }
  for (int l = 0; l < kMaxLevels; ++l) {
    cudaFree(L[l].vals);
    cudaFree(L[l].cols);
    cudaFree(L[l].vals16);
    cudaFree(L[l].r64);
    cudaFree(L[l].r32);
  }
  for (double *ptr : stage) cudaFree(ptr);
  for (void *ptr : halo_bases) cudaFree(ptr);
  for (int h = 0; h < 2; ++h) {
    if (pin_copied[h]) cudaEventDestroy(pin_copied[h]);
    if (pin_vals[h]) cudaFreeHost(pin_vals[h]);
    if (pin_cols[h]) cudaFreeHost(pin_cols[h]);
  }
  for (void *ptr : {(void *)b, (void *)x, (void *)r, (void *)r32, (void *)Ap, (void *)tmp,
                    (void *)result,
                    (void *)st, (void *)gsum, (void *)red.partials, (void *)red.counter})
    cudaFree(ptr);
  if (gen) general_destroy(gen);
  if (own_stream) cudaStreamDestroy(own_stream);
}

namespace {

#define HANDLE(p)                                                          \
  do {                                                                     \
    if (!(p)) return fail(HPCGX_EINVAL, "null problem handle");            \
    cudaError_t e_ = cudaSetDevice((p)->device);                          \
    if (e_ != cudaSuccess) return cuda_fail(e_);                        \
  } while (0)

int check_level(hpcgx_problem *p, int level) {
  if (level < 0 || level >= p->nlev)
    return fail(HPCGX_EINVAL, "level " + std::to_string(level) + " out of range");
  return HPCGX_OK;
}

// Operators that exist only for the 27-point stencil layout.
int stencil_only(hpcgx_problem *p, const char *what) {
  if (p->gen)
    return fail(HPCGX_ESTATE, std::string(what) + " is not available on a general-pattern problem");
  return HPCGX_OK;
}

int general_ready_or_fail(hpcgx_problem *p) {
  if (!general_ready(p->gen)) return fail(HPCGX_ESTATE, "not every level is loaded");
  return HPCGX_OK;
}

// Runs f(begin, end) over [0, n) on the host's cores.
template <class F>
void parallel_for(int64_t n, F f) {
  const unsigned hw = std::thread::hardware_concurrency();
  const int64_t nt = std::max<int64_t>(1, std::min<int64_t>(hw ? hw : 1, 64));
  if (n < 65536 || nt == 1) {
    f(0, n, 0);
    return;
  }
  std::vector<std::thread> ts;
  const int64_t chunk = (n + nt - 1) / nt;
  for (int64_t t = 0; t < nt; ++t) {
    const int64_t a = t * chunk, b = std::min(n, a + chunk);
    if (a < b) ts.emplace_back(f, a, b, (int)t);
  }
  for (auto &th : ts) th.join();
}

// Natural row of storage row k, or -1 for a row that only pads a colour to a
// multiple of 32 (the inverse of storage_row_host).
int64_t natural_row_host(const LevelDev &A, int64_t k, int &ix, int &iy, int &iz) {
  for (int c = 0; c < 8; ++c) {
    if (k < A.cstart[c] || k >= A.cstart[c] + A.ccount[c]) continue;
    const int px = c & 1, q = c >> 1;
    const int64_t off = k - A.cstart[c], len = A.cls[q].len[px];
    const int64_t j = off / len;
    ix = (int)(2 * (off - j * len) + px);
    const int64_t jz = j / A.cls[q].nyq;
    iy = (int)(2 * (j - jz * A.cls[q].nyq) + (q & 1));
    iz = (int)(2 * jz + (q >> 1));
    return ix + A.nx * (iy + (int64_t)A.ny * iz);
  }
  return -1;
}


// Shared body of the two host loaders: get(i, j, col, val) yields entry j of
// row i.  The level is filled in chunks of 4096 slices in storage order: the
// host's cores validate and scatter the rows of one chunk into pinned
// staging while the previous chunk is copied to the device.  On a malformed
// row the load stops, the level is left unloaded, and the failing row with
// the lowest index is reported.
template <class Nnz, class Get>
int load_level_impl(hpcgx_problem *p, int level, Nnz nnz_of, Get get) {
  TRY(check_level(p, level));
  LevelDev &A = p->L[level];
  // One row: validates it and writes its 27 slots through put(s, col, val);
  // returns an empty string or what is wrong with the row.
  auto scan_row = [&](int64_t row, auto put) -> std::string {
    const int ix = (int)(row % A.nx), iy = (int)((row / A.nx) % A.ny),
              iz = (int)(row / ((int64_t)A.nx * A.ny));
    for (int s = 0; s < HPCGX_STENCIL; ++s) put(s, (int32_t)row, 0.0);
    const int nz = nnz_of(row);
    if (nz < 1 || nz > HPCGX_STENCIL) return std::to_string(nz) + " entries";
    int last = -1;
    bool diag = false;
    for (int j = 0; j < nz; ++j) {
      int32_t col;
      double v;
      get(row, j, col, v);
      if (col < 0 || col >= A.n) return "column out of range";
      const int jx = col % A.nx, jy = (col / A.nx) % A.ny,
                jz = (int)(col / ((int64_t)A.nx * A.ny));
      const int dx = jx - ix, dy = jy - iy, dz = jz - iz;
      if (dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 || dz > 1)
        return "column " + std::to_string(col) + " is not a stencil neighbour";
      const int s = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
      if (s <= last) return "entries not in stencil order";
      last = s;
      diag |= (s == HPCGX_DIAG_SLOT);
      put(s, col, v);
    }
    if (!diag) return "no diagonal";
    return std::string();
  };
  // The common case without a division per entry: walk the 27 slots once,
  // matching each entry's column to the next slot whose neighbour exists.
  // Columns of existing neighbours are distinct, so this accepts exactly the
  // rows scan_row accepts; a row it rejects goes to scan_row for the message.
  int64_t off[HPCGX_STENCIL];
  for (int s = 0; s < HPCGX_STENCIL; ++s)
    off[s] = (s % 3 - 1) + (int64_t)A.nx * ((s / 3) % 3 - 1 + (int64_t)A.ny * (s / 9 - 1));
  auto fast_row = [&](int64_t row, int ix, int iy, int iz, auto put) -> bool {
    for (int s = 0; s < HPCGX_STENCIL; ++s) put(s, (int32_t)row, 0.0);
    const int nz = nnz_of(row);
    if (nz < 1 || nz > HPCGX_STENCIL) return false;
    const bool okx[3] = {ix > 0, true, ix + 1 < A.nx}, oky[3] = {iy > 0, true, iy + 1 < A.ny},
               okz[3] = {iz > 0, true, iz + 1 < A.nz};
    int s = 0;
    bool diag = false;
    for (int j = 0; j < nz; ++j) {
      int32_t col;
      double v;
      get(row, j, col, v);
      for (;; ++s) {
        if (s == HPCGX_STENCIL) return false;
        if (okx[s % 3] && oky[(s / 3) % 3] && okz[s / 9] && row + off[s] == col) break;
      }
      diag |= (s == HPCGX_DIAG_SLOT);
      put(s, col, v);
      ++s;
    }
    return diag;
  };
  p->loaded[level] = false;
  p->mixed_stale = true;
  const int64_t slices = A.storage_rows / HPCGX_SLICE;
  TRY(p->pinned_staging());
  bool pending[2] = {false, false};
  bool failed = false;
  std::vector<char> bad(64);
  for (int64_t c0 = 0, it = 0; c0 < slices && !failed; c0 += kPinnedSlices, ++it) {
    const int h = (int)(it & 1);
    double *bv = p->pin_vals[h];
    int32_t *bc = p->pin_cols[h];
    if (pending[h]) CK(cudaEventSynchronize(p->pin_copied[h]));
    pending[h] = false;
    const int64_t c1 = std::min(slices, c0 + kPinnedSlices);
    const int64_t k0 = c0 * HPCGX_SLICE, e0 = c0 * kSliceElems;
    parallel_for((c1 - c0) * HPCGX_SLICE, [&](int64_t a, int64_t e, int t) {
      for (int64_t k = k0 + a; k < k0 + e; ++k) {
        int ix, iy, iz;
        const int64_t row = natural_row_host(A, k, ix, iy, iz);
        if (row < 0) {   // padding: value 0, column 0
          for (int s = 0; s < HPCGX_STENCIL; ++s) {
            bv[vidx(k, s) - e0] = 0.0;
            bc[cidx(k, s) - e0] = 0;
          }
          continue;
        }
        auto put = [&](int s, int32_t col, double v) {
          bv[vidx(k, s) - e0] = v;
          bc[cidx(k, s) - e0] = col;
        };
        if (!fast_row(row, ix, iy, iz, put) && !scan_row(row, put).empty()) {
          bad[t] = 1;
          return;
        }
      }
    });
    for (char f : bad) failed |= f != 0;
    if (failed) break;
    const size_t ne = (size_t)(c1 - c0) * kSliceElems;
    CK(cudaMemcpyAsync(A.vals + e0, bv, ne * sizeof(double), cudaMemcpyHostToDevice, p->stream));
    CK(cudaMemcpyAsync(A.cols + e0, bc, ne * sizeof(int32_t), cudaMemcpyHostToDevice,
                       p->stream));
    CK(cudaEventRecord(p->pin_copied[h], p->stream));
    pending[h] = true;
  }
  CK(cudaStreamSynchronize(p->stream));
  if (failed) {
    // the lowest failing row: each thread's first in natural order
    std::vector<int64_t> first(64, -1);
    std::vector<std::string> msg(64);
    parallel_for(A.n, [&](int64_t a, int64_t e, int t) {
      for (int64_t row = a; row < e; ++row) {
        const std::string m = scan_row(row, [](int, int32_t, double) {});
        if (!m.empty()) {
          first[t] = row;
          msg[t] = m;
          return;
        }
      }
    });
    for (int t = 0; t < 64; ++t)
      if (first[t] >= 0) return fail(HPCGX_ELAYOUT, "row " + std::to_string(first[t]) + ": " + msg[t]);
    return fail(HPCGX_ELAYOUT, "malformed row");
  }
  p->loaded[level] = true;
  return HPCGX_OK;
}

}  // namespace

// ======================================================================
// Sharding backends.
//
// NCCL is opened at run time -- the library torch.distributed already loaded
// when there is one, else the system's -- so single-GPU users of libhpcgx need
// no NCCL; only the types come from nccl.h.
struct NcclApi {
  ncclResult_t (*GetUniqueId)(ncclUniqueId *) = nullptr;
  ncclResult_t (*CommInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*Send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*Recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*AllReduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                            cudaStream_t) = nullptr;
  ncclResult_t (*GroupStart)() = nullptr;
  ncclResult_t (*GroupEnd)() = nullptr;
  const char *(*GetErrorString)(ncclResult_t) = nullptr;
  ncclResult_t (*CommInitRankConfig)(ncclComm_t *, int, ncclUniqueId, int, ncclConfig_t *) = nullptr;
  ncclResult_t (*CommGetAsyncError)(ncclComm_t, ncclResult_t *) = nullptr;
  ncclResult_t (*CommAbort)(ncclComm_t) = nullptr;
};

static NcclApi *nccl_api() {
  static NcclApi api;
  static bool ok = false;
  static std::once_flag once;
  std::call_once(once, []() {
    void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
    if (!h) return;
    api.GetUniqueId = (decltype(api.GetUniqueId))dlsym(h, "ncclGetUniqueId");
    api.CommInitRank = (decltype(api.CommInitRank))dlsym(h, "ncclCommInitRank");
    api.CommDestroy = (decltype(api.CommDestroy))dlsym(h, "ncclCommDestroy");
    api.Send = (decltype(api.Send))dlsym(h, "ncclSend");
    api.Recv = (decltype(api.Recv))dlsym(h, "ncclRecv");
    api.AllReduce = (decltype(api.AllReduce))dlsym(h, "ncclAllReduce");
    api.GroupStart = (decltype(api.GroupStart))dlsym(h, "ncclGroupStart");
    api.GroupEnd = (decltype(api.GroupEnd))dlsym(h, "ncclGroupEnd");
    api.GetErrorString = (decltype(api.GetErrorString))dlsym(h, "ncclGetErrorString");
    api.CommInitRankConfig =
        (decltype(api.CommInitRankConfig))dlsym(h, "ncclCommInitRankConfig");
    api.CommGetAsyncError = (decltype(api.CommGetAsyncError))dlsym(h, "ncclCommGetAsyncError");
    api.CommAbort = (decltype(api.CommAbort))dlsym(h, "ncclCommAbort");
    ok = api.GetUniqueId && api.CommInitRank && api.CommDestroy && api.Send && api.Recv &&
         api.AllReduce && api.GroupStart && api.GroupEnd && api.GetErrorString &&
         api.CommInitRankConfig && api.CommGetAsyncError && api.CommAbort;
  });
  return ok ? &api : nullptr;
}

// The communicator is non-blocking (ncclConfig_t::blocking = 0): a call may
// return ncclInProgress, and the communicator's state is then polled with
// ncclCommGetAsyncError until it settles -- for at most HPCGX_WAIT_TIMEOUT_S,
// after which the communicator is aborted (ncclCommAbort, which also stops
// its kernels) and the call returns HPCGX_ETIMEOUT instead of blocking
// behind a peer that has failed.  The reference aborts on a failed exchange
// too (src/ExchangeHalo.cpp:102-104).
struct NcclLink {
  ncclComm_t comm = nullptr;
  bool aborted = false;
};

double wait_limit_s() {
  static const double limit = [] {
    const char *e = std::getenv("HPCGX_WAIT_TIMEOUT_S");
    const double v = e ? std::atof(e) : 0.0;
    return v > 0.0 ? v : 600.0;
  }();
  return limit;
}

void nccl_abort(NcclLink *link) {
  if (link->comm && !link->aborted && nccl_api()) nccl_api()->CommAbort(link->comm);
  link->aborted = true;
}

void nccl_release(NcclLink *link) {
  if (link->comm && !link->aborted && nccl_api()) nccl_api()->CommDestroy(link->comm);
  delete link;
}

// Waits (bounded) until the communicator has settled after a call that
// returned r; aborts it on a timeout or an error.
// Fault injection for tests, on the host: HPCGX_FAULT_NCCL_STALL=k makes the
// first k settles of the process see a communicator that never leaves
// ncclInProgress, as behind a peer that has died (no GPU fault involved).
bool nccl_fake_stall() {
  static std::atomic<int> left{env_int("HPCGX_FAULT_NCCL_STALL", 0)};
  return left.fetch_sub(1) > 0;
}

int nccl_settle(NcclLink *link, ncclResult_t r, const char *what) {
  NcclApi *api = nccl_api();
  const double t0 = now_s();
  const bool stall = (r == ncclSuccess || r == ncclInProgress) && nccl_fake_stall();
  if (stall) r = ncclInProgress;
  for (int polls = 0; r == ncclInProgress; ++polls) {
    if (api->CommGetAsyncError(link->comm, &r) != ncclSuccess) r = ncclInternalError;
    if (stall && r == ncclSuccess) r = ncclInProgress;
    if (r != ncclInProgress) break;
    if (now_s() - t0 > wait_limit_s()) {
      nccl_abort(link);
      return fail(HPCGX_ETIMEOUT, std::string(what) +
                                      ": the NCCL communicator did not settle within "
                                      "HPCGX_WAIT_TIMEOUT_S; it was aborted");
    }
    if (polls > 2000) std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  if (r != ncclSuccess) {
    nccl_abort(link);
    return fail(HPCGX_ECOMM, std::string(what) + ": " + api->GetErrorString(r) +
                                 " (the communicator was aborted)");
  }
  return HPCGX_OK;
}

#define NCCLCK(link, call) TRY(nccl_settle((link), (call), #call))

namespace {

// Halo exchange of one level vector of a z-slab over NCCL: this rank's first
// plane to the rank below (its upper halo), its last plane to the rank above
// (its lower halo), and the converse into this rank's halo planes.
int nccl_halo(hpcgx_problem *p, int l, void *v, int esize, cudaStream_t s) {
  const LevelDev &A = p->L[l];
  if (!A.zlo && !A.zhi) return HPCGX_OK;
  NcclApi *api = nccl_api();
  const size_t plane = (size_t)A.nx * A.ny;
  const ncclDataType_t t = esize == 8 ? ncclFloat64 : ncclFloat32;
  char *b = static_cast<char *>(v);
  NcclLink *link = p->nccl;
  ncclComm_t c = link->comm;
  // inside a group the calls only record the operations; GroupEnd issues them
  ncclResult_t r = api->GroupStart();
  if (A.zlo && (r == ncclSuccess || r == ncclInProgress)) {
    r = api->Send(b, plane, t, p->rank - 1, c, s);
    if (r == ncclSuccess || r == ncclInProgress)
      r = api->Recv(b - plane * esize, plane, t, p->rank - 1, c, s);
  }
  if (A.zhi && (r == ncclSuccess || r == ncclInProgress)) {
    r = api->Send(b + (A.n - (int64_t)plane) * esize, plane, t, p->rank + 1, c, s);
    if (r == ncclSuccess || r == ncclInProgress)
      r = api->Recv(b + A.n * esize, plane, t, p->rank + 1, c, s);
  }
  const ncclResult_t e = api->GroupEnd();
  if (r == ncclSuccess || r == ncclInProgress) r = e;
  NCCLCK(link, r);
  return HPCGX_OK;
}

// The same exchange through the caller's halo function.
int callback_halo(hpcgx_problem *p, int l, void *v, int esize) {
  const LevelDev &A = p->L[l];
  if (!A.zlo && !A.zhi) return HPCGX_OK;
  const int64_t plane = (int64_t)A.nx * A.ny;
  char *b = static_cast<char *>(v);
  void *send_lo = A.zlo ? b : nullptr;
  void *recv_lo = A.zlo ? b - plane * esize : nullptr;
  void *send_hi = A.zhi ? b + (A.n - plane) * esize : nullptr;
  void *recv_hi = A.zhi ? b + A.n * esize : nullptr;
  if (p->comm_halo(p->comm_ctx, send_lo, recv_lo, send_hi, recv_hi, plane, esize,
                   static_cast<void *>(p->stream)) != 0)
    return fail(HPCGX_ECOMM, "the halo function failed");
  return HPCGX_OK;
}

// Runs one rank's plan: halo steps and sums of the deferred totals over the
// attached backend (NCCL or the caller's functions).  Without one (one rank)
// both are no-ops.
int run_plan(hpcgx_problem *p, Plan &pl) {
  if (p->nccl && p->nccl->aborted)
    return fail(HPCGX_ESTATE, "the NCCL communicator was aborted after a timeout or an error; "
                              "attach a new one (hpcgx_attach_nccl)");
  for (Step &s : pl) {
    if (s.kind == STEP_LAUNCH) {
      TRY(s.launch());
    } else if (s.kind == STEP_HALO) {
      if (p->nccl && s.interior) {
        // the exchange on the side stream once x is complete; the interior
        // work beside it; the rest of the plan after it
        TRY(p->overlap_streams());
        CK(cudaEventRecord(p->ev_ready, p->stream));
        CK(cudaStreamWaitEvent(p->comm_stream, p->ev_ready, 0));
        TRY(nccl_halo(p, s.level, s.vec, s.esize, p->comm_stream));
        CK(cudaEventRecord(p->ev_halo, p->comm_stream));
        TRY(s.interior());
        CK(cudaStreamWaitEvent(p->stream, p->ev_halo, 0));
        continue;
      }
      if (p->nccl) TRY(nccl_halo(p, s.level, s.vec, s.esize, p->stream));
      else if (p->comm_halo) TRY(callback_halo(p, s.level, s.vec, s.esize));
      if (s.interior) TRY(s.interior());
    } else {
      if (p->nccl)
        NCCLCK(p->nccl, nccl_api()->AllReduce(p->gsum, p->gsum, s.nv, ncclFloat64, ncclSum,
                                              p->nccl->comm, p->stream));
      else if (p->comm_sum &&
               p->comm_sum(p->comm_ctx, p->gsum, s.nv, static_cast<void *>(p->stream)) != 0)
        return fail(HPCGX_ECOMM, "the sum function failed");
      if (s.fin >= 0) p->note(launch_finish(s.fin, s.nv, p->gsum, p->st, p->stream));
    }
  }
  CK(cudaGetLastError());
  return HPCGX_OK;
}

}  // namespace

// Every rank of a z-slab decomposition held by one process on one GPU and one
// stream: the ranks' plans run step by step in lockstep, halo steps become
// device copies between the ranks' vectors and sums add the ranks' totals in
// rank order.  It runs the multi-rank algorithm on a single GPU (tests,
// emulation) without kernels that wait on each other.
struct hpcgx_group {
  std::vector<hpcgx_problem *> ranks;
  std::vector<cudaStream_t> saved;   // each rank's stream before the group
  double **bufs = nullptr;           // device array of every rank's gsum
  ~hpcgx_group() {
    if (bufs) cudaFree(bufs);
  }
};

namespace {

using Runner = std::function<int(std::vector<Plan> &)>;

int group_run(hpcgx_group *g, std::vector<Plan> &plans) {
  const int P = (int)g->ranks.size();
  const size_t ns = plans[0].size();
  for (const Plan &pl : plans)
    if (pl.size() != ns) return fail(HPCGX_ESTATE, "ranks planned different step sequences");
  hpcgx_problem *p0 = g->ranks[0];
  cudaStream_t s = p0->stream;
  for (size_t i = 0; i < ns; ++i) {
    const Step &s0 = plans[0][i];
    for (int r = 1; r < P; ++r)
      if (plans[r][i].kind != s0.kind) return fail(HPCGX_ESTATE, "ranks planned different steps");
    if (s0.kind == STEP_LAUNCH) {
      for (int r = 0; r < P; ++r) TRY(plans[r][i].launch());
    } else if (s0.kind == STEP_HALO) {
      for (int r = 0; r < P; ++r) {
        const Step &st = plans[r][i];
        const LevelDev &A = g->ranks[r]->L[st.level];
        const int64_t plane = (int64_t)A.nx * A.ny;
        const size_t pb = (size_t)plane * st.esize;
        const char *v = static_cast<const char *>(st.vec);
        if (r + 1 < P)   // last plane -> lower halo of the rank above
          CK(cudaMemcpyAsync(static_cast<char *>(plans[r + 1][i].vec) - pb,
                             v + (A.n - plane) * st.esize, pb, cudaMemcpyDeviceToDevice, s));
        if (r > 0)       // first plane -> upper halo of the rank below
          CK(cudaMemcpyAsync(static_cast<char *>(plans[r - 1][i].vec) + A.n * st.esize, v, pb,
                             cudaMemcpyDeviceToDevice, s));
      }
      for (int r = 0; r < P; ++r)
        if (plans[r][i].interior) TRY(plans[r][i].interior());
    } else {
      p0->note(launch_rank_sum(P, g->bufs, s0.nv, s));
      if (s0.fin >= 0)
        for (hpcgx_problem *pr : g->ranks)
          pr->note(launch_finish(s0.fin, s0.nv, pr->gsum, pr->st, s));
    }
  }
  CK(cudaGetLastError());
  return HPCGX_OK;
}

Runner single_runner(hpcgx_problem *p) {
  return [p](std::vector<Plan> &plans) { return run_plan(p, plans[0]); };
}
Runner group_runner(hpcgx_group *g) {
  return [g](std::vector<Plan> &plans) { return group_run(g, plans); };
}

// Waits for the work queued on s, for at most HPCGX_WAIT_TIMEOUT_S seconds
// (environment, default 600): on a sharded problem a rank whose peer has
// failed then returns HPCGX_ETIMEOUT instead of blocking for ever behind an
// exchange.  The queued work itself is left to finish.
int bounded_wait(hpcgx_problem *p) {
  const double limit = wait_limit_s();
  cudaStream_t s = p->stream;
  cudaEvent_t ev;
  CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  cudaError_t e = cudaEventRecord(ev, s);
  const double t0 = now_s();
  for (int polls = 0; e == cudaSuccess; ++polls) {
    const cudaError_t q = cudaEventQuery(ev);
    if (q != cudaErrorNotReady) {   // finished, or a real error
      e = q;
      break;
    }
    if (now_s() - t0 > limit) {
      cudaEventDestroy(ev);
      cudaGetLastError();           // the not-ready status of the last query
      // an NCCL kernel waiting for a failed peer would never finish: abort the
      // communicator, which ends its kernels (attach a new one to go on)
      const bool nccl = p->nccl && !p->nccl->aborted;
      if (nccl) nccl_abort(p->nccl);
      return fail(HPCGX_ETIMEOUT, "sharded work did not finish within HPCGX_WAIT_TIMEOUT_S = " +
                                      std::to_string(limit) + " s" +
                                      (nccl ? "; the NCCL communicator was aborted" : ""));
    }
    if (polls > 2000) std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  cudaEventDestroy(ev);
  if (e != cudaSuccess) return cuda_fail(e);
  // a query that found the work unfinished leaves cudaErrorNotReady as the
  // thread's last error, which is a status, not a failure: clear it
  const cudaError_t last = cudaGetLastError();
  if (last != cudaSuccess && last != cudaErrorNotReady)
    return cuda_fail(last);
  return HPCGX_OK;
}

// CG over the ranks (src/CG.cpp:76-130 with the reductions of every rank
// summed): the same iteration as the one-GPU solver, run step by step; the
// host reads the stop flag (identical on every rank) once per iteration.
int sharded_cg(const std::vector<hpcgx_problem *> &ps, const Runner &run, int kind,
               const double *const *b, double *const *x, int max_iter, double tol, int *niters,
               double *normr, double *normr0) {
  if (max_iter < 0) return fail(HPCGX_EINVAL, "max_iter < 0");
  const size_t P = ps.size();
  CgState h;
  std::memset(&h, 0, sizeof(h));
  h.tol = tol;
  h.max_iter = max_iter;
  h.flexible = kind == G_MIXED;
  std::vector<Plan> init(P), iter(P);
  for (size_t r = 0; r < P; ++r) {
    hpcgx_problem *p = ps[r];
    TRY(p->check_ready(kind == G_MIXED));
    if (!b[r] || !x[r]) return fail(HPCGX_EINVAL, "null vector");
    CK(cudaMemcpyAsync(p->st, &h, sizeof(h), cudaMemcpyHostToDevice, p->stream));
    CK(cudaMemcpyAsync(p->x, x[r], p->L[0].n * sizeof(double), cudaMemcpyDeviceToDevice,
                       p->stream));
    p->plan_cg_init(init[r], kind, b[r]);
    p->plan_cg_iteration(iter[r], kind);
  }
  TRY(run(init));
  hpcgx_problem *p0 = ps[0];
  while (true) {
    // wait (bounded) first: a copy to pageable host memory would block
    // without limit until the stream drains
    TRY(bounded_wait(p0));
    CK(cudaMemcpyAsync(&h, p0->st, sizeof(h), cudaMemcpyDeviceToHost, p0->stream));
    CK(cudaStreamSynchronize(p0->stream));   // idle stream: returns at once
    if (h.done) break;
    TRY(run(iter));
  }
  // the last iteration's x += alpha p, deferred by k_cg_p
  for (hpcgx_problem *p : ps)
    p->note(launch_cg_xflush(p->L[0].n, p->p, p->x, p->st, p->stream));
  for (size_t r = 0; r < P; ++r)
    CK(cudaMemcpyAsync(x[r], ps[r]->x, ps[r]->L[0].n * sizeof(double), cudaMemcpyDeviceToDevice,
                       ps[r]->stream));
  for (hpcgx_problem *p : ps) TRY(bounded_wait(p));
  if (niters) *niters = h.niters;
  if (normr) *normr = h.normr;
  if (normr0) *normr0 = h.normr0;
  if (h.nonfinite) return fail(HPCGX_ENONFINITE, "CG: residual norm is not finite");
  return HPCGX_OK;
}

// A one-step operator (SpMV / SYMGS / V-cycle) over the ranks.
template <class BUILD>
int sharded_op(const std::vector<hpcgx_problem *> &ps, const Runner &run, BUILD build) {
  std::vector<Plan> plans(ps.size());
  for (size_t r = 0; r < ps.size(); ++r) TRY(build(ps[r], plans[r], (int)r));
  TRY(run(plans));
  for (hpcgx_problem *p : ps) TRY(bounded_wait(p));
  CK(cudaGetLastError());
  return HPCGX_OK;
}

// The per-problem operators of a sharded problem run over its communicator.
int need_comm(hpcgx_problem *p) {
  if (p->nranks > 1 && !p->nccl && !p->comm_halo)
    return fail(HPCGX_ESTATE, "sharded problem: attach a communicator or use a group");
  return HPCGX_OK;
}

int group_kind(int mode, int *kind) {
  switch (mode) {
    case HPCGX_CG_PLAIN: *kind = G_FP64_NOPREC; return HPCGX_OK;
    case HPCGX_CG_MG: *kind = G_FP64_PREC; return HPCGX_OK;
    case HPCGX_CG_MIXED: *kind = G_MIXED; return HPCGX_OK;
    default: return fail(HPCGX_EINVAL, "unknown CG mode");
  }
}

}  // namespace

extern "C" {

const char *hpcgx_last_error(void) { return g_err.c_str(); }

int hpcgx_version(void) { return 2; }   // 2: sharding (slabs, NCCL, groups)

int hpcgx_init_device(int device) {
  NvtxRange range_("hpcgx_init_device");
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaFree(nullptr);   // forces the context into existence
  return e == cudaSuccess ? HPCGX_OK : cuda_fail(e);
}

int hpcgx_create(int device, int nx, int ny, int nz, int levels, hpcgx_problem **out) {
  return hpcgx_create_slab(device, nx, ny, nz, levels, 1, 0, out);
}

int hpcgx_create_slab(int device, int nx, int ny, int nz, int levels, int nranks, int rank,
                      hpcgx_problem **out) {
  NvtxRange range_("hpcgx_create_slab");
  if (!out) return fail(HPCGX_EINVAL, "out is NULL");
  *out = nullptr;
  if (nx < 1 || ny < 1 || nz < 1 || levels < 1 || levels > kMaxLevels)
    return fail(HPCGX_EINVAL, "bad geometry or level count");
  if (nranks < 1 || rank < 0 || rank >= nranks) return fail(HPCGX_EINVAL, "bad rank or rank count");
  if ((int64_t)nx * ny * (nz + 2) >= (int64_t)1 << 31)
    return fail(HPCGX_EINVAL, "more than 2^31 rows: column indices are int32");
  for (int l = 0; l + 1 < levels; ++l)
    if (((nx >> l) & 1) || ((ny >> l) & 1) || ((nz >> l) & 1))
      return fail(HPCGX_EINVAL, "level dimensions must be even to coarsen");
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(e);
  hpcgx_problem *p = new hpcgx_problem;
  p->device = device;
  p->nlev = levels;
  p->nranks = nranks;
  p->rank = rank;
  int rc = HPCGX_OK;
  auto bail = [&](int code) {
    delete p;
    return code;
  };
  e = cudaStreamCreateWithFlags(&p->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return bail(cuda_fail(e));
  p->stream = p->own_stream;
  // reduction scratch: up to two values per block of any reducing launch,
  // plus two per group of 1024 blocks
  auto red_need = [](int64_t blocks) { return 2 * blocks + 2 * ((blocks + 1023) / 1024); };
  int64_t red_cap = 0;
  for (int l = 0; l < levels; ++l) {
    LevelDev &A = p->L[l];
    plan_level(A, nx >> l, ny >> l, nz >> l);
    A.zlo = rank > 0;
    A.zhi = rank + 1 < nranks;
    const size_t slots = (size_t)A.storage_rows * HPCGX_STENCIL;
    if ((rc = p->alloc((void **)&A.vals, slots * sizeof(double)))) return bail(rc);
    if ((rc = p->alloc((void **)&A.cols, slots * sizeof(int32_t)))) return bail(rc);
    const int64_t plane = (int64_t)A.nx * A.ny;
    if (l > 0) {
      if ((rc = p->alloc((void **)&A.r64, A.n * sizeof(double)))) return bail(rc);
      if ((rc = p->alloc_halo((void **)&A.x64, A.n, sizeof(double), plane))) return bail(rc);
      if ((rc = p->alloc((void **)&A.r32, A.n * sizeof(float)))) return bail(rc);
      if ((rc = p->alloc_halo((void **)&A.x32, A.n, sizeof(float), plane))) return bail(rc);
    }
    red_cap = std::max<int64_t>(red_cap, red_need(A.spmv_blocks));
    for (int q = 0; q < 4; ++q)
      red_cap = std::max<int64_t>(red_cap, red_need(A.blocks[q]));
  }
  const int64_t n = p->L[0].n;
  red_cap = std::max<int64_t>(red_cap, red_need(vector_blocks(n)));
  const int64_t plane0 = (int64_t)p->L[0].nx * p->L[0].ny;
  for (double **v : {&p->b, &p->x, &p->r, &p->Ap, &p->tmp})
    if ((rc = p->alloc((void **)v, n * sizeof(double)))) return bail(rc);
  for (double **v : {&p->z, &p->p})
    if ((rc = p->alloc_halo((void **)v, n, sizeof(double), plane0))) return bail(rc);
  if ((rc = p->alloc_halo((void **)&p->z32, n, sizeof(float), plane0))) return bail(rc);
  if ((rc = p->alloc((void **)&p->r32, n * sizeof(float)))) return bail(rc);
  if ((rc = p->alloc((void **)&p->gsum, 2 * sizeof(double)))) return bail(rc);
  if ((rc = p->alloc((void **)&p->result, 4 * sizeof(double)))) return bail(rc);
  if ((rc = p->alloc((void **)&p->st, sizeof(CgState)))) return bail(rc);
  if ((rc = p->alloc((void **)&p->red.partials, red_cap * sizeof(double)))) return bail(rc);
  const int64_t ncounters = 1 + (red_cap + 1023) / 1024;   // top counter + one per group
  if ((rc = p->alloc((void **)&p->red.counter, ncounters * sizeof(unsigned int)))) return bail(rc);
  p->red.capacity = red_cap;
  e = cudaMemsetAsync(p->red.counter, 0, ncounters * sizeof(unsigned int), p->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
  if (e != cudaSuccess) return bail(cuda_fail(e));
  *out = p;
  return HPCGX_OK;
}

int hpcgx_create_general(int device, int levels, hpcgx_problem **out) {
  NvtxRange range_("hpcgx_create_general");
  if (!out) return fail(HPCGX_EINVAL, "null output");
  *out = nullptr;
  if (levels < 1 || levels > kMaxLevels) return fail(HPCGX_EINVAL, "bad level count");
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(e);
  hpcgx_problem *p = new hpcgx_problem;
  p->device = device;
  p->nlev = levels;
  e = cudaStreamCreateWithFlags(&p->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete p;
    return cuda_fail(e);
  }
  p->stream = p->own_stream;
  p->gen = general_create(levels, p->stream);
  *out = p;
  return HPCGX_OK;
}

int hpcgx_load_level_general(hpcgx_problem *p, int level, int64_t nrows, const char *nnz,
                             const int32_t *const *cols, const double *const *vals,
                             const int32_t *f2c, int64_t nc) {
  NvtxRange range_("hpcgx_load_level_general");
  HANDLE(p);
  if (!p->gen) return fail(HPCGX_ESTATE, "not a general-pattern problem (hpcgx_create_general)");
  TRY(check_level(p, level));
  if (!nnz || !cols || !vals) return fail(HPCGX_EINVAL, "null row arrays");
  CK(cudaSetDevice(p->device));
  const char *why = nullptr;
  const int rc = general_load_level(p->gen, level, nrows, nnz, cols, vals, f2c, nc, &why);
  if (rc == HPCGX_ELAYOUT) return fail(rc, why ? why : "matrix rejected");
  if (rc != HPCGX_OK) return rc;
  p->L[level].n = nrows;
  if (level == 0) {
    // the vectors and reduction scratch of the shared entry points (host
    // staging, dot, WAXPBY, residual, CG's b and x)
    for (double **v : {&p->b, &p->x})
      TRY(p->alloc((void **)v, nrows * sizeof(double)));
    TRY(p->alloc((void **)&p->result, 4 * sizeof(double)));
    const int64_t blocks = vector_blocks(nrows);
    const int64_t cap = 2 * blocks + 2 * ((blocks + 1023) / 1024);
    TRY(p->alloc((void **)&p->red.partials, cap * sizeof(double)));
    const int64_t counters = 1 + (cap + 1023) / 1024;
    TRY(p->alloc((void **)&p->red.counter, counters * sizeof(unsigned int)));
    p->red.capacity = cap;
    CK(cudaMemsetAsync(p->red.counter, 0, counters * sizeof(unsigned int), p->stream));
    CK(cudaStreamSynchronize(p->stream));
  }
  p->loaded[level] = true;
  return HPCGX_OK;
}

int hpcgx_colours(hpcgx_problem *p, int level) {
  HANDLE(p);
  TRY(check_level(p, level));
  if (!p->gen) return 8;   // the stencil layout's parity colouring
  return general_colours(p->gen, level);
}

int hpcgx_destroy(hpcgx_problem *p) {
  if (!p) return HPCGX_OK;
  delete p;
  return HPCGX_OK;
}

int64_t hpcgx_rows(hpcgx_problem *p, int level) {
  if (!p || level < 0 || level >= p->nlev) return -1;
  return p->L[level].n;
}

int hpcgx_load_level(hpcgx_problem *p, int level, const uint8_t *nnz, const int32_t *cols,
                     const double *vals) {
  NvtxRange range_("hpcgx_load_level");
  HANDLE(p);
  TRY(stencil_only(p, "hpcgx_load_level"));
  if (p->nranks > 1) return fail(HPCGX_ESTATE, "sharded problems are generated on the device");
  if (!nnz || !cols || !vals) return fail(HPCGX_EINVAL, "null host array");
  return load_level_impl(
      p, level, [&](int64_t i) { return (int)nnz[i]; },
      [&](int64_t i, int j, int32_t &c, double &v) {
        c = cols[i * HPCGX_STENCIL + j];
        v = vals[i * HPCGX_STENCIL + j];
      });
}

int hpcgx_load_level_rows(hpcgx_problem *p, int level, const char *nnz,
                          const int32_t *const *cols, const double *const *vals) {
  NvtxRange range_("hpcgx_load_level_rows");
  HANDLE(p);
  TRY(stencil_only(p, "hpcgx_load_level_rows"));
  if (p->nranks > 1) return fail(HPCGX_ESTATE, "sharded problems are generated on the device");
  if (!nnz || !cols || !vals) return fail(HPCGX_EINVAL, "null host array");
  return load_level_impl(
      p, level, [&](int64_t i) { return (int)(unsigned char)nnz[i]; },
      [&](int64_t i, int j, int32_t &c, double &v) {
        c = cols[i][j];
        v = vals[i][j];
      });
}

int hpcgx_check_f2c(hpcgx_problem *p, int level, const int32_t *f2c, int64_t nc) {
  HANDLE(p);
  TRY(stencil_only(p, "hpcgx_check_f2c"));
  TRY(check_level(p, level));
  if (level + 1 >= p->nlev) return fail(HPCGX_EINVAL, "coarsest level has no injection");
  const LevelDev &F = p->L[level];
  const int nxc = F.nx / 2, nyc = F.ny / 2, nzc = F.nz / 2;
  if (nc != (int64_t)nxc * nyc * nzc) return fail(HPCGX_ELAYOUT, "f2c length mismatch");
  for (int64_t ic = 0; ic < nc; ++ic) {
    const int64_t ixc = ic % nxc, iyc = (ic / nxc) % nyc, izc = ic / ((int64_t)nxc * nyc);
    const int64_t f = (2 * izc) * (int64_t)F.nx * F.ny + (2 * iyc) * (int64_t)F.nx + 2 * ixc;
    if (f2c[ic] != f) return fail(HPCGX_ELAYOUT, "f2c is not the geometric injection");
  }
  return HPCGX_OK;
}

int hpcgx_generate(hpcgx_problem *p, int kind, uint64_t seed, double sigma) {
  NvtxRange range_("hpcgx_generate");
  HANDLE(p);
  TRY(stencil_only(p, "hpcgx_generate"));
  for (int l = 0; l < p->nlev; ++l) {
    if (kind == HPCGX_GEN_HPCG) {
      p->note(launch_generate_hpcg(p->L[l], p->stream));
    } else if (kind == HPCGX_GEN_VARCOEF) {
      if (p->nranks > 1) return fail(HPCGX_EINVAL, "variable coefficients: one rank only");
      p->note(launch_generate_varcoef(p->L[l], l, p->L[0].nx, p->L[0].ny, seed, sigma, p->stream));
    } else {
      return fail(HPCGX_EINVAL, "unknown generator kind");
    }
    p->loaded[l] = true;
  }
  CK(cudaStreamSynchronize(p->stream));
  CK(cudaGetLastError());
  p->mixed_stale = true;
  return HPCGX_OK;
}

int hpcgx_build_mixed(hpcgx_problem *p) {
  NvtxRange range_("hpcgx_build_mixed");
  HANDLE(p);
  TRY(stencil_only(p, "the mixed-precision solver"));
  p->mixed_stale = true;
  TRY(p->check_ready(true));
  CK(cudaStreamSynchronize(p->stream));
  return HPCGX_OK;
}

int hpcgx_set_stencil_columns(hpcgx_problem *p, int on) {
  HANDLE(p);
  TRY(stencil_only(p, "hpcgx_set_stencil_columns"));
  for (int l = 0; l < p->nlev; ++l) p->L[l].stencil_cols = on != 0;
  // the FP64 iteration graphs hold the other kernels: rebuild them on next use
  for (int k : {G_FP64_PREC, G_FP64_NOPREC})
    if (p->graph[k]) {
      CK(cudaGraphExecDestroy(p->graph[k]));
      p->graph[k] = nullptr;
      p->probes[k].clear();
    }
  return HPCGX_OK;
}

int hpcgx_set_diagonal_host(hpcgx_problem *p, int level, const double *diag) {
  HANDLE(p);
  if (p->gen) {
    TRY(check_level(p, level));
    TRY(general_ready_or_fail(p));
    return general_set_diagonal(p->gen, level, diag);
  }
  TRY(check_level(p, level));
  const LevelDev &A = p->L[level];
  CK(cudaMemcpyAsync(p->tmp, diag, A.n * sizeof(double), cudaMemcpyHostToDevice, p->stream));
  p->note(launch_set_diagonal(A, p->tmp, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  p->mixed_stale = true;
  return HPCGX_OK;
}

int hpcgx_get_diagonal_host(hpcgx_problem *p, int level, double *diag) {
  HANDLE(p);
  if (p->gen) {
    TRY(check_level(p, level));
    TRY(general_ready_or_fail(p));
    return general_get_diagonal(p->gen, level, diag);
  }
  TRY(check_level(p, level));
  const LevelDev &A = p->L[level];
  p->note(launch_get_diagonal(A, p->tmp, p->stream));
  CK(cudaMemcpyAsync(diag, p->tmp, A.n * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  return HPCGX_OK;
}

int hpcgx_set_values(hpcgx_problem *p, int level, const double *vals27, int recoarsen) {
  NvtxRange range_("hpcgx_set_values");
  HANDLE(p);
  TRY(stencil_only(p, "hpcgx_set_values"));
  TRY(check_level(p, level));
  p->note(launch_set_values(p->L[level], vals27, p->stream));
  p->loaded[level] = true;
  if (recoarsen)
    for (int l = level; l + 1 < p->nlev; ++l) {
      p->note(launch_coarsen_varcoef(p->L[l], p->L[l + 1], p->stream));
      p->loaded[l + 1] = true;
    }
  CK(cudaStreamSynchronize(p->stream));
  CK(cudaGetLastError());
  p->mixed_stale = true;
  return HPCGX_OK;
}

int hpcgx_get_values(hpcgx_problem *p, int level, double *vals27, int32_t *cols27) {
  HANDLE(p);
  TRY(stencil_only(p, "hpcgx_get_values"));
  TRY(check_level(p, level));
  p->note(launch_get_values(p->L[level], vals27, cols27, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  return HPCGX_OK;
}

int hpcgx_memory_bytes(hpcgx_problem *p, double *bytes) {
  if (!p || !bytes) return fail(HPCGX_EINVAL, "null argument");
  *bytes = (double)p->bytes + (p->gen ? general_bytes(p->gen) : 0.0);
  return HPCGX_OK;
}

int hpcgx_spmv(hpcgx_problem *p, int level, const double *x, double *y) {
  NvtxRange range_("hpcgx_spmv");
  HANDLE(p);
  if (p->gen) {
    TRY(check_level(p, level));
    TRY(general_ready_or_fail(p));
    return general_spmv(p->gen, level, x, y);
  }
  TRY(check_level(p, level));
  if (!p->loaded[level]) return fail(HPCGX_ESTATE, "level not loaded");
  if (p->sharded()) {
    TRY(need_comm(p));
    return sharded_op({p}, single_runner(p), [&](hpcgx_problem *q, Plan &pl, int) {
      return q->plan_spmv(pl, level, x, y);
    });
  }
  p->note(launch_spmv(p->L[level], x, y, nullptr, 0, nullptr, nullptr, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  CK(cudaGetLastError());
  return HPCGX_OK;
}

int hpcgx_spmv_stencil(hpcgx_problem *p, int level, const double *x, double *y) {
  NvtxRange range_("hpcgx_spmv_stencil");
  HANDLE(p);
  TRY(stencil_only(p, "hpcgx_spmv_stencil"));
  if (p->nranks > 1) return fail(HPCGX_ESTATE, "not available on a sharded problem");
  TRY(check_level(p, level));
  if (!p->loaded[level]) return fail(HPCGX_ESTATE, "level not loaded");
  p->note(launch_spmv(p->L[level], x, y, nullptr, 0, nullptr, nullptr, p->stream, true));
  CK(cudaStreamSynchronize(p->stream));
  CK(cudaGetLastError());
  return HPCGX_OK;
}

int hpcgx_symgs(hpcgx_problem *p, int level, const double *r, double *x) {
  NvtxRange range_("hpcgx_symgs");
  HANDLE(p);
  if (p->gen) {
    TRY(check_level(p, level));
    TRY(general_ready_or_fail(p));
    return general_symgs(p->gen, level, r, x);
  }
  TRY(check_level(p, level));
  if (!p->loaded[level]) return fail(HPCGX_ESTATE, "level not loaded");
  if (p->sharded()) {
    TRY(need_comm(p));
    return sharded_op({p}, single_runner(p), [&](hpcgx_problem *q, Plan &pl, int) {
      return q->plan_symgs(pl, level, r, x);
    });
  }
  TRY((p->symgs<double, double>(level, r, x)));
  CK(cudaStreamSynchronize(p->stream));
  CK(cudaGetLastError());
  return HPCGX_OK;
}

int hpcgx_mg(hpcgx_problem *p, const double *r, double *x) {
  NvtxRange range_("hpcgx_mg");
  HANDLE(p);
  if (p->gen) {
    TRY(general_ready_or_fail(p));
    return general_mg(p->gen, r, x);
  }
  TRY(p->check_ready(false));
  if (p->sharded()) {
    TRY(need_comm(p));
    return sharded_op({p}, single_runner(p), [&](hpcgx_problem *q, Plan &pl, int) {
      return q->plan_mg(pl, r, x);
    });
  }
  TRY((p->vcycle<double, double>(r, x, nullptr)));
  CK(cudaStreamSynchronize(p->stream));
  CK(cudaGetLastError());
  return HPCGX_OK;
}

int hpcgx_spmv_mixed(hpcgx_problem *p, int level, const float *x, float *y) {
  NvtxRange range_("hpcgx_spmv_mixed");
  HANDLE(p);
  TRY(stencil_only(p, "the mixed-precision solver"));
  if (p->nranks > 1) return fail(HPCGX_ESTATE, "not available on a sharded problem");
  TRY(check_level(p, level));
  TRY(p->check_ready(true));
  p->note(launch_spmv32(p->L[level], x, y, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  CK(cudaGetLastError());
  return HPCGX_OK;
}

int hpcgx_symgs_mixed(hpcgx_problem *p, int level, const double *r64, const float *r32,
                      float *x) {
  NvtxRange range_("hpcgx_symgs_mixed");
  HANDLE(p);
  TRY(stencil_only(p, "the mixed-precision solver"));
  if (p->nranks > 1) return fail(HPCGX_ESTATE, "not available on a sharded problem");
  TRY(check_level(p, level));
  TRY(p->check_ready(true));
  if ((r64 == nullptr) == (r32 == nullptr)) return fail(HPCGX_EINVAL, "give exactly one of r64, r32");
  if (r64)
    TRY((p->symgs<float, double>(level, r64, x)));
  else
    TRY((p->symgs<float, float>(level, r32, x)));
  CK(cudaStreamSynchronize(p->stream));
  CK(cudaGetLastError());
  return HPCGX_OK;
}

int hpcgx_mg_mixed(hpcgx_problem *p, const double *r, float *x) {
  NvtxRange range_("hpcgx_mg_mixed");
  HANDLE(p);
  TRY(stencil_only(p, "the mixed-precision solver"));
  if (p->nranks > 1) return fail(HPCGX_ESTATE, "not available on a sharded problem");
  TRY(p->check_ready(true));
  TRY((p->vcycle<float, double>(r, x, nullptr)));
  CK(cudaStreamSynchronize(p->stream));
  CK(cudaGetLastError());
  return HPCGX_OK;
}

int hpcgx_restriction(hpcgx_problem *p, int level, const double *rf, const double *Axf,
                      double *rc) {
  HANDLE(p);
  TRY(stencil_only(p, "hpcgx_restriction"));
  TRY(check_level(p, level));
  if (level + 1 >= p->nlev) return fail(HPCGX_EINVAL, "coarsest level has no restriction");
  p->note(launch_restriction(p->L[level + 1].n, p->L[level], rf, Axf, rc, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  CK(cudaGetLastError());
  return HPCGX_OK;
}

int hpcgx_prolongation(hpcgx_problem *p, int level, const double *xc, double *xf) {
  HANDLE(p);
  TRY(stencil_only(p, "hpcgx_prolongation"));
  TRY(check_level(p, level));
  if (level + 1 >= p->nlev) return fail(HPCGX_EINVAL, "coarsest level has no prolongation");
  p->note(launch_prolongation(p->L[level + 1].n, p->L[level], xc, xf, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  CK(cudaGetLastError());
  return HPCGX_OK;
}

int hpcgx_dot(hpcgx_problem *p, int64_t n, const double *x, const double *y, double *result) {
  HANDLE(p);
  if (n < 0 || n > p->L[0].n || !result) return fail(HPCGX_EINVAL, "bad dot arguments");
  p->note(launch_dot(n, x, y, p->red, p->result, p->stream));
  CK(cudaMemcpyAsync(result, p->result, sizeof(double), cudaMemcpyDeviceToHost, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  return HPCGX_OK;
}

int hpcgx_waxpby(hpcgx_problem *p, int64_t n, double alpha, const double *x, double beta,
                 const double *y, double *w) {
  HANDLE(p);
  if (n < 0) return fail(HPCGX_EINVAL, "negative length");
  p->note(launch_waxpby(n, alpha, x, beta, y, w, nullptr, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  CK(cudaGetLastError());
  return HPCGX_OK;
}

int hpcgx_residual(hpcgx_problem *p, int64_t n, const double *v1, const double *v2,
                   double *result) {
  HANDLE(p);
  if (n < 0 || n > p->L[0].n || !result) return fail(HPCGX_EINVAL, "bad residual arguments");
  p->note(launch_absmax_diff(n, v1, v2, p->red, p->result, p->stream));
  CK(cudaMemcpyAsync(result, p->result, sizeof(double), cudaMemcpyDeviceToHost, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  return HPCGX_OK;
}

int hpcgx_cg(hpcgx_problem *p, const double *b, double *x, int max_iter, double tolerance,
             int precond, int *niters, double *normr, double *normr0, double *times) {
  NvtxRange range_("hpcgx_cg");
  HANDLE(p);
  if (p->gen) {
    TRY(general_ready_or_fail(p));
    return general_cg(p->gen, b, x, max_iter, tolerance, precond, niters, normr, normr0, times);
  }
  if (p->sharded()) {
    TRY(need_comm(p));
    return sharded_cg({p}, single_runner(p), precond ? G_FP64_PREC : G_FP64_NOPREC, &b, &x,
                      max_iter, tolerance, niters, normr, normr0);
  }
  return p->cg(precond ? G_FP64_PREC : G_FP64_NOPREC, b, x, max_iter, tolerance, niters, normr,
               normr0, times);
}

int hpcgx_cg_mixed(hpcgx_problem *p, const double *b, double *x, int max_iter, double tolerance,
                   int *niters, double *normr, double *normr0, double *times) {
  NvtxRange range_("hpcgx_cg_mixed");
  HANDLE(p);
  TRY(stencil_only(p, "the mixed-precision solver"));
  if (p->sharded()) {
    TRY(need_comm(p));
    return sharded_cg({p}, single_runner(p), G_MIXED, &b, &x, max_iter, tolerance, niters, normr,
                      normr0);
  }
  return p->cg(G_MIXED, b, x, max_iter, tolerance, niters, normr, normr0, times);
}

int hpcgx_cg_host(hpcgx_problem *p, int mode, const double *b_host, double *x_host, int max_iter,
                  double tolerance, int *niters, double *normr, double *normr0, double *times) {
  NvtxRange range_("hpcgx_cg_host");
  HANDLE(p);
  const int64_t n = p->L[0].n;
  int kind;
  switch (mode) {
    case HPCGX_CG_PLAIN: kind = G_FP64_NOPREC; break;
    case HPCGX_CG_MG: kind = G_FP64_PREC; break;
    case HPCGX_CG_MIXED: kind = G_MIXED; break;
    default: return fail(HPCGX_EINVAL, "unknown CG mode");
  }
  if (p->gen && kind == G_MIXED) return stencil_only(p, "the mixed-precision solver");
  if (p->gen) TRY(general_ready_or_fail(p));
  CK(cudaMemcpyAsync(p->b, b_host, n * sizeof(double), cudaMemcpyHostToDevice, p->stream));
  CK(cudaMemcpyAsync(p->x, x_host, n * sizeof(double), cudaMemcpyHostToDevice, p->stream));
  if (p->gen) {
    TRY(general_cg(p->gen, p->b, p->x, max_iter, tolerance, kind == G_FP64_PREC, niters, normr,
                   normr0, times));
  } else if (p->sharded()) {
    TRY(need_comm(p));
    const double *bd = p->b;
    double *xd = p->x;
    TRY(sharded_cg({p}, single_runner(p), kind, &bd, &xd, max_iter, tolerance, niters, normr,
                   normr0));
  } else {
    TRY(p->cg(kind, p->b, p->x, max_iter, tolerance, niters, normr, normr0, times));
  }
  CK(cudaMemcpyAsync(x_host, p->x, n * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  return HPCGX_OK;
}

int hpcgx_spmv_host(hpcgx_problem *p, int level, const double *x, double *y) {
  HANDLE(p);
  TRY(check_level(p, level));
  TRY(p->staging());
  const int64_t n = p->L[level].n;
  TRY(p->up(p->stage[0], x, n));
  TRY(hpcgx_spmv(p, level, p->stage[0], p->stage[1]));
  return p->down(y, p->stage[1], n);
}

int hpcgx_symgs_host(hpcgx_problem *p, int level, const double *r, double *x) {
  HANDLE(p);
  TRY(check_level(p, level));
  TRY(p->staging());
  const int64_t n = p->L[level].n;
  TRY(p->up(p->stage[0], r, n));
  TRY(p->up(p->stage[1], x, n));
  TRY(hpcgx_symgs(p, level, p->stage[0], p->stage[1]));
  return p->down(x, p->stage[1], n);
}

int hpcgx_mg_host(hpcgx_problem *p, const double *r, double *x) {
  HANDLE(p);
  TRY(p->staging());
  const int64_t n = p->L[0].n;
  TRY(p->up(p->stage[0], r, n));
  TRY(hpcgx_mg(p, p->stage[0], p->stage[1]));
  return p->down(x, p->stage[1], n);
}

int hpcgx_dot_host(hpcgx_problem *p, int64_t n, const double *x, const double *y,
                   double *result) {
  HANDLE(p);
  if (n < 0 || n > p->L[0].n) return fail(HPCGX_EINVAL, "bad dot length");
  TRY(p->staging());
  TRY(p->up(p->stage[0], x, n));
  if (y != x) TRY(p->up(p->stage[1], y, n));
  return hpcgx_dot(p, n, p->stage[0], y == x ? p->stage[0] : p->stage[1], result);
}

int hpcgx_waxpby_host(hpcgx_problem *p, int64_t n, double alpha, const double *x, double beta,
                      const double *y, double *w) {
  HANDLE(p);
  if (n < 0 || n > p->L[0].n) return fail(HPCGX_EINVAL, "bad waxpby length");
  TRY(p->staging());
  TRY(p->up(p->stage[0], x, n));
  TRY(p->up(p->stage[1], y, n));
  TRY(hpcgx_waxpby(p, n, alpha, p->stage[0], beta, p->stage[1], p->stage[2]));
  return p->down(w, p->stage[2], n);
}

int hpcgx_adjoint_grad(hpcgx_problem *p, const double *lambda, const double *x, double *grad) {
  NvtxRange range_("hpcgx_adjoint_grad");
  HANDLE(p);
  TRY(stencil_only(p, "hpcgx_adjoint_grad"));
  if (p->nranks > 1) return fail(HPCGX_ESTATE, "not available on a sharded problem");
  p->note(launch_adjoint_grad(p->L[0], lambda, x, grad, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  CK(cudaGetLastError());
  return HPCGX_OK;
}

int hpcgx_fill_uniform(hpcgx_problem *p, int64_t n, uint64_t seed, double lo, double hi,
                       double *v) {
  HANDLE(p);
  // a finest-level vector of a z-slab holds entries rank*n .. of the global one
  const uint64_t offset = n == p->L[0].n ? (uint64_t)p->rank * (uint64_t)n : 0;
  p->note(launch_fill_uniform(n, seed, offset, lo, hi, v, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  CK(cudaGetLastError());
  return HPCGX_OK;
}

int hpcgx_fill_normal(hpcgx_problem *p, int64_t n, uint64_t seed, uint64_t offset, double *v) {
  HANDLE(p);
  p->note(launch_fill_normal(n, seed, offset, v, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  CK(cudaGetLastError());
  return HPCGX_OK;
}

int hpcgx_set_probe(hpcgx_problem *p, int probe_mask) {
  HANDLE(p);
  if (probe_mask < 0 || probe_mask > 7) return fail(HPCGX_EINVAL, "unknown probe mask");
  p->probe = probe_mask;
  return HPCGX_OK;
}

int hpcgx_probe_read(hpcgx_problem *p, int kind, double *ms, int64_t *launches, double *bytes,
                     int reset) {
  if (!p) return fail(HPCGX_EINVAL, "null problem handle");
  if (kind != HPCGX_PROBE_GS_FINE && kind != HPCGX_PROBE_SPMV_FINE &&
      kind != HPCGX_PROBE_GS_FINE_BWD)
    return fail(HPCGX_EINVAL, "probe_read takes a single probe kind");
  const int slot = probe_slot(kind);
  if (ms) *ms = p->probe_ms[slot];
  if (launches) *launches = p->probe_launches[slot];
  if (bytes) *bytes = p->probe_bytes[slot];
  if (reset) {
    p->probe_ms[slot] = 0.0;
    p->probe_bytes[slot] = 0.0;
    p->probe_launches[slot] = 0;
  }
  return HPCGX_OK;
}

int64_t hpcgx_launch_count(hpcgx_problem *p) {
  return p ? p->launches + (p->gen ? general_launches(p->gen) : 0) : -1;
}

int hpcgx_iteration_bytes(hpcgx_problem *p, int mode, double *bytes) {
  HANDLE(p);
  if (!bytes) return fail(HPCGX_EINVAL, "null output");
  int kind = 0;
  TRY(group_kind(mode, &kind));
  if (!p->graph[kind]) return fail(HPCGX_ESTATE, "no solve of this mode has run on the problem yet");
  *bytes = p->graph_bytes[kind];
  return HPCGX_OK;
}

int hpcgx_set_stream(hpcgx_problem *p, void *stream) {
  HANDLE(p);
  CK(cudaStreamSynchronize(p->stream));
  p->stream = stream ? static_cast<cudaStream_t>(stream) : p->own_stream;
  if (p->gen) general_set_stream(p->gen, p->stream);
  return HPCGX_OK;
}

int hpcgx_synchronize(hpcgx_problem *p) {
  HANDLE(p);
  CK(cudaStreamSynchronize(p->stream));
  return HPCGX_OK;
}

int hpcgx_check_status(void) {
  CK(cudaDeviceSynchronize());
  unsigned long long rec = 0ull;
  const int e = read_check_record(&rec);
  if (e != 0) return cuda_fail((cudaError_t)e);
  if (rec == 0ull) return HPCGX_OK;
  static const char *sites[] = {"?", "SpMV row", "SpMV column", "Gauss-Seidel row",
                                "Gauss-Seidel column", "coarse row", "restriction row",
                                "restriction column"};
  const int site = (int)(rec >> 56);
  const long long index = (long long)(rec & ((1ull << 56) - 1));
  return fail(HPCGX_ECHECK, std::string("index check: ") + (site < 8 ? sites[site] : "?") +
                                " index " + std::to_string(index) + " out of range");
}

// ---- sharding
int hpcgx_nccl_unique_id(void *id, int bytes) {
  if (!id || bytes < (int)sizeof(ncclUniqueId)) return fail(HPCGX_EINVAL, "id buffer too small");
  NcclApi *api = nccl_api();
  if (!api) return fail(HPCGX_ECOMM, "NCCL (libnccl.so.2) could not be loaded");
  ncclUniqueId u;
  const ncclResult_t r = api->GetUniqueId(&u);
  if (r != ncclSuccess) return fail(HPCGX_ECOMM, std::string("ncclGetUniqueId: ") + api->GetErrorString(r));
  std::memcpy(id, &u, sizeof(u));
  return HPCGX_OK;
}

int hpcgx_attach_nccl(hpcgx_problem *p, const void *id, int bytes) {
  NvtxRange range_("hpcgx_attach_nccl");
  HANDLE(p);
  TRY(stencil_only(p, "sharding"));
  if (!id || bytes < (int)sizeof(ncclUniqueId)) return fail(HPCGX_EINVAL, "id buffer too small");
  if (p->nccl && p->nccl->aborted) {   // a communicator aborted on a timeout: replace it
    nccl_release(p->nccl);
    p->nccl = nullptr;
  }
  if (p->nccl || p->comm_halo) return fail(HPCGX_ESTATE, "a communicator is attached already");
  NcclApi *api = nccl_api();
  if (!api) return fail(HPCGX_ECOMM, "NCCL (libnccl.so.2) could not be loaded");
  ncclUniqueId u;
  std::memcpy(&u, id, sizeof(u));
  CK(cudaSetDevice(p->device));
  NcclLink *link = new NcclLink;
  ncclConfig_t config = NCCL_CONFIG_INITIALIZER;
  config.blocking = 0;
  ncclResult_t r = api->CommInitRankConfig(&link->comm, p->nranks, u, p->rank, &config);
  if (r != ncclSuccess && r != ncclInProgress) {
    delete link;
    return fail(HPCGX_ECOMM, std::string("ncclCommInitRankConfig: ") + api->GetErrorString(r));
  }
  const int rc = nccl_settle(link, r, "ncclCommInitRankConfig");
  if (rc != HPCGX_OK) {
    nccl_release(link);
    return rc;
  }
  p->nccl = link;
  return HPCGX_OK;
}

int hpcgx_attach_comm(hpcgx_problem *p, hpcgx_halo_fn halo, hpcgx_sum_fn sum, void *ctx) {
  HANDLE(p);
  TRY(stencil_only(p, "sharding"));
  if (!halo || !sum) return fail(HPCGX_EINVAL, "both functions are needed");
  if (p->nccl || p->comm_halo) return fail(HPCGX_ESTATE, "a communicator is attached already");
  p->comm_halo = halo;
  p->comm_sum = sum;
  p->comm_ctx = ctx;
  return HPCGX_OK;
}

int hpcgx_group_create(hpcgx_problem *const *ranks, int nranks, hpcgx_group **out) {
  if (!out || !ranks || nranks < 1) return fail(HPCGX_EINVAL, "bad group arguments");
  *out = nullptr;
  for (int r = 0; r < nranks; ++r) {
    hpcgx_problem *p = ranks[r];
    if (!p) return fail(HPCGX_EINVAL, "null rank");
    if (p->nranks != nranks || p->rank != r)
      return fail(HPCGX_EINVAL, "rank r of the group must be slab r of nranks");
    if (p->device != ranks[0]->device || p->nlev != ranks[0]->nlev ||
        p->L[0].nx != ranks[0]->L[0].nx || p->L[0].ny != ranks[0]->L[0].ny ||
        p->L[0].nz != ranks[0]->L[0].nz)
      return fail(HPCGX_EINVAL, "group ranks differ in device or geometry");
    if (p->nccl || p->comm_halo) return fail(HPCGX_ESTATE, "rank has a communicator attached");
  }
  CK(cudaSetDevice(ranks[0]->device));
  std::unique_ptr<hpcgx_group> g(new hpcgx_group);
  g->ranks.assign(ranks, ranks + nranks);
  CK(cudaMalloc(&g->bufs, nranks * sizeof(double *)));
  std::vector<double *> h(nranks);
  for (int r = 0; r < nranks; ++r) h[r] = ranks[r]->gsum;
  CK(cudaMemcpy(g->bufs, h.data(), nranks * sizeof(double *), cudaMemcpyHostToDevice));
  // a pageable copy may still be in flight on the legacy stream, which the
  // ranks' non-blocking streams do not wait for
  CK(cudaDeviceSynchronize());
  // one stream for every rank: the lockstep order is the stream order
  for (int r = 0; r < nranks; ++r) {
    CK(cudaStreamSynchronize(ranks[r]->stream));
    g->saved.push_back(ranks[r]->stream);
  }
  for (int r = 0; r < nranks; ++r) ranks[r]->stream = ranks[0]->stream;
  *out = g.release();
  return HPCGX_OK;
}

int hpcgx_group_destroy(hpcgx_group *g) {
  if (!g) return HPCGX_OK;
  if (!g->ranks.empty()) cudaStreamSynchronize(g->ranks[0]->stream);
  for (size_t r = 0; r < g->ranks.size(); ++r) g->ranks[r]->stream = g->saved[r];
  delete g;
  return HPCGX_OK;
}

int hpcgx_group_spmv(hpcgx_group *g, int level, const double *const *x, double *const *y) {
  NvtxRange range_("hpcgx_group_spmv");
  if (!g || !x || !y) return fail(HPCGX_EINVAL, "null argument");
  for (hpcgx_problem *p : g->ranks) {
    TRY(check_level(p, level));
    if (!p->loaded[level]) return fail(HPCGX_ESTATE, "level not loaded");
  }
  return sharded_op(g->ranks, group_runner(g), [&](hpcgx_problem *q, Plan &pl, int r) {
    return q->plan_spmv(pl, level, x[r], y[r]);
  });
}

int hpcgx_group_symgs(hpcgx_group *g, int level, const double *const *r, double *const *x) {
  NvtxRange range_("hpcgx_group_symgs");
  if (!g || !r || !x) return fail(HPCGX_EINVAL, "null argument");
  for (hpcgx_problem *p : g->ranks) {
    TRY(check_level(p, level));
    if (!p->loaded[level]) return fail(HPCGX_ESTATE, "level not loaded");
  }
  return sharded_op(g->ranks, group_runner(g), [&](hpcgx_problem *q, Plan &pl, int k) {
    return q->plan_symgs(pl, level, r[k], x[k]);
  });
}

int hpcgx_group_mg(hpcgx_group *g, const double *const *r, double *const *x) {
  NvtxRange range_("hpcgx_group_mg");
  if (!g || !r || !x) return fail(HPCGX_EINVAL, "null argument");
  for (hpcgx_problem *p : g->ranks) TRY(p->check_ready(false));
  return sharded_op(g->ranks, group_runner(g), [&](hpcgx_problem *q, Plan &pl, int k) {
    return q->plan_mg(pl, r[k], x[k]);
  });
}

int hpcgx_group_cg(hpcgx_group *g, int mode, const double *const *b, double *const *x,
                   int max_iter, double tolerance, int *niters, double *normr, double *normr0) {
  NvtxRange range_("hpcgx_group_cg");
  if (!g || !b || !x) return fail(HPCGX_EINVAL, "null argument");
  int kind = 0;
  TRY(group_kind(mode, &kind));
  return sharded_cg(g->ranks, group_runner(g), kind, b, x, max_iter, tolerance, niters, normr,
                    normr0);
}

}  // extern "C"
