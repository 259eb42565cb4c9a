// common.cuh -- shared types and device helpers of libhpcgx.
//
// Device layout of one multigrid level ("colour-sorted sliced ELL"):
//   * rows are stored colour-major: colour c = (ix&1) + 2(iy&1) + 4(iz&1), the
//     8-colouring that the reference's greedy multicolouring produces on the
//     27-point stencil (src/OptimizeProblem.cpp:43-96); inside a colour, rows
//     keep natural order, so each colour is a list of x-lines (fixed iy, iz)
//     holding every other point;
//   * every colour starts on a 32-row boundary; rows are grouped in slices of
//     32 rows x 27 slots.  Inside a slice the slots are grouped per stencil
//     z-plane (9 slots each) and, inside a plane, interleaved across the 32
//     rows in short vectors: FP64 values in pairs of slots (one 16-byte load
//     per row and pair), int32 columns and BF16 values in quads (one 16- or
//     8-byte load), plus one single slot per plane.  A warp's load of one
//     group for its 32 rows is one contiguous 512 / 256-byte segment, and a
//     row needs 15 value loads and 9 column loads instead of 27 + 27;
//   * slot s is the stencil offset (dz+1)*9 + (dy+1)*3 + (dx+1); slot 13 is the
//     diagonal.  Absent neighbours (boundary rows) hold value 0 and column =
//     the row itself.  Present entries therefore appear in exactly the
//     (sz, sy, sx) order the reference generator emits
//     (src/GenerateProblem_ref.cpp:152-172), which makes every row sum below
//     round exactly as the reference's;
//   * columns are int32 natural row indices, read by the FP64 sweeps and the
//     plain solver's SpMV; the mixed V-cycle and the mixed solver's FP64 SpMV
//     derive them from the stencil offsets instead (row + offset), so the
//     BF16 copy holds values only; vectors stay in natural order.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#define HPCGX_STENCIL 27
#define HPCGX_SLICE 32
#define HPCGX_DIAG_SLOT 13

namespace hpcgx {

// Largest number of multigrid levels (the reference fixes 4, src/main.cpp:139).
constexpr int kMaxLevels = 4;

// Division of n in [0, 2^31) by a fixed d >= 1 with one multiply-high, one
// add and one shift (the round-up method of Granlund and Montgomery,
// "Division by invariant integers using multiplication", 1994): the kernels
// map a thread to its line and row without integer division instructions.
struct FastDiv {
  uint32_t d, m, s;
};
inline FastDiv make_fastdiv(uint32_t d) {
  FastDiv f{d, 0u, 0u};
  if (d == 0) return f;
  while ((1ull << f.s) < d) ++f.s;
  f.m = (uint32_t)(((1ull << 32) * ((1ull << f.s) - d)) / d + 1);
  return f;
}
__host__ __device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv &f) {
#ifdef __CUDA_ARCH__
  const uint32_t hi = __umulhi(n, f.m);
#else
  const uint32_t hi = (uint32_t)(((uint64_t)n * f.m) >> 32);
#endif
  return (uint32_t)(((uint64_t)hi + n) >> f.s);
}

// The four x-line classes of a level: class q = (iy&1) + 2(iz&1).  Class q
// holds colours 2q (even ix) and 2q+1 (odd ix).
struct ClassInfo {
  int q, py, pz;
  int nyq;          // lines of this class along y
  int lines;        // lines of this class
  int len[2];       // rows per line for px = 0 / 1
  int64_t start[2]; // storage row of the first row of colour 2q+px
  FastDiv dlen[2];  // division by len[px]
  FastDiv dnyq;     // division by nyq
};

// What a kernel needs to know about one level's matrix.
template <class VT>
struct LevelMat {
  const VT *vals;
  const int32_t *cols;
  int nx, ny, nz;
  int64_t n;
  // z-slab halo planes present below / above (a neighbouring rank there), and
  // the index range [lo, lo + span) of the vector including them
  int zlo, zhi;
  int lo, span;
  int64_t srows;   // storage rows (colours padded to 32)
  // Stencil offsets: slot s of row i holds column i + off[s] whenever the row
  // has that neighbour (the layout enforces it when a level is loaded), and
  // column i with value 0 otherwise.  The mixed-precision V-cycle and the
  // mixed solver's SpMV derive their columns from these instead of reading
  // `cols`.
  int off[HPCGX_STENCIL];
};

// Elements of one 32-row slice and of one z-plane inside it.
constexpr int kSliceElems = HPCGX_STENCIL * HPCGX_SLICE;  // 864
constexpr int kPlaneElems = 9 * HPCGX_SLICE;              // 288

// Index of (storage row k, slot s) in the FP64 value array: per plane, slots
// r = 0..7 in interleaved pairs, slot r = 8 alone.
__host__ __device__ inline int64_t vidx(int64_t k, int s) {
  const int p = s / 9, r = s - 9 * p;
  const int64_t base = (k >> 5) * kSliceElems + p * kPlaneElems;
  const int lane = (int)(k & 31);
  return r < 8 ? base + (r >> 1) * 64 + lane * 2 + (r & 1) : base + 256 + lane;
}
// Index of (storage row k, slot s) in the column and BF16 value arrays: per
// plane, slots r = 0..7 in interleaved quads, slot r = 8 alone.
__host__ __device__ inline int64_t cidx(int64_t k, int s) {
  const int p = s / 9, r = s - 9 * p;
  const int64_t base = (k >> 5) * kSliceElems + p * kPlaneElems;
  const int lane = (int)(k & 31);
  return r < 8 ? base + (r >> 2) * 128 + lane * 4 + (r & 3) : base + 256 + lane;
}

// Colour of the neighbour in slot s of a row of colour c.
__host__ __device__ constexpr int slot_mask(int s) {
  return ((s % 3) != 1 ? 1 : 0) | (((s / 3) % 3) != 1 ? 2 : 0) | ((s / 9) != 1 ? 4 : 0);
}

// Arithmetic with one rounding per operation and no contraction into FMA,
// so that device sums reproduce the reference's x86-64 rounding bit for bit.
__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double rn_div(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float rn_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rn_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float rn_div(float a, float b) { return __fdiv_rn(a, b); }

// Accumulation steps s + a b and s - a b.  FP64 rounds the product and the
// sum separately, as the reference's x86-64 build does (it emits no FMA), so
// the FP64 path stays bit-exact with it; the FP32 arithmetic of the mixed
// V-cycle (no reference counterpart) uses one fused multiply-add, as its
// oracle does with C's fmaf.
__device__ __forceinline__ double mac_add(double s, double a, double b) {
  return __dadd_rn(s, __dmul_rn(a, b));
}
__device__ __forceinline__ double mac_sub(double s, double a, double b) {
  return __dsub_rn(s, __dmul_rn(a, b));
}
__device__ __forceinline__ float mac_add(float s, float a, float b) { return __fmaf_rn(a, b, s); }
__device__ __forceinline__ float mac_sub(float s, float a, float b) { return __fmaf_rn(-a, b, s); }

// Matrix value -> arithmetic type.
__device__ __forceinline__ double to_arith(double v, double) { return v; }
__device__ __forceinline__ float to_arith(uint16_t h, float) {
  return __uint_as_float(((uint32_t)h) << 16);
}
// Vector value -> arithmetic type (the finest level of the mixed V-cycle
// reads its FP64 right-hand side and rounds it to FP32 where it is read).
__device__ __forceinline__ double vec_to(double v, double) { return v; }
__device__ __forceinline__ float vec_to(double v, float) { return __double2float_rn(v); }
__device__ __forceinline__ float vec_to(float v, float) { return v; }

// FP64 -> BF16 exactly as the oracle does: round to FP32, then round the FP32
// bit pattern to BF16 (nearest-even); NaN stays a quiet NaN.
__host__ __device__ inline uint16_t bf16_from_double(double v) {
  float f = (float)v;
  uint32_t u;
#ifdef __CUDA_ARCH__
  u = __float_as_uint(f);
#else
  __builtin_memcpy(&u, &f, 4);
#endif
  if ((u & 0x7f800000u) == 0x7f800000u && (u & 0x007fffffu)) return (uint16_t)((u >> 16) | 0x40);
  uint32_t lsb = (u >> 16) & 1u;
  u += 0x7fffu + lsb;
  return (uint16_t)(u >> 16);
}

// SplitMix64 (Steele, Lea, Flood 2014) and the counter-based draws built on
// it; the oracle implements the same functions on the host.
__host__ __device__ inline uint64_t splitmix64(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__host__ __device__ inline double uniform01(uint64_t seed, uint64_t i) {
  uint64_t h = splitmix64(splitmix64(seed) + i);
  return (double)(h >> 11) * 0x1.0p-53;
}

}  // namespace hpcgx
