// k_staged.cu -- plane integrals with the volume staged in shared memory.
//
// Geometry.  The lattice rows of radon_grid's planes (fixed i, running j,
// radon_grid/src/integral.c:43-55) run along v2 = normal x v1 =
// (-sin phi, cos phi, 0): every row is horizontal, so all samples of a row
// share one z coordinate and therefore one pair of z-layers of the node grid
// and one z interpolation weight.  The kernel is organised around that:
//
//   work item = (request, z-layer iz, y-tile, chunk of directions).
//   The CTA stages the layer pair (iz, iz+1) of its y-tile into shared memory
//   as one float4 per (cell x, node row y):
//       (v0, v0(x+1) - v0, v1 - v0, (v1 - v0)(x+1) - (v1 - v0))
//   (v0/v1 = node values on layers iz/iz+1), so a trilinear sample is two
//   16-byte loads (node rows y and y+1) and a handful of FMAs.  Two cells of
//   zeros pad every staged row on both sides in x, so samples just outside
//   the cube's x faces read zeros and need no bounds test.  The warps take the
//   chunk's directions one at a time, enumerate every lattice row (shift s,
//   index i) of that direction whose z falls in layer iz, and walk them kGroup
//   rows at a time, 32/kGroup lanes of a row on consecutive samples (those
//   lanes read the same or adjacent cells, so bank conflicts come only from
//   different rows in one quarter-warp; a warp's 16-byte shared load costs
//   four wavefronts however much its lanes overlap).
//   Persistent CTAs (one per SM) pull items from a global counter; the host
//   orders items by estimated cost, largest first.
//
// Nearest sampler (zero_interp, radon_grid/src/interp.c:63-87, the
// reference's default): the same items, rows, classification and sums over
// the n^3 cells instead of the n - 1 node intervals (h = n/2 cells per unit
// length); a row's samples lie in one cell layer, whose y-tile is staged as
// one FP32 value per cell from the volume's z-major copy (all 128 rows of a
// layer fit at n = 128), and a sample is one 4-byte load of cell
// round(q - 1/2) = floor(q).  Guard-band samples take the reference's FP64
// zero_interp arithmetic.
//
// Arithmetic: coordinates and interpolation use the packed FP32 pair
// instructions of sm_100 (fma/add/sub .f32x2) on (x, y) and on the quad
// halves.
//
// Numerics (same contract as the plain kernel, wrt_internal.cuh): FP32 cell
// coordinates; a sample whose x or y cell fraction, or a row whose z cell
// fraction, lies within the guard band of a cell boundary is re-evaluated with
// the reference's FP64 arithmetic from global memory (in a second pass over
// the rows that have such samples, outside the hot loop).  Every row belongs
// to exactly one layer and every sample to exactly one tile, decided by the
// same FP32 expressions everywhere.  The lanes of a row sum its samples in
// FP32 and combine in a fixed tree; the row total is added to its plane as a
// 64-bit fixed-point integer (scale 2^k from max|f| so that no sum can
// overflow): the result does not depend on the order in which rows, items and
// atomics complete -- bitwise identical alone or in a batch.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <tuple>
#include <vector>

#include "wrt_internal.cuh"

namespace {

constexpr unsigned kFull = 0xffffffffu;
// x + 1.5 * 2^23 rounds x to an integer held in the low mantissa bits
// (|x| < 2^22); subtracting the constant's bit pattern recovers it.
constexpr float kMagic = 12582912.0f;
constexpr int kMagicBits = 0x4B400000;
constexpr int kPadX = 2;  // zero cells staged left and right of every row
// Rows whose FP64 z cell coordinate lies within this distance of a node layer
// take the FP64 reference path: their z is the reference's up to a few FP64
// roundings, so only rows on a node layer (where the reference's cell index
// and fraction can disagree) fall in it.
constexpr double kZBand = 1e-9;

// ---- packed FP32 pairs (f32x2 arithmetic of sm_100)
typedef unsigned long long u64;
__device__ __forceinline__ u64 pk2(float lo, float hi) {
  u64 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void upk2(u64 r, float &lo, float &hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(r));
}
__device__ __forceinline__ u64 fma2(u64 a, u64 b, u64 c) {
  u64 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ u64 add2(u64 a, u64 b) {
  u64 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ u64 sub2(u64 a, u64 b) {
  u64 d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
// FP64 scalar from shared memory, re-read at every use (keeps row-geometry
// constants out of the registers the sample loop needs)
__device__ __forceinline__ double ldsd(const double *p) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"((unsigned)__cvta_generic_to_shared(p)));
  return v;
}

// z cell coordinate of lattice row i of (shift s, direction): w = (s nz + i
// delta v1z + 1) h, in FP64 with explicit roundings (the same value wherever
// it is computed: the layer a row belongs to and its z weight agree).
__device__ __forceinline__ double row_w(double s, double nz, double a1z, double di, double h) {
  return __dmul_rn(__dadd_rn(__fma_rn(di, a1z, __dmul_rn(s, nz)), 1.0), h);
}

// Rows i in [imin, imax] of (direction, shift) whose z cell coordinate w lies
// in [wlo, whi) -- w decreases with i (a1z = -sin(theta) delta < 0).  Returns
// the count, first index in *ia.
__device__ __forceinline__ int rows_in_layer(double s, double nz, double a1z, double inv_a1z,
                                             double h, double inv_h, double wlo, double whi,
                                             int imin, int imax, int *ia) {
  if (imin > imax || !(a1z < 0.0)) return 0;
  // real-valued inverses of w(i), then exact fix-up with row_w itself
  const double base = __dmul_rn(s, nz);
  double i_hi = ((wlo * inv_h - 1.0) - base) * inv_a1z;  // w(i) >= wlo  <=>  i <= i_hi
  double i_lo = ((whi * inv_h - 1.0) - base) * inv_a1z;  // w(i) <  whi  <=>  i >  i_lo
  i_hi = fmin(fmax(i_hi, (double)imin - 4.0), (double)imax + 4.0);
  i_lo = fmin(fmax(i_lo, (double)imin - 4.0), (double)imax + 4.0);
  int a = (int)floor(i_lo) + 1, b = (int)floor(i_hi);
  for (int k = 0; k < 4 && row_w(s, nz, a1z, (double)a, h) >= whi; ++k) ++a;
  for (int k = 0; k < 4 && row_w(s, nz, a1z, (double)(a - 1), h) < whi; ++k) --a;
  for (int k = 0; k < 4 && row_w(s, nz, a1z, (double)b, h) < wlo; ++k) --b;
  for (int k = 0; k < 4 && row_w(s, nz, a1z, (double)(b + 1), h) >= wlo; ++k) ++b;
  a = max(a, imin);
  b = min(b, imax);
  *ia = a;
  return b >= a ? b - a + 1 : 0;
}

// j-range with q0 + j dq in [lo, hi] (inv = 1/dq), widened by less than one
// sample on each side: with |dq| < 1/2 the samples kept lie within half a cell
// of [lo, hi] (the staged rows' zero padding relies on this).
__device__ __forceinline__ bool clip_lin(float q0, float dq, float inv, float lo, float hi,
                                         int &jlo, int &jhi) {
  if (dq == 0.0f) return q0 >= lo && q0 <= hi;
  float a = (lo - q0) * inv, b = (hi - q0) * inv;
  if (a > b) {
    const float t = a;
    a = b;
    b = t;
  }
  a = fmaxf(a, (float)jlo) - 0.25f;
  b = fminf(b, (float)jhi) + 0.25f;
  jlo = max(jlo, (int)floorf(a));
  jhi = min(jhi, (int)ceilf(b));
  return jlo <= jhi;
}

// Cell row of sample j of a row, relative to the tile (the fast loop's
// expression bit for bit: q_y = fma(j, dv, vb) rounded once, then rounded to
// an integer by the magic constant).  Monotone in j: non-decreasing for
// dv >= 0, non-increasing for dv < 0.
__device__ __forceinline__ int row_cell_y(int j, float vb, float dv, int yoff) {
  return __float_as_int(__fadd_rn(__fmaf_rn((float)j, dv, vb), kMagic)) - yoff;
}

// First j in [lo, hi] with sgn * (row_cell_y(j) - c) >= 0 (hi + 1 if none);
// the predicate is false then true as j grows.  jest: real-valued estimate of
// the switch, corrected by at most three steps each way and verified against
// its neighbours; a bisection settles the cases it does not (directions with
// dv ~ 0, where the estimate means nothing).
__device__ __forceinline__ int first_at_or_past(int lo, int hi, float jest, int c, int sgn,
                                             float vb, float dv, int yoff) {
  auto at = [&](int j) { return sgn * (row_cell_y(j, vb, dv, yoff) - c) >= 0; };
  int j = (int)fminf(fmaxf(ceilf(jest), (float)lo), (float)hi + 1.0f);  // NaN -> lo
  for (int k = 0; k < 3 && j > lo && at(j - 1); ++k) --j;
  for (int k = 0; k < 3 && j <= hi && !at(j); ++k) ++j;
  if ((j == lo || !at(j - 1)) && (j > hi || at(j))) return j;
  int a = lo, b = hi + 1;
  for (int k = 0; k < 32 && a < b; ++k) {
    const int m = (a + b) >> 1;
    if (at(m)) b = m;
    else a = m + 1;
  }
  return a;
}

__device__ __noinline__ double exact_sample(const wrt::StagedReq &R, int d, int is, int i, int j) {
  const double *D = R.dir + 9 * (size_t)d;
  const double s = R.shift[is];
  const double delta = 1.0 / R.n;
  const double di = (double)i, dj = (double)j;
  const double px = __dadd_rn(__dadd_rn(__dmul_rn(s, D[0]), __dmul_rn(__dmul_rn(delta, D[3]), di)),
                              __dmul_rn(__dmul_rn(delta, D[6]), dj));
  const double py = __dadd_rn(__dadd_rn(__dmul_rn(s, D[1]), __dmul_rn(__dmul_rn(delta, D[4]), di)),
                              __dmul_rn(__dmul_rn(delta, D[7]), dj));
  const double pz = __dadd_rn(__dadd_rn(__dmul_rn(s, D[2]), __dmul_rn(__dmul_rn(delta, D[5]), di)),
                              __dmul_rn(__dmul_rn(delta, D[8]), dj));
  if (R.nearest) return wrtd::exact_nearest(static_cast<const float *>(R.vol), R.n, px, py, pz);
  return R.storage == WRT_STORAGE_BF16
             ? wrtd::exact_trilinear(static_cast<const __nv_bfloat16 *>(R.vol), R.n, px, py, pz)
             : wrtd::exact_trilinear(static_cast<const float *>(R.vol), R.n, px, py, pz);
}

// Sample classification shared by the fast walk and the guard-band walk (the
// two must agree bit for bit).  q = (x, y) cell coordinates minus 1/2.
struct SampleC {
  u64 s;       // q + 1.5 * 2^23 (integer cells in the low mantissa bits)
  u64 t;       // cell fractions (tx, ty)
  bool band;   // within the guard band in x or y
};
__device__ __forceinline__ SampleC classify(u64 q, u64 magic2, u64 half2, float halfband) {
  SampleC c;
  c.s = add2(q, magic2);
  const u64 d = sub2(q, sub2(c.s, magic2));  // q - round(q), in [-1/2, 1/2]
  c.t = add2(d, half2);
  float dx, dy;
  upk2(d, dx, dy);
  c.band = fmaxf(fabsf(dx), fabsf(dy)) > halfband;
  return c;
}

// One sample of the fast loop, written in PTX so that it compiles to the
// instructions it names (the same computation in C++ came out ~8 instructions
// longer per sample): position q = j (du, dv) + qb, the classification of
// classify() bit for bit, the row-end test and the guard-band test as one
// predicate `fast`, the shared address (bits(y' + magic) * 16 qp +
// 16 bits(x' + magic) + abase, or the zero quad), two 16-byte loads (node
// rows y, y+1), the z-lerp of both quad halves as pairs, the x- and y-lerps,
// the running sum.
// A sample that is not fast (past its row's end, or in the guard band) reads
// the zero padding quad instead.  cnt counts the lane's fast samples; a row
// whose lanes count fewer than its length has guard-band samples.
#define WRT_SAMPLE_STEP_PTX                                                          \
  "{\n\t"                                                                            \
  ".reg .b64 q, s, r, d, t, a01, a23, b01, b23, za, zb;\n\t"                         \
  ".reg .f32 dx, dy, m, jf, jfh, tx, ty, ca, cxa, cb, cxb, va, vb, df;\n\t"          \
  ".reg .b32 sxb, syb, addr, addr2, ax;\n\t"                                         \
  ".reg .pred live, fast;\n\t"                                                       \
  "fma.rn.f32x2 q, %2, %3, %4;\n\t"                                                  \
  "add.rn.f32x2 s, q, %5;\n\t"                                                       \
  "sub.rn.f32x2 r, s, %5;\n\t"                                                       \
  "sub.rn.f32x2 d, q, r;\n\t"                                                        \
  "add.rn.f32x2 t, d, %6;\n\t"                                                       \
  "mov.b64 {dx, dy}, d;\n\t"                                                         \
  "abs.f32 dx, dx;\n\t"                                                              \
  "abs.f32 dy, dy;\n\t"                                                              \
  "max.f32 m, dx, dy;\n\t"                                                           \
  "mov.b64 {jf, jfh}, %2;\n\t"                                                       \
  "setp.le.f32 live, jf, %8;\n\t"                                                    \
  "setp.le.and.f32 fast, m, %7, live;\n\t"                                           \
  "@fast add.u32 %1, %1, 1;\n\t"                                                     \
  "mov.b64 {sxb, syb}, s;\n\t"                                                       \
  "shl.b32 ax, sxb, 4;\n\t"                                                          \
  "mad.lo.u32 addr, syb, %9, %10;\n\t"                                               \
  "add.u32 addr, addr, ax;\n\t"                                                      \
  "selp.b32 addr, addr, %12, fast;\n\t"                                              \
  "add.u32 addr2, addr, %9;\n\t"                                                     \
  "ld.shared.v2.b64 {a01, a23}, [addr];\n\t"                                         \
  "ld.shared.v2.b64 {b01, b23}, [addr2];\n\t"                                        \
  "fma.rn.f32x2 za, a23, %11, a01;\n\t"                                              \
  "fma.rn.f32x2 zb, b23, %11, b01;\n\t"                                              \
  "mov.b64 {ca, cxa}, za;\n\t"                                                       \
  "mov.b64 {cb, cxb}, zb;\n\t"                                                       \
  "mov.b64 {tx, ty}, t;\n\t"                                                         \
  "fma.rn.f32 va, tx, cxa, ca;\n\t"                                                  \
  "fma.rn.f32 vb, tx, cxb, cb;\n\t"                                                  \
  "sub.rn.f32 df, vb, va;\n\t"                                                       \
  "fma.rn.f32 va, ty, df, va;\n\t"                                                   \
  "add.rn.f32 %0, %0, va;\n\t"                                                       \
  "}"

__device__ __forceinline__ void sample_step(u64 jj, u64 duv, u64 qb, u64 magic2, u64 half2,
                                            float halfband, float jbf, unsigned qp16,
                                            unsigned abase, unsigned zaddr, u64 tz2, float &part,
                                            unsigned &cnt) {
  asm(WRT_SAMPLE_STEP_PTX
      : "+f"(part), "+r"(cnt)
      : "l"(jj), "l"(duv), "l"(qb), "l"(magic2), "l"(half2), "f"(halfband), "f"(jbf), "r"(qp16),
        "r"(abase), "l"(tz2), "r"(zaddr));
}
#undef WRT_SAMPLE_STEP_PTX

// The nearest sampler's sample (zero_interp): the same position and
// classification, the cell round(q) (that is floor of the cell coordinate),
// one 4-byte load of the staged cell value (or of the zero cell), the sum.
#define WRT_NEAREST_STEP_PTX                                                         \
  "{\n\t"                                                                            \
  ".reg .b64 q, s, r, d;\n\t"                                                        \
  ".reg .f32 dx, dy, m, jf, jfh, v;\n\t"                                             \
  ".reg .b32 sxb, syb, addr, ax;\n\t"                                                \
  ".reg .pred live, fast;\n\t"                                                       \
  "fma.rn.f32x2 q, %2, %3, %4;\n\t"                                                  \
  "add.rn.f32x2 s, q, %5;\n\t"                                                       \
  "sub.rn.f32x2 r, s, %5;\n\t"                                                       \
  "sub.rn.f32x2 d, q, r;\n\t"                                                        \
  "mov.b64 {dx, dy}, d;\n\t"                                                         \
  "abs.f32 dx, dx;\n\t"                                                              \
  "abs.f32 dy, dy;\n\t"                                                              \
  "max.f32 m, dx, dy;\n\t"                                                           \
  "mov.b64 {jf, jfh}, %2;\n\t"                                                       \
  "setp.le.f32 live, jf, %7;\n\t"                                                    \
  "setp.le.and.f32 fast, m, %6, live;\n\t"                                           \
  "@fast add.u32 %1, %1, 1;\n\t"                                                     \
  "mov.b64 {sxb, syb}, s;\n\t"                                                       \
  "shl.b32 ax, sxb, 2;\n\t"                                                          \
  "mad.lo.u32 addr, syb, %8, %9;\n\t"                                                \
  "add.u32 addr, addr, ax;\n\t"                                                      \
  "selp.b32 addr, addr, %10, fast;\n\t"                                              \
  "ld.shared.f32 v, [addr];\n\t"                                                     \
  "add.rn.f32 %0, %0, v;\n\t"                                                        \
  "}"

__device__ __forceinline__ void nearest_step(u64 jj, u64 duv, u64 qb, u64 magic2, float halfband,
                                             float jbf, unsigned qp4, unsigned abase,
                                             unsigned zaddr, float &part, unsigned &cnt) {
  asm(WRT_NEAREST_STEP_PTX
      : "+f"(part), "+r"(cnt)
      : "l"(jj), "l"(duv), "l"(qb), "l"(magic2), "f"(halfband), "f"(jbf), "r"(qp4), "r"(abase),
        "r"(zaddr));
}
#undef WRT_NEAREST_STEP_PTX

// FP64 reference evaluation of `count` queued guard-band samples of direction
// d, one per lane, each added to its plane as a fixed-point integer.  Returns
// the number of samples this lane evaluated.
__device__ __forceinline__ int exact_queue_flush(const wrt::StagedReq &R, int d,
                                                 const int2 *q, int count, int lane) {
  if (lane >= count) return 0;
  const int2 e = q[lane];
  const int i = (int)(short)((unsigned)e.y >> 16), j = (int)(short)((unsigned)e.y & 0xFFFFu);
  const long long v = __double2ll_rn(exact_sample(R, d, e.x, i, j) * R.scale);
  if (v != 0) atomicAdd(R.acc + (size_t)e.x * R.ndir + d, (unsigned long long)v);
  return 1;
}

// kThreads: CTA size (one CTA per SM); kGroup: lattice rows a warp walks at
// once (32/kGroup lanes per row, on consecutive samples); kShiftsPerLane:
// shifts a lane enumerates per pass (a pass covers 32*kShiftsPerLane shifts);
// kCount: count the samples evaluated (measurement build); kNear: the nearest
// sampler (n cells per axis, one staged FP32 value per cell of a z-layer,
// rows grouped by the cell layer of their z) instead of trilinear (n - 1
// cells between nodes, layer pairs staged as quads).
template <int kThreads, int kGroup, int kShiftsPerLane, bool kCount, bool kNear = false>
__global__ void __launch_bounds__(kThreads, 1)
    plane_staged_kernel(const wrt::StagedReq *__restrict__ reqs,
                        const wrt::StagedItem *__restrict__ items,
                        const int *__restrict__ nitems_ptr, int *__restrict__ next_item,
                        unsigned long long *__restrict__ counter) {
  constexpr int kLanesPerRow = 32 / kGroup;
  constexpr int kWarps = kThreads / 32;
  // dynamic shared memory: per warp a row table and a guard-band queue, then
  // the staged tile
  extern __shared__ float4 dyn_smem[];
  // the warp's rows: [0][slot] = (q0x, q0y, tz, ja), [1][slot] = (jb, shift
  // index, i | jlo, jhi | flags); the two halves apart, so that a half-warp's
  // 4 rows read words that fall in any of the 8 bank groups
  float4(*s_rows)[2][32] = reinterpret_cast<float4(*)[2][32]>(dyn_smem);
  // guard-band samples waiting for the FP64 path: (shift index, i << 16 | j)
  int2(*s_xq)[64] = reinterpret_cast<int2(*)[64]>(dyn_smem + kWarps * 64);
  float4 *quads = dyn_smem + kWarps * wrt::kStagedWarpSmemQuads;
  __shared__ int s_item, s_dir;
  // FP64 row geometry: per item (h, 1/h, layer bounds) and per warp's direction
  // (normal, delta v1, 1/(delta v1z))
  __shared__ double s_item_geo[4];
  __shared__ double s_dir_geo[kWarps][8];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int pos = lane % kLanesPerRow;  // position of this lane within its row
  const unsigned smem0 = (unsigned)__cvta_generic_to_shared(quads);
  unsigned long long evaluated = 0;
  const u64 magic2 = pk2(kMagic, kMagic), half2 = pk2(0.5f, 0.5f);
  const u64 step2 = pk2((float)kLanesPerRow, (float)kLanesPerRow);
  const int nitems = __ldg(nitems_ptr);
  for (;;) {
    if (tid == 0) {
      s_item = atomicAdd(next_item, 1);
      s_dir = 0;
    }
    __syncthreads();
    const int it = s_item;
    if (it >= nitems) break;
    const wrt::StagedItem item = items[it];
    const wrt::StagedReq &R = reqs[item.req];
    const int n = R.n, W = kNear ? n : n - 1;  // cells per axis
    const int qp = R.qpitch;
    const int y0 = item.tile * R.tile_h;
    const int H = min(R.tile_h, W - y0);
    // layer bounds of the row enumeration; rows within kZBand of a node layer
    // (or of the cube's z faces) are evaluated exactly (visible to all warps
    // after the staging barrier below)
    if (tid == 0) {
      const double h64 = 0.5 * (double)W;
      s_item_geo[0] = h64;
      s_item_geo[1] = 1.0 / h64;
      s_item_geo[2] = item.layer == 0 ? -kZBand : (double)item.layer;
      s_item_geo[3] = item.layer == W - 1 ? (double)W + kZBand : (double)(item.layer + 1);
    }
    // ---- stage layer pair (iz, iz+1), node rows y0 .. y0+H, cells -2 .. W+1
    // (nearest: cell layer iz, cell rows y0 .. y0+H-1, one float per cell)
    if (kNear) {
      const float *src = static_cast<const float *>(R.pairs) +
                         ((size_t)item.layer * n * R.pitch2 + (size_t)y0 * R.pitch2);
      float *cells = reinterpret_cast<float *>(quads);
      const int wide = W + 2 * kPadX;
      const int total = H * wide;
      for (int k = tid; k < total; k += kThreads) {
        const int yy = k / wide, xc = k - yy * wide, x = xc - kPadX;
        cells[yy * qp + xc] = (x >= 0 && x < W) ? __ldg(src + (size_t)yy * R.pitch2 + x) : 0.0f;
      }
    } else {
      const size_t base = (size_t)item.layer * n * R.pitch2 + (size_t)y0 * R.pitch2;
      const float2 *src = static_cast<const float2 *>(R.pairs) + base;
      const __nv_bfloat162 *src16 = static_cast<const __nv_bfloat162 *>(R.pairs) + base;
      const bool bf16 = R.storage == WRT_STORAGE_BF16;
      const int wide = W + 2 * kPadX;
      const int total = (H + 1) * wide;
      for (int k = tid; k < total; k += kThreads) {
        const int yy = k / wide, xc = k - yy * wide, x = xc - kPadX;
        float4 q = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (x >= 0 && x < W) {
          const size_t o = (size_t)yy * R.pitch2 + x;
          const float2 a = bf16 ? __bfloat1622float2(__ldg(src16 + o)) : __ldg(src + o);
          const float2 b = bf16 ? __bfloat1622float2(__ldg(src16 + o + 1)) : __ldg(src + o + 1);
          const float dz0 = a.y - a.x, dz1 = b.y - b.x;
          q = make_float4(a.x, b.x - a.x, dz0, dz1 - dz0);
        }
        quads[yy * qp + xc] = q;
      }
    }
    __syncthreads();
    const float delta = 1.0f / (float)n, nf = (float)n;
    const float g = R.guard;
    const float halfband = 0.5f - g;
    const float rc2 = R.crop_r2;
    const int L = R.L;
    // Cell coordinates are held relative to the grid's centre cell C (halves
    // their magnitude and so their FP32 rounding, which sets the guard band).
    const int C = W / 2;
    // shared address of cell (x, row y) = sbase + E * (yrel * qp + bits(x' + magic)),
    // yrel = bits(y' + magic) - yoff, E the element size (16, nearest 4); as
    // one expression (mod 2^32):
    //   bits(y' + magic) * E qp + E bits(x' + magic) + abase
    constexpr unsigned kElem = kNear ? 4u : 16u;
    const unsigned sbase = smem0 + kElem * (unsigned)(kPadX + C - kMagicBits);
    const unsigned qp16 = kElem * (unsigned)qp;
    const int yoff = kMagicBits - C + y0;
    const unsigned abase = sbase - qp16 * (unsigned)yoff;
    for (;;) {
      int dl = 0;
      if (lane == 0) dl = atomicAdd(&s_dir, 1);
      dl = __shfl_sync(kFull, dl, 0);
      if (dl >= item.ndir) break;
      const int d = item.dir0 + dl;
      const double *Dd = R.dir + 9 * (size_t)d;
      double *G = s_dir_geo[warp];
      {
        const double delta64 = 1.0 / (double)n;
        if (lane < 6) G[lane] = __ldg(Dd + lane) * (lane >= 3 ? delta64 : 1.0);
        if (lane == 6) G[6] = 1.0 / (__ldg(Dd + 5) * delta64);
        __syncwarp();
      }
      // per-sample steps in cell units, rounded once to FP32
      const float du = (float)(__ldg(Dd + 6) * (1.0 / (double)n) * ldsd(&s_item_geo[0]));
      const float dv = (float)(__ldg(Dd + 7) * (1.0 / (double)n) * ldsd(&s_item_geo[0]));
      const float inv_du = du != 0.0f ? 1.0f / du : 0.0f;
      const float inv_dv = dv != 0.0f ? 1.0f / dv : 0.0f;
      const u64 duv = pk2(du, dv);
      int xq_n = 0;  // queued guard-band samples of this direction (warp-uniform)
      for (int sb = 0; sb < R.nshift; sb += 32 * kShiftsPerLane) {
        // ---- enumerate rows of this layer: lane owns shifts sb + lane*K + k
        int cnt[kShiftsPerLane], ia[kShiftsPerLane];
        int lane_total = 0;
#pragma unroll
        for (int k = 0; k < kShiftsPerLane; ++k) {
          const int is = sb + lane * kShiftsPerLane + k;
          cnt[k] = 0;
          ia[k] = 0;
          if (is < R.nshift) {
            const float s = __ldg(R.shift32 + is);
            const float rem = rc2 - s * s;
            if (rem >= 0.0f) {
              // |i| <= sqrt(rem) / delta; +1 covers the rounding of sqrt and n
              const int im = (int)floorf(sqrtf(rem) * nf) + 1;
              cnt[k] = rows_in_layer(__ldg(R.shift + is), ldsd(G + 2), ldsd(G + 5), ldsd(G + 6),
                                     ldsd(&s_item_geo[0]), ldsd(&s_item_geo[1]),
                                     ldsd(&s_item_geo[2]), ldsd(&s_item_geo[3]), max(-L, -im),
                                     min(L - 1, im), &ia[k]);
            }
          }
          lane_total += cnt[k];
        }
        int incl = lane_total;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int t = __shfl_up_sync(kFull, incl, o);
          if (lane >= o) incl += t;
        }
        const int excl = incl - lane_total;
        const int total = __shfl_sync(kFull, incl, 31);
        for (int r0 = 0; r0 < total; r0 += 32) {
          const int r = r0 + lane;
          // ---- locate row r: owner lane (largest lane with excl <= r), then its shift
          int owner = 0;
#pragma unroll
          for (int step = 16; step > 0; step >>= 1) {
            const int cand = owner + step;
            const int ex = __shfl_sync(kFull, excl, cand);
            if (cand < 32 && ex <= r) owner = cand;
          }
          int off = r - __shfl_sync(kFull, excl, owner);
          int is = -1, i = 0;
#pragma unroll
          for (int k = 0; k < kShiftsPerLane; ++k) {
            const int c = __shfl_sync(kFull, cnt[k], owner);
            const int a = __shfl_sync(kFull, ia[k], owner);
            if (is < 0 && off < c) {
              is = sb + owner * kShiftsPerLane + k;
              i = a + off;
            }
            if (is < 0) off -= c;
          }
          const bool valid = r < total && is >= 0;
          // ---- row set-up (one lane per row): [jlo, jhi] holds every sample
          // of the row that this tile may have to evaluate; [ja, jb] is the
          // exact run of samples whose FP32 cell row lies in the tile (the fast
          // loop walks it without a per-sample tile test)
          int jlo = 1, jhi = 0, ja = 1, jb = 0;
          float ub = 0.f, vb = 0.f, tz = 0.f;
          bool zexact = false, edge = false;
          if (valid) {
            const float s = __ldg(R.shift32 + is);
            const double s64 = __ldg(R.shift + is), di64 = (double)i;
            const float di = (float)i;
            const double h64 = ldsd(&s_item_geo[0]);
            const double tz64 = row_w(s64, ldsd(G + 2), ldsd(G + 5), di64, h64) - (double)item.layer;
            tz = (float)tz64;
            zexact = tz64 < kZBand || tz64 > 1.0 - kZBand;
            // row origin in cell units relative to the centre (q - 1/2 - C at
            // j = 0), FP64 then rounded once
            ub = (float)((fma(di64, ldsd(G + 3), s64 * ldsd(G + 0)) + 1.0) * h64 - (0.5 + C));
            vb = (float)((fma(di64, ldsd(G + 4), s64 * ldsd(G + 1)) + 1.0) * h64 - (0.5 + C));
            const float rem = rc2 - s * s - (delta * di) * (delta * di);
            if (rem >= 0.0f) {
              const int jm = (int)floorf(sqrtf(rem) * nf) + 1;
              jlo = max(-L, -jm);
              jhi = min(L - 1, jm);
              if (!clip_lin(ub, du, inv_du, -1.5f - C, (float)(W + 1 - C) - 0.5f, jlo, jhi) ||
                  !clip_lin(vb, dv, inv_dv, (float)(y0 - C) - 1.5f, (float)(y0 + H - C) + 0.5f,
                            jlo, jhi)) {
                jlo = 1;
                jhi = 0;
              }
            }
            if (jlo <= jhi && zexact) {
              ja = jlo;  // a row in the z band has no fast samples
              jb = jlo - 1;
            } else if (jlo <= jhi) {
              const float yb = (float)(y0 - C) - 0.5f;  // q_y at the tile's first cell row
              if (dv >= 0.0f) {
                ja = first_at_or_past(jlo, jhi, (yb - vb) * inv_dv, 0, 1, vb, dv, yoff);
                jb = first_at_or_past(jlo, jhi, (yb + (float)H - vb) * inv_dv, H, 1, vb, dv,
                                      yoff) - 1;
              } else {
                ja = first_at_or_past(jlo, jhi, (yb + (float)H - vb) * inv_dv, H - 1, -1, vb,
                                      dv, yoff);
                jb = first_at_or_past(jlo, jhi, (yb - vb) * inv_dv, -1, -1, vb, dv, yoff) - 1;
              }
              // A guard-band sample just outside a y face of the grid has its
              // cell row clamped into the edge tile by the guard-band pass; the
              // fast loop does not see it, so the row asks for that pass here.
              // Only the samples next to [ja, jb] (or the ends of an empty run)
              // can lie within the guard band of a face: cell rows are
              // monotone in j and |dv| < 1/2.
              const int c1 = ja <= jb ? ja - 1 : jlo, c2 = ja <= jb ? jb + 1 : jhi;
#pragma unroll
              for (int e = 0; e < 2; ++e) {
                const int jc = e ? c2 : c1;
                if (jc < jlo || jc > jhi) continue;
                const SampleC cc = classify(fma2(pk2((float)jc, (float)jc), pk2(du, dv),
                                                 pk2(ub, vb)),
                                            magic2, half2, halfband);
                float csx, csy;
                upk2(cc.s, csx, csy);
                const int cy = min(max(__float_as_int(csy) - kMagicBits + C, 0), W - 1) - y0;
                edge |= cc.band & ((unsigned)cy < (unsigned)H);
              }
            }
          }
          // ---- rows with fast samples or guard-band work, longest fast run
          // first (rows walked together then have similar lengths), kGroup at
          // a time
          const bool live_row = valid && jlo <= jhi && (ja <= jb || zexact || edge);
          const int nrows = __popc(__ballot_sync(kFull, live_row));
          if (live_row) {
            // i, j in [-L, L) fit 16 bits (L <= 8 n and n < 3600 for a staged tile)
            s_rows[warp][0][lane] = make_float4(ub, vb, tz, __int_as_float(ja));
            s_rows[warp][1][lane] = make_float4(
                __int_as_float(jb), __int_as_float(is),
                __int_as_float((int)(((unsigned)i << 16) | ((unsigned)jlo & 0xFFFFu))),
                __int_as_float((int)(((unsigned)jhi << 16) | (unsigned)zexact |
                                     ((unsigned)edge << 1))));
          }
          // bitonic sort of (fast length, lane) keys, descending; empty slots last
          unsigned key =
              live_row ? ((unsigned)(max(jb - ja + 1, 0) + 1) << 5) | (unsigned)lane : 0u;
#pragma unroll
          for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
            for (int j = k >> 1; j > 0; j >>= 1) {
              const unsigned other = __shfl_xor_sync(kFull, key, j);
              const bool up = ((lane & k) == 0) == ((lane & j) == 0);
              key = up ? max(key, other) : min(key, other);
            }
          }
          __syncwarp();
          for (int g0 = 0; g0 < nrows; g0 += kGroup) {
            const int kr = g0 + lane / kLanesPerRow;
            const bool rvalid = kr < nrows;
            const int slot = (int)(__shfl_sync(kFull, key, rvalid ? kr : 0) & 31u);
            const float4 r0v = s_rows[warp][0][slot], r1v = s_rows[warp][1][slot];
            const float k_ubm = r0v.x, k_vbm = r0v.y;  // q - 1/2 at j = 0
            const float k_tz = r0v.z;
            const int k_ja = __float_as_int(r0v.w);
            const int k_jb = rvalid ? __float_as_int(r1v.x) : k_ja - 1;
            const int k_is = __float_as_int(r1v.y);
            const int k_pz = __float_as_int(r1v.z), k_pw = __float_as_int(r1v.w);
            const int k_i = k_pz >> 16, k_jlo = (int)(short)(k_pz & 0xFFFF);
            const int k_jhi = rvalid ? (k_pw >> 16) : k_jlo - 1;
            const bool k_zx = rvalid && (k_pw & 1) != 0;
            const bool k_edge = rvalid && (k_pw & 2) != 0;
            const u64 qb = pk2(k_ubm, k_vbm), tz2 = pk2(k_tz, k_tz);
            const int len = k_jb - k_ja + 1;
            const int trips = (int)__reduce_max_sync(
                kFull, (unsigned)((max(len, 0) + kLanesPerRow - 1) / kLanesPerRow));
            const float jbf = (float)k_jb;
            const float jf0 = (float)(k_ja + pos);
            bool any_band = k_zx | k_edge;
            float part = 0.0f;
            {
              // branch-free: a lane past its row's end or on a guard-band
              // sample reads the zero quads of the padding column (staged
              // column 0, node rows 0 and 1) and adds 0
              unsigned cnt = 0;
              u64 jj = pk2(jf0, jf0);
              if (kNear) {
#pragma unroll 4
                for (int t = 0; t < trips; ++t, jj = add2(jj, step2))
                  nearest_step(jj, duv, qb, magic2, halfband, jbf, qp16, abase, smem0, part, cnt);
              } else {
#pragma unroll 4
                for (int t = 0; t < trips; ++t, jj = add2(jj, step2))
                  sample_step(jj, duv, qb, magic2, half2, halfband, jbf, qp16, abase, smem0, tz2,
                              part, cnt);
              }
              // samples j = ja + pos + t kLanesPerRow <= jb of this lane
              const int mine = k_jb - k_ja - pos >= 0 ? (k_jb - k_ja - pos) / kLanesPerRow + 1 : 0;
              any_band |= (int)cnt < mine;
              if (kCount) evaluated += cnt;
            }
            // ---- guard-band samples (and whole rows in the z band) go to the
            // warp's queue; full warps of them take the FP64 path below
            if (__any_sync(kFull, any_band)) {
              // walks the row's whole candidate range [jlo, jhi]
              const int blen = k_jhi - k_jlo + 1;
              const int btrips = (int)__reduce_max_sync(
                  kFull, (unsigned)((max(blen, 0) + kLanesPerRow - 1) / kLanesPerRow));
              const float jhif = (float)k_jhi;
              const float bj0 = (float)(k_jlo + pos);
              u64 jj = pk2(bj0, bj0);
              for (int t = 0; t < btrips; ++t, jj = add2(jj, step2)) {
                float jf, jf_hi;
                upk2(jj, jf, jf_hi);
                const SampleC c = classify(fma2(jj, duv, qb), magic2, half2, halfband);
                float sx, sy;
                upk2(c.s, sx, sy);
                // a guard-band sample belongs to the tile of its FP32 cell row,
                // clamped to the grid (samples within the band outside a face
                // are evaluated, and cut off, by the FP64 reference arithmetic)
                const int cy = min(max(__float_as_int(sy) - kMagicBits + C, 0), W - 1) - y0;
                const bool want = (jf <= jhif) & (c.band | k_zx) & ((unsigned)cy < (unsigned)H);
                const unsigned m = __ballot_sync(kFull, want);
                if (m) {
                  if (want)
                    s_xq[warp][xq_n + __popc(m & ((1u << lane) - 1u))] =
                        make_int2(k_is, (int)(((unsigned)k_i << 16) | ((unsigned)(int)jf & 0xFFFFu)));
                  xq_n += __popc(m);
                  __syncwarp();
                  if (xq_n >= 32) {
                    const int ev = exact_queue_flush(R, d, s_xq[warp], 32, lane);
                    if (kCount) evaluated += ev;
                    if (lane < xq_n - 32) s_xq[warp][lane] = s_xq[warp][lane + 32];
                    xq_n -= 32;
                    __syncwarp();
                  }
                }
              }
            }
            // ---- row sums over the row's lanes, fixed point, one atomic per row
#pragma unroll
            for (int o = kLanesPerRow / 2; o > 0; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
            const long long v = rvalid ? __double2ll_rn((double)part * R.scale) : 0LL;
            if (pos == 0 && v != 0)
              atomicAdd(R.acc + (size_t)k_is * R.ndir + d, (unsigned long long)v);
          }
          __syncwarp();
        }
      }
      if (xq_n > 0) {
        const int ev = exact_queue_flush(R, d, s_xq[warp], xq_n, lane);
        if (kCount) evaluated += ev;
        __syncwarp();
      }
    }
    __syncthreads();
  }
  if (kCount) {
    for (int o = 16; o > 0; o >>= 1) evaluated += __shfl_xor_sync(kFull, evaluated, o);
    if (lane == 0 && evaluated) atomicAdd(counter, evaluated);
  }
}

// out[p] = acc[p] / scale * delta^2, in place (acc aliases out).
__global__ void plane_finalize_kernel(double *out, long long count, double factor) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < count;
       k += (long long)gridDim.x * blockDim.x) {
    const long long v = reinterpret_cast<const long long *>(out)[k];
    out[k] = (double)v * factor;
  }
}

}  // namespace

namespace wrt {

int staged_smem_bytes(int n, int *tile_h, int *qpitch) {
  const int W = n - 1;
  int qp = W + 2 * kPadX;
  while (qp % 8 != 3) ++qp;  // 16-byte words: rows offset by 3 bank groups
  const int budget = kStagedSmemMax;
  int rows_max = budget / (qp * 16);  // node rows that fit
  if (rows_max < 3) return -1;
  int ntiles = (W + (rows_max - 1) - 1) / (rows_max - 1);
  int th = (W + ntiles - 1) / ntiles;  // balanced tiles of <= rows_max-1 cells
  *tile_h = th;
  *qpitch = qp;
  return (th + 1) * qp * 16;
}

int staged_smem_bytes_nearest(int n, int *tile_h, int *qpitch) {
  int qp = n + 2 * kPadX;
  if (!(qp & 1)) ++qp;  // odd pitch: a row of cells and the next start in different banks
  const int rows_max = kStagedSmemMax / (qp * 4);  // cell rows that fit
  if (rows_max < 2) return -1;
  const int ntiles = (n + rows_max - 1) / rows_max;
  const int th = (n + ntiles - 1) / ntiles;  // balanced tiles of <= rows_max cell rows
  *tile_h = th;
  *qpitch = qp;
  return th * qp * 4;
}

namespace {
template <int T, int G, int K, bool NEAR = false>
int launch_cfg(wrt_ctx *ctx, cudaStream_t stream, const StagedReq *d_reqs,
               const StagedItem *d_items, const int *d_nitems, int max_smem, int *d_next) {
  const bool count = ctx->d_counter != nullptr;
  auto kern = count ? plane_staged_kernel<T, G, K, true, NEAR>
                    : plane_staged_kernel<T, G, K, false, NEAR>;
  max_smem += (T / 32) * wrt::kStagedWarpSmemQuads * 16;  // per-warp row tables and queues
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "staged kernel smem attribute");
  e = cudaMemsetAsync(d_next, 0, sizeof(int), stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "staged counter reset");
  kern<<<ctx->sm_count, T, max_smem, stream>>>(d_reqs, d_items, d_nitems, d_next,
                                               ctx->d_counter);
  ctx->launches++;
  return check_launch(ctx, "plane_staged_kernel");
}
}  // namespace

// The tile shapes the autotuner chooses among: (CTA threads, lattice rows a
// warp walks at once, shifts per lane per enumeration pass).
// Entry 0 is the default (no tuning: the serving loop, untuned contexts); it
// was the fastest at 96^3, 128^3 and 256^3 on B200.
const StagedConfig kStagedConfigs[] = {
    {1024, 8, 2}, {768, 8, 2}, {768, 4, 2}, {1024, 4, 2}, {768, 2, 2}, {1024, 1, 2}, {512, 8, 4},
};
const int kNumStagedConfigs = sizeof(kStagedConfigs) / sizeof(kStagedConfigs[0]);

int plane_staged_launch(wrt_ctx *ctx, cudaStream_t stream, const StagedReq *d_reqs,
                        const StagedItem *d_items, const int *d_nitems, int max_smem,
                        int *d_next) {
  const int c = (ctx->staged_config >= 0 && ctx->staged_config < kNumStagedConfigs)
                    ? ctx->staged_config : 0;
  switch (c) {
    case 0: return launch_cfg<1024, 8, 2>(ctx, stream, d_reqs, d_items, d_nitems, max_smem, d_next);
    case 1: return launch_cfg<768, 8, 2>(ctx, stream, d_reqs, d_items, d_nitems, max_smem, d_next);
    case 2: return launch_cfg<768, 4, 2>(ctx, stream, d_reqs, d_items, d_nitems, max_smem, d_next);
    case 3: return launch_cfg<1024, 4, 2>(ctx, stream, d_reqs, d_items, d_nitems, max_smem, d_next);
    case 4: return launch_cfg<768, 2, 2>(ctx, stream, d_reqs, d_items, d_nitems, max_smem, d_next);
    case 5: return launch_cfg<1024, 1, 2>(ctx, stream, d_reqs, d_items, d_nitems, max_smem, d_next);
    default: return launch_cfg<512, 8, 4>(ctx, stream, d_reqs, d_items, d_nitems, max_smem, d_next);
  }
}

int plane_staged_launch_nearest(wrt_ctx *ctx, cudaStream_t stream, const StagedReq *d_reqs,
                                const StagedItem *d_items, const int *d_nitems, int max_smem,
                                int *d_next) {
  return launch_cfg<1024, 8, 2, true>(ctx, stream, d_reqs, d_items, d_nitems, max_smem, d_next);
}

int plane_finalize(wrt_ctx *ctx, double *out, long long count, double factor) {
  const int blocks = ctx->sm_count * 4;
  plane_finalize_kernel<<<blocks, 256, 0, ctx->stream>>>(out, count, factor);
  ctx->launches++;
  return check_launch(ctx, "plane_finalize_kernel");
}

// Work items of one request, largest estimated cost first.  Cost of a
// (layer, tile): voxels of the tile's slab inside the crop radius.
void staged_items_costed(int req, int n, int tile_h, float crop_r2, int ndir, int dir_chunk,
                         double weight, std::vector<std::pair<double, StagedItem>> &out,
                         bool nearest) {
  const int W = nearest ? n : n - 1;  // cells per axis
  const int ntiles = (W + tile_h - 1) / tile_h;
  const double h = 2.0 / W;
  for (int iz = 0; iz < W; ++iz) {
    const double z = -1.0 + h * (iz + 0.5);
    for (int t = 0; t < ntiles; ++t) {
      double cost = 0.0;
      for (int y = t * tile_h; y < std::min(W, (t + 1) * tile_h); ++y) {
        const double yy = -1.0 + h * (y + 0.5);
        const double r = crop_r2 - z * z - yy * yy;
        if (r > 0) cost += 2.0 * sqrt(r);
      }
      if (cost <= 0.0) continue;
      for (int d0 = 0; d0 < ndir; d0 += dir_chunk) {
        StagedItem it;
        it.req = req;
        it.layer = iz;
        it.tile = t;
        it.dir0 = d0;
        it.ndir = std::min(dir_chunk, ndir - d0);
        out.push_back({cost * it.ndir * weight, it});
      }
    }
  }
}

void staged_items(int req, int n, int tile_h, float crop_r2, int ndir, int dir_chunk,
                  std::vector<StagedItem> &out, bool nearest) {
  std::vector<std::pair<double, StagedItem>> v;
  staged_items_costed(req, n, tile_h, crop_r2, ndir, dir_chunk, 1.0, v, nearest);
  std::stable_sort(v.begin(), v.end(),
                   [](const std::pair<double, StagedItem> &a,
                      const std::pair<double, StagedItem> &b) { return a.first > b.first; });
  for (auto &c : v) out.push_back(c.second);
}

namespace {
struct ItemList {
  void *d = nullptr;
  int count = 0;
  size_t bytes = 0;
};
struct StagedCache {
  std::map<std::tuple<int, int, unsigned, int, bool>, ItemList> lists;
};
}  // namespace

// Device copy of the item list of one geometry: a 16-byte header holding the
// item count (the kernel reads it from there), then the items.
int staged_items_cached(wrt_ctx *ctx, int n, int tile_h, float crop_r2, int ndir,
                        StagedItem **d_items, const int **d_nitems, int *nitems, bool nearest) {
  if (!ctx->staged_cache) ctx->staged_cache = new StagedCache();
  StagedCache *c = static_cast<StagedCache *>(ctx->staged_cache);
  unsigned bits;
  memcpy(&bits, &crop_r2, sizeof(bits));
  const auto key = std::make_tuple(n, tile_h, bits, ndir, nearest);
  auto it = c->lists.find(key);
  if (it == c->lists.end()) {
    if (c->lists.size() > 64) {  // bounded: drop everything, rebuild on demand
      cudaStreamSynchronize(ctx->stream);
      for (auto &kv : c->lists) ctx_free(ctx, kv.second.d, kv.second.bytes);
      c->lists.clear();
    }
    std::vector<StagedItem> items;
    staged_items(0, n, tile_h, crop_r2, ndir, kStagedDirChunk, items, nearest);
    ItemList l;
    l.count = (int)items.size();
    l.bytes = 16 + sizeof(StagedItem) * items.size();
    std::vector<char> host(l.bytes, 0);
    memcpy(host.data(), &l.count, sizeof(int));
    if (!items.empty()) memcpy(host.data() + 16, items.data(), sizeof(StagedItem) * items.size());
    int st = ctx_alloc(ctx, (void **)&l.d, l.bytes);
    if (st) return st;
    cudaError_t e = cudaMemcpy(l.d, host.data(), l.bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      ctx_free(ctx, l.d, l.bytes);
      return cuda_fail(ctx, e, "staged items");
    }
    it = c->lists.emplace(key, l).first;
  }
  *d_nitems = reinterpret_cast<const int *>(it->second.d);
  *d_items = reinterpret_cast<StagedItem *>(reinterpret_cast<char *>(it->second.d) + 16);
  *nitems = it->second.count;
  return WRT_OK;
}

int staged_scratch(wrt_ctx *ctx, size_t req_bytes) {
  if (!ctx->staged_next) {
    int st = ctx_alloc(ctx, (void **)&ctx->staged_next, sizeof(int));
    if (st) return st;
  }
  if (ctx->staged_req_bytes < req_bytes) {
    if (ctx->staged_req) {
      cudaStreamSynchronize(ctx->stream);
      ctx_free(ctx, ctx->staged_req, ctx->staged_req_bytes);
      ctx->staged_req = nullptr;
    }
    int st = ctx_alloc(ctx, &ctx->staged_req, req_bytes);
    if (st) return st;
    ctx->staged_req_bytes = req_bytes;
  }
  return WRT_OK;
}

void staged_release(wrt_ctx *ctx) {
  if (ctx->staged_cache) {
    StagedCache *c = static_cast<StagedCache *>(ctx->staged_cache);
    for (auto &kv : c->lists) ctx_free(ctx, kv.second.d, kv.second.bytes);
    delete c;
    ctx->staged_cache = nullptr;
  }
  ctx_free(ctx, ctx->staged_req, ctx->staged_req_bytes);
  ctx->staged_req = nullptr;
  ctx_free(ctx, ctx->staged_next, sizeof(int));
  ctx->staged_next = nullptr;
}

}  // namespace wrt
