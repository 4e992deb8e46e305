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
//   as one float4 per cell (x, y):
//       (v0, v1 - v0, v0(x+1) - v0, (v1 - v0)(x+1) - (v1 - v0))
//   (v0/v1 = node values on layers iz/iz+1), so a trilinear sample is two
//   16-byte loads (rows y and y+1) and eight FMAs.  Its warps then take the
//   chunk's directions one at a time, enumerate every lattice row (shift s,
//   index i) of that direction whose z falls in layer iz, and walk them with
//   one lane per row.
//   Persistent CTAs (one per SM) pull items from a global counter; the host
//   orders items by estimated cost, largest first.
//
// Numerics (same contract as the plain kernel, wrt_internal.cuh): FP32 cell
// coordinates; a sample whose x or y cell fraction, or a row whose z cell
// fraction, lies within the guard band of a cell boundary is re-evaluated with
// the reference's FP64 arithmetic from global memory.  Every row belongs to
// exactly one layer and every sample to exactly one tile, decided by the same
// FP32 expressions everywhere.  Row sums are FP64; they are accumulated per
// plane as 64-bit fixed-point integers (scale 2^k chosen from max|f| so that no
// sum can overflow), which makes the result independent of the order in which
// items, warps and atomics complete: bitwise identical alone or in a batch.
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

__device__ __forceinline__ float row_w(float s, float nz, float a1z, float di, float h) {
  return (fmaf(di, a1z, s * nz) + 1.0f) * h;
}

// Rows i of (direction, shift) whose z cell coordinate w lies in
// [wlo, whi) -- w decreases with i.  Returns count, first index in *ia.
__device__ __forceinline__ int rows_in_layer(float s, float nz, float a1z, float h, float wlo,
                                             float whi, int imin, int imax, int *ia) {
  if (imin > imax) return 0;
  // real-valued inverses of w(i) = (s nz + i a1z + 1) h, then exact fix-up
  const float base = s * nz;
  float i_hi = ((wlo / h - 1.0f) - base) / a1z;  // w(i) >= wlo  <=>  i <= i_hi
  float i_lo = ((whi / h - 1.0f) - base) / a1z;  // w(i) <  whi  <=>  i >  i_lo
  i_hi = fminf(fmaxf(i_hi, (float)imin - 4.0f), (float)imax + 4.0f);
  i_lo = fminf(fmaxf(i_lo, (float)imin - 4.0f), (float)imax + 4.0f);
  int a = (int)floorf(i_lo) + 1, b = (int)floorf(i_hi);
  for (int k = 0; k < 4 && row_w(s, nz, a1z, (float)a, h) >= whi; ++k) ++a;
  for (int k = 0; k < 4 && row_w(s, nz, a1z, (float)(a - 1), h) < whi; ++k) --a;
  for (int k = 0; k < 4 && row_w(s, nz, a1z, (float)b, h) < wlo; ++k) --b;
  for (int k = 0; k < 4 && row_w(s, nz, a1z, (float)(b + 1), h) >= wlo; ++k) ++b;
  a = max(a, imin);
  b = min(b, imax);
  *ia = a;
  return b >= a ? b - a + 1 : 0;
}

__device__ __forceinline__ bool clip_lin(float q0, float dq, float lo, float hi, int &jlo,
                                         int &jhi) {
  // conservative j-range with q0 + j dq in [lo, hi]
  if (dq == 0.0f) return q0 >= lo && q0 <= hi;
  float a = (lo - q0) / dq, b = (hi - q0) / dq;
  if (a > b) {
    float t = a;
    a = b;
    b = t;
  }
  a = fmaxf(a, (float)jlo) - 1.0f;
  b = fminf(b, (float)jhi) + 1.0f;
  jlo = max(jlo, (int)floorf(a));
  jhi = min(jhi, (int)ceilf(b));
  return jlo <= jhi;
}

struct DirF {
  float nx, ny, nz, a1x, a1y, a1z, a2x, a2y;
};

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
  return wrtd::exact_trilinear(R.vol, R.n, px, py, pz);
}

// kThreads: CTA size (one CTA per SM); kGroup: rows a warp walks together
// (32/kGroup lanes per row); kShiftsPerLane: shifts a lane enumerates per
// pass (a pass covers 32*kShiftsPerLane shifts).
template <int kThreads, int kGroup, int kShiftsPerLane>
__global__ void __launch_bounds__(kThreads, 1)
    plane_staged_kernel(const wrt::StagedReq *__restrict__ reqs,
                        const wrt::StagedItem *__restrict__ items, int nitems,
                        int *__restrict__ next_item, unsigned long long *__restrict__ counter) {
  constexpr int kLanesPerRow = 32 / kGroup;
  extern __shared__ float4 quads[];
  __shared__ int s_item, s_dir;
  const int tid = threadIdx.x, lane = tid & 31;
  unsigned long long evaluated = 0;
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
    const int n = R.n, W = n - 1;
    const int qp = R.qpitch;
    const int y0 = item.tile * R.tile_h;
    const int H = min(R.tile_h, W - y0);
    // ---- stage layer pair (iz, iz+1), quad rows y0 .. y0+H
    {
      const float2 *src = R.pairs + (size_t)item.layer * n * R.pitch2 + (size_t)y0 * R.pitch2;
      const int total = (H + 1) * W;
      for (int k = tid; k < total; k += kThreads) {
        const int yy = k / W, x = k - yy * W;
        const float2 *row = src + (size_t)yy * R.pitch2;
        const float2 a = __ldg(row + x), b = __ldg(row + x + 1);
        const float dz0 = a.y - a.x, dz1 = b.y - b.x;
        quads[yy * qp + x] = make_float4(a.x, dz0, b.x - a.x, dz1 - dz0);
      }
    }
    __syncthreads();
    const float h = 0.5f * (float)W;
    const float delta = 1.0f / (float)n;
    const float g = R.guard;
    const float halfband = 0.5f - g;
    const float wlo = item.layer == 0 ? -g : (float)item.layer;
    const float whi = item.layer == W - 1 ? (float)W + g : (float)(item.layer + 1);
    const float rc2 = R.crop_r2;
    const int L = R.L;
    for (;;) {
      int dl = 0;
      if (lane == 0) dl = atomicAdd(&s_dir, 1);
      dl = __shfl_sync(kFull, dl, 0);
      if (dl >= item.ndir) break;
      const int d = item.dir0 + dl;
      const float *Df = R.dir32 + 8 * (size_t)d;
      DirF D;
      D.nx = __ldg(Df + 0);
      D.ny = __ldg(Df + 1);
      D.nz = __ldg(Df + 2);
      D.a1x = __ldg(Df + 3) * delta;
      D.a1y = __ldg(Df + 4) * delta;
      D.a1z = __ldg(Df + 5) * delta;
      D.a2x = __ldg(Df + 6) * delta;
      D.a2y = __ldg(Df + 7) * delta;
      const float du = D.a2x * h, dv = D.a2y * h;
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
              const int im = (int)floorf(sqrtf(rem) / delta) + 1;
              cnt[k] = rows_in_layer(s, D.nz, D.a1z, h, wlo, whi, max(-L, -im), min(L - 1, im), &ia[k]);
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
          // ---- row set-up
          int jlo = 1, jhi = 0;
          float ub = 0.f, vb = 0.f, tz = 0.f;
          bool zexact = false;
          if (valid) {
            const float s = __ldg(R.shift32 + is);
            const float di = (float)i;
            const float w = row_w(s, D.nz, D.a1z, di, h);
            tz = w - (float)item.layer;
            zexact = fabsf(tz - 0.5f) > halfband;
            ub = (fmaf(di, D.a1x, s * D.nx) + 1.0f) * h;
            vb = (fmaf(di, D.a1y, s * D.ny) + 1.0f) * h;
            const float rem = rc2 - s * s - (delta * di) * (delta * di);
            if (rem >= 0.0f) {
              const int jm = (int)floorf(sqrtf(rem) / delta) + 1;
              jlo = max(-L, -jm);
              jhi = min(L - 1, jm);
              if (!clip_lin(ub, du, -1.0f, (float)n, jlo, jhi) ||
                  !clip_lin(vb, dv, (float)y0 - 1.0f, (float)(y0 + H) + 1.0f, jlo, jhi)) {
                jlo = 1;
                jhi = 0;
              }
            }
          }
          // ---- walk the rows in groups of kGroup, kLanesPerRow lanes per row,
          // consecutive samples on consecutive lanes of a row
          const int nrows = min(32, total - r0);
          for (int g0 = 0; g0 < nrows; g0 += kGroup) {
            const int rr = g0 + lane / kLanesPerRow, pos = lane % kLanesPerRow;
            const bool rvalid = rr < nrows;
            const int src = rvalid ? rr : 0;
            const int k_is = __shfl_sync(kFull, is, src), k_i = __shfl_sync(kFull, i, src);
            const int k_jlo = __shfl_sync(kFull, jlo, src);
            const int jhi_src = __shfl_sync(kFull, jhi, src);
            const int k_jhi = rvalid ? jhi_src : k_jlo - 1;
            const float k_ubm = __shfl_sync(kFull, ub, src) - 0.5f;  // q - 1/2 at j = 0
            const float k_vbm = __shfl_sync(kFull, vb, src) - 0.5f;
            const float k_tz = __shfl_sync(kFull, tz, src);
            const bool k_zx = __shfl_sync(kFull, (int)zexact, src) != 0;
            const int len = max(0, k_jhi - k_jlo + 1);
            const int trips = (int)__reduce_max_sync(kFull, (unsigned)((len + kLanesPerRow - 1) / kLanesPerRow));
            const float jhif = (float)k_jhi;
            float jf = (float)(k_jlo + pos);
            float part = 0.0f;
            double xacc = 0.0;  // guard-band samples, FP64
            for (int t = 0; t < trips; ++t, jf += (float)kLanesPerRow) {
              if (jf <= jhif) {
                // cell = round-to-nearest(q - 1/2) via the 1.5 * 2^23 shift (no
                // float-to-int conversion instructions); d = frac(q) - 1/2
                const float qx = fmaf(jf, du, k_ubm), qy = fmaf(jf, dv, k_vbm);
                const float sx = qx + kMagic, sy = qy + kMagic;
                const float fx = sx - kMagic, fy = sy - kMagic;
                const float dx = qx - fx, dy = qy - fy;
                const int ix = __float_as_int(sx) - kMagicBits;
                const int iy = __float_as_int(sy) - kMagicBits - y0;
                const bool band = k_zx | (fmaxf(fabsf(dx), fabsf(dy)) > halfband);
                if (!band) {
                  if ((unsigned)ix < (unsigned)W && (unsigned)iy < (unsigned)H) {
                    const float tx = dx + 0.5f, ty = dy + 0.5f;
                    const float4 *q = quads + iy * qp + ix;
                    const float4 a = q[0], b = q[qp];
                    const float va = fmaf(tx, fmaf(k_tz, a.w, a.z), fmaf(k_tz, a.y, a.x));
                    const float vb2 = fmaf(tx, fmaf(k_tz, b.w, b.z), fmaf(k_tz, b.y, b.x));
                    part += fmaf(ty, vb2 - va, va);
                    ++evaluated;
                  }
                } else {
                  // a guard-band sample belongs to the tile of its FP32 cell row,
                  // clamped to the grid (samples within the band outside a face
                  // are evaluated, and cut off, by the FP64 reference arithmetic)
                  const int cy = min(max(iy + y0, 0), W - 1) - y0;
                  if ((unsigned)cy < (unsigned)H) {
                    xacc += exact_sample(R, d, k_is, k_i, (int)jf);
                    ++evaluated;
                  }
                }
              }
            }
            // ---- fixed-point accumulation, segmented by plane over the warp
            // (rows are ordered by shift, so lanes of one plane are contiguous)
            const double row_acc = xacc + (double)part;
            long long v = rvalid ? __double2ll_rn(row_acc * R.scale) : 0LL;
            const int key = rvalid ? k_is : -1;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
              const long long tv = __shfl_up_sync(kFull, v, o);
              const int k2 = __shfl_up_sync(kFull, key, o);
              if (lane >= o && k2 == key) v += tv;
            }
            const int knext = __shfl_down_sync(kFull, key, 1);
            if (rvalid && (lane == 31 || knext != key) && v != 0)
              atomicAdd(R.acc + (size_t)k_is * R.ndir + d, (unsigned long long)v);
          }
        }
      }
    }
    __syncthreads();
  }
  if (counter) {
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
  int qp = W;
  while (qp % 8 != 3) ++qp;  // 16-byte words: rows offset by 3 bank groups
  const int budget = 200 * 1024;
  int rows_max = budget / (qp * 16);  // quad rows that fit
  if (rows_max < 3) return -1;
  int ntiles = (W + (rows_max - 1) - 1) / (rows_max - 1);
  int th = (W + ntiles - 1) / ntiles;  // balanced tiles of <= rows_max-1 cells
  *tile_h = th;
  *qpitch = qp;
  return (th + 1) * qp * 16;
}

namespace {
template <int T, int G, int K>
int launch_cfg(wrt_ctx *ctx, const StagedReq *d_reqs, const StagedItem *d_items, int nitems,
               int max_smem, int *d_next) {
  cudaError_t e = cudaFuncSetAttribute(plane_staged_kernel<T, G, K>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "staged kernel smem attribute");
  e = cudaMemsetAsync(d_next, 0, sizeof(int), ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "staged counter reset");
  plane_staged_kernel<T, G, K><<<ctx->sm_count, T, max_smem, ctx->stream>>>(
      d_reqs, d_items, nitems, d_next, ctx->d_counter);
  ctx->launches++;
  return check_launch(ctx, "plane_staged_kernel");
}
}  // namespace

// The tile shapes the autotuner chooses among: (CTA threads, rows per warp
// group, shifts per lane per enumeration pass).
const StagedConfig kStagedConfigs[] = {
    {512, 4, 4}, {512, 8, 4}, {512, 2, 4}, {640, 4, 2}, {768, 4, 2}, {768, 8, 2},
};
const int kNumStagedConfigs = sizeof(kStagedConfigs) / sizeof(kStagedConfigs[0]);

int plane_staged_launch(wrt_ctx *ctx, const StagedReq *d_reqs, const StagedItem *d_items,
                        int nitems, int max_smem, int *d_next) {
  const int c = (ctx->staged_config >= 0 && ctx->staged_config < kNumStagedConfigs)
                    ? ctx->staged_config : 0;
  switch (c) {
    case 0: return launch_cfg<512, 4, 4>(ctx, d_reqs, d_items, nitems, max_smem, d_next);
    case 1: return launch_cfg<512, 8, 4>(ctx, d_reqs, d_items, nitems, max_smem, d_next);
    case 2: return launch_cfg<512, 2, 4>(ctx, d_reqs, d_items, nitems, max_smem, d_next);
    case 3: return launch_cfg<640, 4, 2>(ctx, d_reqs, d_items, nitems, max_smem, d_next);
    case 4: return launch_cfg<768, 4, 2>(ctx, d_reqs, d_items, nitems, max_smem, d_next);
    default: return launch_cfg<768, 8, 2>(ctx, d_reqs, d_items, nitems, max_smem, d_next);
  }
}

int plane_finalize(wrt_ctx *ctx, double *out, long long count, double factor) {
  const int blocks = ctx->sm_count * 4;
  plane_finalize_kernel<<<blocks, 256, 0, ctx->stream>>>(out, count, factor);
  ctx->launches++;
  return check_launch(ctx, "plane_finalize_kernel");
}

// Work items of one request, largest estimated cost first.  Cost of a
// (layer, tile): voxels of the tile's slab inside the crop radius.
void staged_items(int req, int n, int tile_h, float crop_r2, int ndir, int dir_chunk,
                  std::vector<StagedItem> &out) {
  const int W = n - 1;
  const int ntiles = (W + tile_h - 1) / tile_h;
  const double h = 2.0 / (n - 1);
  struct C {
    double cost;
    StagedItem it;
  };
  std::vector<C> v;
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
        v.push_back({cost * it.ndir, it});
      }
    }
  }
  std::stable_sort(v.begin(), v.end(), [](const C &a, const C &b) { return a.cost > b.cost; });
  for (auto &c : v) out.push_back(c.it);
}

double fixed_point_scale(float maxabs, int L) {
  // |row sum| <= maxabs * 2L and |plane sum| <= maxabs * (2L)^2: scale so the
  // plane sum stays below 2^61 in magnitude
  if (!(maxabs > 0.0f) || !isfinite(maxabs)) return 1.0;
  const double bound = (double)maxabs * (2.0 * L + 1.0) * (2.0 * L + 1.0);
  const int k = (int)floor(log2(ldexp(1.0, 61) / bound));
  return ldexp(1.0, std::max(-200, std::min(200, k)));
}

namespace {
struct ItemList {
  StagedItem *d = nullptr;
  int count = 0;
  size_t bytes = 0;
};
struct StagedCache {
  std::map<std::tuple<int, int, unsigned, int>, ItemList> lists;
};
}  // namespace

int staged_items_cached(wrt_ctx *ctx, int n, int tile_h, float crop_r2, int ndir,
                        StagedItem **d_items, int *nitems) {
  if (!ctx->staged_cache) ctx->staged_cache = new StagedCache();
  StagedCache *c = static_cast<StagedCache *>(ctx->staged_cache);
  unsigned bits;
  memcpy(&bits, &crop_r2, sizeof(bits));
  const auto key = std::make_tuple(n, tile_h, bits, ndir);
  auto it = c->lists.find(key);
  if (it == c->lists.end()) {
    if (c->lists.size() > 64) {  // bounded: drop everything, rebuild on demand
      cudaStreamSynchronize(ctx->stream);
      for (auto &kv : c->lists) ctx_free(ctx, kv.second.d, kv.second.bytes);
      c->lists.clear();
    }
    std::vector<StagedItem> items;
    const int chunk = 512;  // directions per item
    staged_items(0, n, tile_h, crop_r2, ndir, chunk, items);
    ItemList l;
    l.count = (int)items.size();
    l.bytes = sizeof(StagedItem) * std::max<size_t>(1, items.size());
    int st = ctx_alloc(ctx, (void **)&l.d, l.bytes);
    if (st) return st;
    if (!items.empty()) {
      cudaError_t e = cudaMemcpy(l.d, items.data(), sizeof(StagedItem) * items.size(),
                                 cudaMemcpyHostToDevice);
      if (e != cudaSuccess) {
        ctx_free(ctx, l.d, l.bytes);
        return cuda_fail(ctx, e, "staged items");
      }
    }
    it = c->lists.emplace(key, l).first;
  }
  *d_items = it->second.d;
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
