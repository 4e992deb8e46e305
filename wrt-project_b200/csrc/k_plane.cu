// k_plane.cu -- plane integrals (radon_grid/src/integral.c:26-58), plain
// kernel, and its exact transpose.
//
// Plane (shift s, direction d) is the reference's lattice
//     p(i, j) = s*normal + delta*i*v1 + delta*j*v2,  delta = 1/n,  i, j in [-L, L)
// summed with weight delta^2 (L = 2n in the reference).  One warp per plane,
// one lattice row (fixed i) per lane.  Rows and row segments that cannot hold
// a non-zero sample are skipped:
//   * |p|^2 = s^2 + delta^2 (i^2 + j^2) > crop_r2  (the volume's non-zero
//     nodes all lie within sqrt(crop_r2) minus one cell diagonal);
//   * the sample is outside [-1,1]^3, where both samplers return 0.
// Both cuts drop only samples whose value is exactly 0.
//
// Numerics: FP32 cell coordinates with the guard band of wrt_internal.cuh;
// samples inside the band are re-evaluated with the reference's FP64
// arithmetic.  Sums: FP32 over chunks of 32 samples of one row, FP64 across
// chunks, rows and lanes; the FP64 total is scaled by delta^2 once.
#include "wrt_internal.cuh"

namespace {

struct RowGeom {
  double bx, by, bz;     // row base point (j = 0), reference arithmetic
  int jlo, jhi;          // samples to visit
};

// Conservative j-range with |b + t*j| <= 1 (+ tolerance); false if empty.
__device__ __forceinline__ bool clip_axis(double b, double t, int &lo, int &hi) {
  const double eps = 1e-13;
  if (t == 0.0) return fabs(b) <= 1.0 + eps;
  double k0 = (-1.0 - eps - b) / t, k1 = (1.0 + eps - b) / t;
  if (k0 > k1) {
    double s = k0;
    k0 = k1;
    k1 = s;
  }
  double flo = fmax(floor(k0) - 2.0, (double)lo), fhi = fmin(ceil(k1) + 2.0, (double)hi);
  if (!(flo <= fhi)) return false;
  lo = (int)flo;
  hi = (int)fhi;
  return true;
}

struct PlaneConsts {
  double snx, sny, snz;  // shift*normal
  double a1x, a1y, a1z;  // delta*v1
  double a2x, a2y, a2z;  // delta*v2
  double delta, rem;     // rem = crop_r2 - s^2
};

__device__ __forceinline__ PlaneConsts plane_consts(const wrt::PlaneJob &job, int is, int d) {
  const double *D = job.dir + 9 * (size_t)d;
  const double s = job.shift[is];
  PlaneConsts c;
  c.delta = 1.0 / job.n;  // integral.c:38
  c.snx = __dmul_rn(s, D[0]);
  c.sny = __dmul_rn(s, D[1]);
  c.snz = __dmul_rn(s, D[2]);
  c.a1x = __dmul_rn(c.delta, D[3]);
  c.a1y = __dmul_rn(c.delta, D[4]);
  c.a1z = __dmul_rn(c.delta, D[5]);
  c.a2x = __dmul_rn(c.delta, D[6]);
  c.a2y = __dmul_rn(c.delta, D[7]);
  c.a2z = __dmul_rn(c.delta, D[8]);
  // every sample farther than sqrt(r2) + margin from the origin has only
  // zero corners; nothing outside radius sqrt(3) is inside the cube
  double crop_r2 = 3.0 + 1e-9;
  if (job.r2bits) {
    const double r = sqrt((double)__uint_as_float(__ldg(job.r2bits))) + job.margin;
    crop_r2 = fmin(r * r, crop_r2);
  }
  c.rem = crop_r2 - s * s;
  return c;
}

__device__ __forceinline__ bool row_geom(const PlaneConsts &c, int L, int i, RowGeom &r) {
  const double di = (double)i;
  r.bx = __dadd_rn(c.snx, __dmul_rn(c.a1x, di));
  r.by = __dadd_rn(c.sny, __dmul_rn(c.a1y, di));
  r.bz = __dadd_rn(c.snz, __dmul_rn(c.a1z, di));
  double remj = c.rem - (c.delta * di) * (c.delta * di);
  if (remj < 0.0) return false;
  int jm = (int)floor(sqrt(remj) / c.delta) + 1;
  r.jlo = max(-L, -jm);
  r.jhi = min(L - 1, jm);
  if (r.jlo > r.jhi) return false;
  if (!clip_axis(r.bx, c.a2x, r.jlo, r.jhi)) return false;
  if (!clip_axis(r.by, c.a2y, r.jlo, r.jhi)) return false;
  if (!clip_axis(r.bz, c.a2z, r.jlo, r.jhi)) return false;
  return true;
}

__device__ __forceinline__ void row_range(const PlaneConsts &c, int L, int &ilo, int &ihi) {
  int im = (int)floor(sqrt(fmax(c.rem, 0.0)) / c.delta) + 1;
  ilo = max(-L, -im);
  ihi = min(L - 1, im);
}

template <int SAMPLER>
__global__ void __launch_bounds__(256) plane_plain_kernel(wrt::PlaneJob job, float guard) {
  const int lane = threadIdx.x & 31;
  const long long plane = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (plane >= (long long)job.ndir * job.nshift) return;
  const int is = (int)(plane / job.ndir), d = (int)(plane % job.ndir);
  const int n = job.n;
  const PlaneConsts c = plane_consts(job, is, d);
  double acc = 0.0;
  int evaluated = 0;
  if (c.rem >= 0.0) {
    // cells per unit length of the sampler's grid
    const double h = SAMPLER == WRT_SAMPLER_TRILINEAR ? 0.5 * (n - 1) : 0.5 * n;
    const float du = (float)(c.a2x * h), dv = (float)(c.a2y * h), dw = (float)(c.a2z * h);
    const float qmax = SAMPLER == WRT_SAMPLER_TRILINEAR ? (float)(n - 1) : (float)n;
    int ilo, ihi;
    row_range(c, job.L, ilo, ihi);
    for (int i = ilo + lane; i <= ihi; i += 32) {
      RowGeom r;
      if (!row_geom(c, job.L, i, r)) continue;
      const float ub = (float)((r.bx + 1.0) * h), vb = (float)((r.by + 1.0) * h),
                  wb = (float)((r.bz + 1.0) * h);
      for (int j0 = r.jlo; j0 <= r.jhi; j0 += 32) {
        const int j1 = min(r.jhi, j0 + 31);
        float part = 0.0f;
        for (int j = j0; j <= j1; ++j) {
          const float jf = (float)j;
          const float qx = fmaf(jf, du, ub), qy = fmaf(jf, dv, vb), qz = fmaf(jf, dw, wb);
          if (wrtd::in_band(qx, guard) | wrtd::in_band(qy, guard) | wrtd::in_band(qz, guard)) {
            const double dj = (double)j;
            const double px = __dadd_rn(r.bx, __dmul_rn(c.a2x, dj));
            const double py = __dadd_rn(r.by, __dmul_rn(c.a2y, dj));
            const double pz = __dadd_rn(r.bz, __dmul_rn(c.a2z, dj));
            acc += SAMPLER == WRT_SAMPLER_TRILINEAR ? wrtd::exact_trilinear(job.vol, n, px, py, pz)
                                                    : wrtd::exact_nearest(job.vol, n, px, py, pz);
            ++evaluated;
          } else if (qx > 0.0f && qy > 0.0f && qz > 0.0f && qx < qmax && qy < qmax &&
                     qz < qmax) {
            ++evaluated;
            if (SAMPLER == WRT_SAMPLER_TRILINEAR) {
              part += wrtd::tri32(job.vol, n, qx, qy, qz);
            } else {
              part += wrtd::ldv(job.vol, n, (int)qx, (int)qy, (int)qz);
            }
          }
        }
        acc += (double)part;
      }
    }
  }
  acc = wrtd::warp_sum(acc);
  if (lane == 0) job.out[plane] = acc * c.delta * c.delta;
  if (job.counter) {
    for (int o = 16; o > 0; o >>= 1) evaluated += __shfl_xor_sync(0xffffffffu, evaluated, o);
    if (lane == 0) atomicAdd(job.counter, (unsigned long long)evaluated);
  }
}

// layers[iz][iy][ix] = v[ix][iy][iz] (the staged nearest sampler's cell layers)
__global__ void volume_layers_kernel(const float *__restrict__ v, int n,
                                     float *__restrict__ layers) {
  const size_t total = (size_t)n * n * n;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total;
       k += (size_t)gridDim.x * blockDim.x) {
    const int ix = (int)(k % n), iy = (int)((k / n) % n), iz = (int)(k / ((size_t)n * n));
    layers[k] = v[((size_t)ix * n + iy) * n + iz];
  }
}

// Exact transpose: every sample of every plane scatters g[plane] * delta^2 *
// (its sampling weights) into an FP64 volume.  Weights follow the forward
// kernel sample by sample (FP32 fractions outside the band, the reference's
// FP64 fractions inside it).
__device__ __forceinline__ void scatter_tri(double *acc, int n, int ix, int iy, int iz, double tx,
                                            double ty, double tz, double g) {
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int e = 0; e < 2; ++e) {
        double wgt = (a ? tx : 1.0 - tx) * (b ? ty : 1.0 - ty) * (e ? tz : 1.0 - tz);
        atomicAdd(acc + ((size_t)(ix + a) * n + (iy + b)) * n + (iz + e), g * wgt);
      }
}

template <int SAMPLER>
__global__ void __launch_bounds__(256) plane_transpose_kernel(wrt::PlaneJob job, float guard,
                                                              const double *__restrict__ g,
                                                              double *__restrict__ vol64) {
  const int lane = threadIdx.x & 31;
  const long long plane = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (plane >= (long long)job.ndir * job.nshift) return;
  const int is = (int)(plane / job.ndir), d = (int)(plane % job.ndir);
  const int n = job.n;
  const PlaneConsts c = plane_consts(job, is, d);
  if (c.rem < 0.0) return;
  const double gw = g[plane] * c.delta * c.delta;
  if (gw == 0.0) return;
  const double h = SAMPLER == WRT_SAMPLER_TRILINEAR ? 0.5 * (n - 1) : 0.5 * n;
  const float du = (float)(c.a2x * h), dv = (float)(c.a2y * h), dw = (float)(c.a2z * h);
  const float qmax = SAMPLER == WRT_SAMPLER_TRILINEAR ? (float)(n - 1) : (float)n;
  int ilo, ihi;
  row_range(c, job.L, ilo, ihi);
  for (int i = ilo + lane; i <= ihi; i += 32) {
    RowGeom r;
    if (!row_geom(c, job.L, i, r)) continue;
    const float ub = (float)((r.bx + 1.0) * h), vb = (float)((r.by + 1.0) * h),
                wb = (float)((r.bz + 1.0) * h);
    for (int j = r.jlo; j <= r.jhi; ++j) {
      const float jf = (float)j;
      const float qx = fmaf(jf, du, ub), qy = fmaf(jf, dv, vb), qz = fmaf(jf, dw, wb);
      if (wrtd::in_band(qx, guard) | wrtd::in_band(qy, guard) | wrtd::in_band(qz, guard)) {
        const double dj = (double)j;
        const double x = __dadd_rn(r.bx, __dmul_rn(c.a2x, dj));
        const double y = __dadd_rn(r.by, __dmul_rn(c.a2y, dj));
        const double z = __dadd_rn(r.bz, __dmul_rn(c.a2z, dj));
        if ((fabs(x) > 1.0) || (fabs(y) > 1.0) || (fabs(z) > 1.0)) continue;
        if (SAMPLER == WRT_SAMPLER_TRILINEAR) {
          const double delta = __ddiv_rn(2.0, (double)(n - 1));
          const double x1 = __dadd_rn(x, 1.0), y1 = __dadd_rn(y, 1.0), z1 = __dadd_rn(z, 1.0);
          int ix = (int)__ddiv_rn(x1, delta), iy = (int)__ddiv_rn(y1, delta),
              iz = (int)__ddiv_rn(z1, delta);
          double cx = __ddiv_rn(fmod(x1, delta), delta), cy = __ddiv_rn(fmod(y1, delta), delta),
                 cz = __ddiv_rn(fmod(z1, delta), delta);
          if (ix == n - 1) { ix -= 1; cx = 1.0; }
          if (iy == n - 1) { iy -= 1; cy = 1.0; }
          if (iz == n - 1) { iz -= 1; cz = 1.0; }
          scatter_tri(vol64, n, ix, iy, iz, cx, cy, cz, gw);
        } else {
          const double delta = __ddiv_rn(2.0, (double)n);
          int ix = (int)__ddiv_rn(__dadd_rn(x, 1.0), delta),
              iy = (int)__ddiv_rn(__dadd_rn(y, 1.0), delta),
              iz = (int)__ddiv_rn(__dadd_rn(z, 1.0), delta);
          if (ix == n) ix -= 1;
          if (iy == n) iy -= 1;
          if (iz == n) iz -= 1;
          atomicAdd(vol64 + ((size_t)ix * n + iy) * n + iz, gw);
        }
      } else if (qx > 0.0f && qy > 0.0f && qz > 0.0f && qx < qmax && qy < qmax && qz < qmax) {
        const float fx = floorf(qx), fy = floorf(qy), fz = floorf(qz);
        if (SAMPLER == WRT_SAMPLER_TRILINEAR) {
          scatter_tri(vol64, n, (int)fx, (int)fy, (int)fz, qx - fx, qy - fy, qz - fz, gw);
        } else {
          atomicAdd(vol64 + ((size_t)(int)fx * n + (int)fy) * n + (int)fz, gw);
        }
      }
    }
  }
}

}  // namespace

namespace wrt {

static float guard_band(int n) { return 4.8e-7f * (float)(n > 64 ? n : 64); }

int volume_layers(wrt_ctx *ctx, const float *d_vol, int n, float *d_layers) {
  volume_layers_kernel<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(d_vol, n, d_layers);
  ctx->launches++;
  return check_launch(ctx, "volume_layers_kernel");
}

int plane_forward_plain(wrt_ctx *ctx, const PlaneJob &job) {
  const long long nplanes = (long long)job.ndir * job.nshift;
  if (nplanes == 0) return WRT_OK;
  const int threads = 256;
  const long long blocks = (nplanes + 7) / 8;
  if (blocks > 0x7fffffffLL) return fail(ctx, WRT_ERR_INVALID_ARGUMENT, "too many planes");
  const float g = guard_band(job.n);
  if (job.sampler == WRT_SAMPLER_TRILINEAR)
    plane_plain_kernel<WRT_SAMPLER_TRILINEAR><<<(unsigned)blocks, threads, 0, ctx->stream>>>(job, g);
  else
    plane_plain_kernel<WRT_SAMPLER_NEAREST><<<(unsigned)blocks, threads, 0, ctx->stream>>>(job, g);
  ctx->launches++;
  return check_launch(ctx, "plane_plain_kernel");
}

int plane_transpose(wrt_ctx *ctx, const PlaneJob &job, const double *d_g, double *d_vol64) {
  const long long nplanes = (long long)job.ndir * job.nshift;
  if (nplanes == 0) return WRT_OK;
  const long long blocks = (nplanes + 7) / 8;
  const float g = guard_band(job.n);
  if (job.sampler == WRT_SAMPLER_TRILINEAR)
    plane_transpose_kernel<WRT_SAMPLER_TRILINEAR><<<(unsigned)blocks, 256, 0, ctx->stream>>>(
        job, g, d_g, d_vol64);
  else
    plane_transpose_kernel<WRT_SAMPLER_NEAREST><<<(unsigned)blocks, 256, 0, ctx->stream>>>(
        job, g, d_g, d_vol64);
  ctx->launches++;
  return check_launch(ctx, "plane_transpose_kernel");
}

}  // namespace wrt
