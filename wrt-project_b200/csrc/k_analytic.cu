// k_analytic.cu -- plane and ray integrals of analytic test functions
// (radon_analytic/src/integral.c:25-57, ray_analytic/integral.c:10-48), the
// reference's programs that integrate a compiled-in function instead of a
// sampled volume.  The function families are those of the reference's
// example files, with their constants as parameters:
//   exponential bump (radon_analytic/examples-test-functions/exponential_bump.c)
//     f = exp(-1 / (R2 - |x - c|^2)) where |x - c|^2 < R2 - eps, else 0;
//   sine bumps (.../sinusoidal_bump.c): a sum of balls, each
//     amplitude                         for r < rin,
//     amplitude/(20 pi) (-sin 6t / 3 + 3 sin 4t - 15 sin 2t + 20 t),
//       t = pi (r - rout)/(rout - rin)  for rin < r < rout,
//     0                                 otherwise (r = |x - c|).
// Lattices as the reference's: plane points s n + delta (i v1 + j v2), i, j in
// [-2n, 2n), ray points (s cos phi, s sin phi, z) + delta k (cos(phi + pi/2),
// sin(phi + pi/2), 0), k in [-2n, 2n], delta = 1/(n - 1), weights delta^2 and
// delta.
//
// Each term of the function vanishes outside its ball, so a plane integral is
// the sum over balls of the lattice points inside the ball's disk on the
// plane (a ray: inside its chord); only those points are visited.  Values are
// FP32; a point whose FP32 squared radius lies within a guard band of a
// discontinuity (rin^2, rout^2, R2 - eps) is re-evaluated with the
// reference's FP64 expressions.  Sums: FP32 per lattice row, FP64 across rows,
// one warp per plane (deterministic order).
#include <string.h>

#include <vector>

#include "wrt_internal.cuh"

namespace {

constexpr int kMaxBalls = WRT_FUNCTION_MAX_BALLS;

struct Ball {                  // one term of the function
  double c[3];                 // centre
  double rho2;                 // squared support radius (rout^2, or R2 - eps)
  double amp, rin, rout, R2;   // the reference's constants (FP64 evaluation)
  float famp, frin, frout, fR2, flim;  // the same in FP32
};
struct Func {
  int kind, count;
  Ball b[kMaxBalls];
};

constexpr float kBand = 2e-6f;  // guard band on squared radii (FP32 error ~1e-7)

// FP64 value of term k at point p, the reference's expressions.
__device__ double term64(const Func &F, int k, double x, double y, double z) {
  const Ball &B = F.b[k];
  const double dx = x - B.c[0], dy = y - B.c[1], dz = z - B.c[2];
  if (F.kind == WRT_FUNCTION_EXP_BUMP) {
    const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
    return r2 < B.rho2 ? exp(-1.0 / (__dsub_rn(__dsub_rn(__dsub_rn(B.R2, __dmul_rn(dx, dx)),
                                                          __dmul_rn(dy, dy)),
                                                __dmul_rn(dz, dz))))
                       : 0.0;
  }
  const double r = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
  const double rin = B.rin, rout = B.rout, amp = B.amp;
  if (r > rout) return 0.0;
  if (r < rout && r > rin) {
    const double t = WRT_PI * (r - rout) / (rout - rin);
    return (amp / (20 * WRT_PI)) * (-sin(6 * t) / 3 + 3 * sin(4 * t) - 15 * sin(2 * t) + 20 * t);
  }
  if (r < rin) return amp;
  return 0.0;
}

// FP32 value of term k at offset q from its centre (squared radius r2);
// *band when the point needs the FP64 evaluation instead.
__device__ __forceinline__ float term32(const Func &F, int k, float r2, bool *band) {
  const Ball &B = F.b[k];
  if (F.kind == WRT_FUNCTION_EXP_BUMP) {
    *band = fabsf(r2 - B.flim) < kBand;
    return r2 < B.flim ? expf(-1.0f / (B.fR2 - r2)) : 0.0f;
  }
  const float rin2 = B.frin * B.frin, rout2 = B.frout * B.frout;
  *band = (fabsf(r2 - rin2) < kBand) | (fabsf(r2 - rout2) < kBand);
  if (r2 >= rout2) return 0.0f;
  if (r2 <= rin2) return B.famp;
  const float r = sqrtf(r2);
  const float t = (float)WRT_PI * (r - B.frout) / (B.frout - B.frin);
  // sin 4t and sin 6t from sin 2t and cos 2t (double- and triple-angle identities)
  float s2, c2;
  sincosf(2.0f * t, &s2, &c2);
  const float s4 = 2.0f * s2 * c2, s6 = s2 * (3.0f - 4.0f * s2 * s2);
  return (B.famp / (20.0f * (float)WRT_PI)) * (-s6 / 3.0f + 3.0f * s4 - 15.0f * s2 + 20.0f * t);
}

// Plane integrals: one warp per plane (order [is][iphi][itheta]); per ball,
// the lattice rows crossing the ball's disk, 32 consecutive j per lane pass.
__global__ void __launch_bounds__(256) analytic_plane_kernel(Func F, int n, const double *dir,
                                                             const double *shift, int ndir,
                                                             int nshift, double *out) {
  const long long nplanes = (long long)ndir * nshift;
  const int lane = threadIdx.x & 31;
  const double delta = (2.0 / (n - 1)) / 2.0;  // integral.c:38
  const int half = 2 * n;
  for (long long pl = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / 32; pl < nplanes;
       pl += (long long)gridDim.x * blockDim.x / 32) {
    const int d = (int)(pl % ndir);
    const double s = shift[pl / ndir];
    const double *D = dir + 9 * (size_t)d;  // normal, v1, v2 (integral.c:26-36)
    double total = 0.0;
    for (int k = 0; k < F.count; ++k) {
      const Ball &B = F.b[k];
      // centre relative to the plane's origin s n, in lattice units
      const double ox = s * D[0] - B.c[0], oy = s * D[1] - B.c[1], oz = s * D[2] - B.c[2];
      const double dist = -(ox * D[0] + oy * D[1] + oz * D[2]);
      const double r2 = (B.rho2 - dist * dist) / (delta * delta);
      if (r2 < 0.0) continue;
      const double a1 = -(ox * D[3] + oy * D[4] + oz * D[5]) / delta;
      const double a2 = -(ox * D[6] + oy * D[7] + oz * D[8]) / delta;
      const double rr = sqrt(r2) + 1.0;
      const int ilo = max(-half, (int)floor(a1 - rr)), ihi = min(half - 1, (int)ceil(a1 + rr));
      const float ex = (float)(delta * D[6]), ey = (float)(delta * D[7]), ez = (float)(delta * D[8]);
      for (int i = ilo; i <= ihi; ++i) {
        const double w2 = rr * rr - (i - a1) * (i - a1);
        if (w2 < 0.0) continue;
        const double w = sqrt(w2);
        const int jlo = max(-half, (int)floor(a2 - w)), jhi = min(half - 1, (int)ceil(a2 + w));
        // offset from the centre at j = 0 of this row
        const float bx = (float)(ox + delta * D[3] * i), by = (float)(oy + delta * D[4] * i),
                    bz = (float)(oz + delta * D[5] * i);
        float part = 0.0f;
        for (int j = jlo + lane; j <= jhi; j += 32) {
          const float jf = (float)j;
          const float qx = fmaf(jf, ex, bx), qy = fmaf(jf, ey, by), qz = fmaf(jf, ez, bz);
          const float q2 = fmaf(qx, qx, fmaf(qy, qy, qz * qz));
          bool band = false;
          const float v = term32(F, k, q2, &band);
          if (band) {
            // integral.c:44-47, FP64 in the reference's order
            const double px = __dadd_rn(__dadd_rn(__dmul_rn(s, D[0]), __dmul_rn(__dmul_rn(delta, D[3]), (double)i)),
                                        __dmul_rn(__dmul_rn(delta, D[6]), (double)j));
            const double py = __dadd_rn(__dadd_rn(__dmul_rn(s, D[1]), __dmul_rn(__dmul_rn(delta, D[4]), (double)i)),
                                        __dmul_rn(__dmul_rn(delta, D[7]), (double)j));
            const double pz = __dadd_rn(__dadd_rn(__dmul_rn(s, D[2]), __dmul_rn(__dmul_rn(delta, D[5]), (double)i)),
                                        __dmul_rn(__dmul_rn(delta, D[8]), (double)j));
            total += term64(F, k, px, py, pz);  // lane-local; summed over the warp below
          } else {
            part += v;
          }
        }
        total += (double)part;
      }
    }
    total = wrtd::warp_sum(total);
    if (lane == 0) out[pl] = total * delta * delta;
  }
}

// Ray integrals: one thread per ray, order [iz][is][iphi] (ray_analytic.c:254-272).
__global__ void __launch_bounds__(256) analytic_ray_kernel(Func F, int n, const double *tab,
                                                           int nshift, int nphi, double *out) {
  const long long nrays = (long long)n * nshift * nphi;
  const double delta = (2.0 / (n - 1)) / 2.0;  // integral.c:29
  const int half = 2 * n;
  for (long long ray = blockIdx.x * (long long)blockDim.x + threadIdx.x; ray < nrays;
       ray += (long long)gridDim.x * blockDim.x) {
    const int ip = (int)(ray % nphi), is = (int)((ray / nphi) % nshift),
              iz = (int)(ray / ((long long)nphi * nshift));
    const double z = (-1.0) + iz * 2.0 / (n - 1);  // ray_analytic.c:255
    const double s = tab[is];
    const double *T = tab + nshift + 4 * (size_t)ip;  // cos phi, sin phi, cos, sin (phi + pi/2)
    const double o[3] = {s * T[0], s * T[1], z};
    double total = 0.0;
    for (int k = 0; k < F.count; ++k) {
      const Ball &B = F.b[k];
      const double ox = o[0] - B.c[0], oy = o[1] - B.c[1], oz = o[2] - B.c[2];
      const double kc = -(ox * T[2] + oy * T[3]) / delta;  // closest point, in steps
      const double p2 = ox * ox + oy * oy + oz * oz - (kc * delta) * (kc * delta);
      const double w2 = (B.rho2 - p2) / (delta * delta);
      if (w2 < 0.0) continue;
      const double w = sqrt(w2) + 1.0;
      const int klo = max(-half, (int)floor(kc - w)), khi = min(half, (int)ceil(kc + w));
      const float bx = (float)ox, by = (float)oy, bz = (float)oz;
      const float ex = (float)(delta * T[2]), ey = (float)(delta * T[3]);
      float part = 0.0f;
      for (int kk = klo; kk <= khi; ++kk) {
        const float qx = fmaf((float)kk, ex, bx), qy = fmaf((float)kk, ey, by);
        const float q2 = fmaf(qx, qx, fmaf(qy, qy, bz * bz));
        bool band = false;
        const float v = term32(F, k, q2, &band);
        if (band) {
          // integral.c:37-40, FP64 in the reference's order
          const double px = __dadd_rn(o[0], __dmul_rn(__dmul_rn(delta, T[2]), (double)kk));
          const double py = __dadd_rn(o[1], __dmul_rn(__dmul_rn(delta, T[3]), (double)kk));
          const double pz = __dadd_rn(o[2], __dmul_rn(__dmul_rn(delta, 0.0), (double)kk));
          total += term64(F, k, px, py, pz);
        } else {
          part += v;
        }
      }
      total += (double)part;
    }
    out[ray] = total * delta;
  }
}

int make_func(wrt_ctx *ctx, const wrt_function *f, Func *F) {
  memset(F, 0, sizeof(*F));
  F->kind = f->kind;
  if (f->kind == WRT_FUNCTION_EXP_BUMP) {
    const double R2 = f->p[3], eps = f->p[4];
    if (!(R2 > 0.0) || !(eps >= 0.0) || !(R2 - eps > 0.0))
      return wrt::fail(ctx, WRT_ERR_INVALID_ARGUMENT, "exponential bump: need R2 > eps >= 0");
    F->count = 1;
    Ball &B = F->b[0];
    for (int a = 0; a < 3; ++a) B.c[a] = f->p[a];
    B.rho2 = R2 - eps;  // exponential_bump.c:11, (0.5 - eps)
    B.R2 = R2;
    B.fR2 = (float)R2;
    B.flim = (float)B.rho2;
    return WRT_OK;
  }
  if (f->kind != WRT_FUNCTION_SINE_BUMPS || f->count < 1 || f->count > kMaxBalls)
    return wrt::fail(ctx, WRT_ERR_INVALID_ARGUMENT, "analytic function: bad kind or ball count");
  F->count = f->count;
  for (int k = 0; k < f->count; ++k) {
    const double *q = f->p + 6 * k;
    if (!(q[4] >= 0.0) || !(q[5] > q[4]))
      return wrt::fail(ctx, WRT_ERR_INVALID_ARGUMENT, "sine bump %d: need 0 <= rin < rout", k);
    Ball &B = F->b[k];
    for (int a = 0; a < 3; ++a) B.c[a] = q[a];
    B.amp = q[3];
    B.rin = q[4];
    B.rout = q[5];
    B.famp = (float)q[3];
    B.frin = (float)q[4];
    B.frout = (float)q[5];
    B.rho2 = q[5] * q[5] * (1.0 + 1e-12);  // the term vanishes beyond rout
  }
  return WRT_OK;
}

}  // namespace

extern "C" {

int wrt_radon_analytic(wrt_ctx *ctx, const wrt_function *f, int ngrid, int nphi, int ntheta,
                       int nshift, double *out) {
  if (!ctx || !f || !out || ngrid < 2 || ngrid > 8192 || nphi < 1 || ntheta < 1 || nshift < 2)
    return ctx ? wrt::fail(ctx, WRT_ERR_INVALID_ARGUMENT, "radon_analytic: bad arguments")
               : WRT_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return wrt::cuda_fail(ctx, e, "cudaSetDevice");
  Func F;
  int st = make_func(ctx, f, &F);
  if (st) return st;
  wrt_grid *grid = nullptr;
  st = wrt_grid_create(ctx, nphi, ntheta, nshift, &grid);
  if (st) return st;
  const size_t nout = (size_t)nphi * ntheta * nshift;
  void *dout = nullptr;
  st = wrt::ws_get(ctx, wrt::WS_OUT, sizeof(double) * nout, &dout);
  if (!st) {
    const double *d_dir = nullptr, *d_shift = nullptr;
    wrt::grid_tables(grid, &d_dir, &d_shift);
    analytic_plane_kernel<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(
        F, ngrid, d_dir, d_shift, nphi * ntheta, nshift, static_cast<double *>(dout));
    ctx->launches++;
    st = wrt::check_launch(ctx, "analytic_plane_kernel");
  }
  if (!st) {
    e = cudaMemcpyAsync(out, dout, sizeof(double) * nout, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) st = wrt::cuda_fail(ctx, e, "radon_analytic result");
  }
  wrt_grid_destroy(grid);
  return st;
}

int wrt_ray_analytic(wrt_ctx *ctx, const wrt_function *f, int ngrid, int nshift, int nphi,
                     double *out) {
  if (!ctx || !f || !out || ngrid < 2 || ngrid > 8192 || nphi < 1 || nshift < 2)
    return ctx ? wrt::fail(ctx, WRT_ERR_INVALID_ARGUMENT, "ray_analytic: bad arguments")
               : WRT_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return wrt::cuda_fail(ctx, e, "cudaSetDevice");
  Func F;
  int st = make_func(ctx, f, &F);
  if (st) return st;
  std::vector<double> tab((size_t)nshift + 4 * (size_t)nphi);
  wrt::ray_tables(nshift, nphi, tab.data());  // ray_analytic/init.c:85-101, integral.c:14-22
  const size_t nout = (size_t)ngrid * nshift * nphi;
  void *dtab = nullptr, *dout = nullptr;
  st = wrt::ws_get(ctx, wrt::WS_TABLE, sizeof(double) * tab.size(), &dtab);
  if (!st) st = wrt::ws_get(ctx, wrt::WS_OUT, sizeof(double) * nout, &dout);
  if (st) return st;
  e = cudaMemcpyAsync(dtab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice,
                      ctx->stream);
  if (e != cudaSuccess) return wrt::cuda_fail(ctx, e, "ray_analytic tables");
  analytic_ray_kernel<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(
      F, ngrid, static_cast<const double *>(dtab), nshift, nphi, static_cast<double *>(dout));
  ctx->launches++;
  st = wrt::check_launch(ctx, "analytic_ray_kernel");
  if (st) return st;
  e = cudaMemcpyAsync(out, dout, sizeof(double) * nout, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? WRT_OK : wrt::cuda_fail(ctx, e, "ray_analytic result");
}

}  // extern "C"
