// k_grid.cu -- the Gauss-uniform sphere grid.
//
// Latitude nodes: n-point Gauss-Legendre rule in FP64 on the GPU, Newton's
// method on P_n with the three-term recurrence, replacing
// gsl_integration_glfixed_* at radon_grid/src/init.c:180-187 (and the same
// call in radon_reduction/init.c:213-220 and backprojection/C/src/init.c:
// 238-245).  This file is compiled with -fmad=false and uses only IEEE basic
// operations, in a fixed order, so the nodes are bit-identical to those of the
// host-side generator that the tests use as the oracle.
//
// Directions: theta = acos(node), phi = 2 pi k / nphi, and the plane basis
// normal / v1 / v2 are evaluated on the host with libm in the reference's own
// expression order (radon_grid/src/init.c:165-189, integral.c:10-36), so the
// FP64 lattice points the kernels re-evaluate in their guard band are the
// reference's points to the last bit.
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <vector>

#include "wrt_internal.cuh"

namespace {

__host__ __device__ double series_cos(double a) {
  double a2 = a * a, term = 1.0, sum = 1.0;
  for (int k = 1; k <= 30; ++k) {
    double den = (double)((2 * k - 1) * (2 * k));
    term = ((-term) * a2) / den;
    sum = sum + term;
  }
  return sum;
}

__host__ __device__ void legendre_pair(int n, double x, double *pn, double *pnm1) {
  double p0 = 1.0, p1 = x;
  if (n == 0) {
    *pn = 1.0;
    *pnm1 = 0.0;
    return;
  }
  for (int k = 1; k < n; ++k) {
    double kd = (double)k;
    double a = 2.0 * kd + 1.0;
    double t = (a * x) * p1;
    double num = t - kd * p0;
    double p2 = num / (kd + 1.0);
    p0 = p1;
    p1 = p2;
  }
  *pn = p1;
  *pnm1 = p0;
}

__host__ __device__ double legendre_deriv(int n, double r, double pn, double pnm1) {
  double num = (double)n * (r * pn - pnm1);
  double den = r * r - 1.0;
  return num / den;
}

// Root k (1 <= k <= n/2) and its weight; k = n/2 + 1 for odd n: the middle
// node.  Writes the mirrored pair into x / w (ascending order).
__host__ __device__ void gl_root(int n, int k, double *x, double *w) {
  const int m = n / 2;
  if (k <= m) {
    double ang = (WRT_PI * ((double)k - 0.25)) / ((double)n + 0.5);
    double r = series_cos(ang);
    double pn, pnm1, dp;
    for (int it = 0; it < 100; ++it) {
      legendre_pair(n, r, &pn, &pnm1);
      dp = legendre_deriv(n, r, pn, pnm1);
      double dr = pn / dp;
      r = r - dr;
      if (fabs(dr) <= 1e-16 * fabs(r)) break;
    }
    legendre_pair(n, r, &pn, &pnm1);
    dp = legendre_deriv(n, r, pn, pnm1);
    double wk = 2.0 / (((1.0 - r * r) * dp) * dp);
    x[k - 1] = -r;
    w[k - 1] = wk;
    x[n - k] = r;
    w[n - k] = wk;
  } else if (k == m + 1 && (n & 1)) {
    double pn, pnm1;
    legendre_pair(n, 0.0, &pn, &pnm1);
    double dp = legendre_deriv(n, 0.0, pn, pnm1);
    x[m] = 0.0;
    w[m] = 2.0 / ((1.0 * dp) * dp);
  }
}

// One thread per positive root (k = 1..n/2) plus one for the middle node.
__global__ void gl_nodes_kernel(int n, double *x, double *w) {
  gl_root(n, blockIdx.x * blockDim.x + threadIdx.x + 1, x, w);
}

}  // namespace

namespace wrt {

int gauss_legendre_device(wrt_ctx *ctx, int n, double *x_host, double *w_host) {
  if (n < 1 || n > 1 << 20) return fail(ctx, WRT_ERR_INVALID_ARGUMENT, "gauss_legendre: n=%d", n);
  double *d = nullptr;
  int st = ctx_alloc(ctx, (void **)&d, sizeof(double) * 2 * (size_t)n);
  if (st) return st;
  int threads = 128, blocks = (n / 2 + 1 + threads - 1) / threads;
  gl_nodes_kernel<<<blocks, threads, 0, ctx->stream>>>(n, d, d + n);
  ctx->launches++;
  st = check_launch(ctx, "gl_nodes_kernel");
  if (!st) {
    cudaError_t e = cudaMemcpyAsync(x_host, d, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(w_host, d + n, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) st = cuda_fail(ctx, e, "gauss_legendre copy");
  }
  ctx_free(ctx, d, sizeof(double) * 2 * (size_t)n);
  return st;
}

int sphere_grid(wrt_ctx *ctx, int nphi, int ntheta, int nshift, double *phi, double *theta,
                double *theta_w, double *shift) {
  if (nphi < 1 || ntheta < 1 || nshift < 2)
    return fail(ctx, WRT_ERR_INVALID_ARGUMENT, "sphere grid: nphi=%d ntheta=%d nshift=%d", nphi,
                ntheta, nshift);
  // radon_grid/src/init.c:167-176
  const double dphi = (2 * M_PI) / nphi;
  for (int i = 0; i < nphi; ++i) phi[i] = dphi * i;
  const double dshift = 2.0 / (nshift - 1);
  for (int i = 0; i < nshift; ++i) shift[i] = (-1.0) + i * dshift;
  std::vector<double> x(ntheta), w(ntheta);
  int st = gauss_legendre_device(ctx, ntheta, x.data(), w.data());
  if (st) return st;
  for (int i = 0; i < ntheta; ++i) {
    theta[i] = acos(x[i]);  // radon_grid/src/init.c:184
    if (theta_w) theta_w[i] = w[i];
  }
  return WRT_OK;
}

// The same rule on the host (the host compiler emits no fused multiply-add
// here, so the nodes are those of gl_nodes_kernel bit for bit); used where a
// caller's path may not allocate device memory.
void gauss_legendre_host(int n, double *x, double *w) {
  for (int k = 1; k <= n / 2 + 1; ++k) gl_root(n, k, x, w);
}

// Backprojection direction table: dirw[ip*ntheta + it] = (omega / h,
// dphi * w_theta) with omega = (sin t cos p, sin t sin p, cos t) in the
// reference's expression order (backprojection/C/src/integral.c:11-18) and
// h = 2/(nshift-1), so that <x, omega>/h + 1/h is a voxel's knot position.
void adjoint_directions(int nphi, int ntheta, int nshift, const double *phi, const double *theta,
                        const double *theta_w, double4 *dirw) {
  const double dphi = 2 * M_PI / nphi;
  const double inv_h = 0.5 * (double)(nshift - 1);
  for (int ip = 0; ip < nphi; ++ip)
    for (int it = 0; it < ntheta; ++it)
      dirw[(size_t)ip * ntheta + it] =
          make_double4(sin(theta[it]) * cos(phi[ip]) * inv_h, sin(theta[it]) * sin(phi[ip]) * inv_h,
                       cos(theta[it]) * inv_h, dphi * theta_w[it]);
}

// radon_grid/src/integral.c:10-36: normal = omega(phi, theta),
// v1 = omega(phi, theta + pi/2), v2 = normal x v1.
void plane_directions(int nphi, const double *phi, int ntheta, const double *theta,
                      double *dir9) {
  for (int ip = 0; ip < nphi; ++ip) {
    for (int it = 0; it < ntheta; ++it) {
      double *D = dir9 + 9 * ((size_t)ip * ntheta + it);
      const double p = phi[ip], t = theta[it];
      double nx = sin(t) * cos(p), ny = sin(t) * sin(p), nz = cos(t);
      double t2 = t + M_PI / 2;
      double ax = sin(t2) * cos(p), ay = sin(t2) * sin(p), az = cos(t2);
      D[0] = nx;
      D[1] = ny;
      D[2] = nz;
      D[3] = ax;
      D[4] = ay;
      D[5] = az;
      D[6] = ny * az - nz * ay;
      D[7] = -(nx * az - nz * ax);
      D[8] = nx * ay - ny * ax;
    }
  }
}

}  // namespace wrt
