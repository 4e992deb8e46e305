// spline_dev.cuh -- device bodies shared by the single-request and the batched
// spline / adjoint kernels (k_spline.cu, batch.cu).
//
// Natural cubic spline in the shift variable over uniform knots s_i = -1 +
// i h, h = 2/(ns-1), end conditions M_0 = M_{ns-1} = 0: the reference builds
// one with GSL for every single evaluation (radon_reduction/slicing.c:45-61,
// radon_inversion/backprojection/C/src/interp.c:13-25); here a line's spline
// is built once and stored per knot interval as the float4
// (y_i, y_{i+1}, M_i, M_{i+1}), so an evaluation is one 16-byte load and
//   S(s) = a y_i + b y_{i+1} + ((a^3 - a) M_i + (b^3 - b) M_{i+1}) h^2 / 6,
//   b = (s - s_i)/h, a = 1 - b.
#pragma once
#include <cuda_runtime.h>

namespace wrtd {

// Tridiagonal solve of one line (Thomas algorithm in FP64).  y(i) is element
// i of the line, read through y + i * se.  cp / den: the line-independent
// forward-elimination coefficients of M_{i-1} + 4 M_i + M_{i+1} = rhs_i.
// scale: a weight the stored values and curvatures are multiplied by in FP64
// before their rounding to FP32 (the spline of scale * y; 1 for plain lines).
__device__ __forceinline__ void spline_line(const double *__restrict__ y, long long se, int ns,
                                            double h, const double *__restrict__ cp,
                                            const double *__restrict__ den,
                                            double *__restrict__ M, float4 *__restrict__ o,
                                            double scale = 1.0) {
  M[0] = 0.0;
  M[ns - 1] = 0.0;
  const double six_h2 = 6.0 / (h * h);
  double prev = 0.0;
  for (int i = 1; i + 1 < ns; ++i) {
    const double rhs = six_h2 * (y[(i + 1) * se] - 2.0 * y[i * se] + y[(i - 1) * se]);
    const double dpi = (rhs - (i > 1 ? prev : 0.0)) / den[i];
    M[i] = dpi;
    prev = dpi;
  }
  for (int i = ns - 3; i >= 1; --i) M[i] = M[i] - cp[i] * M[i + 1];
  for (int i = 0; i + 1 < ns; ++i)
    o[i] = make_float4((float)(scale * y[i * se]), (float)(scale * y[(i + 1) * se]),
                       (float)(scale * M[i]), (float)(scale * M[i + 1]));
}

// The same at a knot position q given in FP64, 0 <= q <= ns - 1 (the
// caller's range test): fraction taken in FP64, then rounded once.  For rough
// data the spline is steep, and an FP32 position error of 1e-7 * (ns - 1)
// knots would move the value by that much times the slope.
__device__ __forceinline__ float spline_eval_q64(const float4 *__restrict__ line, int ns,
                                                 double q, float h2_6) {
  const int i = min(__double2int_rz(q), ns - 2);  // floor (q >= 0); q = ns - 1: b = 1
  const float b = (float)(q - (double)i), a = 1.0f - b;
  const float4 c = __ldg(line + i);
  return fmaf(a, c.x, b * c.y) + ((a * a - 1.0f) * a * c.z + (b * b - 1.0f) * b * c.w) * h2_6;
}

__device__ __forceinline__ float spline_eval(const float4 *__restrict__ line, int ns, float q,
                                             float h2_6) {
  // q = (s + 1)/h in knot units
  float fi = floorf(q);
  fi = fminf(fmaxf(fi, 0.0f), (float)(ns - 2));
  const float b = q - fi, a = 1.0f - b;
  const float4 c = __ldg(line + (int)fi);
  return fmaf(a, c.x, b * c.y) + ((a * a - 1.0f) * a * c.z + (b * b - 1.0f) * b * c.w) * h2_6;
}

// Backprojection (radon_inversion/backprojection/C/src/integral.c:6-24,
// output order [iz][ix][iy] at cell centres, radon3d_ajoint.c:240-254):
//   R*g(x) = sum over directions d of dphi*w_theta * S_d(<x, omega_d>), S_d = 0
//   beyond |s| > 1.
// One thread takes kAdjVoxels voxels along x, (iz, ix0 + v, iy): per direction
// it reads dirw once and steps the knot position q = (s + 1)/h from voxel to
// voxel by one FP64 add, q and its fraction in FP64 (dirw holds the
// reference's FP64 omega; a few FP64 roundings from the direct dot product,
// 1e-14 knots at most), the spline value in FP32 (each direction's weight is
// folded into its line's values and curvatures in FP64 when the line is
// built), the sum over directions in FP64.  |s| <= 1 is tested as
// 0 <= q <= ns - 1.  Threads of a warp take consecutive iy: one direction's
// 32 lanes read neighbouring knot intervals of one line.
constexpr int kAdjVoxels = 4;

// thread items of an n^3 adjoint: (iz, ix group, iy), iy fastest
__host__ __device__ inline long long adjoint_items(int n) {
  return (long long)n * n * ((n + kAdjVoxels - 1) / kAdjVoxels);
}

__device__ __forceinline__ void adjoint_item(const float4 *__restrict__ lines, int ndir, int ns,
                                             const double4 *__restrict__ dirw, int n,
                                             long long t, double *__restrict__ out) {
  const int ngx = (n + kAdjVoxels - 1) / kAdjVoxels;
  const int iy = (int)(t % n), ix0 = (int)((t / n) % ngx) * kAdjVoxels,
            iz = (int)(t / ((long long)n * ngx));
  const double x0 = (-1.0) + (1.0 / n) + ix0 * (2.0 / n);
  const double y = (-1.0) + (1.0 / n) + iy * (2.0 / n);
  const double z = (-1.0) + (1.0 / n) + iz * (2.0 / n);
  const float hs = 2.0f / (float)(ns - 1);
  const double inv_hs = 0.5 * (double)(ns - 1), qmax = (double)(ns - 1);
  const double qdx = (2.0 / n) * inv_hs;  // knot step per voxel along x, per unit omega_x
  const float h2_6 = hs * hs / 6.0f;
  const size_t line_len = (size_t)(ns - 1);
  double acc[kAdjVoxels];
#pragma unroll
  for (int v = 0; v < kAdjVoxels; ++v) acc[v] = 0.0;
#pragma unroll 4
  for (int d = 0; d < ndir; ++d) {
    const double2 w01 = __ldg(reinterpret_cast<const double2 *>(dirw + d));
    const double2 w23 = __ldg(reinterpret_cast<const double2 *>(dirw + d) + 1);
    const double q0 = fma(fma(x0, w01.x, fma(y, w01.y, z * w23.x)), inv_hs, inv_hs);
    const double qs = qdx * w01.x;
    const float4 *line = lines + d * line_len;
#pragma unroll
    for (int v = 0; v < kAdjVoxels; ++v) {
      const double q = fma((double)v, qs, q0);
      if (q >= 0.0 && q <= qmax)
        acc[v] += (double)spline_eval_q64(line, ns, q, h2_6);  // line holds w_d * S_d
    }
  }
  const size_t base = ((size_t)iz * n + ix0) * n + iy;
#pragma unroll
  for (int v = 0; v < kAdjVoxels; ++v)
    if (ix0 + v < n) out[base + (size_t)v * n] = acc[v];
}

}  // namespace wrtd
