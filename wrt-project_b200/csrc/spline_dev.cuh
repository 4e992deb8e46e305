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
__device__ __forceinline__ void spline_line(const double *__restrict__ y, long long se, int ns,
                                            double h, const double *__restrict__ cp,
                                            const double *__restrict__ den,
                                            double *__restrict__ M, float4 *__restrict__ o) {
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
    o[i] = make_float4((float)y[i * se], (float)y[(i + 1) * se], (float)M[i], (float)M[i + 1]);
}

// The same at a knot position q given in FP64 (fraction taken in FP64, then
// rounded once): for rough data the spline is steep, and an FP32 position
// error of 1e-7 * (ns - 1) knots would move the value by that much times the
// slope.
__device__ __forceinline__ float spline_eval_q64(const float4 *__restrict__ line, int ns,
                                                 double q, float h2_6) {
  double fi = floor(q);
  fi = fmin(fmax(fi, 0.0), (double)(ns - 2));
  const float b = (float)(q - fi), a = 1.0f - b;
  const float4 c = __ldg(line + (int)fi);
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

// Backprojection of one voxel k (output order [iz][ix][iy], cell centres,
// radon_inversion/backprojection/C/src/radon3d_ajoint.c:240-254):
//   sum over directions d of dphi*w_theta * S_d(<x, omega_d>), S_d = 0 beyond |s| > 1
// (backprojection/C/src/integral.c:6-24).  The plane coordinate s = <x, omega>
// and its knot position are FP64 (dirw holds the reference's FP64 omega); the
// spline value and the weighted sum are FP32, compensated (Kahan) per latitude
// ring, FP64 over rings: Radon data of mixed signs cancel strongly in this
// sum, and a plain FP32 accumulator would lose up to ~1e-5 of the result.
__device__ __forceinline__ double adjoint_voxel(const float4 *__restrict__ lines, int ndir,
                                                int ntheta, int ns,
                                                const double4 *__restrict__ dirw, int n,
                                                long long k) {
  const int iy = (int)(k % n), ix = (int)((k / n) % n), iz = (int)(k / ((long long)n * n));
  const double x = (-1.0) + (1.0 / n) + ix * (2.0 / n);
  const double y = (-1.0) + (1.0 / n) + iy * (2.0 / n);
  const double z = (-1.0) + (1.0 / n) + iz * (2.0 / n);
  const float hs = 2.0f / (float)(ns - 1);
  const double inv_hs = 0.5 * (double)(ns - 1);
  const float h2_6 = hs * hs / 6.0f;
  const size_t line_len = (size_t)(ns - 1);
  double acc = 0.0;
  for (int d0 = 0; d0 < ndir; d0 += ntheta) {
    float part = 0.0f, comp = 0.0f;  // running sum and its lost low-order part
    const int d1 = min(ndir, d0 + ntheta);
    for (int d = d0; d < d1; ++d) {
      const double2 w01 = __ldg(reinterpret_cast<const double2 *>(dirw + d));
      const double2 w23 = __ldg(reinterpret_cast<const double2 *>(dirw + d) + 1);
      const double4 w = make_double4(w01.x, w01.y, w23.x, w23.y);
      const double s = fma(x, w.x, fma(y, w.y, z * w.z));
      if (fabs(s) <= 1.0) {
        const float term = __fmul_rn(
            (float)w.w, spline_eval_q64(lines + d * line_len, ns, fma(s, inv_hs, inv_hs), h2_6));
        const float yk = __fsub_rn(term, comp);
        const float t = __fadd_rn(part, yk);
        comp = __fsub_rn(__fsub_rn(t, part), yk);
        part = t;
      }
    }
    acc += (double)part - (double)comp;
  }
  return acc;
}

}  // namespace wrtd
