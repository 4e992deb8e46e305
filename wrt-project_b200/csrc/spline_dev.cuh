// spline_dev.cuh -- device bodies shared by the single-request and the batched
// spline / adjoint kernels (k_spline.cu, batch.cu, k_noalloc.cu).
//
// Natural cubic spline in the shift variable over uniform knots s_i = -1 +
// i h, h = 2/(ns-1), end conditions M_0 = M_{ns-1} = 0: the reference builds
// one with GSL for every single evaluation (radon_reduction/slicing.c:45-61,
// radon_inversion/backprojection/C/src/interp.c:13-25); here a line's spline
// is built once and stored per knot interval as one float4, so an evaluation
// is one 16-byte load.  Two forms of the interval record:
//   reduction lines  (y_i, y_{i+1}, M_i, M_{i+1}):
//     S = a y_i + b y_{i+1} + ((a^3 - a) M_i + (b^3 - b) M_{i+1}) h^2 / 6,
//     b = (s - s_i)/h, a = 1 - b;
//   adjoint lines    (c0, c1, c2, c3), the same cubic in the centred variable
//     u = b - 1/2 in [-1/2, 1/2]:  S = c0 + u (c1 + u (c2 + u c3)),
//     coefficients formed in FP64 and rounded once.
#pragma once
#include <cuda_runtime.h>

namespace wrtd {

// Tridiagonal solve of one line (Thomas algorithm in FP64).  y(i) is element
// i of the line, read through y + i * se.  cp / den: the line-independent
// forward-elimination coefficients of M_{i-1} + 4 M_i + M_{i+1} = rhs_i.
__device__ __forceinline__ void spline_solve(const double *__restrict__ y, long long se, int ns,
                                             double h, const double *__restrict__ cp,
                                             const double *__restrict__ den,
                                             double *__restrict__ M) {
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
}

// Reduction lines: (y_i, y_{i+1}, M_i, M_{i+1}) per interval.
__device__ __forceinline__ void spline_line(const double *__restrict__ y, long long se, int ns,
                                            double h, const double *__restrict__ cp,
                                            const double *__restrict__ den,
                                            double *__restrict__ M, float4 *__restrict__ o) {
  spline_solve(y, se, ns, h, cp, den, M);
  for (int i = 0; i + 1 < ns; ++i)
    o[i] = make_float4((float)y[i * se], (float)y[(i + 1) * se], (float)M[i], (float)M[i + 1]);
}

// Adjoint lines: the centred power form of the spline of scale * y (scale is
// the direction's quadrature weight, multiplied in FP64 before rounding).
// With A = (y1 - y0) - h^2 (2 M0 + M1)/6, B = h^2 M0 / 2, C = h^2 (M1 - M0)/6
// the interval's cubic is y0 + A b + B b^2 + C b^3; substituting b = u + 1/2:
//   c0 = y0 + A/2 + B/4 + C/8, c1 = A + B + 3C/4, c2 = B + 3C/2, c3 = C.
__device__ __forceinline__ void spline_line_centred(const double *__restrict__ y, long long se,
                                                    int ns, double h,
                                                    const double *__restrict__ cp,
                                                    const double *__restrict__ den,
                                                    double *__restrict__ M,
                                                    float4 *__restrict__ o, double scale) {
  spline_solve(y, se, ns, h, cp, den, M);
  const double h2 = h * h;
  for (int i = 0; i + 1 < ns; ++i) {
    const double y0 = scale * y[i * se], y1 = scale * y[(i + 1) * se];
    const double m0 = scale * M[i], m1 = scale * M[i + 1];
    const double A = (y1 - y0) - h2 * (2.0 * m0 + m1) / 6.0;
    const double B = 0.5 * h2 * m0;
    const double C = h2 * (m1 - m0) / 6.0;
    o[i] = make_float4((float)(y0 + 0.5 * A + 0.25 * B + 0.125 * C),
                       (float)(A + B + 0.75 * C), (float)(B + 1.5 * C), (float)C);
  }
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

__device__ __forceinline__ float cubic_centred(const float4 c, float u) {
  return fmaf(u, fmaf(u, fmaf(u, c.w, c.z), c.y), c.x);
}

// ------------------------------------------------------------ backprojection
// radon_inversion/backprojection/C/src/integral.c:6-24, output order
// [iz][ix][iy] at cell centres (radon3d_ajoint.c:240-254):
//   R*g(x) = sum over directions d of dphi*w_theta * S_d(<x, omega_d>),
//   S_d = 0 beyond |s| > 1.
// The direction table holds g_d = (omega_d / h, dphi * w_theta) in FP64
// (h = 2/(ns-1)), so a voxel's knot position is q = <x, g_d> + 1/h and the
// interval record of knot floor(q) gives the value (the weight is folded into
// the adjoint lines).
//
// Work split: a warp owns a block of 8 (y) x 4 (z) voxel columns and V
// consecutive voxels along x in each (lane = one column, V voxels).  For one
// direction the 32 columns' knot positions lie within (7 |g_y| + 3 |g_z|) * 2/n
// knots of each other, so the warp's loads touch two or three 128-byte lines
// of the direction's spline; the V voxels of a lane step q by dq = (2/n) g_x.
//
// Per (lane, direction), in FP64: q0 = q - 1/2 of the lane's first voxel,
// split exactly into the integer i0 = rint(q0) and the FP32 remainder f0 in
// [-1/2, 1/2] (the 1.5 * 2^52 rounding constant), the same split of the
// per-voxel step dq = di + df, and the range of the V positions.  When all of
// them lie at least kAdjGuard knots inside [0, ns-1] (|s| < 1 with margin),
// each voxel costs FP32 work only: f = f0 + v df (|f| <= 2), k = rint(f) and
// u = f - k by the 1.5 * 2^23 rounding constant, the record at knot
// i0 + v di + k (in [0, ns-2] by the margin), and a Horner cubic in u.  The
// FP32 error of f is below 3e-7 knots.  A lane whose positions come within
// the guard band of |s| = 1, where S_d jumps to zero, evaluates that
// direction in FP64 per voxel with the exact range test; a lane entirely
// outside skips it.  Values are summed in FP32 over chunks of kAdjChunk
// directions and the chunk sums in FP64, in a fixed order: a voxel's result
// does not depend on how requests are batched.
constexpr int kAdjLanesY = 8, kAdjLanesZ = 4;
constexpr int kAdjChunk = 32;
constexpr double kAdjGuard = 1e-4;

// voxels per lane along x (4: 80 registers, three 256-thread blocks per SM;
// 8 voxels need 110 registers and halve the resident warps)
__host__ __device__ inline int adjoint_vox(int) { return 4; }

__host__ __device__ inline long long adjoint_warps(int n) {
  const int V = adjoint_vox(n);
  return (long long)((n + kAdjLanesY - 1) / kAdjLanesY) * ((n + kAdjLanesZ - 1) / kAdjLanesZ) *
         ((n + V - 1) / V);
}

template <int V>
__device__ __forceinline__ void adjoint_block_v(const float4 *__restrict__ lines, int ndir, int ns,
                                                const double4 *__restrict__ dirw, int n,
                                                long long w, int lane,
                                                double *__restrict__ out) {
  const int nby = (n + kAdjLanesY - 1) / kAdjLanesY, nbz = (n + kAdjLanesZ - 1) / kAdjLanesZ;
  const int by = (int)(w % nby);
  const long long r = w / nby;
  const int bz = (int)(r % nbz), ixg = (int)(r / nbz);
  const int iy = by * kAdjLanesY + lane % kAdjLanesY;
  const int iz = bz * kAdjLanesZ + lane / kAdjLanesY;
  const int ix0 = ixg * V;
  if (iy >= n || iz >= n) return;  // no warp-collective operations below
  // cell centres, radon3d_ajoint.c:248-250
  const double x0 = (-1.0) + (1.0 / n) + ix0 * (2.0 / n);
  const double y = (-1.0) + (1.0 / n) + iy * (2.0 / n);
  const double z = (-1.0) + (1.0 / n) + iz * (2.0 / n);
  const double qoff = 0.5 * (double)(ns - 1) - 0.5;  // 1/h - 1/2
  const double qmax = (double)(ns - 1);
  const double dx = 2.0 / n;
  const double fast_lo = kAdjGuard - 0.5, fast_hi = qmax - 0.5 - kAdjGuard;
  const double out_lo = -0.5 - kAdjGuard, out_hi = qmax - 0.5 + kAdjGuard;
  const size_t line_len = (size_t)(ns - 1);
  double tot[V];
#pragma unroll
  for (int v = 0; v < V; ++v) tot[v] = 0.0;
  for (int d0 = 0; d0 < ndir; d0 += kAdjChunk) {
    const int d1 = min(ndir, d0 + kAdjChunk);
    float acc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) acc[v] = 0.0f;
#pragma unroll 2
    for (int d = d0; d < d1; ++d) {
      const double2 gxy = __ldg(reinterpret_cast<const double2 *>(dirw + d));
      const double gz = __ldg(reinterpret_cast<const double *>(dirw + d) + 2);
      const double q0 = fma(x0, gxy.x, fma(y, gxy.y, fma(z, gz, qoff)));
      const double dq = dx * gxy.x;
      const double qe = fma((double)(V - 1), dq, q0);
      const double lo = fmin(q0, qe), hi = fmax(q0, qe);
      const float4 *line = lines + (size_t)d * line_len;
      if (lo > fast_lo && hi < fast_hi) {
        const double t64 = q0 + 6755399441055744.0;  // 1.5 * 2^52
        const int i0 = __double2loint(t64);           // rint(q0)
        const float f0 = (float)(q0 - (t64 - 6755399441055744.0));
        const double ts = dq + 6755399441055744.0;
        const int di = __double2loint(ts);            // rint(dq)
        const float dqf = (float)(dq - (ts - 6755399441055744.0));
        const float4 *base = line + (i0 - 0x4B400000);
#pragma unroll
        for (int v = 0; v < V; ++v) {
          // q - 1/2 = i0 + v di + f, |f| <= 1/2 + v/2
          const float f = fmaf((float)v, dqf, f0);
          const float t = f + 12582912.0f;  // 1.5 * 2^23: rint(f) in the low bits
          const float u = f - (t - 12582912.0f);
          const float4 c = __ldg(base + (__float_as_int(t) + v * di));
          acc[v] += cubic_centred(c, u);
        }
      } else if (hi >= out_lo && lo <= out_hi) {
#pragma unroll
        for (int v = 0; v < V; ++v) {
          const double q = fma((double)v, dq, q0) + 0.5;
          if (q >= 0.0 && q <= qmax) {  // |s| <= 1 (interp.c:9-11)
            const int i = min(__double2int_rz(q), ns - 2);
            const float u = (float)((q - (double)i) - 0.5);
            acc[v] += cubic_centred(__ldg(line + i), u);
          }
        }
      }
    }
#pragma unroll
    for (int v = 0; v < V; ++v) tot[v] += (double)acc[v];
  }
  const size_t o = ((size_t)iz * n + ix0) * n + iy;
#pragma unroll
  for (int v = 0; v < V; ++v)
    if (ix0 + v < n) out[o + (size_t)v * n] = tot[v];
}

// Warp w (0 <= w < adjoint_warps(n)) of an n^3 backprojection.
__device__ __forceinline__ void adjoint_block(const float4 *__restrict__ lines, int ndir, int ns,
                                              const double4 *__restrict__ dirw, int n,
                                              long long w, int lane, double *__restrict__ out) {
  adjoint_block_v<4>(lines, ndir, ns, dirw, n, w, lane, out);
}

}  // namespace wrtd
