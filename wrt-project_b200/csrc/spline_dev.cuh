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
#include <math.h>
#include <string.h>

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

// Value of reduction record c at fraction b of its knot interval.
__device__ __forceinline__ float spline_value(const float4 c, float b, float h2_6) {
  const float a = 1.0f - b;
  return fmaf(a, c.x, b * c.y) + ((a * a - 1.0f) * a * c.z + (b * b - 1.0f) * b * c.w) * h2_6;
}


__device__ __forceinline__ float cubic_centred(const float4 c, float u) {
  return fmaf(u, fmaf(u, fmaf(u, c.w, c.z), c.y), c.x);
}

// ------------------------------------------------------------ reduction
// The Radon sample that thread t of a reduction computes: threads run over
// the shifts fastest, so a warp's 32 samples share (iphi, itheta) and their
// slices lie side by side (neighbouring spline records of the same layers);
// the output keeps the reference's order (is, iphi, itheta).
__host__ __device__ inline long long reduction_sample_of(long long t, int nshift, int nphi,
                                                         int ntheta) {
  const long long is = t % nshift, r = t / nshift;
  const long long it = r % ntheta, ip = r / ntheta;
  return (is * nphi + ip) * ntheta + it;
}

// radon_reduction (radon_reduction/slicing.c:80-119) of Radon sample k
// (is, iphi, itheta), order of reduction.c:215-229, from the reduction lines
// [iz][iphi][ns_ray-1] of the ray data, by one thread: geometry in FP64 with
// the reference's expressions, spline values and the quadratic in z
// (slicing.c:62-74) in FP32, summed in FP64 in tau order.  No conversion
// instructions in the sample loop: the layer index and the knot interval are
// rounded by the 1.5 * 2^52 and 1.5 * 2^23 constants.  Returns the integral;
// *evaluated counts the slice samples taken.
__device__ __forceinline__ double reduction_one(const float4 *__restrict__ lines, int ngrid,
                                                int ns_ray, int nphi,
                                                const double *__restrict__ shift,
                                                const double *__restrict__ cs, int ntheta,
                                                long long k, int *evaluated_out) {
  const int it = (int)(k % ntheta), ip = (int)((k / ntheta) % nphi),
            is = (int)(k / ((long long)ntheta * nphi));
  const double p = shift[is], ct = cs[2 * it], st = cs[2 * it + 1];
  const double dtau = (2.0 / (ngrid - 1)) / (2.0);  // slicing.c:88
  const double delta_z = 2.0 / (ngrid - 1);         // slicing.c:18
  const double inv_dz = 0.5 * (ngrid - 1);
  const float hs = 2.0f / (float)(ns_ray - 1);
  const float inv_hs = 1.0f / hs;
  const float h2_6 = hs * hs / 6.0f;
  const float last = (float)(ns_ray - 2);
  constexpr double kMagic52 = 6755399441055744.0;  // 1.5 * 2^52
  constexpr float kMagic23 = 12582912.0f;          // 1.5 * 2^23
  const int half = 2 * ngrid;
  // |tau| <= sqrt(1 - p^2) bounds the samples that pass slicing.c:110
  int kmax = half;
  {
    double r = 1.0 - p * p;
    if (r < 0.0) kmax = -1;
    else kmax = min(half, (int)floor(sqrt(r) / dtau) + 1);
  }
  double acc = 0.0;
  int evaluated = 0;
  const size_t line_len = (size_t)(ns_ray - 1);
  const size_t layer = (size_t)nphi * line_len;
  for (int itau = -kmax; itau <= kmax; ++itau) {
    const double tau = __dmul_rn((double)itau, dtau);
    const double z = __dadd_rn(__dmul_rn(p, ct), __dmul_rn(tau, st));
    const double s = __dsub_rn(__dmul_rn(p, st), __dmul_rn(tau, ct));
    if ((fabs(__dadd_rn(__dmul_rn(tau, tau), __dmul_rn(p, p))) > 1.0) || (fabs(z) > 1.0) ||
        (fabs(s) > 1.0))
      continue;
    // layer index of slicing.c:15-20, (int)((z + 1) / delta_z): the
    // reciprocal's quotient qz >= 0 rounded by the 1.5 * 2^52 constant and
    // corrected down when below its rounding, and the division itself where
    // qz lies within 1e-9 of an integer (the reciprocal's error is ~1e-14)
    const double z1 = __dadd_rn(z, 1.0), qz = z1 * inv_dz;
    const double tq = qz + kMagic52;
    const double dq = qz - (tq - kMagic52);  // qz - round(qz), exact
    int iz = __double2loint(tq) - (dq < 0.0 ? 1 : 0);
    if (fabs(dq) < 1e-9) iz = (int)__ddiv_rn(z1, delta_z);
    if (iz == ngrid - 1) iz -= 1;
    const double z0 = __dadd_rn(-1.0, __dmul_rn(delta_z, (double)iz));
    const float f = (float)((z - z0) * inv_dz);
    // knot interval floor(q) clamped to the line and the fraction b, q = (s + 1)/h
    // in knot units (round(q - 1/2) = floor(q) but at the knots, where both
    // neighbouring intervals give the knot's value)
    const float q = (float)(s + 1.0) * inv_hs;
    const float fi = fminf(fmaxf(((q - 0.5f) + kMagic23) - kMagic23, 0.0f), last);
    const float b = q - fi;
    const float4 *rec = lines + ((size_t)iz * nphi + ip) * line_len +
                        (__float_as_int(fi + kMagic23) - 0x4B400000);
    const float4 c0 = __ldg(rec), c1 = __ldg(rec + layer);
    const float4 c2 = iz >= ngrid - 2 ? make_float4(0.f, 0.f, 0.f, 0.f) : __ldg(rec + 2 * layer);
    const float v0 = spline_value(c0, b, h2_6), v1 = spline_value(c1, b, h2_6);
    const float v2 = iz >= ngrid - 2 ? 0.0f : spline_value(c2, b, h2_6);
    // quadratic through (z0, v0), (z0+dz, v1), (z0+2dz, v2) at z0 + f dz
    const float val = v0 + f * (v1 - v0) + 0.5f * f * (f - 1.0f) * (v2 - 2.0f * v1 + v0);
    acc += (double)val;
    ++evaluated;
  }
  *evaluated_out = evaluated;
  return acc * dtau;
}

// ------------------------------------------------------------ backprojection
// radon_inversion/backprojection/C/src/integral.c:6-24, output order
// [iz][ix][iy] at cell centres (radon3d_ajoint.c:240-254):
//   R*g(x) = sum over directions d of dphi*w_theta * S_d(<x, omega_d>),
//   S_d = 0 beyond |s| > 1.
// With g_d = omega_d / h (h = 2/(ns-1)) a voxel's knot position is
// q = <x, g_d> + 1/h, and the interval record of knot floor(q) gives the
// value (the direction's weight is folded into its adjoint line).
//
// Direction constants reach the kernel through its parameter space (the
// constant bank, read once per warp) in launches of kAdjDirsPerLaunch
// directions: per direction g_d in FP64 and a header for the volume's edge n,
// so the L1 data path carries only the spline records.  The voxel sums are
// carried from launch to launch in the output buffer (FP64).
//
// Work split: a warp owns a block of 8 (y) x 4 (z) voxel columns and V
// consecutive voxels along x in each (lane = one column, V voxels).  For one
// direction the 32 columns' knot positions lie within (7 |g_y| + 3 |g_z|) * 2/n
// knots of each other, so the warp's loads touch two or three 128-byte lines
// of the direction's spline.
//
// Per (lane, direction), in FP64: q0 = q - 1/2 of the lane's first voxel and
// its exact split into the integer i0 = rint(q0) and the FP32 remainder f0 in
// [-1/2, 1/2] (1.5 * 2^52 rounding constant).  The per-voxel step
// dq = (2/n) g_x is split the same way on the host, dq = di + df.  Voxel v
// then has q - 1/2 = i0 + v di + f_v, f_v = f0 + v df, |f_v| <= V/2.  When
// i0 lies in the header's window [lo, lo + span] every one of the V positions
// is at least one knot inside [0, ns-1] (|s| < 1), and each voxel costs FP32
// work only, two voxels per packed f32x2 instruction: f_v, k = rint(f_v) and
// u = f_v - k by the 1.5 * 2^23 rounding constant, the record at knot
// i0 + v di + k (in [1, ns-3] by the window), a Horner cubic in u.  The FP32
// error of f_v is below 3e-7 knots.  Other lanes test the range exactly per
// voxel in FP64 (where S_d jumps to zero at |s| = 1), or skip the direction
// when the window shows every position outside.  Values are summed in FP32
// over chunks of kAdjChunk directions and the chunk sums in FP64, in a fixed
// order: a voxel's result does not depend on how requests are batched.
constexpr int kAdjLanesY = 8, kAdjLanesZ = 4;
constexpr int kAdjChunk = 32;
constexpr int kAdjDirsPerLaunch = 768;  // a multiple of kAdjChunk

struct AdjDirs {             // one launch's direction constants (30 KB of parameters)
  double g[kAdjDirsPerLaunch][3];  // omega / h
  int4 hd[kAdjDirsPerLaunch];      // float bits of df, di, lo, span
};

// voxels per lane along x: 8 from edge 192 up (fewer direction set-ups per
// evaluation), 4 below (more warps for smaller volumes)
__host__ __device__ inline int adjoint_vox(int n) { return n >= 192 ? 8 : 4; }

__host__ __device__ inline long long adjoint_warps(int n) {
  const int V = adjoint_vox(n);
  return (long long)((n + kAdjLanesY - 1) / kAdjLanesY) * ((n + kAdjLanesZ - 1) / kAdjLanesZ) *
         ((n + V - 1) / V);
}

// Header of direction g (x component gx) for edge n, ns shifts, V voxels:
// df, di, and the window [lo, lo + span] of i0 for which every position
// q_v - 1/2 = i0 + v di + f_v (|f_v| <= V/2) satisfies 1 <= q_v <= ns - 2.
inline void adjoint_header(double gx, int n, int ns, int V, int4 *hd) {
  const double dq = (2.0 / n) * gx;
  const double ts = dq + 6755399441055744.0;
  const long long di = llrint(ts - 6755399441055744.0);
  const float df = (float)(dq - (ts - 6755399441055744.0));
  const long long mn = di < 0 ? (V - 1) * di : 0, mx = di > 0 ? (V - 1) * di : 0;
  long long lo = V / 2 + 1 - mn, hi = (long long)ns - 3 - V / 2 - mx;
  int span = (int)(hi - lo);
  if (hi < lo) {  // no lane can take the FP32 path for this direction
    lo = 0x40000000;
    span = 0;
  }
  int dfb;
  memcpy(&dfb, &df, sizeof(dfb));
  *hd = make_int4(dfb, (int)di, (int)lo, span);
}

typedef unsigned long long adj_u64;
__device__ __forceinline__ adj_u64 adj_pk(float lo, float hi) {
  adj_u64 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void adj_upk(adj_u64 r, float &lo, float &hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(r));
}
__device__ __forceinline__ adj_u64 adj_fma2(adj_u64 a, adj_u64 b, adj_u64 c) {
  adj_u64 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ adj_u64 adj_add2(adj_u64 a, adj_u64 b) {
  adj_u64 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ adj_u64 adj_sub2(adj_u64 a, adj_u64 b) {
  adj_u64 d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

// Warp w (0 <= w < adjoint_warps(n)) over directions [dbeg, dbeg + nd) of an
// n^3 backprojection; lines[d] holds direction d's ns-1 records.
template <int V, int U = 1>
__device__ __forceinline__ void adjoint_block(const float4 *__restrict__ lines, int ns, int dbeg,
                                              int nd, const AdjDirs &dirs, int n, long long w,
                                              int lane, double *__restrict__ out) {
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
  const size_t line_len = (size_t)(ns - 1);
  const size_t o = ((size_t)iz * n + ix0) * n + iy;
  double tot[V];
#pragma unroll
  for (int v = 0; v < V; ++v) tot[v] = (dbeg == 0 || ix0 + v >= n) ? 0.0 : out[o + (size_t)v * n];
  const adj_u64 MM = adj_pk(12582912.0f, 12582912.0f);  // 1.5 * 2^23
  for (int j0 = 0; j0 < nd; j0 += kAdjChunk) {
    const int j1 = min(nd, j0 + kAdjChunk);
    float acc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) acc[v] = 0.0f;
#pragma unroll U
    for (int j = j0; j < j1; ++j) {
      const float4 *line = lines + (size_t)(dbeg + j) * line_len;
      const int4 hd = dirs.hd[j];
      const double q0 = fma(x0, dirs.g[j][0], fma(y, dirs.g[j][1], fma(z, dirs.g[j][2], qoff)));
      const double t64 = q0 + 6755399441055744.0;  // 1.5 * 2^52
      const int i0 = __double2loint(t64);           // rint(q0)
      if ((unsigned)(i0 - hd.z) <= (unsigned)hd.w) {
        const float f0 = (float)(q0 - (t64 - 6755399441055744.0));
        const float df = __int_as_float(hd.x);
        const int di = hd.y;
        const float4 *base = line + (i0 - 0x4B400000);
        const adj_u64 F0 = adj_pk(f0, f0), DF = adj_pk(df, df);
#pragma unroll
        for (int v = 0; v < V; v += 2) {
          const adj_u64 f = adj_fma2(adj_pk((float)v, (float)(v + 1)), DF, F0);
          const adj_u64 t = adj_add2(f, MM);
          const adj_u64 u = adj_sub2(f, adj_sub2(t, MM));
          float ta, tb, ua, ub;
          adj_upk(t, ta, tb);
          adj_upk(u, ua, ub);
          const float4 ca = __ldg(base + (__float_as_int(ta) + v * di));
          const float4 cb = __ldg(base + (__float_as_int(tb) + (v + 1) * di));
          acc[v] += cubic_centred(ca, ua);
          acc[v + 1] += cubic_centred(cb, ub);
        }
      } else {
        const int di = hd.y;
        const int mn = min(0, (V - 1) * di), mx = max(0, (V - 1) * di);
        // every position certainly outside [0, ns-1]: nothing to add
        if (!(i0 + mx <= -V / 2 - 1 || i0 + mn >= ns + V / 2 - 1)) {
          const double dq = dx * dirs.g[j][0];
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
    }
#pragma unroll
    for (int v = 0; v < V; ++v) tot[v] += (double)acc[v];
  }
#pragma unroll
  for (int v = 0; v < V; ++v)
    if (ix0 + v < n) out[o + (size_t)v * n] = tot[v];
}

}  // namespace wrtd
