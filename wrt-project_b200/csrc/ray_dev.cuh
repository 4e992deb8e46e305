// ray_dev.cuh -- the device body of the layer-by-layer ray integral
// (ray_grid/src/integral.c:11-50), shared by the single-request kernel
// (k_ray.cu) and the batched one (batch.cu).
//
// Ray (z, s, phi): p(k) = (s cos phi, s sin phi, z) + delta*k*(cos(phi+pi/2),
// sin(phi+pi/2), 0), delta = 1/(n-1), k in [-2n, 2n], weight delta, trilinear
// sampler.  With a frame F every point is mapped to F p(k) (the layer scheme
// about another axis; F = identity reproduces the reference).
//
// One lane per ray; the kernels choose which rays share a warp (k_ray.cu: a
// tile of consecutive shifts x consecutive angles of one layer).  Samples
// farther than sqrt(crop_r2) from the origin or outside the cube are skipped
// (their value is exactly 0).  Numerics: FP32 cell coordinates with the guard
// band of wrt_internal.cuh.  In the reference frame the z coordinate of a ray
// is one FP64 number for all its samples, so its cell and fraction are
// computed once per ray with the reference's own arithmetic
// (cube_trilinear_interp, radon_grid/src/interp.c:33-53) and used by every
// FP32 sample of the ray.
#pragma once
#include "wrt_internal.cuh"

namespace wrtd {

// Guard band (cells) of the ray kernels' FP32 cell coordinates.
__host__ __device__ inline float ray_guard(int n) { return 4.8e-7f * (float)(n > 64 ? n : 64); }


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

__device__ __forceinline__ double rot_row(const double *F, int r, double x, double y, double z) {
  return __dadd_rn(__dadd_rn(__dmul_rn(F[3 * r], x), __dmul_rn(F[3 * r + 1], y)),
                   __dmul_rn(F[3 * r + 2], z));
}

// The octet of cell c as one 32-byte load (one L1 request per sample instead
// of two on the same sector); octet arrays come from cudaMalloc, so oct + 2c
// is 32-byte aligned as the vector load requires.
__device__ __forceinline__ void ld_octet(const float4 *oct, size_t c, float4 &lo, float4 &hi) {
  asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(lo.x), "=f"(lo.y), "=f"(lo.z), "=f"(lo.w), "=f"(hi.x), "=f"(hi.y), "=f"(hi.z),
        "=f"(hi.w)
      : "l"(oct + 2 * c));
}

// Trilinear value from a cell octet (lo: x side, hi: x+1 side, each
// (v(y,z), v(y,z+1), v(y+1,z), v(y+1,z+1))): x, then y, then z, the order of
// wrtd::tri32.
__device__ __forceinline__ float octet_lerp(float4 lo, float4 hi, float tx, float ty, float tz) {
  // (a0, b0) = lerp_x of (v(x,y,z), v(x,y,z+1)); (a1, b1) of the y+1 pair
  const float a0 = lerp32(tx, lo.x, hi.x), b0 = lerp32(tx, lo.y, hi.y);
  const float a1 = lerp32(tx, lo.z, hi.z), b1 = lerp32(tx, lo.w, hi.w);
  const float e0 = lerp32(ty, a0, a1), e1 = lerp32(ty, b0, b1);
  return lerp32(tz, e0, e1);
}

constexpr float kRayMagic = 12582912.0f;  // 1.5 * 2^23
constexpr unsigned kRayMagicBits = 0x4B400000u;

// A sample's cell: bits of round(q') + 1.5 * 2^23 per axis (q' = the FP32
// cell coordinate minus 1/2, so round(q') = floor of the coordinate outside
// the guard band), the fractions t = q' - round(q') + 1/2, whether the
// coordinate lies within the guard band of a cell boundary, and whether the
// cell is inside the node grid.
struct RayCell {
  unsigned bx, by, bz;
  float tx, ty, tz;
  bool band, in;
};

// Ray number `ray` (0 <= ray < nslices * nshift * nphi, shift fastest) of a job.
template <bool FRAME>
__device__ __forceinline__ void ray_one(const wrt::RayJob &job, long long ray, float guard) {
  const int is = (int)(ray % job.nshift);
  const int ip = (int)((ray / job.nshift) % job.nphi);
  const int iz = (int)(ray / ((long long)job.nphi * job.nshift));
  const int n = job.n;
  const double *T = job.trig + 4 * ip;
  const double s = job.shift[is];
  const double dz = 2.0 / (job.nslices - 1);                     // ray_grid.c:244
  const double zslice = __dadd_rn(-1.0, __dmul_rn((double)iz, dz));  // ray_grid.c:247
  const double delta = (2.0 / (n - 1)) / (2.0);                  // integral.c:32
  const double p0x = __dmul_rn(s, T[0]), p0y = __dmul_rn(s, T[1]), p0z = zslice;
  const double ax = __dmul_rn(delta, T[2]), ay = __dmul_rn(delta, T[3]);  // delta*direction
  double acc = 0.0;

  double crop_r2 = 3.0 + 1e-9;
  if (job.r2bits) {
    const double r = sqrt((double)__uint_as_float(__ldg(job.r2bits))) + job.margin;
    crop_r2 = fmin(r * r, crop_r2);
  }
  const double rem = crop_r2 - s * s - zslice * zslice;
  const int half = 2 * n;  // nsize/2 with nsize = 4n
  int klo = -half, khi = half;
  bool any = rem >= 0.0;
  if (any) {
    int km = (int)floor(sqrt(rem) / delta) + 1;
    klo = max(klo, -km);
    khi = min(khi, km);
    any = klo <= khi;
  }
  const double h = 0.5 * (n - 1);
  const double *F = job.frame;  // kernel parameter space
  if (any && !FRAME) {
    any = clip_axis(p0x, ax, klo, khi) && clip_axis(p0y, ay, klo, khi) && fabs(zslice) <= 1.0;
  } else if (any) {
    double bx = rot_row(F, 0, p0x, p0y, p0z), by = rot_row(F, 1, p0x, p0y, p0z),
           bz = rot_row(F, 2, p0x, p0y, p0z);
    double tx = F[0] * ax + F[1] * ay, ty = F[3] * ax + F[4] * ay, tz = F[6] * ax + F[7] * ay;
    any = clip_axis(bx, tx, klo, khi) && clip_axis(by, ty, klo, khi) && clip_axis(bz, tz, klo, khi);
  }
  if (any) {
    float ub, vb, wb, du, dv, dw;
    int zc = 0;
    float tzc = 0.0f;
    if (!FRAME) {
      ub = (float)((p0x + 1.0) * h);
      vb = (float)((p0y + 1.0) * h);
      du = (float)(ax * h);
      dv = (float)(ay * h);
      wb = 0.0f;
      dw = 0.0f;
      // z cell of the whole ray, reference arithmetic (interp.c:32-53)
      const double dlt = 2.0 / (n - 1);
      const double z1 = __dadd_rn(zslice, 1.0);
      zc = (int)__ddiv_rn(z1, dlt);
      double cz = __ddiv_rn(fmod(z1, dlt), dlt);
      if (zc == n - 1) {
        zc -= 1;
        cz = 1.0;
      }
      tzc = (float)cz;
    } else {
      const double bx = rot_row(F, 0, p0x, p0y, p0z), by = rot_row(F, 1, p0x, p0y, p0z),
                   bz = rot_row(F, 2, p0x, p0y, p0z);
      ub = (float)((bx + 1.0) * h);
      vb = (float)((by + 1.0) * h);
      wb = (float)((bz + 1.0) * h);
      du = (float)((F[0] * ax + F[1] * ay) * h);
      dv = (float)((F[3] * ax + F[4] * ay) * h);
      dw = (float)((F[6] * ax + F[7] * ay) * h);
    }
    // FP64 reference evaluation of sample k (interp.c:25-60 at F p(k))
    auto exact_at = [&](int k) {
      const double dk = (double)k;
      double px = __dadd_rn(p0x, __dmul_rn(ax, dk));
      double py = __dadd_rn(p0y, __dmul_rn(ay, dk));
      double pz = __dadd_rn(p0z, __dmul_rn(__dmul_rn(delta, 0.0), dk));
      if (FRAME) {
        const double wx = rot_row(F, 0, px, py, pz), wy = rot_row(F, 1, px, py, pz),
                     wz = rot_row(F, 2, px, py, pz);
        px = wx;
        py = wy;
        pz = wz;
      }
      return wrtd::exact_trilinear(job.vol, n, px, py, pz);
    };
    // Every path locates a sample the same way and interpolates its 8
    // corners in one order (octet_lerp: x, then y, then z), whether the
    // corners come from the cell octets, the layer pairs or the volume, so a
    // ray's value does not depend on which of them the job carries.
    // q' = q - 1/2 at k = 0 (one more rounding of at most half an ulp, well
    // inside the guard band's allowance for the FP32 coordinates)
    ub -= 0.5f;
    vb -= 0.5f;
    wb -= 0.5f;
    const float halfband = 0.5f - guard;
    const unsigned mb = kRayMagicBits, um = (unsigned)(n - 1);
    auto locate = [&](int k) {
      RayCell c;
      const float kf = (float)k;
      const float qx = fmaf(kf, du, ub), qy = fmaf(kf, dv, vb);
      const float sx = qx + kRayMagic, sy = qy + kRayMagic;
      const float ex = qx - (sx - kRayMagic), ey = qy - (sy - kRayMagic);
      c.bx = __float_as_uint(sx);
      c.by = __float_as_uint(sy);
      c.tx = ex + 0.5f;
      c.ty = ey + 0.5f;
      float m = fmaxf(fabsf(ex), fabsf(ey));
      c.in = (c.bx - mb < um) & (c.by - mb < um);
      if (FRAME) {
        const float qz = fmaf(kf, dw, wb), sz = qz + kRayMagic;
        const float ez = qz - (sz - kRayMagic);
        c.bz = __float_as_uint(sz);
        c.tz = ez + 0.5f;
        m = fmaxf(m, fabsf(ez));
        c.in &= c.bz - mb < um;
      } else {
        c.bz = mb + (unsigned)zc;  // the ray's z cell, reference arithmetic
        c.tz = tzc;
      }
      c.band = m > halfband;
      return c;
    };
    // the 8 corners of an inside cell in octet order
    auto gather = [&](const RayCell &c, float4 &lo, float4 &hi) {
      const unsigned ix = c.bx - mb, iy = c.by - mb, izc = c.bz - mb;
      if (job.oct) {
        ld_octet(job.oct, ((size_t)izc * (n - 1) + iy) * (n - 1) + ix, lo, hi);
      } else if (!FRAME && job.pairs) {
        // one z-layer pair: rows contiguous in x
        const float2 *p = job.pairs + ((size_t)izc * n + iy) * job.pitch + ix;
        const float2 a = __ldg(p), b = __ldg(p + job.pitch), d = __ldg(p + 1),
                     e = __ldg(p + job.pitch + 1);
        lo = make_float4(a.x, a.y, b.x, b.y);
        hi = make_float4(d.x, d.y, e.x, e.y);
      } else {
        const float *p = job.vol + ((size_t)ix * n + iy) * n + izc;
        const size_t sx = (size_t)n * n;
        lo = make_float4(__ldg(p), __ldg(p + 1), __ldg(p + n), __ldg(p + n + 1));
        hi = make_float4(__ldg(p + sx), __ldg(p + sx + 1), __ldg(p + sx + n),
                         __ldg(p + sx + n + 1));
      }
    };
    // sample k: the guard-band path (FP64, the reference's arithmetic) or the
    // FP32 trilinear value; 0 outside the cube
    auto sample = [&](int k, float &part) {
      const RayCell c = locate(k);
      if (c.band) {
        acc += exact_at(k);
      } else if (c.in) {
        float4 lo, hi;
        gather(c, lo, hi);
        part += octet_lerp(lo, hi, c.tx, c.ty, c.tz);
      }
    };
    for (int k0 = klo; k0 <= khi; k0 += 32) {
      const int k1 = min(khi, k0 + 31);
      float part = 0.0f;
      int k = k0;
      // with the cell octets: four samples at a time with all their loads
      // issued together (the same values, added in the same order, as one at
      // a time); a group with a guard-band sample takes the one-at-a-time path
      if (job.oct) {
        for (; k + 3 <= k1; k += 4) {
          RayCell c[4];
          bool band = false;
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            c[u] = locate(k + u);
            band |= c[u].band;
          }
          if (band) {
#pragma unroll 1
            for (int u = 0; u < 4; ++u) sample(k + u, part);
            continue;
          }
          float4 lo[4], hi[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            lo[u] = hi[u] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (c[u].in) gather(c[u], lo[u], hi[u]);
          }
#pragma unroll
          for (int u = 0; u < 4; ++u)
            if (c[u].in) part += octet_lerp(lo[u], hi[u], c[u].tx, c[u].ty, c[u].tz);
        }
      }
      for (; k <= k1; ++k) sample(k, part);
      acc += (double)part;
    }
  }
  if (job.counter && any) atomicAdd(job.counter, (unsigned long long)(khi - klo + 1));
  job.out[((long long)iz * job.nshift + is) * job.nphi + ip] = acc * delta;
}


}  // namespace wrtd
