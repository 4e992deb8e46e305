/* wrt_oracle.c -- FP64 CPU restatement of the reference hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle).  See wrt_oracle.h for the layouts
 * and for what may call this file.  Compile with -O2 -ffp-contract=off so that
 * no multiply-add is fused: the reference is built that way (plain gcc, no
 * -march), and the bit-for-bit pins depend on it.
 *
 * Each function names the reference function it restates.  Arithmetic is
 * written in the reference's evaluation order; only the data structures
 * differ (flat arrays instead of double***), plus two exact work-savers that
 * cannot change any result:
 *   - plane and ray lattice samples outside [-1,1]^3 return exactly 0 in the
 *     reference's samplers, so rows are clipped to the cube (with a margin of
 *     two lattice steps, the exact per-sample test still decides);
 *   - the reference rebuilds a natural cubic spline for every sample
 *     (radon_reduction/slicing.c:45-61, backprojection/C/src/interp.c:41-45);
 *     the spline of a line depends only on that line, so it is built once per
 *     line here.  The evaluation is the same arithmetic on the same numbers.
 */
#include "wrt_oracle.h"
#include "orc_math.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define VOL(v, n, ix, iy, iz) ((v)[((size_t)(ix) * (n) + (iy)) * (n) + (iz)])

static void set_threads(int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
}

int orc_gauss_legendre(int n, double *x, double *w) { return orc_gl_nodes(n, x, w); }

void orc_radon_grid_init(int nphi, int ntheta, int nshift, double *phi,
                         double *theta, double *theta_w, double *shift) {
  const double dphi = (2 * M_PI) / nphi;
  for (int i = 0; i < nphi; ++i) phi[i] = dphi * i;
  const double dshift = 2.0 / (nshift - 1);
  for (int i = 0; i < nshift; ++i) shift[i] = (-1.0) + i * dshift;
  double *x = malloc(sizeof(double) * ntheta), *w = malloc(sizeof(double) * ntheta);
  orc_gl_nodes(ntheta, x, w);
  for (int i = 0; i < ntheta; ++i) {
    theta[i] = acos(x[i]);
    if (theta_w) theta_w[i] = w[i];
  }
  free(x);
  free(w);
}

void orc_ray_grid_init(int nshift, int nphi, double *shift, double *phi) {
  const double dshift = 2.0 / (nshift - 1);
  for (int i = 0; i < nshift; ++i) shift[i] = (-1.0) + i * dshift;
  const double dphi = (2 * M_PI) / nphi;
  for (int i = 0; i < nphi; ++i) phi[i] = dphi * i;
}

/* ---- samplers: radon_grid/src/interp.c ---------------------------------- */

static double lin(double t, double a, double b) { return ((1 - t) * a + t * b); }

double orc_trilinear(const double *v, int n, double x, double y, double z) {
  if ((fabs(x) > 1) || (fabs(y) > 1) || (fabs(z) > 1)) return 0;
  const double delta = 2.0 / (n - 1);
  int ix = (int)((x + 1.0) / delta), iy = (int)((y + 1.0) / delta),
      iz = (int)((z + 1.0) / delta);
  double cx = fmod((x + 1.0), delta) / delta, cy = fmod((y + 1.0), delta) / delta,
         cz = fmod((z + 1.0), delta) / delta;
  if (ix == (n - 1)) { ix -= 1; cx = 1.0; }
  if (iy == (n - 1)) { iy -= 1; cy = 1.0; }
  if (iz == (n - 1)) { iz -= 1; cz = 1.0; }
  /* corner order and nesting of cell_trilinear_interp (interp.c:14-21,56-58):
   * bilinear(x,y, v000, v100, v110, v010) then bilinear at iz+1, then z. */
  double a0 = lin(cx, VOL(v, n, ix, iy, iz), VOL(v, n, ix + 1, iy, iz));
  double a1 = lin(cx, VOL(v, n, ix, iy + 1, iz), VOL(v, n, ix + 1, iy + 1, iz));
  double c0 = lin(cy, a0, a1);
  double b0 = lin(cx, VOL(v, n, ix, iy, iz + 1), VOL(v, n, ix + 1, iy, iz + 1));
  double b1 = lin(cx, VOL(v, n, ix, iy + 1, iz + 1), VOL(v, n, ix + 1, iy + 1, iz + 1));
  double c1 = lin(cy, b0, b1);
  return lin(cz, c0, c1);
}

double orc_zero_interp(const double *v, int n, double x, double y, double z) {
  if ((fabs(x) > 1) || (fabs(y) > 1) || (fabs(z) > 1)) return 0;
  const double delta = 2.0 / n;
  int ix = (int)((x + 1.0) / delta), iy = (int)((y + 1.0) / delta),
      iz = (int)((z + 1.0) / delta);
  if (ix == n) ix -= 1;
  if (iy == n) iy -= 1;
  if (iz == n) iz -= 1;
  return VOL(v, n, ix, iy, iz);
}

/* Conservative index range [lo, hi] of k such that |b + t*k| <= 1 (the exact
 * test is redone per sample).  Returns 0 if the range is empty. */
static int clip_axis(double b, double t, long *lo, long *hi) {
  /* the sample coordinate b + t*k is rounded, so a point whose exact value is
   * just outside [-1,1] can land on +-1: widen by eps in coordinate space */
  const double eps = 1e-13;
  if (t == 0.0) return fabs(b) <= 1.0 + eps;
  double k0 = (-1.0 - eps - b) / t, k1 = (1.0 + eps - b) / t;
  if (k0 > k1) { double s = k0; k0 = k1; k1 = s; }
  /* clamp in double before converting: k0, k1 can be far outside long range
   * when t is tiny */
  double flo = fmax(floor(k0) - 2, (double)*lo), fhi = fmin(ceil(k1) + 2, (double)*hi);
  if (!(flo <= fhi)) return 0;
  *lo = (long)flo;
  *hi = (long)fhi;
  return 1;
}

/* ---- plane integral: radon_grid/src/integral.c:10-58 -------------------- */

typedef struct { double x, y, z; } v3;

static v3 sph_dir(double phi, double theta) { /* integral.c:10-16 */
  v3 r;
  r.x = sin(theta) * cos(phi);
  r.y = sin(theta) * sin(phi);
  r.z = cos(theta);
  return r;
}

static v3 cross(v3 a, v3 b) { /* integral.c:18-24 */
  v3 r;
  r.x = a.y * b.z - a.z * b.y;
  r.y = -(a.x * b.z - a.z * b.x);
  r.z = a.x * b.y - a.y * b.x;
  return r;
}

double orc_plane_integral(const double *v, int n, double phi, double theta,
                          double shift, int sampler, int L) {
  v3 nrm = sph_dir(phi, theta);
  v3 v1 = sph_dir(phi, theta + M_PI / 2);
  v3 v2 = cross(nrm, v1);
  const double delta = (1.0 / (n));
  double integral = 0;
  for (long i1 = -L; i1 < L; ++i1) {
    /* row base, evaluated exactly as the reference evaluates the first two
     * terms of point.c = shift*normal.c + delta*v1.c*i_v1 + delta*v2.c*i_v2 */
    double bx = shift * nrm.x + delta * v1.x * i1;
    double by = shift * nrm.y + delta * v1.y * i1;
    double bz = shift * nrm.z + delta * v1.z * i1;
    long lo = -L, hi = L - 1;
    if (!clip_axis(bx, delta * v2.x, &lo, &hi)) continue;
    if (!clip_axis(by, delta * v2.y, &lo, &hi)) continue;
    if (!clip_axis(bz, delta * v2.z, &lo, &hi)) continue;
    for (long i2 = lo; i2 <= hi; ++i2) {
      double px = bx + delta * v2.x * i2;
      double py = by + delta * v2.y * i2;
      double pz = bz + delta * v2.z * i2;
      double value = sampler == ORC_SAMPLER_NEAREST ? orc_zero_interp(v, n, px, py, pz)
                                                    : orc_trilinear(v, n, px, py, pz);
      integral += value * delta * delta;
    }
  }
  return integral;
}

void orc_radon_planes(const double *v, int n, int nplanes, const double *phi,
                      const double *theta, const double *shift, int sampler,
                      int L, double *out, int nthreads) {
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4)
  for (int k = 0; k < nplanes; ++k)
    out[k] = orc_plane_integral(v, n, phi[k], theta[k], shift[k], sampler, L);
}

void orc_radon_forward(const double *v, int n, int nphi, int ntheta, int nshift,
                       int sampler, int L, double *out, int nthreads) {
  double *phi = malloc(sizeof(double) * nphi), *theta = malloc(sizeof(double) * ntheta),
         *shift = malloc(sizeof(double) * nshift);
  orc_radon_grid_init(nphi, ntheta, nshift, phi, theta, NULL, shift);
  const long total = (long)nphi * ntheta * nshift;
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4)
  for (long k = 0; k < total; ++k) {
    int it = (int)(k % ntheta), ip = (int)((k / ntheta) % nphi), is = (int)(k / ((long)ntheta * nphi));
    out[k] = orc_plane_integral(v, n, phi[ip], theta[it], shift[is], sampler, L);
  }
  free(phi);
  free(theta);
  free(shift);
}

/* ---- ray transform: ray_grid/src/integral.c:11-50 ----------------------- */

double orc_ray_transform(const double *v, int n, double zslice, double shift,
                         double phi, const double *F) {
  v3 nrm = {cos(phi), sin(phi), 0};
  v3 dir = {cos(phi + M_PI / 2), sin(phi + M_PI / 2), 0};
  v3 p0 = {shift * nrm.x, shift * nrm.y, zslice};
  const double delta = (2.0 / (n - 1)) / (2.0);
  const long half = (4L * n) / 2;
  double integral = 0;
  long lo = -half, hi = half;
  if (!F) {
    if (!clip_axis(p0.x, delta * dir.x, &lo, &hi)) return 0;
    if (!clip_axis(p0.y, delta * dir.y, &lo, &hi)) return 0;
    if (!clip_axis(p0.z, delta * dir.z, &lo, &hi)) return 0;
  }
  for (long k = lo; k <= hi; ++k) {
    double px = p0.x + delta * dir.x * k;
    double py = p0.y + delta * dir.y * k;
    double pz = p0.z + delta * dir.z * k;
    if (F) { /* rotated layer frame: x_world = F x_local */
      double wx = F[0] * px + F[1] * py + F[2] * pz;
      double wy = F[3] * px + F[4] * py + F[5] * pz;
      double wz = F[6] * px + F[7] * py + F[8] * pz;
      px = wx; py = wy; pz = wz;
    }
    double value = orc_trilinear(v, n, px, py, pz);
    integral += value * delta;
  }
  return integral;
}

void orc_ray_forward(const double *v, int n, int nslices, int nshift, int nphi,
                     const double *F, double *out, int nthreads) {
  double *shift = malloc(sizeof(double) * nshift), *phi = malloc(sizeof(double) * nphi);
  orc_ray_grid_init(nshift, nphi, shift, phi);
  const double dz = 2.0 / (nslices - 1);
  const long total = (long)nslices * nshift * nphi;
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
  for (long k = 0; k < total; ++k) {
    int ip = (int)(k % nphi), is = (int)((k / nphi) % nshift), iz = (int)(k / ((long)nphi * nshift));
    double z = (-1.0) + iz * dz;
    out[k] = orc_ray_transform(v, n, z, shift[is], phi[ip], F);
  }
  free(shift);
  free(phi);
}

/* ---- reduction: radon_reduction/slicing.c:5-119 ------------------------- */

typedef struct {
  int ngrid, nshift_ray, nphi;
  double *ray_shift; /* spline knots: the ray offset grid */
  double *val;       /* [iz][iphi][is], the reference's ray_values layout */
  double *M;         /* natural-spline second derivatives, same layout */
} rays_t;

static void rays_build(rays_t *r, const double *rays, int ngrid, int nshift_ray, int nphi) {
  r->ngrid = ngrid;
  r->nshift_ray = nshift_ray;
  r->nphi = nphi;
  r->ray_shift = malloc(sizeof(double) * nshift_ray);
  const double dshift = 2.0 / (nshift_ray - 1);
  for (int i = 0; i < nshift_ray; ++i) r->ray_shift[i] = (-1.0) + i * dshift;
  size_t tot = (size_t)ngrid * nphi * nshift_ray;
  r->val = malloc(sizeof(double) * tot);
  r->M = malloc(sizeof(double) * tot);
  /* file order z, s, phi -> ray_values[iz][iphi][is] (init.c:134-143) */
  for (int iz = 0; iz < ngrid; ++iz)
    for (int is = 0; is < nshift_ray; ++is)
      for (int ip = 0; ip < nphi; ++ip)
        r->val[((size_t)iz * nphi + ip) * nshift_ray + is] =
            rays[((size_t)iz * nshift_ray + is) * nphi + ip];
#pragma omp parallel
  {
    double *work = malloc(sizeof(double) * 2 * nshift_ray);
#pragma omp for
    for (long line = 0; line < (long)ngrid * nphi; ++line)
      orc_spline_natural(r->ray_shift, r->val + line * nshift_ray, nshift_ray,
                         r->M + line * nshift_ray, work);
    free(work);
  }
}

static void rays_free(rays_t *r) {
  free(r->ray_shift);
  free(r->val);
  free(r->M);
}

static double ray_interpolate(const rays_t *r, double slice_z, double slice_shift, int i_phi) {
  if ((fabs(slice_z) > 1.0) || (fabs(slice_shift) > 1.0)) return 0;
  const int ngrid = r->ngrid, ns = r->nshift_ray;
  const double delta_z = 2.0 / (ngrid - 1);
  int iz = (int)((slice_z + 1.0) / delta_z);
  if (iz == (ngrid - 1)) iz -= 1;
  double vals[3], zs[3];
  zs[0] = (-1.0) + delta_z * iz;
  zs[1] = (-1.0) + delta_z * (iz + 1);
  zs[2] = (-1.0) + delta_z * (iz + 2);
  for (int k = 0; k < 3; ++k) {
    if (k == 2 && iz >= (ngrid - 2)) { vals[2] = 0; break; }
    size_t line = ((size_t)(iz + k) * r->nphi + i_phi) * ns;
    vals[k] = orc_spline_eval(r->ray_shift, r->val + line, r->M + line, ns, slice_shift);
  }
  return orc_quadratic(zs, vals, slice_z);
}

static double radon_reduction(const rays_t *r, double p_shift, double p_phi_unused,
                              double p_theta, int i_phi) {
  (void)p_phi_unused;
  const int ngrid = r->ngrid;
  const double dtau = (2.0 / (ngrid - 1)) / (2.0);
  const int nsize = 4 * ngrid;
  double integral_value = 0, add = 0;
  for (int i_tau = -(nsize / 2); i_tau < (nsize / 2) + 1; ++i_tau) {
    double tau = (i_tau) * dtau;
    double slice_z = p_shift * cos(p_theta) + tau * sin(p_theta);
    double slice_shift = p_shift * sin(p_theta) - tau * cos(p_theta);
    if ((fabs(tau * tau + p_shift * p_shift) > 1.0) || (fabs(slice_z) > 1.0) ||
        (fabs(slice_shift) > 1.0))
      add = 0;
    else
      add = ray_interpolate(r, slice_z, slice_shift, i_phi);
    integral_value += (add * dtau);
  }
  return integral_value;
}

void orc_reduction_planes(const double *rays, int ngrid, int nshift_ray, int nphi,
                          int nshift, int ntheta, int nplanes, const int *is,
                          const int *iphi, const int *it, double *out, int nthreads) {
  set_threads(nthreads);
  rays_t r;
  rays_build(&r, rays, ngrid, nshift_ray, nphi);
  double *phi = malloc(sizeof(double) * nphi), *theta = malloc(sizeof(double) * ntheta),
         *shift = malloc(sizeof(double) * nshift);
  orc_radon_grid_init(nphi, ntheta, nshift, phi, theta, NULL, shift);
#pragma omp parallel for schedule(dynamic, 16)
  for (int k = 0; k < nplanes; ++k)
    out[k] = radon_reduction(&r, shift[is[k]], phi[iphi[k]], theta[it[k]], iphi[k]);
  free(phi);
  free(theta);
  free(shift);
  rays_free(&r);
}

void orc_reduction_forward(const double *rays, int ngrid, int nshift_ray, int nphi,
                           int nshift, int ntheta, double *out, int nthreads) {
  set_threads(nthreads);
  rays_t r;
  rays_build(&r, rays, ngrid, nshift_ray, nphi);
  double *phi = malloc(sizeof(double) * nphi), *theta = malloc(sizeof(double) * ntheta),
         *shift = malloc(sizeof(double) * nshift);
  orc_radon_grid_init(nphi, ntheta, nshift, phi, theta, NULL, shift);
  const long total = (long)nshift * nphi * ntheta;
#pragma omp parallel for schedule(dynamic, 16)
  for (long k = 0; k < total; ++k) {
    int t = (int)(k % ntheta), p = (int)((k / ntheta) % nphi), s = (int)(k / ((long)ntheta * nphi));
    out[k] = radon_reduction(&r, shift[s], phi[p], theta[t], p);
  }
  free(phi);
  free(theta);
  free(shift);
  rays_free(&r);
}

/* ---- adjoint: radon_inversion/backprojection/C/src/integral.c:6-24 ------ */

typedef struct {
  int nphi, ntheta, nshift;
  double *phi, *theta, *w, *shift;
  double *val, *M; /* [iphi][itheta][is] (init.c:182-188 layout) */
} radon_t;

static void radon_build(radon_t *R, const double *radon, int nphi, int ntheta, int nshift) {
  R->nphi = nphi;
  R->ntheta = ntheta;
  R->nshift = nshift;
  R->phi = malloc(sizeof(double) * nphi);
  R->theta = malloc(sizeof(double) * ntheta);
  R->w = malloc(sizeof(double) * ntheta);
  R->shift = malloc(sizeof(double) * nshift);
  orc_radon_grid_init(nphi, ntheta, nshift, R->phi, R->theta, R->w, R->shift);
  size_t tot = (size_t)nphi * ntheta * nshift;
  R->val = malloc(sizeof(double) * tot);
  R->M = malloc(sizeof(double) * tot);
  for (int is = 0; is < nshift; ++is)
    for (int ip = 0; ip < nphi; ++ip)
      for (int it = 0; it < ntheta; ++it)
        R->val[((size_t)ip * ntheta + it) * nshift + is] =
            radon[((size_t)is * nphi + ip) * ntheta + it];
#pragma omp parallel
  {
    double *work = malloc(sizeof(double) * 2 * nshift);
#pragma omp for
    for (long line = 0; line < (long)nphi * ntheta; ++line)
      orc_spline_natural(R->shift, R->val + line * nshift, nshift, R->M + line * nshift, work);
    free(work);
  }
}

static void radon_free(radon_t *R) {
  free(R->phi); free(R->theta); free(R->w); free(R->shift); free(R->val); free(R->M);
}

static double adjoint_at(const radon_t *R, double x, double y, double z) {
  const int nphi = R->nphi, ntheta = R->ntheta, nshift = R->nshift;
  double acc = 0;
  const double dphi = 2 * M_PI / nphi;
  for (int ip = 0; ip < nphi; ++ip) {
    for (int it = 0; it < ntheta; ++it) {
      double s = x * sin(R->theta[it]) * cos(R->phi[ip]) +
                 y * sin(R->theta[it]) * sin(R->phi[ip]) + z * cos(R->theta[it]);
      double val = 0.0; /* radon_interpolate_s, interp.c:5-28 */
      if (!(fabs(s) > 1)) {
        size_t line = ((size_t)ip * ntheta + it) * nshift;
        val = orc_spline_eval(R->shift, R->val + line, R->M + line, nshift, s);
      }
      acc += dphi * R->w[it] * val;
    }
  }
  return acc;
}

void orc_adjoint_points(const double *radon, int nphi, int ntheta, int nshift,
                        int npts, const double *x, const double *y, const double *z,
                        double *out, int nthreads) {
  set_threads(nthreads);
  radon_t R;
  radon_build(&R, radon, nphi, ntheta, nshift);
#pragma omp parallel for schedule(dynamic, 16)
  for (int k = 0; k < npts; ++k) out[k] = adjoint_at(&R, x[k], y[k], z[k]);
  radon_free(&R);
}

void orc_adjoint_forward(const double *radon, int nphi, int ntheta, int nshift,
                         int n, double *out, int nthreads) {
  set_threads(nthreads);
  radon_t R;
  radon_build(&R, radon, nphi, ntheta, nshift);
  const long total = (long)n * n * n;
#pragma omp parallel for schedule(dynamic, 64)
  for (long k = 0; k < total; ++k) {
    int iy = (int)(k % n), ix = (int)((k / n) % n), iz = (int)(k / ((long)n * n));
    /* cell centres, radon3d_ajoint.c:248-250 */
    double x = (-1.0) + (1.0 / n) + ix * (2.0 / n), y = (-1.0) + (1.0 / n) + iy * (2.0 / n),
           z = (-1.0) + (1.0 / n) + iz * (2.0 / n);
    out[k] = adjoint_at(&R, x, y, z);
  }
  radon_free(&R);
}

/* ---- exact transpose of orc_radon_forward ------------------------------- */

static void scatter_trilinear(double *acc, int n, double x, double y, double z, double g) {
  if ((fabs(x) > 1) || (fabs(y) > 1) || (fabs(z) > 1)) return;
  const double delta = 2.0 / (n - 1);
  int ix = (int)((x + 1.0) / delta), iy = (int)((y + 1.0) / delta),
      iz = (int)((z + 1.0) / delta);
  double cx = fmod((x + 1.0), delta) / delta, cy = fmod((y + 1.0), delta) / delta,
         cz = fmod((z + 1.0), delta) / delta;
  if (ix == (n - 1)) { ix -= 1; cx = 1.0; }
  if (iy == (n - 1)) { iy -= 1; cy = 1.0; }
  if (iz == (n - 1)) { iz -= 1; cz = 1.0; }
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 2; ++c) {
        double w = (a ? cx : 1 - cx) * (b ? cy : 1 - cy) * (c ? cz : 1 - cz);
        VOL(acc, n, ix + a, iy + b, iz + c) += g * w;
      }
}

static void scatter_nearest(double *acc, int n, double x, double y, double z, double g) {
  if ((fabs(x) > 1) || (fabs(y) > 1) || (fabs(z) > 1)) return;
  const double delta = 2.0 / n;
  int ix = (int)((x + 1.0) / delta), iy = (int)((y + 1.0) / delta),
      iz = (int)((z + 1.0) / delta);
  if (ix == n) ix -= 1;
  if (iy == n) iy -= 1;
  if (iz == n) iz -= 1;
  VOL(acc, n, ix, iy, iz) += g;
}

void orc_radon_transpose(const double *g, int n, int nphi, int ntheta, int nshift,
                         int sampler, int L, double *vol_out) {
  double *phi = malloc(sizeof(double) * nphi), *theta = malloc(sizeof(double) * ntheta),
         *shift = malloc(sizeof(double) * nshift);
  orc_radon_grid_init(nphi, ntheta, nshift, phi, theta, NULL, shift);
  const double delta = 1.0 / n;
  for (int is = 0; is < nshift; ++is)
    for (int ip = 0; ip < nphi; ++ip)
      for (int it = 0; it < ntheta; ++it) {
        double gv = g[((size_t)is * nphi + ip) * ntheta + it] * delta * delta;
        v3 nrm = sph_dir(phi[ip], theta[it]);
        v3 v1 = sph_dir(phi[ip], theta[it] + M_PI / 2);
        v3 v2 = cross(nrm, v1);
        for (long i1 = -L; i1 < L; ++i1) {
          double bx = shift[is] * nrm.x + delta * v1.x * i1;
          double by = shift[is] * nrm.y + delta * v1.y * i1;
          double bz = shift[is] * nrm.z + delta * v1.z * i1;
          long lo = -L, hi = L - 1;
          if (!clip_axis(bx, delta * v2.x, &lo, &hi)) continue;
          if (!clip_axis(by, delta * v2.y, &lo, &hi)) continue;
          if (!clip_axis(bz, delta * v2.z, &lo, &hi)) continue;
          for (long i2 = lo; i2 <= hi; ++i2) {
            double px = bx + delta * v2.x * i2, py = by + delta * v2.y * i2,
                   pz = bz + delta * v2.z * i2;
            if (sampler == ORC_SAMPLER_NEAREST) scatter_nearest(vol_out, n, px, py, pz, gv);
            else scatter_trilinear(vol_out, n, px, py, pz, gv);
          }
        }
      }
  free(phi);
  free(theta);
  free(shift);
}
