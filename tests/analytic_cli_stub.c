/* CPU stand-in for the few libwrt entry points the analytic drop-in programs
 * call (cli/radon_analytic.c, cli/ray_analytic.c), so that the programs'
 * own work -- options, parameter file, grid columns, row order, "%lf"
 * formatting, readme -- can be checked end to end without a GPU against the
 * reference's programs (tests/test_cli_cpu.py).  TEST INFRASTRUCTURE ONLY.
 *
 * The transforms come from the reference's own integrators built with its
 * example functions (oracle/_ref/libref_{radon,ray}_analytic_{exp,sine}.so,
 * directory in WRT_STUB_REF_DIR); the grid from the oracle's restatement of
 * radon_grid_init (liboracle.so).  Before integrating, the wrt_function the
 * program passes is evaluated at 4096 seeded points of [-1,1]^3 with the
 * families' formulas and compared with the reference's example function at
 * the same points, which checks the program's example constants. */
#include <dlfcn.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "wrt.h"
#include "../oracle/wrt_oracle.h"

struct wrt_ctx {
  char last[256];
};

const char *wrt_status_string(int st) { return st ? "stub error" : "ok"; }

int wrt_ctx_create(int device, size_t budget, wrt_ctx **out) {
  (void)device;
  (void)budget;
  *out = calloc(1, sizeof(wrt_ctx));
  return *out ? WRT_OK : WRT_ERR_OUT_OF_MEMORY;
}

int wrt_ctx_destroy(wrt_ctx *ctx) {
  free(ctx);
  return WRT_OK;
}

const char *wrt_ctx_last_error(const wrt_ctx *ctx) { return ctx->last; }

int wrt_radon_grid_init(wrt_ctx *ctx, int nphi, int ntheta, int nshift, double *phi, double *theta,
                        double *w, double *shift) {
  (void)ctx;
  orc_radon_grid_init(nphi, ntheta, nshift, phi, theta, w, shift);
  return WRT_OK;
}

static int fail(wrt_ctx *ctx, const char *msg) {
  snprintf(ctx->last, sizeof ctx->last, "%s", msg);
  return WRT_ERR_INVALID_ARGUMENT;
}

/* the two example families, from their formulas */
static double family_value(const wrt_function *f, double x, double y, double z) {
  if (f->kind == WRT_FUNCTION_EXP_BUMP) {
    const double dx = x - f->p[0], dy = y - f->p[1], dz = z - f->p[2];
    const double r2 = dx * dx + dy * dy + dz * dz;
    return r2 < f->p[3] - f->p[4] ? exp(-1.0 / (f->p[3] - r2)) : 0.0;
  }
  double v = 0.0;
  for (int b = 0; b < f->count; ++b) {
    const double *q = f->p + 6 * b;
    const double r = sqrt((x - q[0]) * (x - q[0]) + (y - q[1]) * (y - q[1]) + (z - q[2]) * (z - q[2]));
    const double amp = q[3], rin = q[4], rout = q[5];
    if (r < rin) {
      v += amp;
    } else if (r < rout) {
      const double t = M_PI * (r - rout) / (rout - rin);
      v += (amp / (20 * M_PI)) * (-sin(6 * t) / 3 + 3 * sin(4 * t) - 15 * sin(2 * t) + 20 * t);
    }
  }
  return v;
}

static void *reference(wrt_ctx *ctx, const char *kind, const wrt_function *f) {
  const char *dir = getenv("WRT_STUB_REF_DIR");
  const char *family = f->kind == WRT_FUNCTION_EXP_BUMP ? "exp" : "sine";
  char path[4096];
  snprintf(path, sizeof path, "%s/libref_%s_analytic_%s.so", dir ? dir : ".", kind, family);
  void *h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!h) {
    fail(ctx, "reference integrator library not found");
    return NULL;
  }
  void (*values)(int, const double *, const double *, const double *, double *) =
      (void (*)(int, const double *, const double *, const double *, double *))dlsym(
          h, "refdrv_analytic_values");
  enum { kPoints = 4096 };
  static double x[kPoints], y[kPoints], z[kPoints], ref[kPoints];
  unsigned long long s = 12345;
  for (int k = 0; k < kPoints; ++k) {
    double *c[3] = {&x[k], &y[k], &z[k]};
    for (int a = 0; a < 3; ++a) {
      s = s * 6364136223846793005ULL + 1442695040888963407ULL;
      *c[a] = -1.0 + 2.0 * (double)(s >> 11) / 9007199254740992.0;
    }
  }
  values(kPoints, x, y, z, ref);
  for (int k = 0; k < kPoints; ++k)
    if (fabs(family_value(f, x[k], y[k], z[k]) - ref[k]) > 1e-9) {
      fail(ctx, "function constants differ from the reference's example");
      dlclose(h);
      return NULL;
    }
  return h;
}

int wrt_radon_analytic(wrt_ctx *ctx, const wrt_function *f, int ngrid, int nphi, int ntheta,
                       int nshift, double *out) {
  void *h = reference(ctx, "radon", f);
  if (!h) return WRT_ERR_INVALID_ARGUMENT;
  void (*planes)(int, int, const double *, const double *, const double *, double *, int) =
      (void (*)(int, int, const double *, const double *, const double *, double *, int))dlsym(
          h, "refdrv_analytic_planes");
  double *phi = malloc(sizeof(double) * nphi), *theta = malloc(sizeof(double) * ntheta),
         *shift = malloc(sizeof(double) * nshift);
  const size_t count = (size_t)nphi * ntheta * nshift;
  double *P = malloc(sizeof(double) * count), *T = malloc(sizeof(double) * count),
         *S = malloc(sizeof(double) * count);
  orc_radon_grid_init(nphi, ntheta, nshift, phi, theta, NULL, shift);
  for (size_t k = 0; k < count; ++k) {  /* out[is][iphi][itheta] */
    P[k] = phi[(k / ntheta) % nphi];
    T[k] = theta[k % ntheta];
    S[k] = shift[k / ((size_t)ntheta * nphi)];
  }
  planes(ngrid, (int)count, P, T, S, out, 0);
  free(phi); free(theta); free(shift); free(P); free(T); free(S);
  dlclose(h);
  return WRT_OK;
}

int wrt_ray_analytic(wrt_ctx *ctx, const wrt_function *f, int ngrid, int nshift, int nphi,
                     double *out) {
  void *h = reference(ctx, "ray", f);
  if (!h) return WRT_ERR_INVALID_ARGUMENT;
  void (*rays)(int, int, const double *, const double *, const double *, double *, int) =
      (void (*)(int, int, const double *, const double *, const double *, double *, int))dlsym(
          h, "refdrv_analytic_rays");
  double *shift = malloc(sizeof(double) * nshift), *phi = malloc(sizeof(double) * nphi);
  const size_t count = (size_t)ngrid * nshift * nphi;
  double *Z = malloc(sizeof(double) * count), *S = malloc(sizeof(double) * count),
         *P = malloc(sizeof(double) * count);
  orc_ray_grid_init(nshift, nphi, shift, phi);
  for (size_t k = 0; k < count; ++k) {  /* out[iz][is][iphi] */
    const size_t iz = k / ((size_t)nshift * nphi);
    Z[k] = (-1.0) + iz * 2.0 / (ngrid - 1);
    S[k] = shift[(k / nphi) % nshift];
    P[k] = phi[k % nphi];
  }
  rays(ngrid, (int)count, Z, S, P, out, 0);
  free(shift); free(phi); free(Z); free(S); free(P);
  dlclose(h);
  return WRT_OK;
}
