/* Flat-array entry points around the reference's radon_grid hot path
 * (radon_grid/src/integral.c, interp.c, init.c compiled unmodified from the
 * reference tree).  TEST INFRASTRUCTURE ONLY: the checker and the CPU
 * baseline call these; the product never does. */
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "init.h"
#include "integral.h"
#include "interp.h"

static double ***view3(const double *v, int n) {
  double ***p = malloc(sizeof(double **) * n);
  for (int i = 0; i < n; ++i) {
    p[i] = malloc(sizeof(double *) * n);
    for (int j = 0; j < n; ++j) p[i][j] = (double *)v + ((size_t)i * n + j) * n;
  }
  return p;
}
static void free3(double ***p, int n) {
  for (int i = 0; i < n; ++i) free(p[i]);
  free(p);
}

int refdrv_radon_grid_init(int nphi, int ntheta, int nshift, double *phi,
                           double *theta, double *shift) {
  return radon_grid_init(nphi, ntheta, nshift, phi, theta, shift);
}

void refdrv_plane_integrals(const double *vol, int n, int nplanes, const double *phi,
                            const double *theta, const double *shift, double *out,
                            int nthreads) {
  double ***v = view3(vol, n);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 4)
  for (int k = 0; k < nplanes; ++k) out[k] = plane_integral(v, n, phi[k], theta[k], shift[k]);
  free3(v, n);
}

void refdrv_samplers(const double *vol, int n, int npts, const double *x, const double *y,
                     const double *z, double *out_nearest, double *out_trilinear) {
  double ***v = view3(vol, n);
  for (int k = 0; k < npts; ++k) {
    out_nearest[k] = zero_interp(v, n, x[k], y[k], z[k]);
    out_trilinear[k] = cube_trilinear_interp(v, n, x[k], y[k], z[k]);
  }
  free3(v, n);
}
