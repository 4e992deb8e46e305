/* Flat-array entry points around the reference's backprojection hot path
 * (radon_inversion/backprojection/C/src/integral.c, interp.c, init.c).  TEST
 * INFRASTRUCTURE ONLY.  Radon data in file order [nshift][nphi][ntheta]. */
#include <stdio.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "init.h"
#include "integral.h"

void refdrv_adjoint_points(const double *radon, int nphi, int ntheta, int nshift, int npts,
                           const double *x, const double *y, const double *z, double *out,
                           int nthreads) {
  double *phi, *theta, *w, *shift, ***R;
  radon_all_alloc(nphi, ntheta, nshift, &phi, &theta, &w, &shift, &R);
  radon_grid_init(nphi, ntheta, nshift, phi, theta, w, shift);
  for (int s = 0; s < nshift; ++s)
    for (int p = 0; p < nphi; ++p)
      for (int t = 0; t < ntheta; ++t) R[p][t][s] = radon[((size_t)s * nphi + p) * ntheta + t];
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 1)
  for (int k = 0; k < npts; ++k)
    out[k] = radon3d_adjoint(R, x[k], y[k], z[k], phi, theta, w, shift, nphi, ntheta, nshift);
  radon_values_clean(R, nphi, ntheta, nshift);
  radon_grid_clean(phi, theta, w, shift);
}

int refdrv_grid(int nphi, int ntheta, int nshift, double *phi, double *theta, double *w,
                double *shift) {
  return radon_grid_init(nphi, ntheta, nshift, phi, theta, w, shift);
}
