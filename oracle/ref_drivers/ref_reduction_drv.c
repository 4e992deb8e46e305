/* Flat-array entry points around the reference's radon_reduction hot path
 * (radon_reduction/slicing.c, interpolation.c, init.c).  TEST
 * INFRASTRUCTURE ONLY.  Rays come in file order [ngrid][nshift][nphi]. */
#include <stdio.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "init.h"
#include "slicing.h"

void refdrv_reduction_planes(const double *rays, int ngrid, int nshift, int nphi,
                             int ntheta, int nplanes, const int *is, const int *ip,
                             const int *it, double *out, int nthreads) {
  double ***rv;
  ray_values_alloc(nshift, nphi, ngrid, &rv);
  for (int z = 0; z < ngrid; ++z)
    for (int s = 0; s < nshift; ++s)
      for (int p = 0; p < nphi; ++p) rv[z][p][s] = rays[((size_t)z * nshift + s) * nphi + p];
  double *shift, *phi, *theta;
  radon_grid_alloc(nshift, nphi, ntheta, &shift, &phi, &theta);
  radon_grid_init(nshift, nphi, ntheta, shift, phi, theta);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 1)
  for (int k = 0; k < nplanes; ++k)
    out[k] = radon_reduction(rv, shift, phi, theta, nshift, nphi, ntheta, ngrid, is[k], ip[k], it[k]);
  radon_grid_clean(shift, phi, theta);
  ray_values_clean(nshift, nphi, ngrid, rv);
}
