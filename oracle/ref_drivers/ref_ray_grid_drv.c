/* Flat-array entry points around the reference's ray_grid hot path
 * (ray_grid/src/integral.c, interp.c, init.c).  TEST INFRASTRUCTURE ONLY. */
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "init.h"
#include "integral.h"

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

/* The loop nest of ray_grid/src/ray_grid.c:243-258, output [z][s][phi]. */
void refdrv_ray_forward(const double *vol, int n, int nslices, int nshift, int nphi,
                        double *out, int nthreads) {
  double ***v = view3(vol, n);
  double *shift, *phi;
  ray_grid_alloc(nshift, nphi, &shift, &phi);
  ray_grid_init(nshift, nphi, shift, phi);
  const double dzslice = 2.0 / (nslices - 1);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 1)
  for (int iz = 0; iz < nslices; ++iz) {
    double zslice = (-1.0) + iz * dzslice;
    for (int is = 0; is < nshift; ++is)
      for (int ip = 0; ip < nphi; ++ip)
        out[((size_t)iz * nshift + is) * nphi + ip] = ray_transform(v, n, zslice, shift[is], phi[ip]);
  }
  ray_grid_clean(shift, phi);
  free3(v, n);
}

/* Arbitrary rays (z[k], s[k], phi[k]). */
void refdrv_rays(const double *vol, int n, int nrays, const double *z, const double *s,
                 const double *phi, double *out, int nthreads) {
  double ***v = view3(vol, n);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 64)
  for (int k = 0; k < nrays; ++k) out[k] = ray_transform(v, n, z[k], s[k], phi[k]);
  free3(v, n);
}
