/* Flat-array entry points around the reference's analytic-function
 * transforms: plane_integral (radon_analytic/src/integral.c:25-57) or
 * ray_integral (ray_analytic/integral.c:10-48) of the test_function the
 * library is compiled with (one of the reference's example functions).
 * TEST INFRASTRUCTURE ONLY. */
#include <stddef.h>
#ifdef _OPENMP
#include <omp.h>
#endif

double test_function(double x, double y, double z);
#ifdef REF_RAY
double ray_integral(double (*function_ptr)(double, double, double), double zslice, double shift,
                    double phi, int ngrid);
/* out[k] = ray integral at (z[k], shift[k], phi[k]) */
void refdrv_analytic_rays(int ngrid, int count, const double *z, const double *shift,
                          const double *phi, double *out, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 16)
  for (int k = 0; k < count; ++k) out[k] = ray_integral(&test_function, z[k], shift[k], phi[k], ngrid);
}
#else
double plane_integral(double (*function_ptr)(double, double, double), int ngrid, double phi,
                      double theta, double shift);
/* out[k] = plane integral at (phi[k], theta[k], shift[k]) */
void refdrv_analytic_planes(int ngrid, int count, const double *phi, const double *theta,
                            const double *shift, double *out, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 4)
  for (int k = 0; k < count; ++k)
    out[k] = plane_integral(&test_function, ngrid, phi[k], theta[k], shift[k]);
}
#endif
/* the test function itself, for point checks */
void refdrv_analytic_values(int count, const double *x, const double *y, const double *z,
                            double *out) {
  for (int k = 0; k < count; ++k) out[k] = test_function(x[k], y[k], z[k]);
}
