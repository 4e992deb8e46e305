/* GSL-compatible spline wrapper (test infrastructure only): a gsl_interp that
 * keeps its own copy of the knots and values. */
#ifndef WRT_GSL_SHIM_SPLINE_H
#define WRT_GSL_SHIM_SPLINE_H
#include "gsl_interp.h"
typedef struct {
  gsl_interp *interp;
  double *x;
  double *y;
  size_t size;
} gsl_spline;

gsl_spline *gsl_spline_alloc(const gsl_interp_type *T, size_t size);
int gsl_spline_init(gsl_spline *spline, const double xa[], const double ya[],
                    size_t size);
double gsl_spline_eval(const gsl_spline *spline, double x, gsl_interp_accel *a);
void gsl_spline_free(gsl_spline *spline);
#endif
