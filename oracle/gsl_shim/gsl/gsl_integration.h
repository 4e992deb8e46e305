/* GSL-compatible fixed-order Gauss-Legendre API (test infrastructure only).
 * Semantics follow the published GSL manual: gsl_integration_glfixed_point
 * returns the i-th node of the n-point rule on [a,b] in ascending order
 * together with its weight.  The nodes are computed by Newton's method on the
 * Legendre three-term recurrence (see gsl_shim.c); no GSL source is used. */
#ifndef WRT_GSL_SHIM_INTEGRATION_H
#define WRT_GSL_SHIM_INTEGRATION_H
#include <stddef.h>
#include "gsl_errno.h"
typedef struct {
  size_t n;
  double *x; /* ascending nodes on [-1,1] */
  double *w; /* matching weights          */
} gsl_integration_glfixed_table;

gsl_integration_glfixed_table *gsl_integration_glfixed_table_alloc(size_t n);
void gsl_integration_glfixed_table_free(gsl_integration_glfixed_table *t);
int gsl_integration_glfixed_point(double a, double b, size_t i, double *xi,
                                  double *wi,
                                  const gsl_integration_glfixed_table *t);
#endif
