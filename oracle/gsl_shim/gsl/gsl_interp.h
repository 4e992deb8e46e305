/* GSL-compatible 1D interpolation API (test infrastructure only): natural
 * cubic spline ("cspline") and global polynomial interpolation, written from
 * the mathematics.  Out-of-range evaluation prints an error and returns NaN,
 * which is what GSL does with its error handler switched off. */
#ifndef WRT_GSL_SHIM_INTERP_H
#define WRT_GSL_SHIM_INTERP_H
#include <stddef.h>
#include "gsl_errno.h"
typedef struct {
  const char *name;
  unsigned int min_size;
  int kind; /* 1 = natural cubic spline, 2 = polynomial */
} gsl_interp_type;

extern const gsl_interp_type *gsl_interp_cspline;
extern const gsl_interp_type *gsl_interp_polynomial;

typedef struct {
  size_t cache; /* last interval found (hint only) */
} gsl_interp_accel;

typedef struct {
  const gsl_interp_type *type;
  double xmin, xmax;
  size_t size;
  double *work; /* cspline: second derivatives M_i; polynomial: divided differences */
} gsl_interp;

gsl_interp_accel *gsl_interp_accel_alloc(void);
void gsl_interp_accel_free(gsl_interp_accel *a);
gsl_interp *gsl_interp_alloc(const gsl_interp_type *T, size_t n);
int gsl_interp_init(gsl_interp *interp, const double xa[], const double ya[],
                    size_t size);
double gsl_interp_eval(const gsl_interp *interp, const double xa[],
                       const double ya[], double x, gsl_interp_accel *a);
void gsl_interp_free(gsl_interp *interp);
#endif
