/* gsl_shim.c -- just enough of the GSL API for the reference's hot-path
 * sources to compile and run here (GNU GSL is not installed).  TEST
 * INFRASTRUCTURE ONLY: used to build oracle/_ref from the reference sources.
 * Written from the GSL manual's description of each call and from the
 * mathematics in orc_math.c; no GSL source code is used. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "gsl/gsl_integration.h"
#include "gsl/gsl_spline.h"
#include "../orc_math.h"

static const gsl_interp_type cspline_type = {"cspline", 3, 1};
static const gsl_interp_type polynomial_type = {"polynomial", 3, 2};
const gsl_interp_type *gsl_interp_cspline = &cspline_type;
const gsl_interp_type *gsl_interp_polynomial = &polynomial_type;

gsl_integration_glfixed_table *gsl_integration_glfixed_table_alloc(size_t n) {
  gsl_integration_glfixed_table *t = malloc(sizeof(*t));
  if (!t) return NULL;
  t->n = n;
  t->x = malloc(n * sizeof(double));
  t->w = malloc(n * sizeof(double));
  orc_gl_nodes((int)n, t->x, t->w);
  return t;
}

void gsl_integration_glfixed_table_free(gsl_integration_glfixed_table *t) {
  if (!t) return;
  free(t->x);
  free(t->w);
  free(t);
}

int gsl_integration_glfixed_point(double a, double b, size_t i, double *xi,
                                  double *wi,
                                  const gsl_integration_glfixed_table *t) {
  if (i >= t->n) return GSL_EINVAL;
  const double half = (b - a) / 2, mid = (a + b) / 2;
  *xi = mid + half * t->x[i];
  *wi = half * t->w[i];
  return GSL_SUCCESS;
}

gsl_interp_accel *gsl_interp_accel_alloc(void) {
  return calloc(1, sizeof(gsl_interp_accel));
}
void gsl_interp_accel_free(gsl_interp_accel *a) { free(a); }

gsl_interp *gsl_interp_alloc(const gsl_interp_type *T, size_t n) {
  if (n < T->min_size) {
    fprintf(stderr, "gsl_shim: insufficient number of points for %s\n", T->name);
    return NULL;
  }
  gsl_interp *p = malloc(sizeof(*p));
  p->type = T;
  p->size = n;
  p->xmin = p->xmax = 0;
  p->work = malloc(3 * n * sizeof(double));
  return p;
}

int gsl_interp_init(gsl_interp *p, const double xa[], const double ya[],
                    size_t size) {
  if (size != p->size) return GSL_EINVAL;
  for (size_t i = 1; i < size; ++i)
    if (!(xa[i] > xa[i - 1])) return GSL_EINVAL;
  p->xmin = xa[0];
  p->xmax = xa[size - 1];
  if (p->type->kind == 1) orc_spline_natural(xa, ya, size, p->work, p->work + size);
  return GSL_SUCCESS;
}

double gsl_interp_eval(const gsl_interp *p, const double xa[], const double ya[],
                       double x, gsl_interp_accel *a) {
  (void)a;
  if (x < p->xmin || x > p->xmax) {
    /* GSL's default error handler aborts the program here; the shim reports
     * the first occurrence and returns NaN (GSL with the handler off). */
    static int reported = 0;
    if (!reported) {
      reported = 1;
      fprintf(stderr, "gsl_shim: interpolation error (x=%.17g outside [%.17g, %.17g]); "
              "GSL would abort here, the shim returns NaN\n", x, p->xmin, p->xmax);
    }
    return NAN;
  }
  if (p->type->kind == 1) return orc_spline_eval(xa, ya, p->work, p->size, x);
  /* polynomial: the reference only ever uses 3 points */
  if (p->size == 3) return orc_quadratic(xa, ya, x);
  /* general Newton form */
  double *d = p->work;
  for (size_t i = 0; i < p->size; ++i) d[i] = ya[i];
  for (size_t k = 1; k < p->size; ++k)
    for (size_t i = p->size - 1; i >= k; --i)
      d[i] = (d[i] - d[i - 1]) / (xa[i] - xa[i - k]);
  double r = d[p->size - 1];
  for (size_t i = p->size - 1; i-- > 0;) r = d[i] + (x - xa[i]) * r;
  return r;
}

void gsl_interp_free(gsl_interp *p) {
  if (!p) return;
  free(p->work);
  free(p);
}

gsl_spline *gsl_spline_alloc(const gsl_interp_type *T, size_t size) {
  gsl_spline *s = malloc(sizeof(*s));
  s->interp = gsl_interp_alloc(T, size);
  s->x = malloc(size * sizeof(double));
  s->y = malloc(size * sizeof(double));
  s->size = size;
  return s;
}

int gsl_spline_init(gsl_spline *s, const double xa[], const double ya[],
                    size_t size) {
  if (size != s->size) return GSL_EINVAL;
  memcpy(s->x, xa, size * sizeof(double));
  memcpy(s->y, ya, size * sizeof(double));
  return gsl_interp_init(s->interp, s->x, s->y, size);
}

double gsl_spline_eval(const gsl_spline *s, double x, gsl_interp_accel *a) {
  return gsl_interp_eval(s->interp, s->x, s->y, x, a);
}

void gsl_spline_free(gsl_spline *s) {
  if (!s) return;
  gsl_interp_free(s->interp);
  free(s->x);
  free(s->y);
  free(s);
}
