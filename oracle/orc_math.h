/* orc_math.h -- FP64 numerical kernels shared by the oracle restatement and
 * by the GSL-compatible shim that lets the reference's own sources compile.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the CUDA library, the
 * drop-in command-line programs) links or calls this code; the tests and the
 * benchmark's CPU baseline use it as the checker.
 *
 * Everything here is written from the mathematics:
 *   - Gauss-Legendre nodes/weights: Newton iteration on P_n evaluated with the
 *     three-term recurrence (k+1)P_{k+1} = (2k+1)xP_k - kP_{k-1}, derivative
 *     P_n' = n(xP_n - P_{n-1})/(x^2-1), weights 2/((1-x^2)P_n'(x)^2).  This is
 *     what the reference obtains from gsl_integration_glfixed_* at
 *     radon_grid/src/init.c:180-187.
 *   - natural cubic spline (second derivatives M_0 = M_{n-1} = 0, tridiagonal
 *     system solved by forward elimination / back substitution), evaluated
 *     with the standard piecewise-cubic formula; this is the "cspline" the
 *     reference builds at radon_reduction/slicing.c:45-61 and
 *     radon_inversion/backprojection/C/src/interp.c:41-45.
 *   - the 3-point interpolating polynomial in Newton divided-difference form
 *     (radon_reduction/slicing.c:67-72, gsl_interp_polynomial with 3 points).
 */
#ifndef WRT_ORC_MATH_H
#define WRT_ORC_MATH_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* n-point Gauss-Legendre rule on [-1,1]; x ascending, exactly symmetric. */
int orc_gl_nodes(int n, double *x, double *w);

/* Index i in [0, n-2] with x[i] <= t < x[i+1] (clamped at both ends). */
size_t orc_interval(const double *x, size_t n, double t);

/* Natural cubic spline second derivatives M[0..n-1]; work needs 2n doubles. */
void orc_spline_natural(const double *x, const double *y, size_t n, double *M,
                        double *work);

/* Evaluate the spline (x, y, M) at t, t inside [x[0], x[n-1]]. */
double orc_spline_eval(const double *x, const double *y, const double *M,
                       size_t n, double t);

/* Interpolating quadratic through (z[k], v[k]), k = 0..2, evaluated at t. */
double orc_quadratic(const double z[3], const double v[3], double t);

#ifdef __cplusplus
}
#endif
#endif
