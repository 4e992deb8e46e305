/* orc_math.c -- see orc_math.h.  TEST INFRASTRUCTURE ONLY (the oracle). */
#include "orc_math.h"
#include <math.h>

/* The Gauss-Legendre generator uses only IEEE basic operations (+ - * /,
 * fabs) in a fixed order, so that the same algorithm compiled for the GPU
 * (wrt-project_b200/csrc/k_grid.cu, built without fused multiply-add)
 * produces bit-identical nodes and weights.  The initial guess therefore uses
 * a Maclaurin series for the cosine instead of libm. */
static double series_cos(double a) { /* a in [0, pi] */
  double a2 = a * a, term = 1.0, sum = 1.0;
  for (int k = 1; k <= 30; ++k) {
    double den = (double)((2 * k - 1) * (2 * k));
    term = ((-term) * a2) / den;
    sum = sum + term;
  }
  return sum;
}

static void legendre_pair(int n, double x, double *pn, double *pnm1) {
  double p0 = 1.0, p1 = x;
  if (n == 0) { *pn = 1.0; *pnm1 = 0.0; return; }
  for (int k = 1; k < n; ++k) {
    double kd = (double)k;
    double a = 2.0 * kd + 1.0;
    double t = (a * x) * p1;
    double num = t - kd * p0;
    double p2 = num / (kd + 1.0);
    p0 = p1;
    p1 = p2;
  }
  *pn = p1;
  *pnm1 = p0;
}

static double legendre_deriv(int n, double r, double pn, double pnm1) {
  double num = (double)n * (r * pn - pnm1);
  double den = r * r - 1.0;
  return num / den;
}

int orc_gl_nodes(int n, double *x, double *w) {
  if (n < 1) return -1;
  const int m = n / 2; /* number of strictly positive roots */
  for (int k = 1; k <= m; ++k) {
    double ang = (M_PI * ((double)k - 0.25)) / ((double)n + 0.5);
    double r = series_cos(ang); /* k-th largest root, initial guess */
    double pn, pnm1, dp;
    for (int it = 0; it < 100; ++it) {
      legendre_pair(n, r, &pn, &pnm1);
      dp = legendre_deriv(n, r, pn, pnm1);
      double dr = pn / dp;
      r = r - dr;
      if (fabs(dr) <= 1e-16 * fabs(r)) break;
    }
    legendre_pair(n, r, &pn, &pnm1);
    dp = legendre_deriv(n, r, pn, pnm1);
    double wk = 2.0 / (((1.0 - r * r) * dp) * dp);
    /* ascending order: negative roots first, mirrored exactly */
    x[k - 1] = -r;
    w[k - 1] = wk;
    x[n - k] = r;
    w[n - k] = wk;
  }
  if (n & 1) {
    double pn, pnm1;
    legendre_pair(n, 0.0, &pn, &pnm1);
    double dp = legendre_deriv(n, 0.0, pn, pnm1);
    x[m] = 0.0;
    w[m] = 2.0 / ((1.0 * dp) * dp);
  }
  return 0;
}

size_t orc_interval(const double *x, size_t n, double t) {
  size_t lo = 0, hi = n - 1;
  while (hi > lo + 1) {
    size_t mid = (lo + hi) / 2;
    if (x[mid] > t) hi = mid;
    else lo = mid;
  }
  return lo;
}

void orc_spline_natural(const double *x, const double *y, size_t n, double *M,
                        double *work) {
  /* Unknowns M_1..M_{n-2}; row i:
   *   h_{i-1} M_{i-1} + 2(h_{i-1}+h_i) M_i + h_i M_{i+1}
   *     = 6((y_{i+1}-y_i)/h_i - (y_i-y_{i-1})/h_{i-1}).                   */
  double *cp = work;      /* modified super-diagonal */
  double *dp = work + n;  /* modified right-hand side */
  M[0] = 0.0;
  M[n - 1] = 0.0;
  if (n < 3) return;
  for (size_t i = 1; i + 1 < n; ++i) {
    double hl = x[i] - x[i - 1], hr = x[i + 1] - x[i];
    double diag = 2.0 * (hl + hr);
    double rhs = 6.0 * ((y[i + 1] - y[i]) / hr - (y[i] - y[i - 1]) / hl);
    if (i > 1) {
      double den = diag - hl * cp[i - 1];
      cp[i] = hr / den;
      dp[i] = (rhs - hl * dp[i - 1]) / den;
    } else {
      cp[i] = hr / diag;
      dp[i] = rhs / diag;
    }
  }
  M[n - 2] = dp[n - 2];
  for (size_t i = n - 2; i-- > 1;) M[i] = dp[i] - cp[i] * M[i + 1];
}

double orc_spline_eval(const double *x, const double *y, const double *M,
                       size_t n, double t) {
  size_t i = orc_interval(x, n, t);
  double h = x[i + 1] - x[i];
  double a = (x[i + 1] - t) / h, b = (t - x[i]) / h;
  return a * y[i] + b * y[i + 1] +
         ((a * a * a - a) * M[i] + (b * b * b - b) * M[i + 1]) * (h * h) / 6.0;
}

double orc_quadratic(const double z[3], const double v[3], double t) {
  double d01 = (v[1] - v[0]) / (z[1] - z[0]);
  double d12 = (v[2] - v[1]) / (z[2] - z[1]);
  double d012 = (d12 - d01) / (z[2] - z[0]);
  return v[0] + (t - z[0]) * (d01 + (t - z[1]) * d012);
}
