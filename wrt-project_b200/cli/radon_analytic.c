/* radon_analytic -- drop-in for the reference's radon_analytic program
 * (radon_analytic/src/radon_analytic.c): plane integrals of an analytic test
 * function over the Gauss-uniform (shift, phi, theta) grid, on the GPU.
 *
 *   radon_analytic -p PARAMS -o OUT --function exponential_bump|sinusoidal_bump
 *                  [-n THREADS] [--binary]
 *
 * The reference compiles its test function into the program (test_function.c,
 * with two example files); here --function picks one of those examples, with
 * their constants (examples-test-functions/exponential_bump.c,
 * sinusoidal_bump.c).  PARAMS: nphi, ntheta, nshift, ngrid
 * (radon_analytic.c:201-204; ngrid sets the lattice density, delta =
 * 1/(ngrid - 1)).  OUT: lines "%lf, %lf, %lf, %lf" (s, phi, theta, Rf) in
 * the order shift, phi, theta (radon_analytic.c:253-267), plus readme_OUT. */
#include <stdlib.h>

#include "cli_common.h"

typedef struct {
  const double *phi, *theta, *shift, *val;
  int nphi, ntheta;
} rows_t;

static int row(char *buf, size_t k, const void *c) {
  const rows_t *r = c;
  size_t it = k % r->ntheta, ip = (k / r->ntheta) % r->nphi, is = k / ((size_t)r->ntheta * r->nphi);
  return sprintf(buf, "%lf, %lf, %lf, %lf\n", r->shift[is], r->phi[ip], r->theta[it], r->val[k]);
}

int main(int argc, char **argv) {
  cli_args a;
  cli_parse_flags(argc, argv, &a, "-p (filename) -o (filename) -n (number) --function (name)",
                  CLI_FUNCTION);
  int p[4];
  printf("  Reading parameters from %s...", a.params);
  if (cli_read_params(a.params, p)) {
    fprintf(stderr, "Aborting : parameters_init.\n");
    return EXIT_FAILURE;
  }
  printf("Done.\n");
  const int nphi = p[0], ntheta = p[1], nshift = p[2], ngrid = p[3];
  if (nphi < 1 || ntheta < 1 || nshift < 2 || ngrid < 2) {
    fprintf(stderr, "Aborting : invalid grid parameters %d %d %d %d\n", nphi, ntheta, nshift, ngrid);
    return EXIT_FAILURE;
  }
  const size_t nout = (size_t)nphi * ntheta * nshift;
  double *out = malloc(sizeof(double) * nout);
  double *phi = malloc(sizeof(double) * nphi), *theta = malloc(sizeof(double) * ntheta),
         *shift = malloc(sizeof(double) * nshift);
  if (!out || !phi || !theta || !shift) {
    fprintf(stderr, "Aborting : out of host memory\n");
    return EXIT_FAILURE;
  }
  wrt_function f;
  cli_example_function(a.function, &f);
  wrt_ctx *ctx = cli_context(&a);
  printf("  Initializing the grid in Radon space...");
  cli_die_status(ctx, wrt_radon_grid_init(ctx, nphi, ntheta, nshift, phi, theta, NULL, shift),
                 "radon_grid_init");
  printf("Done.\n\n");
  double t0 = cli_now();
  cli_die_status(ctx, wrt_radon_analytic(ctx, &f, ngrid, nphi, ntheta, nshift, out),
                 "radon_analytic");
  printf("  Plane integrals on device %d, elapsed time: %3.3f sec\n", a.device, cli_now() - t0);
  /* radon_analytic.c:54-67 */
  cli_readme(a.output,
             "  Radon transforms in 3D for test-function given in %s\n"
             "  Format of the data: [s], [phi], [theta], [Rf]\n"
             "  Parameters of the data:\n"
             "    number of angles of [phi]  : %d,\n"
             "    number of angles of [theta]: %d,\n"
             "    number of shifts of [s]    : %d.\n",
             a.output, nphi, ntheta, nshift);
  rows_t r = {phi, theta, shift, out, nphi, ntheta};
  if (cli_write_rows(a.output, nout, row, &r, a.nthreads)) return EXIT_FAILURE;
  if (a.binary && cli_write_binary(a.output, out, nout)) return EXIT_FAILURE;
  wrt_ctx_destroy(ctx);
  free(out); free(phi); free(theta); free(shift);
  return EXIT_SUCCESS;
}
