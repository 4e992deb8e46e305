/* ray_analytic -- drop-in for the reference's ray_analytic program
 * (ray_analytic/ray_analytic.c): layer-by-layer ray integrals of an analytic
 * test function, on the GPU.
 *
 *   ray_analytic -p PARAMS -o OUT --function exponential_bump|sinusoidal_bump
 *                [-n THREADS] [--binary]
 *
 * --function picks one of the reference's example test functions
 * (test-functions-examples/exponential_bump.c, sinusoidal_bump.c), which the
 * reference compiles in.  PARAMS: three lines, nshift, nphi, ngrid
 * (ray_analytic.c:201-203; ngrid z-slices z = -1 + 2 iz/(ngrid - 1), and the
 * density of the points on a ray).  OUT: lines "%lf, %lf, %lf, %lf"
 * (z, s, phi, Pf) in the order z, shift, phi (ray_analytic.c:254-274), plus
 * readme_OUT. */
#include <math.h>
#include <stdlib.h>

#include "cli_common.h"

typedef struct {
  const double *shift, *phi, *val;
  int nshift, nphi, nslices;
} rows_t;

static int row(char *buf, size_t k, const void *c) {
  const rows_t *r = c;
  size_t ip = k % r->nphi, is = (k / r->nphi) % r->nshift, iz = k / ((size_t)r->nphi * r->nshift);
  const double z = (-1.0) + iz * 2.0 / (r->nslices - 1);  /* ray_analytic.c:255 */
  return sprintf(buf, "%lf, %lf, %lf, %lf\n", z, r->shift[is], r->phi[ip], r->val[k]);
}

int main(int argc, char **argv) {
  cli_args a;
  cli_parse_flags(argc, argv, &a, "-p (filename) -o (filename) -n (number) --function (name)",
                  CLI_FUNCTION);
  int p[3];
  printf("  Reading parameters from %s...", a.params);
  if (cli_read_params_n(a.params, p, 3)) {
    fprintf(stderr, "Aborting : parameters_init.\n");
    return EXIT_FAILURE;
  }
  printf("Done.\n");
  const int nshift = p[0], nphi = p[1], ngrid = p[2];
  if (nshift < 2 || nphi < 1 || ngrid < 2) {
    fprintf(stderr, "Aborting : invalid grid parameters %d %d %d\n", nshift, nphi, ngrid);
    return EXIT_FAILURE;
  }
  const size_t nout = (size_t)ngrid * nshift * nphi;
  double *out = malloc(sizeof(double) * nout);
  double *shift = malloc(sizeof(double) * nshift), *phi = malloc(sizeof(double) * nphi);
  if (!out || !shift || !phi) {
    fprintf(stderr, "Aborting : out of host memory\n");
    return EXIT_FAILURE;
  }
  /* ray_analytic/init.c:85-101 */
  const double dshift = 2.0 / (nshift - 1), dphi = (2 * M_PI) / nphi;
  for (int i = 0; i < nshift; ++i) shift[i] = (-1.0) + i * dshift;
  for (int i = 0; i < nphi; ++i) phi[i] = dphi * i;
  wrt_function f;
  cli_example_function(a.function, &f);
  wrt_ctx *ctx = cli_context(&a);
  double t0 = cli_now();
  cli_die_status(ctx, wrt_ray_analytic(ctx, &f, ngrid, nshift, nphi, out), "ray_analytic");
  printf("  Ray integrals on device %d, elapsed time: %3.3f sec\n", a.device, cli_now() - t0);
  /* ray_analytic.c:55-71 */
  cli_readme(a.output,
             "  Ray transforms in 3D, output file: %s\n"
             "  Format of the data: [z], [s], [phi], [Pf]\n"
             "  Parameters of the data:\n"
             "     number of z-slices [nz]   : %d,\n"
             "     number of shifts   [s]    : %d.\n"
             "     number of angles   [phi]  : %d,\n",
             a.output, ngrid, nshift, nphi);
  rows_t r = {shift, phi, out, nshift, nphi, ngrid};
  if (cli_write_rows(a.output, nout, row, &r, a.nthreads)) return EXIT_FAILURE;
  if (a.binary && cli_write_binary(a.output, out, nout)) return EXIT_FAILURE;
  wrt_ctx_destroy(ctx);
  free(out); free(shift); free(phi);
  return EXIT_SUCCESS;
}
