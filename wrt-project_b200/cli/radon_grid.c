/* radon_grid -- drop-in for the reference's radon_grid program
 * (radon_grid/src/radon_grid.c): plane integrals of a grid-sampled volume
 * over the Gauss-uniform (shift, phi, theta) grid, on the GPU.
 *
 *   radon_grid -p PARAMS -i VOLUME -o OUT [-n THREADS]
 *              [--sampler nearest|trilinear] [--half-extent L] [--binary]
 *
 * PARAMS: nphi, ntheta, nshift, ngrid (radon_grid.c:182-185).  VOLUME: ngrid^3
 * lines "%lf", x slowest, z fastest.  OUT: lines "%lf, %lf, %lf, %lf"
 * (s, phi, theta, Rf) in the order shift, phi, theta (radon_grid.c:248-258),
 * plus readme_OUT.  Defaults reproduce the reference (nearest sampler,
 * lattice [-2n, 2n)^2 with step 1/n). */
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
  cli_parse(argc, argv, &a, "-p (filename) -i (filename) -o (filename) -n (number)", 0, 1);
  int p[4];
  printf("  Reading parameters from %s...", a.params);
  if (cli_read_params(a.params, p)) {
    fprintf(stderr, "Aborting : parameters_init failed.\n");
    return EXIT_FAILURE;
  }
  printf("Done.\n");
  const int nphi = p[0], ntheta = p[1], nshift = p[2], ngrid = p[3];
  if (nphi < 1 || ntheta < 1 || nshift < 2 || ngrid < 2) {
    fprintf(stderr, "Aborting : invalid grid parameters %d %d %d %d\n", nphi, ntheta, nshift, ngrid);
    return EXIT_FAILURE;
  }
  const size_t nvox = (size_t)ngrid * ngrid * ngrid, nout = (size_t)nphi * ntheta * nshift;
  double *vol = malloc(sizeof(double) * nvox), *out = malloc(sizeof(double) * nout);
  double *phi = malloc(sizeof(double) * nphi), *theta = malloc(sizeof(double) * ntheta),
         *shift = malloc(sizeof(double) * nshift);
  if (!vol || !out || !phi || !theta || !shift) {
    fprintf(stderr, "Aborting : out of host memory\n");
    return EXIT_FAILURE;
  }
  printf("  Initializing data for the test-function...");
  if (cli_read_column(a.input, nvox, vol, a.nthreads)) {
    fprintf(stderr, "Aborting : tfunction_values_init\n");
    return EXIT_FAILURE;
  }
  printf("Done.\n");
  wrt_ctx *ctx = cli_context(&a);
  cli_die_status(ctx, wrt_radon_grid_init(ctx, nphi, ntheta, nshift, phi, theta, NULL, shift),
                 "radon_grid_init");
  wrt_plane_opts o = {0};
  o.sampler = a.sampler;
  o.half_extent = a.half_extent;
  double t0 = cli_now();
  cli_die_status(ctx, wrt_radon_grid(ctx, vol, ngrid, nphi, ntheta, nshift, &o, out), "radon_grid");
  printf("  Plane integrals on device %d, elapsed time: %3.3f sec\n", a.device, cli_now() - t0);
  cli_readme(a.output,
             "  Radon transforms in 3D for test-function given in %s\n"
             "  Format of the data: [s], [phi], [theta], [Rf]\n"
             "  Parameters of the data:\n"
             "    number of grid ponts [ngrid]: %d,\n"
             "    number of angles of [phi]   : %d,\n"
             "    number of angles of [theta] : %d,\n"
             "    number of shifts of [s]     : %d.\n",
             a.output, ngrid, nphi, ntheta, nshift);
  rows_t r = {phi, theta, shift, out, nphi, ntheta};
  if (cli_write_rows(a.output, nout, row, &r, a.nthreads)) return EXIT_FAILURE;
  if (a.binary && cli_write_binary(a.output, out, nout)) return EXIT_FAILURE;
  wrt_ctx_destroy(ctx);
  free(vol); free(out); free(phi); free(theta); free(shift);
  return EXIT_SUCCESS;
}
