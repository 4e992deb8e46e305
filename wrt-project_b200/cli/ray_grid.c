/* ray_grid -- drop-in for the reference's ray_grid program
 * (ray_grid/src/ray_grid.c): layer-by-layer ray integrals of a grid-sampled
 * volume, on the GPU.
 *
 *   ray_grid -p PARAMS -i VOLUME -o OUT [-n THREADS] [--binary]
 *
 * PARAMS: ngrid, nslices, nshift, nphi (ray_grid.c:177-180).  OUT: lines
 * "%lf, %lf, %lf, %lf" (z, s, phi, Pf) in the order z, shift, phi
 * (ray_grid.c:246-255), plus readme_OUT. */
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
  const double dz = 2.0 / (r->nslices - 1);
  const double z = (-1.0) + iz * dz;
  return sprintf(buf, "%lf, %lf, %lf, %lf\n", z, r->shift[is], r->phi[ip], r->val[k]);
}

int main(int argc, char **argv) {
  cli_args a;
  cli_parse(argc, argv, &a, "-p (filename) -i (filename) -o (filename) -n (number)", 0, 0);
  int p[4];
  printf("  Reading parameters from %s...", a.params);
  if (cli_read_params(a.params, p)) {
    fprintf(stderr, "Aborting : parameters_init.\n");
    return EXIT_FAILURE;
  }
  printf("Done.\n");
  const int ngrid = p[0], nslices = p[1], nshift = p[2], nphi = p[3];
  if (ngrid < 2 || nslices < 2 || nshift < 2 || nphi < 1) {
    fprintf(stderr, "Aborting : invalid grid parameters %d %d %d %d\n", ngrid, nslices, nshift, nphi);
    return EXIT_FAILURE;
  }
  const size_t nvox = (size_t)ngrid * ngrid * ngrid, nout = (size_t)nslices * nshift * nphi;
  double *vol = malloc(sizeof(double) * nvox), *out = malloc(sizeof(double) * nout);
  double *shift = malloc(sizeof(double) * nshift), *phi = malloc(sizeof(double) * nphi);
  if (!vol || !out || !shift || !phi) {
    fprintf(stderr, "Aborting : out of host memory\n");
    return EXIT_FAILURE;
  }
  printf("  Initializing test-function data...");
  if (cli_read_column(a.input, nvox, vol, a.nthreads)) {
    fprintf(stderr, "Aborting : tfunction_values_init.\n");
    return EXIT_FAILURE;
  }
  printf("Done.\n");
  /* ray_grid/src/init.c:163-176 */
  const double dshift = 2.0 / (nshift - 1), dphi = (2 * M_PI) / nphi;
  for (int i = 0; i < nshift; ++i) shift[i] = (-1.0) + i * dshift;
  for (int i = 0; i < nphi; ++i) phi[i] = dphi * i;
  wrt_ctx *ctx = cli_context(&a);
  double t0 = cli_now();
  cli_die_status(ctx, wrt_ray_grid(ctx, vol, ngrid, nslices, nshift, nphi, NULL, out), "ray_grid");
  printf("  Ray integrals on device %d, elapsed time: %3.3f sec\n", a.device, cli_now() - t0);
  cli_readme(a.output,
             "  Ray transforms in 3D for test-function given in file %s\n"
             "  Format of the data: [z], [shift], [phi], [Pf]\n"
             "  Parameters of the data:\n"
             "      number of z-slicez OZ direction  [nslices]   : %d,\n"
             "      number of angles on circle       [phi]  : %d,\n"
             "      number of shifts per direciton   [s]    : %d.\n",
             a.output, nslices, nphi, nshift);
  rows_t r = {shift, phi, out, nshift, nphi, nslices};
  if (cli_write_rows(a.output, nout, row, &r, a.nthreads)) return EXIT_FAILURE;
  if (a.binary && cli_write_binary(a.output, out, nout)) return EXIT_FAILURE;
  wrt_ctx_destroy(ctx);
  free(vol); free(out); free(shift); free(phi);
  return EXIT_SUCCESS;
}
