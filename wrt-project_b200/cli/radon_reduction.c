/* radon_reduction -- drop-in for the reference's radon_reduction program
 * (radon_reduction/reduction.c): ray data in layer-by-layer sampling reduced
 * to Radon data on the Gauss-uniform grid, on the GPU.
 *
 *   radon_reduction -p PARAMS -i RAYS [-s] -o OUT [-n THREADS] [--binary]
 *
 * PARAMS: nshift, nphi, ntheta, ngrid (reduction.c:145-148).  RAYS: ngrid x
 * nshift x nphi lines in the order z, shift, phi, either 4 columns
 * "%lf, %lf, %lf, %lf" (ray_grid's output) or, with -s, one column
 * (radon_reduction/init.c:116-164).  OUT: one column "%lf" in the order shift,
 * phi, theta (reduction.c:215-229), plus readme_OUT.  (-s takes no argument;
 * the reference asserts on its missing optarg.) */
#include <stdlib.h>

#include "cli_common.h"

static int row(char *buf, size_t k, const void *c) {
  return sprintf(buf, "%lf\n", ((const double *)c)[k]);
}

int main(int argc, char **argv) {
  cli_args a;
  cli_parse(argc, argv, &a, "-p (filename) -i (filename) [-s] -o (filename) -n (number)", 1, 0);
  int p[4];
  printf("  Reading parameters from %s...", a.params);
  if (cli_read_params(a.params, p)) {
    fprintf(stderr, "Aborting : parameters_init.\n");
    return EXIT_FAILURE;
  }
  printf("Done.\n");
  const int nshift = p[0], nphi = p[1], ntheta = p[2], ngrid = p[3];
  if (nshift < 3 || nphi < 1 || ntheta < 1 || ngrid < 3) {
    fprintf(stderr, "Aborting : invalid grid parameters %d %d %d %d\n", nshift, nphi, ntheta, ngrid);
    return EXIT_FAILURE;
  }
  const size_t nin = (size_t)ngrid * nshift * nphi, nout = (size_t)nshift * nphi * ntheta;
  double *rays = malloc(sizeof(double) * nin), *out = malloc(sizeof(double) * nout);
  if (!rays || !out) {
    fprintf(stderr, "Aborting : out of host memory\n");
    return EXIT_FAILURE;
  }
  printf("  Initializing data for ray transforms...");
  if ((a.small_format ? cli_read_column : cli_read_csv4)(a.input, nin, rays, a.nthreads)) {
    fprintf(stderr, "Aborting : ray_values_init.\n");
    return EXIT_FAILURE;
  }
  printf("Done.\n");
  wrt_ctx *ctx = cli_context(&a);
  double t0 = cli_now();
  cli_die_status(ctx, wrt_radon_reduction(ctx, rays, ngrid, nshift, nphi, nshift, ntheta, out),
                 "radon_reduction");
  printf("  Reduction on device %d, elapsed time: %3.3f sec\n", a.device, cli_now() - t0);
  cli_readme(a.output,
             "  Reduction of (weighted) ray transforms (%s) to (weighted) Radon transforms.\n"
             "  Format of the data: [s], [phi], [theta], [Rf]\n"
             "  Parameters of the data:\n"
             "      number of shifts [s]    : %d.\n"
             "      number of angles [phi]  : %d,\n"
             "      number of angles [theta]: %d,\n",
             a.output, nshift, nphi, ntheta);
  if (cli_write_rows(a.output, nout, row, out, a.nthreads)) return EXIT_FAILURE;
  if (a.binary && cli_write_binary(a.output, out, nout)) return EXIT_FAILURE;
  wrt_ctx_destroy(ctx);
  free(rays); free(out);
  return EXIT_SUCCESS;
}
