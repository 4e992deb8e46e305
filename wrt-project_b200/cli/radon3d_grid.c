/* radon3d_grid -- drop-in for the reference's backprojection program
 * (radon_inversion/backprojection/C/src/radon3d_ajoint.c): the adjoint Radon
 * transform at the cell centres of an ngrid^3 grid, on the GPU.
 *
 *   radon3d_grid -p PARAMS -i RADON -o OUT [-n THREADS] [--binary]
 *
 * PARAMS: nphi, ntheta, nshift, ngrid (radon3d_ajoint.c:181-184).  RADON:
 * nshift x nphi x ntheta lines "%lf, %lf, %lf, %lf" (s, phi, theta, R) in the
 * order shift, phi, theta -- radon_grid's output (backprojection init.c:
 * 117-153).  OUT: one column "%lf" in the order z, x, y
 * (radon3d_ajoint.c:240-254), plus readme_OUT. */
#include <stdlib.h>

#include "cli_common.h"

static int row(char *buf, size_t k, const void *c) {
  return sprintf(buf, "%lf\n", ((const double *)c)[k]);
}

int main(int argc, char **argv) {
  cli_args a;
  cli_parse(argc, argv, &a, "-p (filename) -i (filename) -o (filename) -n (number)", 0, 0);
  int p[4];
  printf("  Reading parameters from %s...", a.params);
  if (cli_read_params(a.params, p)) {
    fprintf(stderr, "Aborting : init_parameters.\n");
    return EXIT_FAILURE;
  }
  printf("Done.\n");
  const int nphi = p[0], ntheta = p[1], nshift = p[2], ngrid = p[3];
  if (nphi < 1 || ntheta < 1 || nshift < 3 || ngrid < 1) {
    fprintf(stderr, "Aborting : invalid grid parameters %d %d %d %d\n", nphi, ntheta, nshift, ngrid);
    return EXIT_FAILURE;
  }
  const size_t nin = (size_t)nshift * nphi * ntheta, nout = (size_t)ngrid * ngrid * ngrid;
  double *radon = malloc(sizeof(double) * nin), *out = malloc(sizeof(double) * nout);
  if (!radon || !out) {
    fprintf(stderr, "Aborting : out of host memory\n");
    return EXIT_FAILURE;
  }
  printf("  Reading Radon transforms...");
  if (cli_read_csv4(a.input, nin, radon, a.nthreads)) {
    fprintf(stderr, "Aborting : radon_values_init.\n");
    return EXIT_FAILURE;
  }
  printf("Done.\n\n");
  wrt_ctx *ctx = cli_context(&a);
  double t0 = cli_now();
  cli_die_status(ctx, wrt_radon3d_adjoint(ctx, radon, nphi, ntheta, nshift, ngrid, out),
                 "radon3d_adjoint");
  printf("  Adjoint on device %d, elapsed time: %3.3f sec\n", a.device, cli_now() - t0);
  cli_readme(a.output,
             "  Radon transforms in 3D were taken in %s\n"
             "  Parameters of the input data:\n"
             "     number of angles of [phi]  : %d\n"
             "     number of angles of [theta]: %d\n"
             "     number of shifts of [s]    : %d\n"
             "  Output of adjoint transform was stored in %s\n"
             "  Parameters of the output data:\n"
             "     number of points on the grid: %d\n",
             a.input, nphi, ntheta, nshift, a.output, ngrid);
  if (cli_write_rows(a.output, nout, row, out, a.nthreads)) return EXIT_FAILURE;
  if (a.binary && cli_write_binary(a.output, out, nout)) return EXIT_FAILURE;
  wrt_ctx_destroy(ctx);
  free(radon); free(out);
  return EXIT_SUCCESS;
}
