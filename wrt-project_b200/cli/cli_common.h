/* cli_common.h -- shared pieces of the drop-in programs.
 *
 * The programs keep the reference's command-line and file contract:
 *   -p FILE   parameter file: four lines "%d <text>" (each line must carry
 *             trailing text; radon_grid/src/init.c:30-77)
 *   -i FILE   input data, one "%lf" per line or 4-column "%lf, %lf, %lf, %lf"
 *   -o FILE   output data; a side file readme_<FILE> describes the grid
 *   -n N      thread count (the reference's OpenMP threads; here the threads
 *             of the text formatter -- the output does not depend on it)
 * Long options work (--parameters, --input, --output, --nthreads, --help;
 * the reference's table maps them to 0 and exits, radon_grid.c:106-113).
 * Errors print a message and exit with EXIT_FAILURE, as the reference does.
 */
#ifndef WRT_CLI_COMMON_H
#define WRT_CLI_COMMON_H
#include <stddef.h>
#include <stdio.h>

#include "wrt.h"

typedef struct {
  const char *params, *input, *output;
  int nthreads;
  int small_format; /* radon_reduction -s: one-column ray data */
  int sampler;      /* radon_grid --sampler */
  int half_extent;  /* radon_grid --half-extent */
  int device;
  int binary;       /* also write OUT.bin: raw little-endian FP64 results */
  int function;     /* radon_analytic / ray_analytic --function: a wrt_function_kind, -1 unset */
} cli_args;

/* usage: program-specific usage text; allow_small enables -s/--small. */
void cli_parse(int argc, char **argv, cli_args *a, const char *usage, int allow_small,
               int allow_sampler);
/* The same with option flags: CLI_SMALL (-s/--small), CLI_SAMPLER (--sampler,
 * --half-extent), CLI_FUNCTION (the analytic programs: no -i, --function
 * required). */
enum { CLI_SMALL = 1, CLI_SAMPLER = 2, CLI_FUNCTION = 4 };
void cli_parse_flags(int argc, char **argv, cli_args *a, const char *usage, int flags);
/* Four integers from a parameter file; returns 0 or -1 (message printed). */
int cli_read_params(const char *path, int p[4]);
/* `count` integers, one per line "%d <text>" (ray_analytic reads three). */
int cli_read_params_n(const char *path, int *p, int count);
/* count doubles, one per line ("%lf\n"), parsed by nthreads threads; 0 or -1. */
int cli_read_column(const char *path, size_t count, double *out, int nthreads);
/* count lines "%lf, %lf, %lf, %lf"; keeps the 4th column; 0 or -1. */
int cli_read_csv4(const char *path, size_t count, double *out, int nthreads);
/* Formats rows with `fmt_row(buf, index, ctx)` in parallel chunks and writes
 * them in order; returns 0 or -1. */
typedef int (*cli_row_fn)(char *buf, size_t index, const void *ctx);
int cli_write_rows(const char *path, size_t count, cli_row_fn row, const void *ctx, int nthreads);
int cli_write_binary(const char *path, const double *v, size_t count);
/* "readme_<output>" with the given text (printf-style). */
void cli_readme(const char *output, const char *fmt, ...);
/* The reference's example test function of this kind (WRT_FUNCTION_*) with
 * the constants of its example file. */
void cli_example_function(int kind, wrt_function *f);
wrt_ctx *cli_context(const cli_args *a);
void cli_die_status(wrt_ctx *ctx, int st, const char *what);
double cli_now(void);

#endif
