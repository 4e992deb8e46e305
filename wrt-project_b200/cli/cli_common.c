/* cli_common.c -- argument parsing, text I/O and a parallel formatter for the
 * drop-in programs.  See cli_common.h for the contract. */
#define _GNU_SOURCE
#include "cli_common.h"

#include <errno.h>
#include <getopt.h>
#include <pthread.h>
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

double cli_now(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return t.tv_sec + 1e-9 * t.tv_nsec;
}

static void usage_exit(const char *prog, const char *usage, int flags, FILE *s, int code) {
  fprintf(s, "Usage: %s %s\n", prog, usage);
  fprintf(s, "   -h --help                 Display this usage information.\n"
             "   -p --parameters filename  Read the grid parameters from file.\n");
  if (!(flags & CLI_FUNCTION))
    fprintf(s, "   -i --input filename       Read input data from file.\n");
  fprintf(s, "   -o --output filename      Write output data to the file.\n"
             "   -n --nthreads number      Number of host threads (text formatting).\n");
  if (flags & CLI_FUNCTION)
    fprintf(s, "      --function name        The test function: exponential_bump or\n"
               "                             sinusoidal_bump (the reference's examples).\n");
  fprintf(s, "      --device N             CUDA device ordinal (default 0).\n"
             "      --binary               Also write OUTPUT.bin (raw FP64 results).\n");
  exit(code);
}

void cli_parse(int argc, char **argv, cli_args *a, const char *usage, int allow_small,
               int allow_sampler) {
  cli_parse_flags(argc, argv, a, usage,
                  (allow_small ? CLI_SMALL : 0) | (allow_sampler ? CLI_SAMPLER : 0));
}

void cli_parse_flags(int argc, char **argv, cli_args *a, const char *usage, int flags) {
  const int allow_small = flags & CLI_SMALL, allow_sampler = flags & CLI_SAMPLER;
  const int allow_function = flags & CLI_FUNCTION;
  memset(a, 0, sizeof(*a));
  a->nthreads = 1;
  a->sampler = WRT_SAMPLER_NEAREST;
  a->function = -1;
  if (argc == 1) {
    fprintf(stderr, "%s: arguments required. Try '-h' or '--help'.\n", argv[0]);
    exit(EXIT_FAILURE);
  }
  enum { OPT_DEVICE = 1000, OPT_BINARY, OPT_SAMPLER, OPT_HALF, OPT_FUNCTION };
  const struct option longopts[] = {
      {"help", no_argument, 0, 'h'},          {"parameters", required_argument, 0, 'p'},
      {"input", required_argument, 0, 'i'},   {"output", required_argument, 0, 'o'},
      {"nthreads", required_argument, 0, 'n'}, {"small", no_argument, 0, 's'},
      {"device", required_argument, 0, OPT_DEVICE}, {"binary", no_argument, 0, OPT_BINARY},
      {"sampler", required_argument, 0, OPT_SAMPLER},
      {"half-extent", required_argument, 0, OPT_HALF},
      {"function", required_argument, 0, OPT_FUNCTION}, {0, 0, 0, 0}};
  /* the analytic programs take no input file (radon_analytic.c:131) */
  const char *shortopts = allow_function ? "hp:o:n:" : allow_small ? "hp:i:so:n:" : "hp:i:o:n:";
  int c;
  while ((c = getopt_long(argc, argv, shortopts, longopts, NULL)) != -1) {
    switch (c) {
      case 'h': usage_exit(argv[0], usage, flags, stdout, 0); break;
      case 'p': a->params = optarg; printf("Parameters file: %s\n", optarg); break;
      case 'i':
        if (allow_function) usage_exit(argv[0], usage, flags, stderr, 1);
        a->input = optarg;
        printf("Input file: %s\n", optarg);
        break;
      case 'o': a->output = optarg; printf("Output file: %s\n", optarg); break;
      case 'n':
        a->nthreads = atoi(optarg);
        if (a->nthreads <= 0) {
          fprintf(stderr, "%s: -n expects a positive number\n", argv[0]);
          exit(EXIT_FAILURE);
        }
        printf("Number of threads: %d\n", a->nthreads);
        break;
      case 's':
        if (!allow_small) usage_exit(argv[0], usage, flags, stderr, 1);
        a->small_format = 1;
        printf("Reading of the input in small format\n");
        break;
      case OPT_DEVICE: a->device = atoi(optarg); break;
      case OPT_BINARY: a->binary = 1; break;
      case OPT_SAMPLER:
        if (!allow_sampler) usage_exit(argv[0], usage, flags, stderr, 1);
        if (!strcmp(optarg, "nearest")) a->sampler = WRT_SAMPLER_NEAREST;
        else if (!strcmp(optarg, "trilinear")) a->sampler = WRT_SAMPLER_TRILINEAR;
        else usage_exit(argv[0], usage, flags, stderr, 1);
        break;
      case OPT_HALF:
        if (!allow_sampler) usage_exit(argv[0], usage, flags, stderr, 1);
        a->half_extent = atoi(optarg);
        break;
      case OPT_FUNCTION:
        if (!allow_function) usage_exit(argv[0], usage, flags, stderr, 1);
        if (!strcmp(optarg, "exponential_bump")) a->function = WRT_FUNCTION_EXP_BUMP;
        else if (!strcmp(optarg, "sinusoidal_bump")) a->function = WRT_FUNCTION_SINE_BUMPS;
        else {
          fprintf(stderr, "%s: unknown test function '%s' (exponential_bump or sinusoidal_bump)\n",
                  argv[0], optarg);
          exit(EXIT_FAILURE);
        }
        printf("Test function: %s\n", optarg);
        break;
      default: usage_exit(argv[0], usage, flags, stderr, 1);
    }
  }
  if (optind < argc) printf("Warning: non-option ARGV-arguments are omitted. See '-h' or '--help'.\n");
  if (allow_function) {
    if (!a->params || !a->output) {
      fprintf(stderr, "%s: -p and -o are required. Try '-h' or '--help'.\n", argv[0]);
      exit(EXIT_FAILURE);
    }
    if (a->function < 0) {
      fprintf(stderr, "%s: --function is required: exponential_bump or sinusoidal_bump (the "
                      "reference compiles its test function in). Try '-h' or '--help'.\n", argv[0]);
      exit(EXIT_FAILURE);
    }
  } else if (!a->params || !a->input || !a->output) {
    fprintf(stderr, "%s: -p, -i and -o are required. Try '-h' or '--help'.\n", argv[0]);
    exit(EXIT_FAILURE);
  }
}

int cli_read_params(const char *path, int p[4]) { return cli_read_params_n(path, p, 4); }

int cli_read_params_n(const char *path, int *p, int count) {
  FILE *f = fopen(path, "r");
  if (!f) {
    fprintf(stderr, "Recieved call %s while opening %s. \n", strerror(errno), path);
    return -1;
  }
  char buffer[4096];
  for (int k = 0; k < count; ++k) {
    const int got = fscanf(f, "%d %4095[^\n]\n", &p[k], buffer);
    if (got == EOF) {
      fprintf(stderr, "Error: fscanf parameters %d : reached end of file before it was expected.\n", k);
      fclose(f);
      return -1;
    } else if (got != 2) {
      fprintf(stderr, "Error: fscanf parameters %d : matching failure, fscanf expected 1 integer value.\n", k);
      fclose(f);
      return -1;
    }
  }
  fclose(f);
  return 0;
}

/* A stream that cannot seek (a pipe, a FIFO, /dev/stdin: the reference's
 * "%lf" loop reads those too), read to its end into a growing buffer. */
static char *slurp_stream(FILE *f, size_t *len) {
  size_t cap = (size_t)1 << 20, n = 0;
  char *buf = malloc(cap + 1);
  while (buf) {
    n += fread(buf + n, 1, cap - n, f);
    if (n < cap) break; /* end of stream or a read error */
    char *nb = realloc(buf, 2 * cap + 1);
    if (!nb) {
      free(buf);
      buf = NULL;
      break;
    }
    buf = nb;
    cap *= 2;
  }
  if (buf && ferror(f)) {
    free(buf);
    buf = NULL;
  }
  if (buf) {
    buf[n] = 0;
    *len = n;
  }
  return buf;
}

/* Whole-file read; returns a NUL-terminated buffer or NULL. */
static char *slurp(const char *path, size_t *len) {
  FILE *f = fopen(path, "rb");
  if (!f) {
    fprintf(stderr, "Recieved call %s while opening %s. \n", strerror(errno), path);
    return NULL;
  }
  long n = -1;
  if (fseek(f, 0, SEEK_END) == 0) {
    n = ftell(f);
    if (fseek(f, 0, SEEK_SET) != 0) n = -1;
  }
  char *buf = NULL;
  if (n < 0) {
    buf = slurp_stream(f, len);
  } else {
    buf = malloc((size_t)n + 1);
    if (buf && fread(buf, 1, (size_t)n, f) == (size_t)n) {
      buf[n] = 0;
      *len = (size_t)n;
    } else {
      free(buf);
      buf = NULL;
    }
  }
  if (!buf) fprintf(stderr, "Error: could not read %s\n", path);
  fclose(f);
  return buf;
}

/* One chunk of the input text, [p, end), parsed on its own thread: every
 * record (one value, or the 4th of four comma-separated values) into a
 * growable array.  err: 0, 1 (matching failure at record `bad`), 2 (no memory). */
typedef struct {
  const char *p, *end;
  int columns;
  double *vals;
  size_t n, cap, bad;
  int err;
} parse_job;

static void *parse_worker(void *arg) {
  parse_job *j = arg;
  const char *p = j->p;
  while (p < j->end && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n')) ++p;
  while (p < j->end) {
    double v = 0;
    for (int c = 0; c < j->columns; ++c) {
      char *stop;
      v = strtod(p, &stop);
      if (stop == p || stop > j->end) {
        j->err = 1;
        j->bad = j->n;
        return NULL;
      }
      p = stop;
      while (*p == ' ' || *p == '\t') ++p;
      if (c + 1 < j->columns) {
        if (*p != ',') {
          j->err = 1;
          j->bad = j->n;
          return NULL;
        }
        ++p;
      }
    }
    if (j->n == j->cap) {
      size_t cap = j->cap ? 2 * j->cap : 1 << 16;
      double *nv = realloc(j->vals, cap * sizeof(double));
      if (!nv) {
        j->err = 2;
        return NULL;
      }
      j->vals = nv;
      j->cap = cap;
    }
    j->vals[j->n++] = v;
    while (p < j->end && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n')) ++p;
  }
  return NULL;
}

/* The first `count` records of the file: the text is cut into nthreads
 * chunks at line ends, parsed in parallel, and the records are taken in file
 * order (the reference's reader is a serial "%lf" loop, init.c:107-139; same
 * values, same error cases). */
static int parse_values(const char *path, size_t count, double *out, int columns, int nthreads) {
  size_t len = 0;
  char *buf = slurp(path, &len);
  if (!buf) return -1;
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  if (len < ((size_t)1 << 20)) nthreads = 1;
  parse_job jobs[256];
  pthread_t th[256];
  const char *cut = buf;
  for (int t = 0; t < nthreads; ++t) {
    const char *e = t + 1 == nthreads ? buf + len : buf + len / nthreads * (t + 1);
    if (e < cut) e = cut;
    while (e < buf + len && *e != '\n') ++e;  /* chunks end at a line end */
    jobs[t] = (parse_job){cut, e, columns, NULL, 0, 0, 0, 0};
    cut = e;
  }
  for (int t = 0; t < nthreads; ++t)
    if (nthreads == 1 || pthread_create(&th[t], NULL, parse_worker, &jobs[t]) != 0) {
      parse_worker(&jobs[t]);
      th[t] = 0;
    }
  for (int t = 0; t < nthreads; ++t)
    if (nthreads > 1 && th[t]) pthread_join(th[t], NULL);
  int rc = 0;
  size_t k = 0;
  for (int t = 0; t < nthreads && k < count && !rc; ++t) {
    size_t take = jobs[t].n < count - k ? jobs[t].n : count - k;
    memcpy(out + k, jobs[t].vals, take * sizeof(double));
    k += take;
    if (jobs[t].err == 1 && k < count) {
      fprintf(stderr, "Error: %s: matching failure at value %zu, expected %d floating-point value(s).\n",
              path, k, columns);
      rc = -1;
    } else if (jobs[t].err == 2) {
      fprintf(stderr, "Error: %s: out of memory while reading\n", path);
      rc = -1;
    }
  }
  if (!rc && k < count) {
    fprintf(stderr,
            "Error: %s: reached the end of file before it was expected (value %zu of %d-column data).\n",
            path, k, columns);
    rc = -1;
  }
  for (int t = 0; t < nthreads; ++t) free(jobs[t].vals);
  free(buf);
  return rc;
}

int cli_read_column(const char *path, size_t count, double *out, int nthreads) {
  return parse_values(path, count, out, 1, nthreads);
}

int cli_read_csv4(const char *path, size_t count, double *out, int nthreads) {
  return parse_values(path, count, out, 4, nthreads);
}

typedef struct {
  size_t lo, hi;
  cli_row_fn row;
  const void *ctx;
  char *buf;
  size_t len;
} fmt_job;

static void *fmt_worker(void *arg) {
  fmt_job *j = arg;
  size_t cap = (j->hi - j->lo) * 64 + 64, len = 0;
  j->buf = malloc(cap);
  for (size_t k = j->lo; k < j->hi && j->buf; ++k) {
    if (cap - len < 256) {
      cap *= 2;
      char *nb = realloc(j->buf, cap);
      if (!nb) {
        free(j->buf);
        j->buf = NULL;
        break;
      }
      j->buf = nb;
    }
    len += (size_t)j->row(j->buf + len, k, j->ctx);
  }
  j->len = len;
  return NULL;
}

int cli_write_rows(const char *path, size_t count, cli_row_fn row, const void *ctx, int nthreads) {
  FILE *f = fopen(path, "w");
  if (!f) {
    fprintf(stderr, "Recieved call %s while opening %s. \n", strerror(errno), path);
    return -1;
  }
  if (nthreads < 1) nthreads = 1;
  const size_t block = 1 << 18;  /* rows per formatting job */
  int rc = 0;
  for (size_t base = 0; base < count && !rc; base += block * (size_t)nthreads) {
    fmt_job jobs[256];
    pthread_t th[256];
    int nj = 0;
    for (int t = 0; t < nthreads && t < 256; ++t) {
      size_t lo = base + (size_t)t * block;
      if (lo >= count) break;
      size_t hi = lo + block < count ? lo + block : count;
      jobs[nj] = (fmt_job){lo, hi, row, ctx, NULL, 0};
      if (nthreads == 1 || pthread_create(&th[nj], NULL, fmt_worker, &jobs[nj]) != 0) {
        fmt_worker(&jobs[nj]);
        th[nj] = 0;
      }
      ++nj;
    }
    for (int t = 0; t < nj; ++t) {
      if (th[t]) pthread_join(th[t], NULL);
      if (!jobs[t].buf || fwrite(jobs[t].buf, 1, jobs[t].len, f) != jobs[t].len) rc = -1;
      free(jobs[t].buf);
    }
  }
  if (fclose(f) != 0) rc = -1;
  if (rc) fprintf(stderr, "Error: failed writing %s\n", path);
  return rc;
}

int cli_write_binary(const char *path, const double *v, size_t count) {
  char name[4096];
  snprintf(name, sizeof(name), "%s.bin", path);
  FILE *f = fopen(name, "wb");
  if (!f) return -1;
  size_t w = fwrite(v, sizeof(double), count, f);
  fclose(f);
  return w == count ? 0 : -1;
}

void cli_readme(const char *output, const char *fmt, ...) {
  char name[4096];
  snprintf(name, sizeof(name), "readme_%s", output);
  FILE *f = fopen(name, "w");
  if (!f) {
    fprintf(stderr, "Warning: could not write %s\n", name);
    return;
  }
  va_list ap;
  va_start(ap, fmt);
  vfprintf(f, fmt, ap);
  va_end(ap);
  fclose(f);
}

void cli_example_function(int kind, wrt_function *f) {
  memset(f, 0, sizeof(*f));
  f->kind = kind;
  if (kind == WRT_FUNCTION_EXP_BUMP) {
    /* examples-test-functions/exponential_bump.c: centre (0.2, 0, 0), 0.5, eps 1e-2 */
    const double p[5] = {0.2, 0.0, 0.0, 0.5, 1e-2};
    f->count = 1;
    memcpy(f->p, p, sizeof(p));
  } else {
    /* examples-test-functions/sinusoidal_bump.c: three balls
     * (centre, amplitude, rin, rout) */
    const double p[18] = {0.0, 0.2, 0.0, 1.0, 0.4, 0.6,  -0.5, 0.0, 0.0, 0.6, 0.3, 0.45,
                          0.0, 0.2, 0.5, 0.3, 0.4, 0.6};
    f->count = 3;
    memcpy(f->p, p, sizeof(p));
  }
}

wrt_ctx *cli_context(const cli_args *a) {
  wrt_ctx *ctx = NULL;
  int st = wrt_ctx_create(a->device, 0, &ctx);
  if (st) {
    fprintf(stderr, "Aborting : no CUDA context on device %d: %s\n", a->device, wrt_status_string(st));
    exit(EXIT_FAILURE);
  }
  return ctx;
}

void cli_die_status(wrt_ctx *ctx, int st, const char *what) {
  if (!st) return;
  fprintf(stderr, "Aborting : %s: %s (%s)\n", what, wrt_status_string(st), wrt_ctx_last_error(ctx));
  exit(EXIT_FAILURE);
}
