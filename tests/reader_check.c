/* CPU check of the drop-in programs' parallel text reader (cli/cli_common.c):
 * files of "%lf" lines and "%lf, %lf, %lf, %lf" lines are read with 1, 3, 8
 * and 16 threads and must give exactly the values of a serial strtod parse;
 * a truncated file and a malformed line must be refused; a FIFO (a stream
 * that cannot seek) must read like the file it carries. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <sys/wait.h>
#include <unistd.h>

#include "cli_common.h"

static int write_file(const char *path, const double *v, size_t n, int columns, int bad_line) {
  FILE *f = fopen(path, "w");
  if (!f) return -1;
  for (size_t k = 0; k < n; ++k) {
    if ((int)k == bad_line) fprintf(f, "x%lf\n", v[k]);
    else if (columns == 1) fprintf(f, "%lf\n", v[k]);
    else fprintf(f, "%lf, %lf, %lf, %lf\n", 0.5 * k, -1.0, 2.0, v[k]);
    if (k % 1000 == 7) fprintf(f, "\n");  /* blank lines are whitespace */
  }
  fclose(f);
  return 0;
}

int main(int argc, char **argv) {
  const char *dir = argc > 1 ? argv[1] : ".";
  char path[4096];
  const size_t n = 600000;
  double *v = malloc(n * sizeof(double)), *got = malloc(n * sizeof(double));
  srand(12345);
  for (size_t k = 0; k < n; ++k) v[k] = (rand() / (double)RAND_MAX - 0.5) * 1e3;
  for (int columns = 1; columns <= 4; columns += 3) {
    snprintf(path, sizeof path, "%s/values_%d.txt", dir, columns);
    write_file(path, v, n, columns, -1);
    /* what "%lf" printed: the expected values */
    double *want = malloc(n * sizeof(double));
    for (size_t k = 0; k < n; ++k) {
      char b[64];
      snprintf(b, sizeof b, "%lf", v[k]);
      want[k] = strtod(b, NULL);
    }
    int threads[] = {1, 3, 8, 16};
    for (int t = 0; t < 4; ++t) {
      memset(got, 0, n * sizeof(double));
      int rc = columns == 1 ? cli_read_column(path, n, got, threads[t])
                            : cli_read_csv4(path, n, got, threads[t]);
      if (rc || memcmp(got, want, n * sizeof(double))) {
        printf("FAIL columns=%d threads=%d rc=%d\n", columns, threads[t], rc);
        return 1;
      }
      /* fewer values than the file holds: the first ones */
      if (cli_read_column(path, 1000, got, threads[t]) && columns == 1) {
        printf("FAIL prefix read\n");
        return 1;
      }
    }
    /* the same text through a FIFO, written by a child process */
    char fifo[4096];
    snprintf(fifo, sizeof fifo, "%s/fifo_%d", dir, columns);
    unlink(fifo);
    if (mkfifo(fifo, 0600) != 0) {
      printf("FAIL mkfifo\n");
      return 1;
    }
    pid_t child = fork();
    if (child == 0) {
      FILE *src = fopen(path, "rb"), *dst = fopen(fifo, "wb");
      char chunk[1 << 16];
      size_t m;
      while (src && dst && (m = fread(chunk, 1, sizeof chunk, src)) > 0) fwrite(chunk, 1, m, dst);
      const int ok = src && dst && fclose(dst) == 0; /* _exit flushes no stdio buffer */
      _exit(ok ? 0 : 1);
    }
    memset(got, 0, n * sizeof(double));
    int frc = columns == 1 ? cli_read_column(fifo, n, got, 8) : cli_read_csv4(fifo, n, got, 8);
    int status = 0;
    waitpid(child, &status, 0);
    unlink(fifo);
    if (frc || memcmp(got, want, n * sizeof(double)) || !WIFEXITED(status) || WEXITSTATUS(status)) {
      printf("FAIL fifo columns=%d rc=%d\n", columns, frc);
      return 1;
    }
    /* more values than the file holds: refused */
    if ((columns == 1 ? cli_read_column(path, n + 1, got, 8) : cli_read_csv4(path, n + 1, got, 8)) == 0) {
      printf("FAIL truncated file accepted\n");
      return 1;
    }
    /* a malformed line in the middle: refused */
    snprintf(path, sizeof path, "%s/bad_%d.txt", dir, columns);
    write_file(path, v, n, columns, (int)(n / 2));
    if ((columns == 1 ? cli_read_column(path, n, got, 8) : cli_read_csv4(path, n, got, 8)) == 0) {
      printf("FAIL malformed line accepted\n");
      return 1;
    }
    free(want);
  }
  printf("ok\n");
  return 0;
}
