/* e13recheck -- drop-in for the reference's recheck (src/recheck.c) on the
   device: reads SURVIVOR lines on stdin, re-runs each machine to stage NMAX
   without hashing and prints "<id>: <verdict>" with recheck's texts, then
   "machines N consistent G failed B" on stderr.
   Usage: e13recheck NMAX < survivors.txt   (E13_DEVICE selects the GPU) */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "e13.h"

int main(int argc, char **argv) {
  int nmax = argc > 1 ? atoi(argv[1]) : 15;
  int cap = 1024, n = 0;
  e13_check_in *in = (e13_check_in *)malloc(sizeof(e13_check_in) * (size_t)cap);
  char line[8192];
  while (fgets(line, sizeof line, stdin)) {
    if (n == cap) {
      cap *= 2;
      in = (e13_check_in *)realloc(in, sizeof(e13_check_in) * (size_t)cap);
    }
    if (e13_parse_survivor_line(line, &in[n])) n++;
  }
  e13_ctx *ctx = NULL;
  const char *d = getenv("E13_DEVICE");
  if (e13_ctx_create(d ? atoi(d) : 0, &ctx)) {
    fprintf(stderr, "e13recheck: no usable CUDA device\n");
    return 1;
  }
  e13_check_out *out = (e13_check_out *)calloc((size_t)(n > 0 ? n : 1), sizeof(e13_check_out));
  int rc = e13_check(ctx, in, n, nmax, E13_CHECK_RECHECK, out);
  if (rc) {
    fprintf(stderr, "e13recheck: device check failed (%d)\n", rc);
    return 1;
  }
  int good = 0;
  char v[8192];
  for (int i = 0; i < n; i++) {
    int ok = e13_format_recheck(&out[i], nmax, v, sizeof v);
    good += ok == 1;
    printf("%d: %s\n", i + 1, v);
  }
  fprintf(stderr, "machines %d consistent %d failed %d\n", n, good, n - good);
  e13_ctx_destroy(ctx);
  free(in);
  free(out);
  return 0;
}
