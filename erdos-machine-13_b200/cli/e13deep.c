/* e13deep -- drop-in for the reference's deep (src/deep.c) on the device:
   per SURVIVOR line on stdin, "survivor <id> (nq=.. st0=..): n1:c@left ..."
   up to stage NMAX or the first failure.
   Usage: e13deep NMAX < survivors.txt   (E13_DEVICE selects the GPU) */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "e13.h"

int main(int argc, char **argv) {
  int nmax = argc > 1 ? atoi(argv[1]) : 16;
  int cap = 1024, n = 0;
  e13_check_in *in = (e13_check_in *)malloc(sizeof(e13_check_in) * (size_t)cap);
  char line[8192];
  while (fgets(line, sizeof line, stdin)) {
    if (!strstr(line, "st0=")) continue;
    if (n == cap) {
      cap *= 2;
      in = (e13_check_in *)realloc(in, sizeof(e13_check_in) * (size_t)cap);
    }
    if (e13_parse_survivor_line(line, &in[n])) n++;
  }
  e13_ctx *ctx = NULL;
  const char *d = getenv("E13_DEVICE");
  if (e13_ctx_create(d ? atoi(d) : 0, &ctx)) {
    fprintf(stderr, "e13deep: no usable CUDA device\n");
    return 1;
  }
  e13_check_out *out = (e13_check_out *)calloc((size_t)(n > 0 ? n : 1), sizeof(e13_check_out));
  if (e13_check(ctx, in, n, nmax, E13_CHECK_DEEP, out)) {
    fprintf(stderr, "e13deep: device check failed\n");
    return 1;
  }
  char v[8192];
  for (int i = 0; i < n; i++) {
    e13_format_deep(&in[i], &out[i], nmax, v, sizeof v);
    printf("survivor %d %s\n", i + 1, v);
  }
  e13_ctx_destroy(ctx);
  free(in);
  free(out);
  return 0;
}
