/* e13check -- drop-in for the reference's `python src/check.py FILE` on one
   B200, over the C-ABI of libe13b200.so.

     e13check survivors.txt

   For every line with "table=" it prints the line and check.py's verdict per
   placement of the halt ("   halt@<place>: PASS|FAIL ..."), computed by the
   device (stage walk to n = 11, crafted stage starts).  Environment:
   E13_DEVICE (CUDA device, default 0).  Without a GPU it exits 1. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "e13.h"

int main(int argc, char **argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: e13check survivors.txt\n");
    return 1;
  }
  FILE *f = fopen(argv[1], "r");
  if (!f) {
    fprintf(stderr, "cannot open %s\n", argv[1]);
    return 1;
  }
  char **lines = NULL;
  int n = 0, cap = 0;
  char buf[1 << 14];
  while (fgets(buf, sizeof buf, f)) {
    if (n == cap) {
      cap = cap ? 2 * cap : 256;
      lines = (char **)realloc(lines, sizeof(char *) * (size_t)cap);
    }
    lines[n++] = strdup(buf);
  }
  fclose(f);
  const char *d = getenv("E13_DEVICE");
  e13_ctx *ctx = NULL;
  int rc = e13_ctx_create(d ? atoi(d) : 0, &ctx);
  if (rc) {
    fprintf(stderr, "e13check: no usable CUDA device (error %d)\n", rc);
    return 1;
  }
  size_t len = 1 << 20, need = 0;
  char *out = (char *)malloc(len);
  rc = e13_check_crafted(ctx, (const char *const *)lines, n, out, len, &need);
  if (rc == E13_ERR_ARG && need > len) {
    out = (char *)realloc(out, need);
    len = need;
    rc = e13_check_crafted(ctx, (const char *const *)lines, n, out, len, &need);
  }
  e13_ctx_destroy(ctx);
  if (rc && rc != E13_ERR_OVERFLOW) {
    fprintf(stderr, "e13check failed (error %d)\n", rc);
    return 1;
  }
  fputs(out, stdout);
  if (rc == E13_ERR_OVERFLOW) fprintf(stderr, "WARNING: a counter exceeded %d cells; its line is not exact\n", E13_CRAFTED_MAX_CELLS);
  for (int i = 0; i < n; i++) free(lines[i]);
  free(lines);
  free(out);
  return rc ? 1 : 0;
}
