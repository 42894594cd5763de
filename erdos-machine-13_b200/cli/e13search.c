/* e13search -- drop-in for the reference's e13search (src/e13search.c:25-45,
   435-513) on one B200, over the C-ABI of libe13b200.so.

     e13search base   machine.txt
     e13search mutant machine.txt
     e13search delete machine.txt FMAX X...
     e13search free machine.txt X CELL...
     e13search freesym machine.txt X LO HI CELL...
     e13search estimate machine.txt PROBES X FMAX LO HI [CELL...]

   Survivors go to stdout in the reference's format, one summary line per X to
   stderr.  estimate prints the reference's four lines; its probes are drawn
   from per-probe streams (at most 2^20 probes), so the numbers are another
   sample of the same estimator: they equal the reference probe for probe, not
   line for line.  Environment: E13_DEVICE (CUDA device, default 0), E13_KERNEL
   (persistent | plain), E13_AUTOTUNE=N (tune the persistent kernel on 1/N of
   the command's jobs before searching; see maybe_autotune).  There is no CPU path:
   without a GPU it exits 1.

   free / freesym keep checkpoints as src/e13gpu.py:349-409 does: E13_CKPT
   names the checkpoint (resumed when it exists), E13_CKPT_SEC the seconds
   between saves (default 1800), and creating <E13_CKPT>.stop stops the run
   cleanly with a checkpoint and exit status 3; the same command resumes it. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "e13.h"

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static e13_ctx *open_ctx(void) {
  const char *d = getenv("E13_DEVICE");
  e13_ctx *ctx = NULL;
  int rc = e13_ctx_create(d ? atoi(d) : 0, &ctx);
  if (rc) {
    fprintf(stderr, "e13search: no usable CUDA device (error %d)\n", rc);
    exit(1);
  }
  return ctx;
}

/* E13_AUTOTUNE=N (N >= 1): before searching, tune the persistent kernel on
   shard 0 of N of each of the command's n jobs, run together (N = 1: the whole
   jobs), and use the result for every search of the command. */
static void maybe_autotune(e13_ctx *ctx, const e13_job *jobs, int n, e13_tuning *tu) {
  const char *a = getenv("E13_AUTOTUNE");
  if (!a || atoi(a) < 1 || n < 1 || tu->kernel != E13_KERNEL_PERSISTENT) return;
  e13_tuning best;
  double ms = 0;
  int rc = e13_autotune_jobs(ctx, jobs, n, atoi(a), tu, &best, &ms);
  if (rc) {
    fprintf(stderr, "autotune failed (error %d): default tuning kept\n", rc);
    return;
  }
  fprintf(stderr,
          "autotune jobs=%d proxy=1/%d: block=%d slice=%d warp_stack=%d pool_low_pct=%d run_skip=%d (%.1f ms)\n", n,
          atoi(a), best.block, best.slice, best.warp_stack, best.pool_low_pct, best.run_skip, ms);
  *tu = best;
}

/* ck: NULL, or the checkpoint of a free / freesym run */
static int run_one(e13_ctx *ctx, const e13_job *job, const e13_tuning *tu, const e13_checkpoint *ck) {
  int cap = 1 << 16;
  e13_survivor *surv = (e13_survivor *)malloc(sizeof(e13_survivor) * (size_t)cap);
  e13_counts c;
  int ns = 0;
  double w0 = now_s(), wall = 0.0;
  int rc;
  if (ck) {
    FILE *pf = fopen(ck->path, "r");
    if (pf) {
      char slot[4] = {0};
      if (fgets(slot, sizeof slot, pf)) fprintf(stderr, "resuming from %s.%c\n", ck->path, slot[0]);
      fclose(pf);
    }
    int64_t left = 0;
    rc = e13_search_resumable(ctx, job, tu, ck, &c, surv, cap, &ns, &wall, &left);
    if (rc == E13_STOPPED) {
      fprintf(stderr, "STOPPED cleanly at wall=%.0fs steps=%.3e survivors=%d stack=%lld; run the same command to "
              "resume\n", wall, (double)c.steps, ns, (long long)left);
      free(surv);
      return E13_STOPPED;
    }
    if (rc == E13_ERR_CKPT) fprintf(stderr, "checkpoint %s is unreadable or for another run\n", ck->path);
  } else {
    rc = e13_search(ctx, job, tu, &c, surv, cap, &ns);
    wall = now_s() - w0;
  }
  if (rc && rc != E13_ERR_SURV_CAP) {
    fprintf(stderr, "X=%d search failed (error %d)\n", job->X, rc);
    free(surv);
    return rc;
  }
  char line[2048];
  int shown = ns < cap ? ns : cap;
  for (int i = 0; i < shown; i++) {
    e13_format_survivor(job, &surv[i], line, sizeof line);
    printf("%s\n", line);
  }
  fflush(stdout);
  e13_format_summary(job, &c, wall, line, sizeof line);
  fprintf(stderr, "%s\n", line);
  if (rc == E13_ERR_SURV_CAP) fprintf(stderr, "WARNING: %d survivors, only %d printed\n", ns, cap);
  fflush(stderr);
  free(surv);
  return 0;
}

int main(int argc, char **argv) {
  if (argc < 3) {
    fprintf(stderr,
            "usage: e13search base|mutant|delete|free|freesym machine.txt [FMAX X...]\n"
            "       e13search estimate machine.txt PROBES X FMAX LO HI [CELL...]   (PROBES <= 1048576; a\n"
            "       different sample than the reference's: equal probe for probe, not line for line)\n");
    return 1;
  }
  int32_t base[E13_MAXCELLS];
  int nq0 = e13_load_machine(argv[2], base);
  if (nq0 < 0) {
    fprintf(stderr, "cannot open %s\n", argv[2]);
    return 1;
  }
  e13_tuning tu;
  e13_default_tuning(&tu);
  const char *k = getenv("E13_KERNEL");
  if (k && !strcmp(k, "plain")) tu.kernel = E13_KERNEL_PLAIN;
  const char *mode = argv[1];

  if (!strcmp(mode, "base") || !strcmp(mode, "mutant")) {
    e13_ctx *ctx = open_ctx();
    if (!strcmp(mode, "base")) {
      int64_t o[7];
      if (e13_run_full(ctx, base, 1, nq0, o)) return 1;
      printf("base states=%d result=%s stage=%lld st0=%lld head0=%lld abs=%lld rel=%lld steps=%lld\n", nq0,
             o[0] ? "SURV" : "DEAD", (long long)o[1], (long long)o[2], (long long)o[3], (long long)o[4],
             (long long)o[5], (long long)o[6]);
    } else {
      int n = 0, cap = 2 * nq0 * (4 * nq0 + 1);
      int32_t *tabs = (int32_t *)malloc(sizeof(int32_t) * E13_MAXCELLS * (size_t)cap);
      int *cell = (int *)malloc(sizeof(int) * (size_t)cap), *val = (int *)malloc(sizeof(int) * (size_t)cap);
      for (int i = 0; i < 2 * nq0; i++)
        for (int v = -1; v < 4 * nq0; v++) {
          if (v == base[i]) continue;
          memcpy(tabs + (size_t)n * E13_MAXCELLS, base, sizeof(int32_t) * E13_MAXCELLS);
          tabs[(size_t)n * E13_MAXCELLS + i] = v;
          cell[n] = i;
          val[n] = v;
          n++;
        }
      int64_t *o = (int64_t *)malloc(sizeof(int64_t) * 7 * (size_t)n);
      if (e13_run_full(ctx, tabs, n, nq0, o)) return 1;
      for (int j = 0; j < n; j++)
        printf("%d %d %lld %lld\n", cell[j], val[j], (long long)o[7 * j + 1], (long long)o[7 * j]);
      free(tabs);
      free(cell);
      free(val);
      free(o);
    }
    e13_ctx_destroy(ctx);
    return 0;
  }
  if (!strcmp(mode, "delete")) {
    if (argc < 5) return 1;
    int fmax = atoi(argv[3]);
    e13_ctx *ctx = open_ctx();
    /* every job set up first, so the autotuner sees them all; the reference's
       messages then come in argument order, between the searches */
    const int na = argc - 4;
    e13_job *jobs = (e13_job *)malloc(sizeof(e13_job) * (size_t)na);
    e13_job *runnable = (e13_job *)malloc(sizeof(e13_job) * (size_t)na);
    int *st = (int *)malloc(sizeof(int) * (size_t)na), n = 0;
    for (int i = 0; i < na; i++) {
      st[i] = e13_setup(base, nq0, atoi(argv[4 + i]), fmax, NULL, -1, -1, &jobs[i]);
      if (st[i] == 0) runnable[n++] = jobs[i];
    }
    maybe_autotune(ctx, runnable, n, &tu);
    for (int i = 0; i < na; i++) {
      if (st[i] == E13_ERR_FMAX) {
        fprintf(stderr, "X=%d forced=%d > fmax\n", jobs[i].X, jobs[i].nforced);
        continue;
      }
      if (st[i]) {
        fprintf(stderr, "X=%d: setup error %d\n", jobs[i].X, st[i]);
        return 1;
      }
      if (run_one(ctx, &jobs[i], &tu, NULL)) return 1;
    }
    free(jobs);
    free(runnable);
    free(st);
    e13_ctx_destroy(ctx);
    return 0;
  }
  if (!strcmp(mode, "free") || !strcmp(mode, "freesym")) {
    if (argc < 4) return 1;
    uint8_t freebase[E13_MAXCELLS] = {0};
    int X = atoi(argv[3]), a0 = 4, lo = -1, hi = -1;
    if (!strcmp(mode, "freesym")) {
      if (argc < 6) return 1;
      lo = atoi(argv[4]);
      hi = atoi(argv[5]);
      a0 = 6;
    }
    for (int i = a0; i < argc; i++) {
      int c = 2 * (argv[i][0] - 'A') + (argv[i][1] - '0');
      if (c >= 0 && c < E13_MAXCELLS) freebase[c] = 1;
    }
    e13_job job;
    int rc = e13_setup(base, nq0, X, 0, freebase, lo, hi, &job);
    if (rc == E13_ERR_SYM_NAMED) {
      fprintf(stderr, "symmetric state is named by a fixed cell or has one\n");
      return 1;
    }
    if (rc == E13_ERR_SYM_START) {
      fprintf(stderr, "start state in the symmetric states\n");
      return 1;
    }
    if (rc) {
      fprintf(stderr, "setup error %d\n", rc);
      return 1;
    }
    /* the run's identity for its checkpoint: mode, arguments and machine file name */
    char config[1024];
    const char *slash = strrchr(argv[2], '/');
    int n = snprintf(config, sizeof config, "%s %s", mode, slash ? slash + 1 : argv[2]);
    for (int i = 3; i < argc && n < (int)sizeof config; i++) n += snprintf(config + n, sizeof config - n, " %s", argv[i]);
    const char *ckpath = getenv("E13_CKPT");
    const char *cksec = getenv("E13_CKPT_SEC");
    e13_checkpoint ck = {ckpath, config, cksec ? atof(cksec) : 1800.0, 0.0};
    e13_ctx *ctx = open_ctx();
    maybe_autotune(ctx, &job, 1, &tu);
    rc = run_one(ctx, &job, &tu, (ckpath && ckpath[0]) ? &ck : NULL);
    e13_ctx_destroy(ctx);
    return rc == E13_STOPPED ? 3 : (rc ? 1 : 0);
  }
  if (!strcmp(mode, "estimate")) {
    /* src/e13search.c:473-510: LO < 0 is no symmetry; cells make it a free search */
    if (argc < 8) return 1;
    long probes = atol(argv[3]);
    int X = atoi(argv[4]), fmax = atoi(argv[5]), lo = atoi(argv[6]), hi = atoi(argv[7]);
    uint8_t freebase[E13_MAXCELLS] = {0};
    for (int i = 8; i < argc; i++) {
      int c = 2 * (argv[i][0] - 'A') + (argv[i][1] - '0');
      if (c >= 0 && c < E13_MAXCELLS) freebase[c] = 1;
    }
    e13_job job;
    int rc = e13_setup(base, nq0, X, fmax, argc > 8 ? freebase : NULL, lo >= 0 ? lo : -1, hi, &job);
    if (rc) return 1;
    const char *seed_env = getenv("E13_SEED");
    e13_ctx *ctx = open_ctx();
    e13_estimate_out eo;
    double w0 = now_s();
    rc = e13_estimate(ctx, &job, probes, seed_env ? strtoull(seed_env, NULL, 10) : 0, &eo, NULL);
    double wall = now_s() - w0;
    e13_ctx_destroy(ctx);
    if (rc) {
      fprintf(stderr, "estimate failed (error %d)\n", rc);
      return 1;
    }
    static const char *name[4] = {"leaves", "nodes", "steps", "survivors"};
    printf("estimate X=%d budget=%d probes=%ld wall=%.1fs\n", X, job.budget, probes, wall);
    for (int j = 0; j < 4; j++)
      printf("  %-9s %.3e  (+- %.1e standard error)\n", name[j], eo.mean[j], eo.std_error[j]);
    return 0;
  }
  fprintf(stderr, "unknown mode %s\n", mode);
  return 1;
}
