/*
 * e13_host.c -- host side of libe13b200.so: Zobrist keys, machine files,
 * candidate construction and the reference's text formats.  No device code.
 *
 * Reference behaviour followed (paths within the reference project):
 *   src/e13search.c :98-103 splitmix, :437-444 KEY/TGT, :105-121 parse/load,
 *                   :317-355 setup, :423-426 set_sym, :179-200 report,
 *                   :413-416 summary line
 *   src/recheck.c   :28-56 survivor-line parsing, :71-99 verdict texts
 *   src/deep.c      :53-81 per-stage text
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "e13.h"

static uint64_t splitmix_step(uint64_t *s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

void e13_keys(uint64_t key[1364], uint64_t tgt[E13_STAGES + 1]) {
  uint64_t s = 20261028ULL; /* the reference's seed (src/e13search.c:437) */
  uint64_t k[1364];
  for (int p = 0; p < 1364; p++) k[p] = splitmix_step(&s);
  if (key) memcpy(key, k, sizeof k);
  if (tgt) {
    tgt[0] = 0;
    for (int n = 1; n <= E13_STAGES; n++) {
      uint64_t h = 0;
      for (int c = -1; c <= (1 << n) - 2; c++) h ^= k[c + E13_TAPE_LEFT];
      tgt[n] = h;
    }
  }
}

int e13_parse_cell(const char *s) {
  if (!s || s[0] == '-') return E13_HALT;
  return (atoi(s + 2) << 2) | ((s[1] == 'R') << 1) | (s[0] - '0');
}

int e13_parse_machine(const char *text, int32_t base[E13_MAXCELLS]) {
  if (!text || !base) return E13_ERR_ARG;
  int nq = 0;
  const char *p = text;
  char a[16], b[16];
  int used;
  for (int i = 0; i < E13_MAXCELLS; i++) base[i] = E13_HALT;
  while (nq < E13_MAXQ && sscanf(p, "%15s %15s%n", a, b, &used) == 2) {
    base[2 * nq] = e13_parse_cell(a);
    base[2 * nq + 1] = e13_parse_cell(b);
    nq++;
    p += used;
  }
  return nq;
}

int e13_load_machine(const char *path, int32_t base[E13_MAXCELLS]) {
  if (!path || !base) return E13_ERR_ARG;
  FILE *f = fopen(path, "r");
  if (!f) return E13_ERR_IO;
  char buf[4096];
  size_t n = fread(buf, 1, sizeof buf - 1, f);
  fclose(f);
  buf[n] = 0;
  return e13_parse_machine(buf, base);
}

int e13_setup(const int32_t *base, int nq0, int X, int fmax, const uint8_t *free_cells, int lo, int hi,
              e13_job *job) {
  if (!base || !job || nq0 < 1 || nq0 > E13_MAXQ || X >= nq0 || X < -1) return E13_ERR_ARG;
  memset(job, 0, sizeof *job);
  for (int i = 0; i < E13_MAXCELLS; i++) job->tab[i] = E13_HALT;
  job->X = X;
  job->nq = nq0 - (X >= 0);
  job->sym_lo = job->sym_hi = -1;
  int nF = 0, row = 0;
  for (int q = 0; q < nq0; q++) {
    if (q == X) continue;
    for (int a = 0; a < 2; a++) {
      int code = base[2 * q + a];
      if (free_cells && free_cells[2 * q + a]) {
        code = E13_FREE;
      } else if (code >= 0 && (code >> 2) == X) {
        code = E13_FREE; /* a rule into the deleted state */
        nF++;
      } else if (code >= 0) {
        int nx = code >> 2;
        if (X >= 0 && nx > X) nx--; /* renumber the states above X */
        code = (nx << 2) | (code & 3);
      }
      job->tab[2 * row + a] = code;
    }
    row++;
  }
  job->nforced = nF;
  /* symmetry is on only if the renumbered LO is >= 0 (src/e13search.c:336,
     :424): with no deleted state (X = -1) LO..HI shift down by one, so LO = 0
     turns it off */
  const int slo = lo >= 0 ? lo - (lo > X) : -1, shi = lo >= 0 ? hi - (hi >= X) : -1;
  if (slo >= 0) {
    int n0 = 0;
    uint8_t named[E13_MAXQ + 1] = {0};
    job->sym_lo = slo;
    job->sym_hi = shi;
    /* an empty range (HI < LO after renumbering) is accepted and changes
       nothing, as in the reference; one past the last state is refused (the
       reference would read past its table there) */
    if (shi >= job->nq) return E13_ERR_ARG;
    /* the reference scans the first 2*(NQ-1) cells, also when X < 0 */
    for (int i = 0; i < 2 * (nq0 - 1); i++) {
      int c = job->tab[i];
      if (c >= 0 && (c >> 2) >= slo && (c >> 2) <= shi) named[(c >> 2) - slo] = 1;
    }
    while (n0 <= shi - slo && named[n0]) n0++;
    for (int q = slo + n0; q <= shi; q++)
      if (named[q - slo] || job->tab[2 * q] != E13_FREE || job->tab[2 * q + 1] != E13_FREE) return E13_ERR_SYM_NAMED;
    if (slo == 0) return E13_ERR_SYM_START;
    job->sym_n0 = n0;
  }
  if (free_cells) fmax = nF; /* free mode: nothing but the free and forced cells changes */
  if (nF > fmax) {
    job->budget = -1;
    return E13_ERR_FMAX;
  }
  job->budget = fmax - nF;
  return E13_OK;
}

static int put_cell(char *b, size_t len, int code) {
  if (code < 0) return snprintf(b, len, "---");
  return snprintf(b, len, "%d%c%d", code & 1, (code & 2) ? 'R' : 'L', code >> 2);
}

int e13_format_survivor(const e13_job *job, const e13_survivor *s, char *buf, size_t len) {
  if (!job || !s || !buf || len < 64) return E13_ERR_ARG;
  int n = snprintf(buf, len, "SURVIVOR X=%d st0=%d head0=%d abs=%d rel=%d steps=%lld table=", job->X, s->st0,
                   s->head0, s->abs_ok, s->rel_ok, (long long)s->steps);
  for (int q = 0; q < job->nq && (size_t)n < len; q++) {
    for (int a = 0; a < 2 && (size_t)n < len; a++) {
      int i = 2 * q + a;
      if (!((s->read_mask >> i) & 1)) n += snprintf(buf + n, len - (size_t)n, "?");
      if ((size_t)n < len) n += put_cell(buf + n, len - (size_t)n, s->tab[i] == E13_FREE ? E13_HALT : s->tab[i]);
      if (a == 0 && (size_t)n < len) n += snprintf(buf + n, len - (size_t)n, " ");
    }
    if (q + 1 < job->nq && (size_t)n < len) n += snprintf(buf + n, len - (size_t)n, "|");
  }
  if ((size_t)n >= len) return E13_ERR_ARG;
  return n;
}

int e13_format_summary(const e13_job *job, const e13_counts *c, double wall_s, char *buf, size_t len) {
  if (!job || !c || !buf) return E13_ERR_ARG;
  int n = snprintf(buf, len, "X=%d budget=%d leaves=%llu survivors=%llu steps=%llu wall=%.1fs dead-at-stage(0..%d):",
                   job->X, job->budget, (unsigned long long)c->leaves, (unsigned long long)c->survivors,
                   (unsigned long long)c->steps, wall_s, E13_STAGES);
  for (int j = 0; j <= E13_STAGES && (size_t)n < len; j++)
    n += snprintf(buf + n, len - (size_t)n, " %llu", (unsigned long long)c->hist[j]);
  return n;
}

void e13_default_tuning(e13_tuning *t) {
  if (!t) return;
  memset(t, 0, sizeof *t);
  t->kernel = E13_KERNEL_PERSISTENT;
  t->block = 768;
  t->slice = 24;  /* iterations of two actions each */
  t->warp_stack = 256;
  t->step_cap = 20000;
  t->batch = 0;
  t->epoch_us = 200000;
  t->epochs_per_graph = 4;
  t->pool_low_pct = 5;
  t->run_skip = 8192;
  t->stack_nodes = 0;
}

int e13_resolve_tuning(const e13_tuning *in, int serve, e13_tuning *out) {
  if (!out) return E13_ERR_ARG;
  e13_tuning t;
  e13_default_tuning(&t);
  if (serve) t.epoch_us = 10000; /* short epochs: jobs join and leave at every epoch boundary */
  if (in) {
    if (in->kernel != E13_KERNEL_PLAIN && in->kernel != E13_KERNEL_PERSISTENT) return E13_ERR_ARG;
    if (in->run_skip < 0) return E13_ERR_ARG;
    if (in->block < 0 || in->slice < 0 || in->warp_stack < 0 || in->step_cap < 0 || in->batch < 0 ||
        in->epoch_us < 0 || in->epochs_per_graph < 0 || in->pool_low_pct < 0 || in->stack_nodes < 0)
      return E13_ERR_ARG;
    t.kernel = in->kernel;
    t.run_skip = in->run_skip;
    if (in->block) t.block = in->block;
    if (in->slice) t.slice = in->slice;
    if (in->warp_stack) t.warp_stack = in->warp_stack;
    if (in->step_cap) t.step_cap = in->step_cap;
    if (in->batch) t.batch = in->batch;
    if (in->epoch_us) t.epoch_us = in->epoch_us;
    if (in->epochs_per_graph) t.epochs_per_graph = in->epochs_per_graph;
    if (in->pool_low_pct) t.pool_low_pct = in->pool_low_pct;
    if (in->stack_nodes) t.stack_nodes = in->stack_nodes;
  }
  if (serve) t.kernel = E13_KERNEL_PERSISTENT;
  if (t.block < 64 || t.block > 768 || t.block % 32) return E13_ERR_ARG;
  if (t.slice > 4096 || t.warp_stack > 4096) return E13_ERR_ARG;
  if (t.epochs_per_graph > 64 || t.pool_low_pct > 100) return E13_ERR_ARG;
  if (t.epoch_us > 60 * 1000 * 1000) return E13_ERR_ARG; /* one epoch at most a minute: checkpoints and stops stay timely */
  *out = t;
  return E13_OK;
}

/* ------------------------------------------------------------------ */
/* checker text formats                                                */

int e13_parse_survivor_line(const char *line, e13_check_in *in) {
  if (!line || !in) return 0;
  const char *tb = strstr(line, "table=");
  if (!tb) return 0;
  memset(in, 0, sizeof *in);
  int st0 = 0, abs_ok = 1, rel_ok = 0;
  long long head0 = -2;
  const char *p;
  if ((p = strstr(line, "st0="))) st0 = atoi(p + 4);
  if ((p = strstr(line, "head0="))) head0 = atoi(p + 6);
  if ((p = strstr(line, "abs="))) abs_ok = atoi(p + 4);
  if ((p = strstr(line, "rel="))) rel_ok = atoi(p + 4);
  in->st0 = st0;
  in->head0 = head0;
  in->rel = !abs_ok && rel_ok;
  char *q = (char *)tb + 6;
  int nq = 0;
  while (*q && *q != '\n' && *q != '\r' && nq < E13_MAXQ) {
    for (int a = 0; a < 2; a++) {
      int i = 2 * nq + a;
      while (*q == ' ') q++;
      int unread = 0;
      if (*q == '?') { unread = 1; q++; }
      if (*q == '-') {
        in->kind[i] = unread ? 2 : 1;
        q += 3;
      } else {
        in->kind[i] = 0;
        in->write[i] = (int8_t)(*q++ - '0');
        in->move[i] = (*q++ == 'R') ? 1 : -1;
        in->next[i] = (int8_t)strtol(q, &q, 10);
      }
    }
    nq++;
    while (*q == ' ') q++;
    if (*q == '|') q++;
    else break;
  }
  in->nq = nq;
  return 1;
}

int e13_survivor_check_in(const e13_job *job, const e13_survivor *s, e13_check_in *in) {
  if (!job || !s || !in || job->nq < 1 || job->nq > E13_MAXQ) return E13_ERR_ARG;
  memset(in, 0, sizeof *in);
  in->nq = job->nq;
  in->st0 = s->st0;
  in->head0 = s->head0;
  in->rel = !s->abs_ok && s->rel_ok;
  for (int i = 0; i < 2 * job->nq; i++) {
    const int c = s->tab[i];
    if (c < 0) {  /* halt or free cell: "---", never read when '?' */
      in->kind[i] = ((s->read_mask >> i) & 1u) ? 1 : 2;
    } else {
      in->kind[i] = 0;
      in->write[i] = (int8_t)(c & 1);
      in->move[i] = (c & 2) ? 1 : -1;
      in->next[i] = (int8_t)(c >> 2);
    }
  }
  return E13_OK;
}

/* counter set of stage n as recheck prints it: "-3,-5," ("" = none) */
static int counter_text(const e13_check_out *o, int n, char *b, size_t len) {
  int w = 0;
  b[0] = 0;
  int k = o->nones[n] < E13_CHECK_MAX_ONES ? o->nones[n] : E13_CHECK_MAX_ONES;
  for (int j = 0; j < k && w < 8000 && (size_t)w < len; j++)
    w += snprintf(b + w, len - (size_t)w, "%d,", o->ones_cells[n][j]);
  return w;
}

int e13_format_recheck(const e13_check_out *o, int nmax, char *buf, size_t len) {
  if (!o || !buf) return E13_ERR_ARG;
  static const int first_of[3] = {1, 3, 9};
  char a[2048], b[2048], c9[2048];
  /* stages before a failure were all consistent, or the loop would have stopped earlier */
  int done = o->stages_done;
  for (int n = 1; n <= done; n++) {
    int c = n <= 2 ? 0 : (n <= 8 ? 1 : 2);
    int first = first_of[c];
    if (n != first) {
      counter_text(o, first, a, sizeof a);
      counter_text(o, n, b, sizeof b);
      if (strcmp(a, b)) {
        snprintf(buf, len, "counter changes at n=%d (%s -> %s)", n, a[0] ? a : "none", b[0] ? b : "none");
        return 0;
      }
    }
  }
  switch (o->status) {
    case E13_CHK_LIMIT: snprintf(buf, len, "stage %d not reached (limit)", o->fail_stage); return 0;
    case E13_CHK_OFFTAPE: snprintf(buf, len, "stage %d: off tape", o->fail_stage); return 0;
    case E13_CHK_FREE_READ:
      snprintf(buf, len, "free cell %c%d read before stage %d", 'A' + o->free_state, o->free_sym, o->fail_stage);
      return 0;
    case E13_CHK_HALT: snprintf(buf, len, "halt before stage %d", o->fail_stage); return 0;
    default: break;
  }
  if (nmax >= 9) {
    counter_text(o, 1, a, sizeof a);
    counter_text(o, 3, b, sizeof b);
    counter_text(o, 9, c9, sizeof c9);
    if (!strcmp(a, b) || !strcmp(b, c9) || !strcmp(a, c9)) {
      snprintf(buf, len, "counter equal for different c");
      return 0;
    }
  } else {
    /* recheck prints ctr[9] even when nmax < 9: a stale buffer there; this
       library prints the empty set */
    c9[0] = 0;
  }
  snprintf(buf, len, "CONSISTENT to n=%d (c2 counter %s)", nmax, c9);
  return 1;
}

int e13_format_deep(const e13_check_in *in, const e13_check_out *o, int nmax, char *buf, size_t len) {
  if (!in || !o || !buf) return E13_ERR_ARG;
  int w = snprintf(buf, len, "(nq=%d st0=%d%s):", in->nq, in->st0, in->rel ? " rel" : "");
  for (int n = 1; n <= o->stages_done && n <= nmax && (size_t)w < len; n++) {
    w += snprintf(buf + w, len - (size_t)w, " n%d:%d", n, o->nones[n]);
    if (o->nones[n] && (size_t)w < len) w += snprintf(buf + w, len - (size_t)w, "@%lld", (long long)o->leftmost[n]);
  }
  if ((size_t)w >= len) return w;
  switch (o->status) {
    case E13_CHK_LIMIT:
      w += snprintf(buf + w, len - (size_t)w, " | stage %d NOT reached (limit, t=%lld)", o->fail_stage,
                    (long long)o->fail_t);
      break;
    case E13_CHK_OFFTAPE:
      w += snprintf(buf + w, len - (size_t)w, " | stage %d: off tape at %lld", o->fail_stage, (long long)o->fail_head);
      break;
    case E13_CHK_FREE_READ:
      w += snprintf(buf + w, len - (size_t)w, " | FREE cell %c%d read before stage %d (t=%lld)", 'A' + o->free_state,
                    o->free_sym, o->fail_stage, (long long)o->fail_t);
      break;
    case E13_CHK_HALT:
      w += snprintf(buf + w, len - (size_t)w, " | HALT before stage %d (t=%lld)", o->fail_stage, (long long)o->fail_t);
      break;
    default: break;
  }
  return w;
}
