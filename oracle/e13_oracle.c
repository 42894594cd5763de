/*
 * e13_oracle.c -- CPU restatement of the reference's tree-normal-form (TNF)
 * search over 2-symbol Turing machines and of its two hash-free survivor
 * checkers.
 *
 * TEST INFRASTRUCTURE ONLY.  The product (libe13b200.so and the e13search
 * drop-in CLI) never links, loads or calls this file.  It is loaded by the
 * tests, by __graft_entry__.smoke() and by bench.py's cpu_baseline leg, and
 * there only as the checker of the CUDA path.
 *
 * Parity of this restatement is pinned two ways: against the result logs the
 * reference ships (fixtures under tests/golden/, made by
 * tests/golden/make_golden.py), and against the reference programs compiled
 * from their own sources into oracle/_ref/ by oracle/Makefile.
 *
 * Reference code restated here (paths within the reference project):
 *   src/e13search.c  splitmix :98-103, KEY/TGT :437-444, parse_cell :105-108,
 *                    sim_init :123-129, run :134-177, sym_next :206-212,
 *                    explore :214-254, setup :317-355, set_sym :423-426,
 *                    run_full :428-433, report :184-200
 *   src/e13search.c  probe :256-313, estimate :473-510 (Knuth size estimate)
 *   src/recheck.c    main :22-103   (exact counter sets per stage)
 *   src/deep.c       main :15-84    (counter size and leftmost one per stage)
 *   src/check.py     :1-173         (stages to 11, crafted stage starts, its text)
 *
 * The structure is this file's own: the DFS keeps whole machine snapshots in
 * its frontier (no replay from the blank tape), and the parallel phase is a
 * pthread pool over that frontier.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define O_STAGES 9          /* stage starts n = 1..9 (e13search.c:58) */
#define O_LEFT 64           /* cells left of 0 kept (e13search.c:59) */
#define O_RIGHT 1300        /* cells from 0 rightwards (e13search.c:60) */
#define O_TAPE (O_LEFT + O_RIGHT)
#define O_MAXQ 16
#define O_FREE (-2)         /* a free cell not yet given a move (e13search.c:66) */
#define O_HALT (-1)

enum { O_DIED = -1, O_SURVIVED = -2 };

/* Step at which erdos_14 reaches each stage start, and the number of
   powers-of-two exceptions seen by stage n (e13search.c:70-71).  These are
   the filter's definition, so they are the same numbers. */
static const long ERDOS14_STAGE_STEP[O_STAGES + 1] = {0, 2, 22, 90, 268, 944, 3434, 13450, 52068, 208864};
static const int EXCEPTIONS_BY_STAGE[O_STAGES + 1] = {0, 0, 0, 1, 1, 1, 1, 1, 1, 2};

static uint64_t g_key[O_TAPE];
static uint64_t g_target[O_STAGES + 1];
static int g_keys_ready;

static uint64_t mix_next(uint64_t *state) {
  /* splitmix64, e13search.c:98-103 */
  uint64_t z = (*state += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

/* Zobrist keys of the 1364 window cells and the hash of each stage-start
   block {-1 .. 2^n - 2} (e13search.c:437-444). */
void oracle_keys(uint64_t *key_out, uint64_t *target_out) {
  if (!g_keys_ready) {
    uint64_t s = 20261028ULL;
    for (int p = 0; p < O_TAPE; p++) g_key[p] = mix_next(&s);
    for (int n = 1; n <= O_STAGES; n++) {
      uint64_t h = 0;
      for (int cell = -1; cell <= (1 << n) - 2; cell++) h ^= g_key[cell + O_LEFT];
      g_target[n] = h;
    }
    g_keys_ready = 1;
  }
  if (key_out) memcpy(key_out, g_key, sizeof g_key);
  if (target_out) memcpy(target_out, g_target, sizeof g_target);
}

/* ------------------------------------------------------------------ */
/* machine tables                                                      */

/* "<w><L|R><next>" or "---" -> (next << 2) | (dir << 1) | write, -1 halt
   (e13search.c:105-108). */
int oracle_parse_cell(const char *s) {
  if (s[0] == '-') return O_HALT;
  int next = atoi(s + 2);
  return (next << 2) | ((s[1] == 'R') ? 2 : 0) | (s[0] - '0');
}

/* Reads up to 16 rows of two cells each (e13search.c:110-121). */
int oracle_load(const char *path, int *base) {
  FILE *f = fopen(path, "r");
  if (!f) return -1;
  char a[16], b[16];
  int nq = 0;
  while (nq < O_MAXQ && fscanf(f, "%15s %15s", a, b) == 2) {
    base[2 * nq] = oracle_parse_cell(a);
    base[2 * nq + 1] = oracle_parse_cell(b);
    nq++;
  }
  fclose(f);
  return nq;
}

/* Candidate construction (e13search.c:317-355 with set_sym :423-426).
   Returns the remaining change budget (>= 0), or
     -1  forced cells exceed fmax (the reference skips this X),
     -3  a symmetric state is named by a fixed cell or has a fixed cell,
     -4  the start state is among the symmetric states.
   lo < 0 turns symmetry off.  freebase (2*nq0 flags, base numbering) selects
   free mode; NULL selects delete mode with fmax. */
int oracle_setup(const int *base, int nq0, int X, int fmax, const unsigned char *freebase, int lo, int hi,
                 int *tab, int *sym_lo, int *sym_hi, int *sym_n0, int *nforced) {
  int nF = 0, s = 0;
  for (int q = 0; q < nq0; q++) {
    if (q == X) continue;
    for (int a = 0; a < 2; a++) {
      int code = base[2 * q + a];
      if (freebase && freebase[2 * q + a]) {
        code = O_FREE;
      } else if (code >= 0 && (code >> 2) == X) {
        code = O_FREE;
        nF++;
      } else if (code >= 0) {
        int next = code >> 2;
        if (X >= 0 && next > X) next--;
        code = (next << 2) | (code & 3);
      }
      tab[2 * s + a] = code;
    }
    s++;
  }
  int slo = -1, shi = -1, n0 = 0;
  if (lo >= 0) {
    slo = lo - (lo > X);
    shi = hi - (hi >= X);
  }
  /* symmetry is on only if the renumbered LO is >= 0 (e13search.c:336): with
     no deleted state (X = -1) the reference shifts LO..HI down by one, so
     LO = 0 turns it off */
  if (slo < 0) {
    slo = shi = -1;
  } else {
    unsigned char named[O_MAXQ + 1] = {0};
    /* the reference scans 2*(NQ-1) cells even when X < 0 (e13search.c:341) */
    for (int i = 0; i < 2 * (nq0 - 1); i++) {
      int c = tab[i];
      if (c >= 0 && (c >> 2) >= slo && (c >> 2) <= shi) named[(c >> 2) - slo] = 1;
    }
    while (n0 <= shi - slo && named[n0]) n0++;
    for (int q = slo + n0; q <= shi; q++)
      if (named[q - slo] || tab[2 * q] != O_FREE || tab[2 * q + 1] != O_FREE) return -3;
    if (slo == 0) return -4;
  }
  if (sym_lo) *sym_lo = slo;
  if (sym_hi) *sym_hi = shi;
  if (sym_n0) *sym_n0 = n0;
  if (nforced) *nforced = nF;
  if (freebase) fmax = nF;
  if (nF > fmax) return -1;
  return fmax - nF;
}

/* ------------------------------------------------------------------ */
/* the filter: one machine on the 1364-cell window                     */

typedef struct {
  int head, st, nt, stage, st0, head0, abs_ok, rel_ok;
  int seen[3];
  long t, deadline;
  uint64_t hb, hc, counter_hash[3];
  unsigned char tape[O_TAPE];
} OSim;

static void osim_blank(OSim *m) {
  /* e13search.c:123-129 */
  memset(m, 0, sizeof *m);
  m->st0 = -1;
  m->abs_ok = m->rel_ok = 1;
  m->nt = 1;
  m->deadline = 4 * ERDOS14_STAGE_STEP[1] + 64;
}

/* Runs until an unread cell is read (returns its index), the machine dies
   (O_DIED) or it reaches the start of stage 9 (O_SURVIVED).  Same order of
   checks per step as e13search.c:134-177. */
static int osim_advance(OSim *m, const int *tab, const unsigned char *read) {
  for (;;) {
    if (m->hb == g_target[m->nt]) {
      int c = EXCEPTIONS_BY_STAGE[m->nt];
      int accept = 1, a_ok = m->abs_ok, r_ok = m->rel_ok;
      if (m->nt > 1) {
        if (m->st != m->st0) accept = 0;
        if (m->head != m->head0) a_ok = 0;
        if (m->head - (1 << m->nt) != m->head0 - 2) r_ok = 0;
        if (!a_ok && !r_ok) accept = 0;
      }
      if (accept) {
        if (m->seen[c] && m->counter_hash[c] != m->hc) return O_DIED;
        for (int j = 0; j < 3; j++)
          if (j != c && m->seen[j] && m->counter_hash[j] == m->hc) return O_DIED;
        m->seen[c] = 1;
        m->counter_hash[c] = m->hc;
        if (m->nt == 1) {
          m->st0 = m->st;
          m->head0 = m->head;
        }
        m->abs_ok = a_ok;
        m->rel_ok = r_ok;
        m->stage = m->nt;
        if (m->nt == O_STAGES) return O_SURVIVED;
        m->nt++;
        m->deadline = 4 * ERDOS14_STAGE_STEP[m->nt] + 64;
      }
    }
    if (m->t > m->deadline) return O_DIED;
    int p = m->head + O_LEFT;
    int sym = m->tape[p];
    int cell = 2 * m->st + sym;
    if (!read[cell]) return cell;
    int code = tab[cell];
    if (code < 0) return O_DIED;
    if ((code & 1) != sym) {
      m->tape[p] = (unsigned char)(code & 1);
      if (m->head >= -2) m->hb ^= g_key[p];
      else m->hc ^= g_key[p];
    }
    m->head += (code & 2) ? 1 : -1;
    if (m->head <= -O_LEFT || m->head >= O_RIGHT - 1) return O_DIED;
    m->st = code >> 2;
    m->t++;
  }
}

/* Runs a fully fixed table from the blank tape (e13search.c:428-433).
   out[0] = 1 survivor / 0 dead, then stage, st0, head0, abs, rel, t. */
void oracle_run_full(const int *tab, int nq, long long *out) {
  oracle_keys(NULL, NULL);
  OSim m;
  unsigned char read[2 * O_MAXQ];
  memset(read, 1, sizeof read);
  (void)nq;
  osim_blank(&m);
  int r = osim_advance(&m, tab, read);
  out[0] = r == O_SURVIVED;
  out[1] = m.stage;
  out[2] = m.st0;
  out[3] = m.head0;
  out[4] = m.abs_ok;
  out[5] = m.rel_ok;
  out[6] = m.t;
}

/* ------------------------------------------------------------------ */
/* the TNF enumeration                                                 */

/* Survivor record: 32 codes (-2 free-unread), read mask, st0, head0,
   abs, rel, steps.  40 ints. */
#define O_REC 40

typedef struct {
  long long leaves, survivors, steps, hist[O_STAGES + 1];
} OCounts;

typedef struct {
  int nq, sym_lo, sym_hi;
  OCounts c;
  int *surv;
  int surv_cap, nsurv;
  pthread_mutex_t *lock; /* guards the shared survivor buffer */
  int *surv_shared_n;
  /* frontier collection */
  int collect_depth;
  struct ONode *front;
  long nfront, capfront;
  OSim stack_sims[2 * O_MAXQ + 3];
} OWalk;

typedef struct ONode {
  OSim sim;
  int tab[2 * O_MAXQ];
  unsigned char read[2 * O_MAXQ];
  int budget, nintro;
} ONode;

/* Relabel symmetry (e13search.c:206-212): the number of symmetric states in
   use after a cell gets `code`, or -1 if the move skips the next unused one. */
static int sym_after(const OWalk *w, int code, int nintro) {
  if (w->sym_lo < 0 || code < 0) return nintro;
  int q = code >> 2;
  if (q < w->sym_lo || q > w->sym_hi) return nintro;
  if (q - w->sym_lo < nintro) return nintro;
  return (q - w->sym_lo == nintro) ? nintro + 1 : -1;
}

static void record_survivor(OWalk *w, const OSim *m, const int *tab, const unsigned char *read) {
  int idx;
  pthread_mutex_lock(w->lock);
  idx = (*w->surv_shared_n)++;
  pthread_mutex_unlock(w->lock);
  if (idx >= w->surv_cap) return;
  int *r = w->surv + (long)O_REC * idx;
  uint32_t mask = 0;
  for (int i = 0; i < 32; i++) {
    r[i] = i < 2 * w->nq ? tab[i] : O_HALT;
    if (i < 2 * w->nq && read[i]) mask |= 1u << i;
  }
  r[32] = (int)mask;
  r[33] = m->st0;
  r[34] = m->head0;
  r[35] = m->abs_ok;
  r[36] = m->rel_ok;
  r[37] = (int)m->t;
  r[38] = 0;
  r[39] = 0;
}

/* DFS below a machine stopped at its first read of `cell`... the children
   are: keep the table's move (unless the cell is free), then while the cell
   is free or budget remains, every other move allowed by the symmetry rule
   (e13search.c:214-254).  Each child starts from a copy of the parent. */
static void walk(OWalk *w, int depth, int *tab, unsigned char *read, int budget, int nintro, int multis) {
  OSim *m = &w->stack_sims[depth];
  long t_start = m->t;
  int r = osim_advance(m, tab, read);
  w->c.steps += m->t - t_start;
  if (r == O_DIED) {
    w->c.hist[m->stage]++;
    w->c.leaves++;
    return;
  }
  if (r == O_SURVIVED) {
    w->c.survivors++;
    w->c.leaves++;
    record_survivor(w, m, tab, read);
    return;
  }
  int cell = r, orig = tab[cell];
  int branching = (orig == O_FREE) || budget > 0;
  if (w->collect_depth >= 0 && multis == w->collect_depth) {
    if (w->nfront == w->capfront) {
      w->capfront = w->capfront ? 2 * w->capfront : 256;
      w->front = (ONode *)realloc(w->front, sizeof(ONode) * (size_t)w->capfront);
      if (!w->front) abort();
    }
    ONode *nd = &w->front[w->nfront++];
    nd->sim = *m;
    memcpy(nd->tab, tab, sizeof nd->tab);
    memcpy(nd->read, read, sizeof nd->read);
    nd->budget = budget;
    nd->nintro = nintro;
    return;
  }
  OSim *child = &w->stack_sims[depth + 1];
  read[cell] = 1;
  if (orig != O_FREE) {
    *child = *m;
    walk(w, depth + 1, tab, read, budget, nintro, multis + branching);
  }
  if (branching) {
    int child_budget = (orig == O_FREE) ? budget : budget - 1;
    for (int v = 0; v < 4 * w->nq; v++) {
      if (v == orig) continue;
      int ni = sym_after(w, v, nintro);
      if (ni < 0) continue;
      tab[cell] = v;
      *child = *m;
      walk(w, depth + 1, tab, read, child_budget, ni, multis + 1);
    }
  }
  tab[cell] = orig;
  read[cell] = 0;
}

typedef struct {
  OWalk *w;
  ONode *front;
  long nfront;
  long *next;
  pthread_mutex_t *qlock;
} OPool;

static void *pool_worker(void *arg) {
  OPool *pl = (OPool *)arg;
  OWalk *w = pl->w;
  for (;;) {
    long k;
    pthread_mutex_lock(pl->qlock);
    k = (*pl->next)++;
    pthread_mutex_unlock(pl->qlock);
    if (k >= pl->nfront) break;
    ONode *nd = &pl->front[k];
    int tab[2 * O_MAXQ];
    unsigned char read[2 * O_MAXQ];
    memcpy(tab, nd->tab, sizeof tab);
    memcpy(read, nd->read, sizeof read);
    w->stack_sims[0] = nd->sim;
    /* the node is stopped at an unread cell: advancing again stops at once
       with no steps, then the children are enumerated */
    walk(w, 0, tab, read, nd->budget, nd->nintro, 0);
  }
  return NULL;
}

/* One share of the search, split the way the reference splits a search over
   threads (e13search.c:222-235, 376-403): a serial walk collects the machines
   at their second branching first read; frontier node k belongs to shard
   k % nshards, and what the serial walk finished itself (leaves, steps,
   survivors) counts in shard 0 only.  So the shards' counts add up to the
   whole search and their survivors together are its survivors.  Arguments
   and outputs as oracle_search. */
int oracle_search_shard(const int *tab0, int nq, int budget, int sym_lo, int sym_hi, int sym_n0, int nthreads,
                        int shard, int nshards, long long *counts_out, int *surv, int surv_cap, int *nsurv);

/* The whole search for one prepared table.  counts_out: leaves, survivors,
   steps, hist[0..9] (13 long longs).  Survivor records (O_REC ints each) go
   to surv (up to surv_cap); *nsurv gets the total found.  nthreads <= 1 runs
   serially. */
int oracle_search(const int *tab0, int nq, int budget, int sym_lo, int sym_hi, int sym_n0, int nthreads,
                  long long *counts_out, int *surv, int surv_cap, int *nsurv) {
  return oracle_search_shard(tab0, nq, budget, sym_lo, sym_hi, sym_n0, nthreads, 0, 1, counts_out, surv, surv_cap,
                             nsurv);
}

int oracle_search_shard(const int *tab0, int nq, int budget, int sym_lo, int sym_hi, int sym_n0, int nthreads,
                        int shard, int nshards, long long *counts_out, int *surv, int surv_cap, int *nsurv) {
  if (nshards < 1 || shard < 0 || shard >= nshards) return -1;
  oracle_keys(NULL, NULL);
  pthread_mutex_t lock = PTHREAD_MUTEX_INITIALIZER, qlock = PTHREAD_MUTEX_INITIALIZER;
  int shared_n = 0;
  int tab[2 * O_MAXQ];
  unsigned char read[2 * O_MAXQ] = {0};
  for (int i = 0; i < 2 * O_MAXQ; i++) tab[i] = i < 2 * nq ? tab0[i] : O_HALT;
  OWalk *top = (OWalk *)calloc(1, sizeof(OWalk));
  top->nq = nq;
  top->sym_lo = sym_lo;
  top->sym_hi = sym_hi;
  top->surv = surv;
  top->surv_cap = surv_cap;
  top->lock = &lock;
  top->surv_shared_n = &shared_n;
  top->collect_depth = (nthreads > 1 || nshards > 1) ? 2 : -1;
  osim_blank(&top->stack_sims[0]);
  walk(top, 0, tab, read, budget, sym_n0, 0);
  OCounts total = top->c;
  if (shard != 0) {
    memset(&total, 0, sizeof total); /* the serial walk's own results belong to shard 0 */
    shared_n = 0;
  }
  if (nshards > 1) { /* keep this shard's frontier nodes, in collection order */
    long n = 0;
    for (long k = shard; k < top->nfront; k += nshards) top->front[n++] = top->front[k];
    top->nfront = n;
  }
  if (top->collect_depth >= 0 && top->nfront > 0) {
    if (nthreads < 1) nthreads = 1;
    long next = 0;
    pthread_t *th = (pthread_t *)calloc((size_t)nthreads, sizeof(pthread_t));
    OWalk *ws = (OWalk *)calloc((size_t)nthreads, sizeof(OWalk));
    OPool *pools = (OPool *)calloc((size_t)nthreads, sizeof(OPool));
    for (int k = 0; k < nthreads; k++) {
      ws[k] = *top;
      memset(&ws[k].c, 0, sizeof ws[k].c);
      ws[k].collect_depth = -1;
      ws[k].front = NULL;
      ws[k].nfront = ws[k].capfront = 0;
      pools[k].w = &ws[k];
      pools[k].front = top->front;
      pools[k].nfront = top->nfront;
      pools[k].next = &next;
      pools[k].qlock = &qlock;
      pthread_create(&th[k], NULL, pool_worker, &pools[k]);
    }
    for (int k = 0; k < nthreads; k++) {
      pthread_join(th[k], NULL);
      total.leaves += ws[k].c.leaves;
      total.survivors += ws[k].c.survivors;
      total.steps += ws[k].c.steps;
      for (int j = 0; j <= O_STAGES; j++) total.hist[j] += ws[k].c.hist[j];
    }
    free(th);
    free(ws);
    free(pools);
  }
  free(top->front);
  free(top);
  counts_out[0] = total.leaves;
  counts_out[1] = total.survivors;
  counts_out[2] = total.steps;
  for (int j = 0; j <= O_STAGES; j++) counts_out[3 + j] = total.hist[j];
  *nsurv = shared_n;
  return 0;
}

/* ------------------------------------------------------------------ */
/* hash-free survivor checkers (recheck.c, deep.c)                     */

/* A survivor table as the checkers read it: per cell a kind (0 move,
   1 halt, 2 free cell never read), write, move (+1 R / -1 L), next. */
typedef struct {
  int nq;
  int kind[32][2], wr[32][2], mv[32][2], nx[32][2];
  int st0, abs_ok, rel_ok;
  long long head0;
  int has_st0, has_head0, has_abs, has_rel;
} OCheckIn;

/* Parses the fields of a SURVIVOR line the way both checkers do
   (recheck.c:31-56, deep.c:22-48). Returns 0 if the line has no table. */
static int parse_survivor_line(const char *line, OCheckIn *in) {
  const char *tb = strstr(line, "table=");
  if (!tb) return 0;
  memset(in, 0, sizeof *in);
  const char *p;
  in->st0 = 0;
  in->head0 = -2;
  in->abs_ok = 1;
  in->rel_ok = 0;
  if ((p = strstr(line, "st0="))) { in->st0 = atoi(p + 4); in->has_st0 = 1; }
  if ((p = strstr(line, "head0="))) { in->head0 = atoi(p + 6); in->has_head0 = 1; }
  if ((p = strstr(line, "abs="))) { in->abs_ok = atoi(p + 4); in->has_abs = 1; }
  if ((p = strstr(line, "rel="))) { in->rel_ok = atoi(p + 4); in->has_rel = 1; }
  char *q = (char *)tb + 6;
  int nq = 0;
  while (*q && *q != '\n' && *q != '\r' && nq < 32) {
    for (int a = 0; a < 2; a++) {
      while (*q == ' ') q++;
      int unread = 0;
      if (*q == '?') { unread = 1; q++; }
      if (*q == '-') {
        in->kind[nq][a] = unread ? 2 : 1;
        q += 3;
      } else {
        in->kind[nq][a] = 0;
        in->wr[nq][a] = *q++ - '0';
        in->mv[nq][a] = (*q++ == 'R') ? 1 : -1;
        in->nx[nq][a] = (int)strtol(q, &q, 10);
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

#define RC_SIDE 4000000LL
static unsigned char *g_rc_tape;
static char g_rc_ctr[20][8192];

/* recheck.c:57-99 for one machine: fills `verdict` with the text recheck
   prints after "<id>: ", and counters[n] (n = 1..nmax) with the exact counter
   set at each stage start ("-3,-4," style, "" for none).  Returns 1 if the
   verdict is CONSISTENT. */
int oracle_recheck_line(const char *line, int nmax, char *verdict, int vlen, char *counters, int clen) {
  OCheckIn in;
  if (!parse_survivor_line(line, &in)) return -1;
  if (!g_rc_tape) g_rc_tape = (unsigned char *)calloc((size_t)(2 * RC_SIDE + 1), 1);
  unsigned char *tp = g_rc_tape;
  memset(tp, 0, (size_t)(2 * RC_SIDE + 1));
#define CELL(c) tp[(c) + RC_SIDE]
  int rel = !in.abs_ok && in.rel_ok;
  long long head = 0, t = 0, minhead = 0, ones = 0;
  int st = 0, failed = 0;
  char v[512] = "";
  for (int n = 1; n <= nmax && !failed; n++) {
    long long blk = 1LL << n;
    long long limit = t + 8LL * (1LL << (2 * n)) + 100000;
    long long want = rel ? in.head0 + blk - 2 : in.head0;
    for (;;) {
      if (st == in.st0 && head == want && ones == blk) {
        int ok = 1;
        for (long long k = -1; k < blk - 1; k++)
          if (!CELL(k)) { ok = 0; break; }
        if (ok) break;
      }
      if (t >= limit) { snprintf(v, sizeof v, "stage %d not reached (limit)", n); failed = 1; break; }
      if (head <= -RC_SIDE + 2 || head >= RC_SIDE - 2) { snprintf(v, sizeof v, "stage %d: off tape", n); failed = 1; break; }
      int s = CELL(head), k = in.kind[st][s];
      if (k == 2) { snprintf(v, sizeof v, "free cell %c%d read before stage %d", 'A' + st, s, n); failed = 1; break; }
      if (k == 1) { snprintf(v, sizeof v, "halt before stage %d", n); failed = 1; break; }
      int w = in.wr[st][s];
      if (w != s) {
        CELL(head) = (unsigned char)w;
        if (head >= -2) ones += w ? 1 : -1;
      }
      head += in.mv[st][s];
      if (head < minhead) minhead = head;
      st = in.nx[st][s];
      t++;
    }
    if (failed) break;
    char *q = g_rc_ctr[n];
    *q = 0;
    int len = 0;
    for (long long k = -3; k >= minhead - 1 && len < 8000; k--)
      if (CELL(k)) len += sprintf(q + len, "%lld,", k);
    int c = n <= 2 ? 0 : (n <= 8 ? 1 : 2);
    int first = c == 0 ? 1 : (c == 1 ? 3 : 9);
    if (n != first && strcmp(g_rc_ctr[n], g_rc_ctr[first])) {
      snprintf(v, sizeof v, "counter changes at n=%d (%s -> %s)", n, g_rc_ctr[first][0] ? g_rc_ctr[first] : "none",
               g_rc_ctr[n][0] ? g_rc_ctr[n] : "none");
      failed = 1;
    }
    if (counters) {
      char *dst = counters + (long)(n - 1) * clen;
      strncpy(dst, g_rc_ctr[n], (size_t)clen - 1);
      dst[clen - 1] = 0;
    }
  }
  if (!failed) {
    if (nmax >= 9 && (!strcmp(g_rc_ctr[1], g_rc_ctr[3]) || !strcmp(g_rc_ctr[3], g_rc_ctr[9]) ||
                      !strcmp(g_rc_ctr[1], g_rc_ctr[9])))
      snprintf(v, sizeof v, "counter equal for different c");
    else
      snprintf(v, sizeof v, "CONSISTENT to n=%d (c2 counter %s)", nmax, g_rc_ctr[9]);
  }
#undef CELL
  strncpy(verdict, v, (size_t)vlen - 1);
  verdict[vlen - 1] = 0;
  return strncmp(v, "CONSISTENT", 10) == 0;
}

/* deep.c:49-81 for one machine: writes the text deep prints after
   "survivor <id> " into out. */
int oracle_deep_line(const char *line, int nmax, char *out, int olen) {
  OCheckIn in;
  if (!parse_survivor_line(line, &in) || !in.has_st0) return -1;
  const long long LEFTC = 4096;
  long long size = LEFTC + (1LL << nmax) + 4096;
  unsigned char *tape = (unsigned char *)calloc((size_t)size, 1);
  int rel = in.has_abs && in.has_rel && !in.abs_ok && in.rel_ok;
  long long head0 = in.has_head0 ? in.head0 : -2;
  long long head = 0, t = 0, ones_ge = 0;
  int st = 0, failed = 0, len = 0;
  len += snprintf(out + len, (size_t)(olen - len), "(nq=%d st0=%d%s):", in.nq, in.st0, rel ? " rel" : "");
  for (int n = 1; n <= nmax && !failed; n++) {
    long long blk = 1LL << n, limit = t + 64LL * (1LL << (2 * n)) + 100000;
    for (;;) {
      if (st == in.st0 && head == (rel ? blk + head0 - 2 : head0) && ones_ge == blk) {
        int ok = 1;
        for (long long k = -1; k < blk - 1; k++)
          if (!tape[LEFTC + k]) { ok = 0; break; }
        if (ok) break;
      }
      if (t >= limit) { len += snprintf(out + len, (size_t)(olen - len), " | stage %d NOT reached (limit, t=%lld)", n, t); failed = 1; break; }
      if (head < -LEFTC + 2 || head > blk + 2000) { len += snprintf(out + len, (size_t)(olen - len), " | stage %d: off tape at %lld", n, head); failed = 1; break; }
      int s = tape[LEFTC + head];
      if (in.kind[st][s] == 2) { len += snprintf(out + len, (size_t)(olen - len), " | FREE cell %c%d read before stage %d (t=%lld)", 'A' + st, s, n, t); failed = 1; break; }
      if (in.kind[st][s]) { len += snprintf(out + len, (size_t)(olen - len), " | HALT before stage %d (t=%lld)", n, t); failed = 1; break; }
      int ww = in.wr[st][s];
      if (ww != s) {
        tape[LEFTC + head] = (unsigned char)ww;
        if (head >= -2) ones_ge += ww ? 1 : -1;
      }
      head += in.mv[st][s];
      st = in.nx[st][s];
      t++;
    }
    if (failed) break;
    int cnt = 0;
    long long lo = 0;
    for (long long k = -3; k >= -LEFTC + 1; k--)
      if (tape[LEFTC + k]) { cnt++; lo = k; }
    len += snprintf(out + len, (size_t)(olen - len), " n%d:%d", n, cnt);
    if (cnt) len += snprintf(out + len, (size_t)(olen - len), "@%lld", lo);
  }
  free(tape);
  return failed ? 0 : 1;
}

/* ------------------------------------------------------------------ */
/* raw simulator (no filter)                                           */

/* Draw k (1-based) of splitmix64 from `seed`: the generator's state after k
   increments is seed + k * golden, so any draw can be made directly. */
/* ------------------------------------------------------------------ */
/* Knuth size estimate (e13search.c:256-313 probe, :473-510 estimate)   */

/* Start of the splitmix64 stream the reference gives OpenMP thread k
   (e13search.c:486-491): the state is the draw at 0x5EED0000 + k + (seed << 20). */
uint64_t oracle_probe_stream(uint64_t seed, uint64_t k) {
  uint64_t s = 0x5EED0000ULL + k + (seed << 20);
  return mix_next(&s);
}

/* One probe: a random root-to-leaf path; every child of a fork on the path
   runs to its next event and the path continues into a live child drawn
   from *rng.  Adds the weighted counts to out[0..3] = leaves, nodes, steps,
   survivors, in the reference's order of additions. */
void oracle_probe(const int *tab0, int nq, int budget, int sym_lo, int sym_hi, int sym_n0, uint64_t *rng,
                  double *out) {
  oracle_keys(NULL, NULL);
  OWalk w;
  memset(&w, 0, sizeof w);
  w.nq = nq;
  w.sym_lo = sym_lo;
  w.sym_hi = sym_hi;
  int tab[2 * O_MAXQ];
  unsigned char read[2 * O_MAXQ];
  for (int i = 0; i < 2 * O_MAXQ; i++) tab[i] = i < 2 * nq ? tab0[i] : O_HALT;
  memset(read, 0, sizeof read);
  int nintro = sym_n0;
  double wt = 1.0;
  OSim *s = (OSim *)malloc(sizeof(OSim) * (4 * O_MAXQ + 2));
  OSim *kids = s + 1;
  osim_blank(s);
  int i = osim_advance(s, tab, read);
  out[1] += 1;
  out[2] += (double)s->t;
  if (i < 0) {
    out[0] += 1;
    if (i == O_SURVIVED) out[3] += 1;
    free(s);
    return;
  }
  for (;;) {
    int orig = tab[i], vals[4 * O_MAXQ + 1], nbs[4 * O_MAXQ + 1], nis[4 * O_MAXQ + 1], k = 0;
    if (orig != O_FREE) {
      vals[k] = orig;
      nbs[k] = budget;
      nis[k] = nintro;
      k++;
    }
    if (orig == O_FREE || budget > 0) {
      for (int v = 0; v < 4 * nq; v++) {
        int ni = sym_after(&w, v, nintro);
        if (v == orig || ni < 0) continue;
        vals[k] = v;
        nbs[k] = orig == O_FREE ? budget : budget - 1;
        nis[k] = ni;
        k++;
      }
    }
    int live[4 * O_MAXQ + 1], nlive = 0;
    read[i] = 1;
    for (int c = 0; c < k; c++) {
      kids[c] = *s;
      tab[i] = vals[c];
      long t0 = kids[c].t;
      int r = osim_advance(&kids[c], tab, read);
      out[1] += wt;
      out[2] += wt * (double)(kids[c].t - t0);
      if (r < 0) {
        out[0] += wt;
        if (r == O_SURVIVED) out[3] += wt;
      } else {
        live[nlive++] = c;
      }
    }
    if (!nlive) break;
    int c = live[mix_next(rng) % (uint64_t)nlive];
    wt *= nlive;
    tab[i] = vals[c];
    budget = nbs[c];
    nintro = nis[c];
    *s = kids[c];
    i = osim_advance(s, tab, read); /* the same unread cell, no steps */
  }
  free(s);
}

static uint64_t mix_draw(uint64_t seed, uint64_t k) {
  uint64_t s = seed + (k - 1) * 0x9E3779B97F4A7C15ULL;
  return mix_next(&s);
}

/* Random tables: machine m, cell i = draw m*2nq + i + 1 mod 4nq, i.e. each
   cell uniform over write x dir x next (no halt).  codes: n * 2nq bytes. */
void oracle_raw_tables(uint64_t seed, long n, int nq, unsigned char *codes) {
  for (long m = 0; m < n; m++)
    for (int i = 0; i < 2 * nq; i++)
      codes[m * 2 * nq + i] = (unsigned char)(mix_draw(seed, (uint64_t)(m * 2 * nq + i + 1)) % (uint64_t)(4 * nq));
}

/* Steps (3)-(7) of run() (src/e13search.c:163-175) with the stage test and
   the deadline removed: a table runs from the blank tape for at most
   max_steps steps and stops when the head leaves the window (head <= -64 or
   >= 1299; that step is not counted, as in run()) or reads a halt.  out (4 per
   machine): steps, status (0 step cap, 1 left the window, 2 halt), final
   head, ones on the tape. */
void oracle_raw_run(const unsigned char *codes, long n, int nq, long max_steps, long long *out) {
  unsigned char tape[O_TAPE];
  for (long m = 0; m < n; m++) {
    const unsigned char *tab = codes + m * 2 * nq;
    memset(tape, 0, sizeof tape);
    int head = 0, st = 0, status = 0;
    long t = 0;
    long long ones = 0;
    while (t < max_steps) {
      int p = head + O_LEFT, sym = tape[p];
      int code = tab[2 * st + sym];
      if (code >= 4 * nq) { status = 2; break; }
      if ((code & 1) != sym) {
        tape[p] = (unsigned char)(code & 1);
        ones += (code & 1) ? 1 : -1;
      }
      head += (code & 2) ? 1 : -1;
      if (head <= -O_LEFT || head >= O_RIGHT - 1) { status = 1; break; }
      st = code >> 2;
      t++;
    }
    out[4 * m] = t;
    out[4 * m + 1] = status;
    out[4 * m + 2] = head;
    out[4 * m + 3] = ones;
  }
}

/* ------------------------------------------------------------------ */
/* check.py: hash-free stages 1..11 and crafted stage starts            */
/* (src/check.py:1-173), with check.py's unbounded tape and its text     */

#define CK_NMAX 11 /* check.py:20 */
#define CK_MMAX 40 /* check.py:21 */

enum { CK_STOP = 0, CK_HALT = 1, CK_LIMIT = 2 };
static const char *const CK_RES[3] = {"stop", "halt", "limit"};

/* a tape that grows to whatever cells the machine visits */
typedef struct {
  unsigned char *b;
  long lo, n; /* cells lo .. lo + n - 1 */
} CkTape;

static int ck_get(const CkTape *t, long c) { return c >= t->lo && c < t->lo + t->n ? t->b[c - t->lo] : 0; }

static void ck_set(CkTape *t, long c, int v) {
  if (c < t->lo || c >= t->lo + t->n) {
    if (!v) return;
    long lo = t->lo, hi = t->lo + t->n;
    long want_lo = c < lo ? c - (t->n + 64) : lo, want_hi = c >= hi ? c + (t->n + 64) : hi;
    unsigned char *nb = (unsigned char *)calloc((size_t)(want_hi - want_lo), 1);
    if (t->n) memcpy(nb + (lo - want_lo), t->b, (size_t)t->n);
    free(t->b);
    t->b = nb;
    t->lo = want_lo;
    t->n = want_hi - want_lo;
  }
  t->b[c - t->lo] = (unsigned char)v;
}

/* the ones at cells < -2, ascending (check.py:51-52) */
static int ck_counter(const CkTape *t, long *cells, int cap) {
  int k = 0;
  for (long c = t->lo; c < -2 && c < t->lo + t->n; c++)
    if (t->b[c - t->lo]) {
      if (k < cap) cells[k] = c;
      k++;
    }
  return k;
}

typedef struct {
  int stage_one; /* stage 1: the block alone (check.py:85-86) */
  int crafted;   /* crafted start: head must be exactly hh (check.py:142-146) */
  long size, h0, hh;
  int s0;
} CkStop;

static int ck_is_block(const CkTape *t, long size, long ones_ge) {
  if (ones_ge != size) return 0;
  for (long c = -1; c < size - 1; c++)
    if (!ck_get(t, c)) return 0;
  return 1;
}

static int ck_stop(const CkTape *t, long ones_ge, long head, int st, const CkStop *s) {
  if (ones_ge != s->size) return 0;
  if (!s->stage_one) {
    if (st != s->s0) return 0;
    if (s->crafted ? head != s->hh : (head != s->h0 && head - s->size != s->h0 - 2)) return 0;
  }
  return ck_is_block(t, s->size, ones_ge);
}

/* run_tracked (check.py:55-77): rows[i] = write | right << 1 | next << 2, or -1 halt */
static int ck_run(const int *rows, CkTape *t, long *head, int *st, const CkStop *s, long limit, long *steps) {
  long ones_ge = 0;
  for (long c = -2; c < t->lo + t->n; c++) ones_ge += ck_get(t, c);
  for (long k = 0; k < limit; k++) {
    if (ck_stop(t, ones_ge, *head, *st, s)) {
      *steps = k;
      return CK_STOP;
    }
    int sym = ck_get(t, *head);
    int r = rows[2 * *st + sym];
    if (r < 0) {
      *steps = k;
      return CK_HALT;
    }
    int w = r & 1;
    if (w && !sym) {
      ck_set(t, *head, 1);
      if (*head >= -2) ones_ge++;
    } else if (sym && !w) {
      ck_set(t, *head, 0);
      if (*head >= -2) ones_ge--;
    }
    *head += (r & 2) ? 1 : -1;
    *st = r >> 2;
  }
  *steps = limit;
  return CK_LIMIT;
}

static int ck_no_two(long m) {
  while (m) {
    if (m % 3 == 2) return 0;
    m /= 3;
  }
  return 1;
}

typedef struct {
  char *s;
  size_t len, cap;
} CkBuf;

static void ck_put(CkBuf *b, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
#include <stdarg.h>
static void ck_put(CkBuf *b, const char *fmt, ...) {
  for (;;) {
    va_list ap;
    va_start(ap, fmt);
    int n = vsnprintf(b->s + b->len, b->cap - b->len, fmt, ap);
    va_end(ap);
    if (n >= 0 && (size_t)n < b->cap - b->len) {
      b->len += (size_t)n;
      return;
    }
    b->cap = 2 * b->cap + (size_t)(n > 0 ? n : 256) + 256;
    b->s = (char *)realloc(b->s, b->cap);
  }
}

/* Python's repr of a tuple of ints */
static void ck_tuple(CkBuf *b, const long *v, int n) {
  ck_put(b, "(");
  for (int i = 0; i < n; i++) ck_put(b, i ? ", %ld" : "%ld", v[i]);
  ck_put(b, n == 1 ? ",)" : ")");
}

#define CK_CAP 4096 /* counter cells kept per stage start */

typedef struct {
  int st;
  long head, total;
  int ncnt;
  long *cnt;
} CkStart;

static int ck_same(const long *a, int na, const long *b, int nb) {
  return na == nb && (na == 0 || !memcmp(a, b, sizeof(long) * (size_t)na));
}

/* One placement: check.py's check() body (:102-162) for a table with its
   halt placed; appends "   halt@<place>: ..." to b. */
static void ck_placement(const int *rows, int place, CkBuf *b) {
  CkTape tp = {0, 0, 0};
  CkStart starts[CK_NMAX + 1];
  int nstarts = 0;
  long head = 0, total = 0;
  int st = 0;
  char place_s[16];
  if (place < 0) snprintf(place_s, sizeof place_s, "None");
  else snprintf(place_s, sizeof place_s, "%d", place);
  for (int n = 1; n <= CK_NMAX; n++) {
    CkStop s = {nstarts == 0, 0, 1L << n, nstarts ? starts[0].head : 0, 0, nstarts ? starts[0].st : 0};
    long t = 0;
    int res = ck_run(rows, &tp, &head, &st, &s, 40L * (1L << (2 * n)) + 1000, &t);
    total += t;
    if (res != CK_STOP) {
      ck_put(b, "   halt@%s: FAIL stage %d: %s at step %ld\n", place_s, n, CK_RES[res], total);
      goto out;
    }
    starts[nstarts].st = st;
    starts[nstarts].head = head;
    starts[nstarts].total = total;
    starts[nstarts].cnt = (long *)malloc(sizeof(long) * CK_CAP);
    starts[nstarts].ncnt = ck_counter(&tp, starts[nstarts].cnt, CK_CAP);
    nstarts++;
  }
  {
    /* counter consistency (:116-126): cnt[c] = the counter at the first start with c */
    int have[3] = {0, 0, 0}, first[3] = {0, 0, 0};
    char bad[96] = "";
    for (int i = 0; i < nstarts; i++) {
      int n = i + 1, c = 0;
      for (int k = 1; k < n; k++) c += ck_no_two(1L << k);
      if (have[c] && !ck_same(starts[first[c]].cnt, starts[first[c]].ncnt, starts[i].cnt, starts[i].ncnt))
        snprintf(bad, sizeof bad, "counter differs within c=%d at n=%d", c, n);
      if (!have[c]) {
        have[c] = 1;
        first[c] = i;
      }
    }
    int ndistinct = 0, nkeys = 0;
    for (int c = 0; c < 3; c++) {
      if (!have[c]) continue;
      nkeys++;
      int dup = 0;
      for (int d = 0; d < c; d++)
        if (have[d] && ck_same(starts[first[d]].cnt, starts[first[d]].ncnt, starts[first[c]].cnt, starts[first[c]].ncnt))
          dup = 1;
      ndistinct += !dup;
    }
    if (ndistinct != nkeys) snprintf(bad, sizeof bad, "counter equal for different c");
    if (bad[0]) {
      ck_put(b, "   halt@%s: FAIL %s\n", place_s, bad);
      goto out;
    }
    const int s0 = starts[0].st;
    const long h0 = starts[0].head;
    int absolute = 1;
    for (int i = 0; i < nstarts; i++)
      if (starts[i].head != h0) absolute = 0;
    /* crafted stage starts (:128-156) */
    CkBuf fails = {0, 0, 0};
    int nfails = 0;
    long *got = (long *)malloc(sizeof(long) * CK_CAP);
    for (int c = 0; c < 3; c++) {
      if (!have[c]) continue;
      for (long m = 2; m <= CK_MMAX; m++) {
        CkTape ct = {0, 0, 0};
        const CkStart *cs = &starts[first[c]];
        for (int i = 0; i < cs->ncnt; i++) ck_set(&ct, cs->cnt[i], 1);
        for (long k = -1; k < m - 1; k++) ck_set(&ct, k, 1);
        long hd = absolute ? h0 : h0 - 2 + m;
        int cst = s0;
        const long nxt = 2 * m;
        const int want_c = ck_no_two(m) ? c + 1 : c;
        const int want_halt = ck_no_two(m) && c == 2;
        CkStop s = {0, 1, nxt, h0, absolute ? h0 : h0 - 2 + nxt, s0};
        long t = 0;
        int res = ck_run(rows, &ct, &hd, &cst, &s, 40 * m * m + 5000, &t);
        char msg[1024] = "";
        if (want_halt) {
          if (res != CK_HALT) snprintf(msg, sizeof msg, "expected halt, got %s", CK_RES[res]);
        } else if (res != CK_STOP) {
          snprintf(msg, sizeof msg, "expected stage 2m, got %s at %ld", CK_RES[res], t);
        } else {
          int ng = ck_counter(&ct, got, CK_CAP);
          if (want_c < 3 && have[want_c]) {
            const CkStart *ts = &starts[first[want_c]];
            if (!ck_same(got, ng, ts->cnt, ts->ncnt)) {
              CkBuf mb = {0, 0, 0};
              ck_put(&mb, "counter ");
              ck_tuple(&mb, got, ng);
              ck_put(&mb, " != c=%d ", want_c);
              ck_tuple(&mb, ts->cnt, ts->ncnt);
              snprintf(msg, sizeof msg, "%s", mb.s);
              free(mb.s);
            }
          } else {
            for (int d = 0; d < 3; d++)
              if (have[d] && ck_same(got, ng, starts[first[d]].cnt, starts[first[d]].ncnt))
                snprintf(msg, sizeof msg, "counter for c=3 equals an earlier one");
          }
        }
        free(ct.b);
        if (msg[0]) {
          if (nfails < 4) ck_put(&fails, nfails ? ", (%d, %ld, '%s')" : "(%d, %ld, '%s')", c, m, msg);
          nfails++;
        }
      }
    }
    free(got);
    ck_put(b, "   halt@%s: %s stages ok to n=%d (step %ld); counters {", place_s, nfails ? "FAIL" : "PASS", CK_NMAX,
           starts[nstarts - 1].total);
    int firstkey = 1;
    for (int c = 0; c < 3; c++) {
      if (!have[c]) continue;
      ck_put(b, firstkey ? "%d: " : ", %d: ", c);
      ck_tuple(b, starts[first[c]].cnt, starts[first[c]].ncnt);
      firstkey = 0;
    }
    ck_put(b, "}; crafted fails %d: [%s]\n", nfails, fails.s ? fails.s : "");
    free(fails.s);
  }
out:
  for (int i = 0; i < nstarts; i++) free(starts[i].cnt);
  free(tp.b);
}

/* check.py's output for one input line (its __main__, :165-173): the line
   (stripped), then a verdict line per placement of the halt.  Returns the
   text length (truncated to outlen - 1), 0 if the line has no table. */
int oracle_check_line(const char *line, char *out, int outlen) {
  const char *tb = strstr(line, "table=");
  if (!tb || outlen < 1) return 0;
  int rows[2 * O_MAXQ], unread[2 * O_MAXQ], nun = 0, ncell = 0, nhalt = 0;
  const char *q = tb + 6;
  while (*q == ' ' || *q == '\t') q++;
  while (*q && *q != '\n' && *q != '\r' && ncell < 2 * O_MAXQ) {
    while (*q == ' ' || *q == '\t') q++;
    if (*q == '|') {
      q++;
      continue;
    }
    if (!*q || *q == '\n' || *q == '\r') break;
    int un = 0;
    if (*q == '?') {
      un = 1;
      q++;
    }
    if (*q == '-') {
      rows[ncell] = -1;
      nhalt++;
      q += 3;
    } else {
      int w = *q++ - '0';
      int right = *q++ == 'R';
      int nx = (int)strtol(q, (char **)&q, 10);
      rows[ncell] = w | (right << 1) | (nx << 2);
    }
    if (un) unread[nun++] = ncell;
    ncell++;
  }
  CkBuf b = {0, 0, 0};
  /* the line, stripped */
  const char *s = line, *e = line + strlen(line);
  while (*s == ' ' || *s == '\t' || *s == '\n' || *s == '\r') s++;
  while (e > s && (e[-1] == ' ' || e[-1] == '\t' || e[-1] == '\n' || e[-1] == '\r')) e--;
  ck_put(&b, "%.*s\n", (int)(e - s), s);
  if (nhalt) {
    ck_placement(rows, -1, &b);
  } else {
    for (int i = 0; i < nun; i++) {
      int r2[2 * O_MAXQ];
      memcpy(r2, rows, sizeof r2);
      r2[unread[i]] = -1;
      ck_placement(r2, unread[i], &b);
    }
  }
  int n = (int)b.len < outlen - 1 ? (int)b.len : outlen - 1;
  memcpy(out, b.s, (size_t)n);
  out[n] = 0;
  free(b.s);
  return n;
}
