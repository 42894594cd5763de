/*
 * e13.h -- C-ABI of libe13b200.so, the B200 (sm_100a) tree-normal-form search
 * over 2-symbol Turing machines near erdos_14.
 *
 * Plain C types only: pointers, sizes and int status codes.  The caller owns
 * every host buffer; a context owns the device memory it allocates.  One host
 * thread per context.  Functions return E13_OK (0) or a negative E13_ERR_*.
 *
 * The reference has no plugin or FFI; its boundary is the e13search process
 * (src/e13search.c:435-513) and the recheck/deep programs.  Each entry point
 * below names the reference code whose behaviour it takes over.
 */
#ifndef E13_H
#define E13_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define E13_MAXQ 16          /* rows a machine file may hold (src/e13search.c:63) */
#define E13_MAXCELLS 32
#define E13_STAGES 9         /* stage starts n = 1..9 (src/e13search.c:58) */
#define E13_TAPE_LEFT 64     /* window: cells -64..1299 (src/e13search.c:59-61) */
#define E13_TAPE_RIGHT 1300

/* cell codes, as in the reference: (next << 2) | (dir << 1) | write, dir 1 = R */
#define E13_HALT (-1)
#define E13_FREE (-2)        /* FORCED in src/e13search.c:66: any move at first read */

enum {
  E13_OK = 0,
  E13_ERR_ARG = -1,          /* bad argument (null pointer, size out of range) */
  E13_ERR_FMAX = -2,         /* forced cells exceed FMAX: the reference skips X (src/e13search.c:353) */
  E13_ERR_SYM_NAMED = -3,    /* symmetric state named by / owning a fixed cell (src/e13search.c:344-348) */
  E13_ERR_SYM_START = -4,    /* start state among the symmetric states (src/e13search.c:349) */
  E13_ERR_CUDA = -5,         /* a CUDA call failed (device, memory, launch) */
  E13_ERR_OVERFLOW = -6,     /* frontier stack capacity exceeded */
  E13_ERR_SURV_CAP = -7,     /* more survivors than the caller's buffer holds (counts stay exact) */
  E13_ERR_NQ = -8,           /* more states than the device path supports (nq <= 16) */
  E13_ERR_IO = -9,           /* machine file missing or unreadable (src/e13search.c:113) */
  E13_ERR_TIMEOUT = -10,     /* a device wait ran out (bounded waits; no hang) */
  E13_ERR_NO_DEVICE = -11,   /* no CUDA device: there is no CPU fallback */
  E13_ERR_NOALLOC_SIZE = -12, /* e13_check_noalloc: more machines (or a larger nmax) than its fixed memory holds */
  E13_ERR_CKPT = -13,        /* checkpoint unreadable, truncated, or of another run or job */
  E13_STOPPED = 3            /* e13_search_resumable: stopped cleanly, checkpoint written (not an error) */
};

/* A prepared candidate family: base machine with state X deleted.
   Built by e13_setup (src/e13search.c:317-355 setup, :423-426 set_sym). */
typedef struct e13_job {
  int32_t X;                 /* deleted base state, -1 = none */
  int32_t nq;                /* states after the deletion */
  int32_t tab[E13_MAXCELLS]; /* codes, renumbered; E13_FREE for free cells */
  int32_t budget;            /* further changes allowed (delete mode); 0 in free mode */
  int32_t nforced;           /* rules into X (nF) */
  int32_t sym_lo, sym_hi;    /* interchangeable states, renumbered; -1 = off */
  int32_t sym_n0;            /* leading symmetric states already named by fixed cells */
} e13_job;

/* Totals of one search (src/e13search.c:413-416 summary line). */
typedef struct e13_counts {
  uint64_t leaves;
  uint64_t survivors;
  uint64_t steps;
  uint64_t hist[E13_STAGES + 1]; /* dead leaves by last stage reached */
} e13_counts;

/* One survivor (src/e13search.c:184-200 report): the table as the search
   left it, with a read mask (bit i: cell i was read, i.e. fixed). */
typedef struct e13_survivor {
  int32_t tab[E13_MAXCELLS]; /* codes; E13_FREE / E13_HALT print as --- */
  uint32_t read_mask;
  int32_t st0, head0, abs_ok, rel_ok;
  int64_t steps;             /* step of the stage-9 start */
} e13_survivor;

/* Search kernels. */
enum {
  E13_KERNEL_PLAIN = 0,      /* one launch per frontier batch, host sync per launch */
  E13_KERNEL_PERSISTENT = 1  /* per-warp DFS with in-kernel work donation, graph-captured epochs */
};

/* Tunables of the device search.  kernel and run_skip are taken as given; in
   every other field 0 means the library default (e13_default_tuning) and a
   negative value is an error.  e13_resolve_tuning states the valid ranges. */
typedef struct e13_tuning {
  int32_t kernel;            /* E13_KERNEL_* */
  int32_t block;             /* lanes (threads) per CTA: 64..768, multiple of 32 */
  int32_t slice;             /* iterations per round between warp-level refills; each iteration takes up
                                to two actions (a step, a run skip, a stage test or a first read) per lane */
  int32_t warp_stack;        /* nodes in each warp's private DFS stack (persistent) */
  int32_t step_cap;          /* plain kernel: steps per work item before it is requeued */
  int32_t batch;             /* nodes taken from the frontier per launch / epoch (0 = auto: the whole
                                frontier for the persistent kernel, 16384 for the plain one) */
  int32_t epoch_us;          /* persistent: wall-clock bound of one epoch, microseconds */
  int32_t epochs_per_graph;  /* persistent: epochs captured in one CUDA graph */
  int32_t pool_low_pct;      /* persistent: warps donate stack nodes while the pool holds fewer than this % of warps */
  int32_t run_skip;          /* advance whole tape words across runs of a self-loop (exact in every form):
                                0 never, 1 always, N >= 2 in the slices of warps where some running
                                machine has made N steps or more (younger machines' runs are short;
                                persistent kernel only: the plain kernel takes N >= 2 as 1, since
                                each of its launches waits for its oldest machine) */
  int64_t stack_nodes;       /* frontier stack capacity in nodes (0 = auto) */
} e13_tuning;

/* Runtime statistics of the last search on a context. */
typedef struct e13_stats {
  double device_ms;          /* CUDA-event time of the search on its stream */
  int64_t launches;          /* kernel launches (all kinds) */
  int64_t epochs;            /* persistent epochs / plain frontier launches */
  int64_t peak_nodes;        /* peak frontier stack */
  int64_t search_kernel_launches;
  double search_kernel_ms;   /* CUDA-event time summed over the search kernel's launches */
  double lane_occupancy;     /* running lanes / 32 averaged over warp rounds */
  int64_t warp_rounds;       /* warp rounds (slice + refill) */
  int64_t donations;         /* persistent: stack nodes donated to the pool */
  int64_t pool_claims;       /* persistent: pool nodes taken by warps without work */
  int64_t idle_polls;        /* persistent: polls by warps waiting for work */
  int64_t h2d_bytes;         /* host-to-device bytes the call copied (roots, control words, checkpoints) */
  int64_t d2h_bytes;         /* device-to-host bytes the call copied (control words, counters, survivors) */
} e13_stats;

typedef struct e13_ctx e13_ctx;

/* ---- host-side helpers (no device needed) ---- */

/* Zobrist keys of the 1364 window cells and stage-start block hashes TGT[0..9]
   (src/e13search.c:98-103, :437-444). */
void e13_keys(uint64_t key[1364], uint64_t tgt[E13_STAGES + 1]);

/* One cell "<w><L|R><next>" or "---" (src/e13search.c:105-108). */
int e13_parse_cell(const char *s);

/* Machine file: up to 16 rows of two cells (src/e13search.c:110-121).
   Returns the number of states, or E13_ERR_IO. */
int e13_load_machine(const char *path, int32_t base[E13_MAXCELLS]);
/* Same from text in memory. */
int e13_parse_machine(const char *text, int32_t base[E13_MAXCELLS]);

/* Candidate construction (src/e13search.c:317-355 setup, :423-426 set_sym).
   free_cells: 2*nq0 flags in base numbering (NULL = delete mode with fmax).
   lo < 0: no symmetry.  LO..HI are renumbered as set_sym() does; a negative
   renumbered LO (LO = 0 with X = -1) also means no symmetry, and an empty
   range changes nothing, both as in the reference.  Returns E13_OK,
   E13_ERR_FMAX, E13_ERR_SYM_NAMED or E13_ERR_SYM_START (E13_ERR_ARG for a
   range past the last state); job is filled as far as the reference gets. */
int e13_setup(const int32_t *base, int nq0, int X, int fmax, const uint8_t *free_cells, int lo, int hi,
              e13_job *job);

/* Survivor line in the reference's format (src/e13search.c:184-200), no
   newline.  Returns the length written (< len) or E13_ERR_ARG. */
int e13_format_survivor(const e13_job *job, const e13_survivor *s, char *buf, size_t len);

/* Summary line (src/e13search.c:413-416) without "split=/front=" (device path)
   and with wall seconds as given.  Returns the length written. */
int e13_format_summary(const e13_job *job, const e13_counts *c, double wall_s, char *buf, size_t len);

/* Fills t with the library defaults for this device. */
void e13_default_tuning(e13_tuning *t);

/* The tuning a search (serve = 0) or a serve session (serve = 1) runs with:
   the defaults, overridden by the nonzero fields of `in` (NULL: defaults; a
   serve session defaults to 10 ms epochs and always uses the persistent
   kernel).  Returns E13_ERR_ARG, and leaves *out alone, unless every field is
   in range: kernel 0..1, run_skip >= 0, block 64..768 and a multiple of 32,
   slice 1..4096, warp_stack 1..4096, epoch_us 1..6e7, epochs_per_graph 1..64,
   pool_low_pct 1..100, and step_cap, batch, stack_nodes >= 0.  Every
   entry point that takes a tuning applies this check first.  No counterpart
   in the reference, whose only knobs are E13_SPLIT (src/e13search.c:47-49)
   and E13_SLICE (src/e13gpu.py:342-346). */
int e13_resolve_tuning(const e13_tuning *in, int serve, e13_tuning *out);

/* ---- device path ---- */

/* Creates a context on CUDA device `device` (allocations happen lazily on
   the first search and are kept for reuse).  Returns E13_OK or an error. */
int e13_ctx_create(int device, e13_ctx **out);
void e13_ctx_destroy(e13_ctx *ctx);

/* The search for one job (src/e13search.c:357-420 run_delete; GPU reference
   src/e13gpu.py:381-461): enumerates every TNF leaf on the device.
   counts: exact totals.  surv: up to surv_cap records; *nsurv = survivors
   found (may exceed surv_cap: E13_ERR_SURV_CAP, counts still exact).
   tuning may be NULL (defaults).  Output order of survivors is undefined, as
   in the reference (src/e13search.c:185): compare sorted lines. */
int e13_search(e13_ctx *ctx, const e13_job *job, const e13_tuning *tuning, e13_counts *counts,
               e13_survivor *surv, int surv_cap, int *nsurv);

/* One share of a search, for spreading one big job over GPUs (one process
   per GPU).  The reference splits a search over OpenMP threads the same way:
   a serial expansion to a frontier, whose nodes are then dealt out
   (src/e13search.c:222-235, 376-403).  Here the plain kernel expands the job
   level by level until the frontier holds 512 nodes per shard.  The frontier
   is put in an order that depends only on its nodes, and shard s in [0,
   nshards) searches nodes s, s + nshards, ...  The leaves, steps and survivors
   that the expansion itself finishes count in shard 0 only.  So the counts
   of all shards add up to e13_search's, and their survivors together are its
   survivors.  Every shard must be given the same job; which nodes a shard
   holds does not depend on the tuning (the expansion uses fixed settings), so
   shards may run with different tunings.  nshards = 1
   is e13_search.  Returns as e13_search; E13_ERR_ARG for a shard out of
   range. */
int e13_search_shard(e13_ctx *ctx, const e13_job *job, const e13_tuning *tuning, int shard, int nshards,
                     e13_counts *counts, e13_survivor *surv, int surv_cap, int *nsurv);

/* ---- checkpoint / resume of one search ---- */

typedef struct e13_checkpoint {
  const char *path;     /* pointer file: names the last complete slot, "a" or "b"; the slots are
                           <path>.a.bin + <path>.a.meta and <path>.b.bin + <path>.b.meta */
  const char *config;   /* identity of the run (the CLI passes its arguments); a checkpoint written
                           under another config, job or node format is refused: E13_ERR_CKPT */
  double interval_s;    /* seconds between checkpoints; <= 0: 1800 (the reference's E13_CKPT_SEC) */
  double stop_after_s;  /* > 0: checkpoint and stop after this many seconds of this call */
} e13_checkpoint;

/* e13_search that survives being stopped (replaces E13_CKPT / E13_CKPT_SEC /
   <ckpt>.stop of src/e13gpu.py:349-409, 462-465).  Between epochs the whole
   state of a search is on the device: the frontier stack, the job's counters
   and its survivor records.  That state is written to the slot the pointer
   file does not name, and only then is the pointer file replaced (write, fsync,
   rename), so a crash during a save keeps the previous checkpoint.  A save
   happens every interval_s, when the file <path>.stop appears (looked for once
   a second; one left from an earlier clean stop is removed at the start), and
   after stop_after_s.  The last two stop the search: E13_STOPPED, with the
   counts so far in *counts and *nsurv.  If the pointer file exists at the
   start, the search resumes from its slot.  A finished search removes the
   checkpoint files and returns as e13_search does.  wall_s (may be NULL): wall
   seconds of the search over all calls; frontier (may be NULL): frontier nodes
   left at the stop (0 when finished). */
int e13_search_resumable(e13_ctx *ctx, const e13_job *job, const e13_tuning *tuning, const e13_checkpoint *ck,
                         e13_counts *counts, e13_survivor *surv, int surv_cap, int *nsurv, double *wall_s,
                         int64_t *frontier);

/* ---- size estimate of a search ---- */

typedef struct e13_estimate_out {
  double mean[4];       /* leaves, nodes, steps, survivors: the average weighted count over the probes */
  double std_error[4];  /* standard error of each mean (the reference's "+-") */
  int64_t probes;
} e13_estimate_out;

/* Knuth's random-probe estimate of the search for `job` (src/e13search.c:256-313
   probe, :473-510 estimate): each probe follows one random path from the
   root, runs every child of every fork on it, and continues into a live
   child drawn at random.  Probe p draws from the splitmix64 stream the
   reference gives its OpenMP thread p (start mix(0x5EED0000 + p + (seed << 20)),
   seed = E13_SEED), so every probe's counts depend only on (seed, p).
   per_probe (may be NULL): 4 doubles per probe, leaves, nodes, steps,
   survivors.  No counterpart of the per-probe layout in the reference, which
   sums per thread.  The reference hands probes to threads dynamically, so its
   printed numbers depend on scheduling; the numbers here are a different
   sample of the same estimator and match the reference probe for probe only
   (each probe's counts equal the oracle's restatement of probe() on the same
   stream), not line for line.  probes is at most E13_ESTIMATE_MAX_PROBES
   (2^20, the stride between the stream starts of seed and seed + 1), else
   E13_ERR_ARG. */
#define E13_ESTIMATE_MAX_PROBES (1LL << 20)
int e13_estimate(e13_ctx *ctx, const e13_job *job, int64_t probes, uint64_t seed, e13_estimate_out *out,
                 double *per_probe);

/* ---- serving: many searches in one persistent kernel ---- */

/* Continuous batching of search jobs (no counterpart in the reference, which
   runs one search per process).  Up to 16 jobs share the persistent kernel:
   every node carries its job's slot, and each job has its own counters and
   survivors.

   Admission is by the frontier memory a job needs.  e13_serve_submit sizes
   each job with the Knuth estimator (e13_estimate, 64 probes, seed 0): the
   frontier of a search never holds more machines than its tree has nodes and
   leaves, so a job whose estimated tree is below one epoch's dump of every
   warp reserves twice its estimate (at least 64 nodes), and a larger job
   reserves that dump bound.  reserve_nodes > 0 replaces the estimate by a
   fixed reservation per job.  First come, first served, a queued job is
   admitted when a slot is free, its submit time has passed and the frontier
   has room for every running job's reservation plus its own; a job alone is
   always admitted.  The serve stack holds tuning->stack_nodes nodes (0 = 16 Mi
   nodes, 5 GB), and a second buffer of the same size lets the frontier be
   regrouped between epochs, the job with the fewest live nodes on top.

   Estimates can be wrong.  When, after an epoch, the frontier leaves less
   room than the next epoch may need, jobs are swapped out, the one with the
   most live nodes first: its nodes and counters go to host memory and it goes
   back to the head of the queue, reserving twice the nodes it had; re-admitted,
   it goes on where it stopped, so its counts stay exact.  A job that does not
   fit even alone ends with status E13_ERR_OVERFLOW, and so does every running
   job when a device wait runs out (E13_ERR_TIMEOUT); the session goes on.

   e13_serve_step admits, runs one epoch (tuning->epoch_us, default 10 ms)
   and returns the jobs that finished in it: a job is finished when none of its
   nodes is left on the frontier.  Each job's counts equal those of e13_search
   on that job alone.  A context runs one serve session at a time and no
   e13_search meanwhile. */
typedef struct e13_serve e13_serve;
typedef struct e13_serve_result {
  int64_t id;
  int32_t status;            /* E13_OK; E13_ERR_SURV_CAP if survivor records were lost; E13_ERR_OVERFLOW /
                                E13_ERR_TIMEOUT if the job was cut short (counts then partial) */
  int32_t nsurv;             /* survivor records kept for e13_serve_survivors */
  e13_counts counts;
  double t_submit, t_start, t_done; /* seconds on the serve clock */
} e13_serve_result;

int e13_serve_create(e13_ctx *ctx, const e13_tuning *tuning, int64_t reserve_nodes, e13_serve **out);
void e13_serve_destroy(e13_serve *s);
/* Seconds since e13_serve_create. */
double e13_serve_clock(const e13_serve *s);
/* Queues a job; t_submit < 0 means now (serve clock).  Unless the session has
   a fixed reservation, runs the job's size estimate on the device first. */
int e13_serve_submit(e13_serve *s, const e13_job *job, int64_t id, double t_submit);
/* Queues one share of a job split over nshards (shard in [0, nshards)), for
   spreading a set of jobs over GPUs with one serve session per GPU: the job's
   frontier is expanded and dealt out as e13_search_shard does, the share then
   joins this session like any job, and the counts and survivors of all shards
   of a job add up to the job's.  The expansion runs here, on the device and on
   buffers of its own, before the call returns.  nshards = 1 is
   e13_serve_submit. */
int e13_serve_submit_shard(e13_serve *s, const e13_job *job, int64_t id, double t_submit, int shard, int nshards);
/* One admission + epoch + completion pass; done needs room for 16 results. */
int e13_serve_step(e13_serve *s, e13_serve_result *done, int cap, int *ndone);
/* Jobs queued or running. */
int64_t e13_serve_pending(const e13_serve *s);
/* Survivors of a finished job (once; *n = all it found). */
int e13_serve_survivors(e13_serve *s, int64_t id, e13_survivor *out, int cap, int *n);
/* CUDA-event time of all epochs, their number, how many times a job was
   swapped out to host memory, the largest frontier after an epoch and the
   largest share of it one job held, in nodes (each pointer may be NULL). */
int e13_serve_stats(const e13_serve *s, double *device_ms, int64_t *epochs, int64_t *swapped_out,
                    int64_t *peak_nodes, int64_t *peak_job_nodes);
/* Preempts a running job between steps: its frontier nodes and counters go
   to host memory and it returns to the head of the queue, to be resumed where
   it stopped when it is admitted again (its counts stay exact).  The same swap
   the session makes by itself when the frontier runs out of room; a caller
   uses it to make room for more urgent jobs.  E13_OK also for a job that is
   queued; E13_ERR_ARG for an unknown or finished id.  No counterpart in the
   reference. */
int e13_serve_preempt(e13_serve *s, int64_t id);

/* Autotuner (no counterpart in the reference, which has one fixed GPU
   launch shape, src/e13gpu.py:342-346, and a fixed serial split depth,
   E13_SPLIT, src/e13search.c:47-49): coordinate descent over block size
   (lanes per CTA, one CTA per SM), slice (iterations between a warp's refill
   rounds), warp_stack (the subtree depth a warp keeps to itself before it
   spills to the frontier or donates) and pool_low_pct (the donation threshold
   at which warps with deep stacks fork work off to idle warps), timing the
   persistent kernel with CUDA events.  The proxy is the workload itself at a
   fraction of its cost: shard 0 of proxy_shards of each of the n jobs
   (e13_serve_submit_shard; 0 or 1 = the whole jobs), all run together in one
   serve session, as a workload of several jobs runs.  Each axis keeps a value
   only if it is at least 3 % faster.  Every candidate must reproduce every
   job's counts, else E13_ERR_CUDA.  start may be NULL (defaults); *best_ms
   (may be NULL) is the best proxy time (epochs only). */
int e13_autotune_jobs(e13_ctx *ctx, const e13_job *jobs, int n, int32_t proxy_shards, const e13_tuning *start,
                      e13_tuning *best, double *best_ms);
/* e13_autotune_jobs for one job. */
int e13_autotune(e13_ctx *ctx, const e13_job *job, int32_t proxy_shards, const e13_tuning *start, e13_tuning *best,
                 double *best_ms);

/* Self-test of the persistent kernel's one device-side wait, for a caller
   (or a test) that wants to see a device wait run out without a hang: runs
   one epoch in which a warp claims a donation-pool slot whose data never
   arrives.  The warp waits wait_us (1 .. 1e6) for it, flags the timeout and
   the epoch ends.  Returns E13_ERR_TIMEOUT when the bounded wait works as it
   should; the context stays usable (the next search starts from a clean
   control block).  No counterpart in the reference, which has no device-side
   waits. */
int e13_selftest_pool_wait(e13_ctx *ctx, int32_t wait_us);

/* Statistics of the last e13_search on this context. */
int e13_last_stats(const e13_ctx *ctx, e13_stats *out);

/* Whole-table runs from the blank tape on the device, one machine per lane
   (src/e13search.c:428-433 run_full; modes base/mutant :447-460).
   tabs: n tables of 2*nq codes (stride E13_MAXCELLS); out: per machine
   {survived, stage, st0, head0, abs, rel, steps} as 7 int64. */
int e13_run_full(e13_ctx *ctx, const int32_t *tabs, int n, int nq, int64_t *out);

/* Raw-simulator throughput set: n whole tables run from the blank tape with
   no filter, at most max_steps steps each, stopping when the head leaves the
   window -64..1299 or reads a halt -- steps (3)-(7) of run()
   (src/e13search.c:163-175) without the stage test and the deadline; the step
   that leaves the window is not counted, as in run().  codes: n * 2*nq bytes
   (0..4nq-1 = moves, anything else = halt), or NULL to draw them on the device:
   cell i of machine m = splitmix64 draw m*2nq+i+1 from `seed`, mod 4nq (each
   cell uniform over write x dir x next).  out (may be NULL): per machine
   {steps, status (0 step cap, 1 left the window, 2 halt), final head, ones}.
   *total_steps (may be NULL) = sum of steps.  Device time: e13_last_stats. */
int e13_raw_run(e13_ctx *ctx, const uint8_t *codes, uint64_t seed, int64_t n, int nq, int64_t max_steps,
                int64_t *out, uint64_t *total_steps);

/* ---- hash-free deep checker (src/recheck.c, src/deep.c) ---- */

enum { E13_CHECK_RECHECK = 0, E13_CHECK_DEEP = 1 };

/* Input: one survivor as the checkers parse it (src/recheck.c:31-56). */
typedef struct e13_check_in {
  int32_t nq;
  int32_t st0;
  int32_t rel;               /* 1: head rule relative to the block end (!abs && rel) */
  int64_t head0;
  int8_t kind[E13_MAXCELLS]; /* 0 move, 1 halt, 2 free cell never read */
  int8_t write[E13_MAXCELLS];
  int8_t move[E13_MAXCELLS]; /* +1 R, -1 L */
  int8_t next[E13_MAXCELLS];
} e13_check_in;

/* Outcome per machine. */
enum {
  E13_CHK_OK = 0,            /* every stage 1..nmax reached */
  E13_CHK_LIMIT = 1,         /* stage not reached within the step limit */
  E13_CHK_OFFTAPE = 2,
  E13_CHK_FREE_READ = 3,     /* a never-read free cell was read */
  E13_CHK_HALT = 4
};

#define E13_CHECK_MAX_NMAX 20
#define E13_CHECK_MAX_ONES 64  /* counter ones recorded per stage start */

typedef struct e13_check_out {
  int32_t status;            /* E13_CHK_* */
  int32_t fail_stage;        /* stage at which it failed (status != OK) */
  int32_t free_state, free_sym; /* for E13_CHK_FREE_READ */
  int64_t fail_t;            /* step at the failure */
  int64_t fail_head;         /* head at the failure (deep's off-tape print) */
  int32_t stages_done;       /* stage starts found */
  int32_t pad;
  int64_t stage_t[E13_CHECK_MAX_NMAX + 1];   /* step of each stage start */
  int64_t minhead[E13_CHECK_MAX_NMAX + 1];   /* leftmost head before each start */
  int32_t nones[E13_CHECK_MAX_NMAX + 1];     /* ones at cells <= -3 (all of them) */
  int64_t leftmost[E13_CHECK_MAX_NMAX + 1];  /* leftmost one at cells <= -3 (0: none) */
  int32_t ones_cells[E13_CHECK_MAX_NMAX + 1][E13_CHECK_MAX_ONES]; /* their cells, -3 downwards */
} e13_check_out;

/* Re-runs machines from the blank tape to stage nmax without hashing, with
   recheck.c's step limit and tape (mode E13_CHECK_RECHECK, src/recheck.c:57-92)
   or deep.c's (E13_CHECK_DEEP, src/deep.c:49-80). */
int e13_check(e13_ctx *ctx, const e13_check_in *in, int n, int nmax, int mode, e13_check_out *out);

/* e13_check without any device allocation, for callers that cannot allocate:
   a process whose GPU memory is all handed out by another allocator (a
   framework's caching allocator or a fixed arena), or a latency-critical loop
   that must not pay cudaMalloc/cudaFree's implicit device synchronisation.
   This entry point has no counterpart in the reference.  The tapes, inputs and
   outputs of at most E13_CHECK_NOALLOC_MAX machines live in fixed device
   arrays compiled into the library (about 16 MB, held by every GPU that loads
   it until the process exits); n above that returns E13_ERR_NOALLOC_SIZE.
   in/out are host arrays of n entries, as for e13_check.  The work runs on a
   non-blocking stream of this entry point's own, one per device, and the call
   returns after synchronising that stream only (no device-wide wait, so a
   kernel the caller runs on another stream is not waited for).  Its first call
   on a device, with that device current, looks up the arrays' device addresses
   (cudaGetSymbolAddress) and creates that stream, once per device even when
   several threads make the first call together; make that first call before
   any stream capture.  All calls share the arrays and keep the last call's
   contents (each call clears what must start at zero): calls that overlap on
   the same GPU (other host threads) race and must be serialised by the
   caller. */
#define E13_CHECK_NOALLOC_MAX 16
int e13_check_noalloc(int device, const e13_check_in *in, int n, int nmax, int mode, e13_check_out *out);

/* Parses a SURVIVOR line into a checker input (src/recheck.c:28-56).
   Returns 1 on success, 0 if the line has no table. */
int e13_parse_survivor_line(const char *line, e13_check_in *in);

/* The checker input of a survivor that a search returned, without going
   through its text: the same input e13_parse_survivor_line gives for the line
   e13_format_survivor prints (the reference pipes e13search's SURVIVOR lines
   into recheck / deep, src/recheck.c:28-56).  Returns E13_OK or E13_ERR_ARG. */
int e13_survivor_check_in(const e13_job *job, const e13_survivor *s, e13_check_in *in);

/* ---- check.py: stages to 11 and crafted stage starts ---- */

#define E13_CRAFTED_MAX_CELLS 256  /* counter cells recorded per stage start */

/* src/check.py on the device, with its text.  lines: survivor lines as
   check.py reads them (lines without "table=" are skipped).  For each, the
   output holds the line (stripped) and one "   halt@<place>: PASS|FAIL ..."
   line per placement of the halt: the table's own halt, else each never-read
   ('?') cell in turn (src/check.py:102-162, :165-173).  out: a buffer of
   out_len bytes, NUL-terminated; *needed (may be NULL) = the bytes the text
   needs.  Returns E13_OK; E13_ERR_ARG if out is too small; E13_ERR_OVERFLOW
   if a counter held more than E13_CRAFTED_MAX_CELLS ones (its text is then
   not exact).  check.py's tape is unbounded; here a stage walk has cells
   -2^22 .. 2^22 and a crafted run -2^18 .. 2^18, and a run that leaves them
   is reported as "off tape" in place of check.py's outcome. */
int e13_check_crafted(e13_ctx *ctx, const char *const *lines, int n, char *out, size_t out_len, size_t *needed);

/* recheck.c's verdict text for one machine (src/recheck.c:71-99) from the
   device result; returns 1 if CONSISTENT. */
int e13_format_recheck(const e13_check_out *o, int nmax, char *buf, size_t len);

/* deep.c's per-machine text after "survivor <id> " (src/deep.c:53-81). */
int e13_format_deep(const e13_check_in *in, const e13_check_out *o, int nmax, char *buf, size_t len);

#ifdef __cplusplus
}
#endif
#endif /* E13_H */
