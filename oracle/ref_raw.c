/* ref_raw.c -- test infrastructure: runs the raw-simulator set through the
 * reference's own step loop, run() of src/e13search.c:134-177, compiled from
 * the reference source where it lies (oracle/Makefile's `ref` target includes
 * it into this file; nothing of it is copied here).
 *
 * The raw set has no filter, and run() always applies one, so the harness
 * switches the filter off from outside: KEY stays all zero (the reference's
 * main() is never called), so the hash hb stays 0, and TGT[] is set to 1, so
 * the stage test (hb == TGT[nt], :136) never fires; the deadline of the Sim is
 * set to max_steps - 1, so run() stops at exactly max_steps steps (:163).
 * Every cell is fixed, so run() never returns a fork.  What is left is steps
 * (3)-(7): read, halt, write, move, window test, state, t++ -- the raw
 * simulator's definition.
 *
 *   ref_raw SEED M0 N NQ MAX_STEPS
 *
 * draws tables M0 .. M0+N-1 of the set (cell i of machine m = splitmix64 draw
 * m*2nq + i + 1 from SEED, taken with the reference's splitmix(), mod 4nq)
 * and writes per machine 4 int64 (steps, status 0 cap / 1 left the window /
 * 2 halt, final head, ones on the tape) to stdout in binary.
 */
#define main e13search_main
#include E13_REF_SOURCE
#undef main

static long long ones_on(const Sim *s) {
  long long n = 0;
  for (int i = 0; i < TAPE; i++) n += s->tape[i];
  return n;
}

int main(int argc, char **argv) {
  if (argc != 6) {
    fprintf(stderr, "usage: ref_raw SEED M0 N NQ MAX_STEPS\n");
    return 1;
  }
  const uint64_t seed = strtoull(argv[1], NULL, 10);
  const long m0 = atol(argv[2]), n = atol(argv[3]);
  const int nq = atoi(argv[4]);
  const long max_steps = atol(argv[5]);
  if (nq < 1 || nq > MAXQ || n < 0 || m0 < 0 || max_steps < 1) return 1;
  for (int i = 0; i <= NS; i++) TGT[i] = 1; /* hb stays 0: no stage start is ever seen */
  int tab[2 * MAXQ];
  unsigned char fixed[2 * MAXQ];
  memset(fixed, 1, sizeof fixed);
  static Sim s;
  for (long m = m0; m < m0 + n; m++) {
    uint64_t state = seed + (uint64_t)(m * 2 * nq) * 0x9E3779B97F4A7C15ULL; /* draw m*2nq+1 comes next */
    for (int i = 0; i < 2 * nq; i++) tab[i] = (int)(splitmix(&state) % (uint64_t)(4 * nq));
    sim_init(&s);
    s.deadline = max_steps - 1;
    const int r = run(&s, tab, fixed);
    long long out[4];
    int status;
    if (r != DEAD) status = -1; /* cannot happen: every cell is fixed and no stage start fires */
    else if (s.t > s.deadline) status = 0;
    else if (s.head <= -LO || s.head >= HI - 1) status = 1;
    else status = 2;
    out[0] = s.t;
    out[1] = status;
    out[2] = s.head;
    out[3] = ones_on(&s);
    fwrite(out, sizeof out, 1, stdout);
  }
  return 0;
}
