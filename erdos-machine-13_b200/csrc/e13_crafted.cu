// e13_crafted.cu -- src/check.py on the device: the hash-free stage walk of a
// survivor to stage 11, and its crafted stage starts.
//
// check.py (src/check.py:1-173) runs every survivor table once per placement
// of its halt: the table's own halt, or each never-read cell in turn.
//   1. From the blank tape, stage n = 1 .. 11 starts at the first step where
//      the ones at cells >= -2 are exactly the block -1 .. 2^n - 2 and (n > 1)
//      the state and head match stage 1 (same cell, or the same offset from the
//      block end); at most 40 * 4^n + 1000 steps per stage.  The ones at cells
//      < -2 (the counter) are recorded at each start.  The counter must depend
//      only on c(n) = #{1 <= k < n : 2^k has no digit 2 in base 3}, and differ
//      between values of c.
//   2. From crafted starts (the counter of c = 0, 1, 2, a block of m = 2 .. 40
//      ones) the machine must halt iff c = 2 and m has no digit 2, and otherwise
//      reach the start with block 2m and the counter of c or c + 1, within
//      40 m^2 + 5000 steps.
//
// Device work: one lane per stage walk (about 3.3e6 steps for erdos_14), one
// lane per crafted run (at most 117 per placement).  Each lane's tape is a bit
// array in HBM with the word under the head kept in a register.  check.py's
// tape is unbounded; here it is cells -2^22 .. 2^22 for the walk and -2^18 ..
// 2^18 for a crafted run (|head - start| <= 69,000 there).  A head that leaves
// it ends the run as "off tape", which check.py cannot print; the verdict line
// then says so.  The host applies check.py's rules to the recorded starts and
// run outcomes and prints its text.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <string>
#include <vector>

#include "e13.h"

namespace {

typedef unsigned int u32;
typedef long long i64;

constexpr int kNmax = 11;   // src/check.py:20
constexpr int kMmax = 40;   // src/check.py:21
constexpr int kCells = E13_CRAFTED_MAX_CELLS;  // counter cells recorded per start
constexpr int kBlock = 64;
constexpr i64 kWalkSide = 1LL << 22;   // stage walk: cells -2^22 .. 2^22 - 1
constexpr i64 kRunSide = 1LL << 18;    // crafted run: cells -2^18 .. 2^18 - 1
constexpr int kWalkBatch = 2048;       // walks per launch (1 MiB of tape each)
constexpr int kRunBatch = 16384;       // crafted runs per launch (64 KiB of tape each)

enum { kStop = 0, kHalt = 1, kLimit = 2, kOff = 3 };
const char *const kResName[4] = {"stop", "halt", "limit", "off tape"};

// a cell entry: bit 0 write, bit 1 right, bits 2..5 next state, bit 7 halt
struct WalkIn {
  unsigned char code[32];
};

struct WalkOut {
  int32_t nstarts, res, fail_n, overflow;
  int64_t fail_total;
  int32_t st[kNmax];
  int64_t head[kNmax];
  int64_t total[kNmax];
  int32_t ncnt[kNmax];
  int32_t cnt[kNmax][kCells];
};

struct RunIn {
  int32_t walk;            // index of the placement (its table)
  int32_t c, m, s0;        // counter class, block size, stage-1 state
  int64_t h0;              // stage-1 head
  int32_t absolute;        // every stage start at head h0
  int32_t cnt_off, ncnt;   // the counter's cells in the shared cell array
  int32_t pad;
};

struct RunOut {
  int32_t res, ncnt, overflow, pad;
  int64_t t;
  int32_t cnt[kCells];
};

struct Stop {
  i64 size, h0, hh;
  int s0;
  int stage_one, crafted;
};

// cells -1 .. size - 2 all ones?  (the rest of the stop test is in run())
__device__ bool block_ok(const u32 *tape, i64 side, i64 size) {
  const i64 a = side - 1, b = side + size - 2;
  for (i64 w = a >> 5; w <= (b >> 5); ++w) {
    u32 mask = ~0u;
    if (w == (a >> 5)) mask &= ~0u << (a & 31);
    if (w == (b >> 5)) mask &= ~0u >> (31 - (b & 31));
    if ((tape[w] & mask) != mask) return false;
  }
  return true;
}

struct Machine {
  i64 head, ones_ge, minhead;
  int st;
};

// run_tracked (src/check.py:55-77): before each of at most `limit` steps,
// the stop test; then a halt cell ends the run, else write, move, next state.
__device__ int run(const u32 *rows, int stride, u32 *tape, i64 side, Machine &M, const Stop &S, i64 limit,
                   i64 &steps) {
  const i64 nwords = (2 * side) >> 5;
  i64 pos = M.head + side;
  i64 ww = pos >> 5;
  int bit = (int)(pos & 31);
  u32 word = tape[ww];
  int res = kLimit;
  i64 k = 0;
  for (;; ++k) {
    if (k == limit) break;
    if (M.ones_ge == S.size &&
        (S.stage_one ||
         (M.st == S.s0 && (S.crafted ? M.head == S.hh : (M.head == S.h0 || M.head - S.size == S.h0 - 2))))) {
      tape[ww] = word;
      if (block_ok(tape, side, S.size)) {
        res = kStop;
        break;
      }
    }
    const u32 sym = (word >> bit) & 1u;
    const u32 e = (rows[M.st * stride] >> (8 * sym)) & 0xFFu;
    if (e & 0x80u) {
      res = kHalt;
      break;
    }
    const u32 w = e & 1u;
    if (w != sym) {
      word ^= 1u << bit;
      if (M.head >= -2) M.ones_ge += w ? 1 : -1;
    }
    M.st = (int)((e >> 2) & 15u);
    if (e & 2u) {
      ++M.head;
      if (++bit == 32) {
        tape[ww] = word;
        bit = 0;
        if (++ww >= nwords) {
          res = kOff;
          ++k;
          break;
        }
        word = tape[ww];
      }
    } else {
      --M.head;
      if (M.head < M.minhead) M.minhead = M.head;
      if (--bit < 0) {
        tape[ww] = word;
        bit = 31;
        if (--ww < 0) {
          res = kOff;
          ++k;
          break;
        }
        word = tape[ww];
      }
    }
  }
  if (res != kOff) tape[ww] = word;
  steps = k;
  return res;
}

// the ones at cells minhead .. -3, ascending (check.py:51-52)
__device__ int counter_cells(const u32 *tape, i64 side, i64 minhead, int32_t *cells, int32_t &overflow) {
  int n = 0;
  const i64 a = (minhead > -side ? minhead : -side) + side, b = side - 3;
  for (i64 w = a >> 5; w <= (b >> 5) && a <= b; ++w) {
    u32 x = tape[w];
    if (w == (a >> 5)) x &= ~0u << (a & 31);
    if (w == (b >> 5)) x &= ~0u >> (31 - (b & 31));
    while (x) {
      const int bpos = __ffs(x) - 1;
      x &= x - 1;
      if (n < kCells) cells[n] = (int32_t)((w << 5) + bpos - side);
      else overflow = 1;
      ++n;
    }
  }
  return n < kCells ? n : kCells;
}

__device__ void load_rows(u32 *rows, int stride, const unsigned char *code) {
  for (int s = 0; s < 16; ++s) rows[s * stride] = (u32)code[2 * s] | ((u32)code[2 * s + 1] << 8);
}

__global__ void __launch_bounds__(kBlock) walk_kernel(const WalkIn *in, int n, u32 *tapes, WalkOut *out) {
  __shared__ u32 s_rows[16 * kBlock];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u32 *rows = s_rows + threadIdx.x;
  load_rows(rows, blockDim.x, in[i].code);
  u32 *tape = tapes + (i64)i * ((2 * kWalkSide) >> 5);
  WalkOut &o = out[i];
  o.nstarts = 0;
  o.res = kStop;
  o.fail_n = 0;
  o.overflow = 0;
  o.fail_total = 0;
  Machine M{0, 0, 0, 0};
  i64 total = 0;
  for (int k = 1; k <= kNmax; ++k) {
    Stop S{1LL << k, k > 1 ? o.head[0] : 0, 0, k > 1 ? o.st[0] : 0, k == 1, 0};
    i64 t = 0;
    const int res = run(rows, blockDim.x, tape, kWalkSide, M, S, 40LL * (1LL << (2 * k)) + 1000, t);
    total += t;
    if (res != kStop) {
      o.res = res;
      o.fail_n = k;
      o.fail_total = total;
      return;
    }
    const int j = o.nstarts++;
    o.st[j] = M.st;
    o.head[j] = M.head;
    o.total[j] = total;
    o.ncnt[j] = counter_cells(tape, kWalkSide, M.minhead, o.cnt[j], o.overflow);
  }
}

__global__ void __launch_bounds__(kBlock) run_kernel(const RunIn *in, int n, const WalkIn *tables,
                                                     const int32_t *cells, u32 *tapes, RunOut *out) {
  __shared__ u32 s_rows[16 * kBlock];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const RunIn &r = in[i];
  u32 *rows = s_rows + threadIdx.x;
  load_rows(rows, blockDim.x, tables[r.walk].code);
  u32 *tape = tapes + (i64)i * ((2 * kRunSide) >> 5);
  RunOut &o = out[i];
  o.overflow = 0;
  o.ncnt = 0;
  // the crafted start (src/check.py:131-135): counter of c, block -1 .. m - 2
  Machine M{r.absolute ? r.h0 : r.h0 - 2 + r.m, r.m, 0, r.s0};
  M.minhead = M.head;
  for (int k = 0; k < r.ncnt; ++k) {
    const i64 c = cells[r.cnt_off + k];
    if (c < -kRunSide) {  // a counter cell beyond this tape: cannot run exactly
      o.res = kOff;
      o.t = 0;
      return;
    }
    const i64 pos = c + kRunSide;
    tape[pos >> 5] |= 1u << (pos & 31);
    if (c < M.minhead) M.minhead = c;
  }
  for (i64 c = -1; c < r.m - 1; ++c) {
    const i64 pos = c + kRunSide;
    tape[pos >> 5] |= 1u << (pos & 31);
  }
  const i64 nxt = 2LL * r.m;
  Stop S{nxt, r.h0, r.absolute ? r.h0 : r.h0 - 2 + nxt, r.s0, 0, 1};
  i64 t = 0;
  o.res = run(rows, blockDim.x, tape, kRunSide, M, S, 40LL * r.m * r.m + 5000, t);
  o.t = t;
  if (o.res == kStop) o.ncnt = counter_cells(tape, kRunSide, M.minhead, o.cnt, o.overflow);
}

// ---- host

bool no_two(i64 m) {
  while (m) {
    if (m % 3 == 2) return false;
    m /= 3;
  }
  return true;
}

// class c(n) of stage n (src/check.py:119)
int stage_class(int n) {
  int c = 0;
  for (int k = 1; k < n; ++k) c += no_two(1LL << k);
  return c;
}

// Python's repr of a tuple of ints
std::string tuple_repr(const int32_t *v, int n) {
  std::string s = "(";
  char b[24];
  for (int i = 0; i < n; ++i) {
    snprintf(b, sizeof b, i ? ", %d" : "%d", v[i]);
    s += b;
  }
  s += n == 1 ? ",)" : ")";
  return s;
}

bool same_cells(const int32_t *a, int na, const int32_t *b, int nb) {
  return na == nb && std::equal(a, a + na, b);
}

struct Line {
  std::string text;  // stripped
  WalkIn table;
  std::vector<int> unread;
  bool has_halt = false;
  bool has_table = false;
};

Line parse_line(const char *line) {
  Line L;
  const char *s = line, *e = line + strlen(line);
  while (*s == ' ' || *s == '\t' || *s == '\n' || *s == '\r') ++s;
  while (e > s && (e[-1] == ' ' || e[-1] == '\t' || e[-1] == '\n' || e[-1] == '\r')) --e;
  L.text.assign(s, e);
  memset(L.table.code, 0x80, sizeof L.table.code);
  const char *tb = strstr(line, "table=");
  if (!tb) return L;
  L.has_table = true;
  const char *q = tb + 6;
  int ncell = 0;
  while (*q && *q != '\n' && *q != '\r' && ncell < 32) {
    while (*q == ' ' || *q == '\t' || *q == '|') ++q;
    if (!*q || *q == '\n' || *q == '\r') break;
    bool un = false;
    if (*q == '?') {
      un = true;
      ++q;
    }
    if (*q == '-') {
      L.table.code[ncell] = 0x80;
      L.has_halt = true;
      q += 3;
    } else {
      const int w = *q++ - '0';
      const int right = *q++ == 'R';
      char *endp = nullptr;
      const long nx = strtol(q, &endp, 10);
      q = endp;
      L.table.code[ncell] = (unsigned char)((w & 1) | (right << 1) | ((nx & 15) << 2));
    }
    if (un) L.unread.push_back(ncell);
    ++ncell;
  }
  return L;
}

struct Placement {
  int line, place;  // place -1: the table as given ("None")
};

}  // namespace

extern "C" int e13_ctx_device(const e13_ctx *c);
extern "C" cudaStream_t e13_ctx_stream(const e13_ctx *c);

#define CKC(x)                                  \
  do {                                          \
    if ((x) != cudaSuccess) {                   \
      rc = E13_ERR_CUDA;                        \
      goto done;                                \
    }                                           \
  } while (0)

extern "C" int e13_check_crafted(e13_ctx *ctx, const char *const *lines, int n, char *out, size_t out_len,
                                 size_t *needed) {
  if (!ctx || (n > 0 && !lines) || n < 0 || (out_len > 0 && !out)) return E13_ERR_ARG;
  if (cudaSetDevice(e13_ctx_device(ctx)) != cudaSuccess) return E13_ERR_CUDA;
  cudaStream_t stream = e13_ctx_stream(ctx);

  // placements of the halt (src/check.py:104-111)
  std::vector<Line> L;
  std::vector<Placement> P;
  std::vector<WalkIn> tables;
  for (int i = 0; i < n; ++i) {
    L.push_back(parse_line(lines[i] ? lines[i] : ""));
    const Line &l = L.back();
    if (!l.has_table) continue;
    if (l.has_halt) {
      P.push_back({i, -1});
      tables.push_back(l.table);
    } else {
      for (int c : l.unread) {
        P.push_back({i, c});
        WalkIn t = l.table;
        t.code[c] = 0x80;
        tables.push_back(t);
      }
    }
  }
  const int np = (int)P.size();
  std::vector<WalkOut> walks(np);
  std::vector<RunIn> runs;
  std::vector<int32_t> cells;
  std::vector<RunOut> runouts;
  std::vector<std::string> verdict(np);
  std::vector<int> run_first(np, -1), run_count(np, 0);
  // per placement: the start index of each class c (first start with that c), -1 if none
  std::vector<std::array<int, 3>> first(np);
  std::vector<int> absolute(np, 1);
  WalkIn *d_tables = nullptr;
  WalkOut *d_walk = nullptr;
  RunIn *d_runs = nullptr;
  RunOut *d_rout = nullptr;
  int32_t *d_cells = nullptr;
  u32 *d_tape = nullptr;
  int rc = E13_OK;
  bool overflow = false;
  std::string text;

  if (np > 0) {
    CKC(cudaMalloc(&d_tables, sizeof(WalkIn) * np));
    CKC(cudaMemcpyAsync(d_tables, tables.data(), sizeof(WalkIn) * np, cudaMemcpyHostToDevice, stream));
    const int wb = std::min(np, kWalkBatch);
    CKC(cudaMalloc(&d_walk, sizeof(WalkOut) * wb));
    CKC(cudaMalloc(&d_tape, (size_t)wb * ((2 * kWalkSide) >> 5) * sizeof(u32)));
    for (int b0 = 0; b0 < np; b0 += kWalkBatch) {
      const int nb = std::min(kWalkBatch, np - b0);
      CKC(cudaMemsetAsync(d_tape, 0, (size_t)nb * ((2 * kWalkSide) >> 5) * sizeof(u32), stream));
      walk_kernel<<<(nb + kBlock - 1) / kBlock, kBlock, 0, stream>>>(d_tables + b0, nb, d_tape, d_walk);
      CKC(cudaGetLastError());
      CKC(cudaMemcpyAsync(walks.data() + b0, d_walk, sizeof(WalkOut) * nb, cudaMemcpyDeviceToHost, stream));
      CKC(cudaStreamSynchronize(stream));
    }
    cudaFree(d_tape);
    d_tape = nullptr;
  }

  // stages and counter classes (src/check.py:112-126), then the crafted runs
  for (int p = 0; p < np; ++p) {
    const WalkOut &w = walks[p];
    char place[16];
    if (P[p].place < 0) snprintf(place, sizeof place, "None");
    else snprintf(place, sizeof place, "%d", P[p].place);
    if (w.overflow) overflow = true;
    if (w.nstarts < kNmax) {
      char b[160];
      snprintf(b, sizeof b, "   halt@%s: FAIL stage %d: %s at step %lld", place, w.fail_n, kResName[w.res],
               (long long)w.fail_total);
      verdict[p] = b;
      continue;
    }
    std::array<int, 3> f = {-1, -1, -1};
    std::string bad;
    for (int j = 0; j < w.nstarts; ++j) {
      const int c = stage_class(j + 1);
      if (f[c] >= 0 && !same_cells(w.cnt[f[c]], w.ncnt[f[c]], w.cnt[j], w.ncnt[j])) {
        char b[96];
        snprintf(b, sizeof b, "counter differs within c=%d at n=%d", c, j + 1);
        bad = b;
      }
      if (f[c] < 0) f[c] = j;
    }
    int keys = 0, distinct = 0;
    for (int c = 0; c < 3; ++c) {
      if (f[c] < 0) continue;
      ++keys;
      bool dup = false;
      for (int d = 0; d < c; ++d)
        if (f[d] >= 0 && same_cells(w.cnt[f[d]], w.ncnt[f[d]], w.cnt[f[c]], w.ncnt[f[c]])) dup = true;
      distinct += !dup;
    }
    if (distinct != keys) bad = "counter equal for different c";
    if (!bad.empty()) {
      verdict[p] = std::string("   halt@") + place + ": FAIL " + bad;
      continue;
    }
    first[p] = f;
    for (int j = 0; j < w.nstarts; ++j)
      if (w.head[j] != w.head[0]) absolute[p] = 0;
    run_first[p] = (int)runs.size();
    for (int c = 0; c < 3; ++c) {
      if (f[c] < 0) continue;
      const int off = (int)cells.size();
      cells.insert(cells.end(), w.cnt[f[c]], w.cnt[f[c]] + w.ncnt[f[c]]);
      for (int m = 2; m <= kMmax; ++m)
        runs.push_back({p, c, m, w.st[0], w.head[0], absolute[p], off, w.ncnt[f[c]], 0});
    }
    run_count[p] = (int)runs.size() - run_first[p];
  }

  if (!runs.empty()) {
    const int nr = (int)runs.size();
    runouts.resize(nr);
    const int rb = std::min(nr, kRunBatch);
    CKC(cudaMalloc(&d_runs, sizeof(RunIn) * nr));
    CKC(cudaMalloc(&d_cells, sizeof(int32_t) * std::max<size_t>(cells.size(), 1)));
    CKC(cudaMalloc(&d_rout, sizeof(RunOut) * rb));
    CKC(cudaMalloc(&d_tape, (size_t)rb * ((2 * kRunSide) >> 5) * sizeof(u32)));
    CKC(cudaMemcpyAsync(d_runs, runs.data(), sizeof(RunIn) * nr, cudaMemcpyHostToDevice, stream));
    if (!cells.empty())
      CKC(cudaMemcpyAsync(d_cells, cells.data(), sizeof(int32_t) * cells.size(), cudaMemcpyHostToDevice, stream));
    for (int b0 = 0; b0 < nr; b0 += kRunBatch) {
      const int nb = std::min(kRunBatch, nr - b0);
      CKC(cudaMemsetAsync(d_tape, 0, (size_t)nb * ((2 * kRunSide) >> 5) * sizeof(u32), stream));
      run_kernel<<<(nb + kBlock - 1) / kBlock, kBlock, 0, stream>>>(d_runs + b0, nb, d_tables, d_cells, d_tape, d_rout);
      CKC(cudaGetLastError());
      CKC(cudaMemcpyAsync(runouts.data() + b0, d_rout, sizeof(RunOut) * nb, cudaMemcpyDeviceToHost, stream));
      CKC(cudaStreamSynchronize(stream));
    }
  }

  // the crafted verdicts (src/check.py:137-162)
  for (int p = 0; p < np; ++p) {
    if (run_first[p] < 0) continue;
    const WalkOut &w = walks[p];
    const std::array<int, 3> &f = first[p];
    int nfails = 0;
    std::string fails;
    for (int k = 0; k < run_count[p]; ++k) {
      const RunIn &r = runs[run_first[p] + k];
      const RunOut &o = runouts[run_first[p] + k];
      if (o.overflow) overflow = true;
      const int c = r.c, m = r.m;
      const int want_c = no_two(m) ? c + 1 : c;
      const bool want_halt = no_two(m) && c == 2;
      std::string msg;
      char b[160];
      if (want_halt) {
        if (o.res != kHalt) msg = std::string("expected halt, got ") + kResName[o.res];
      } else if (o.res != kStop) {
        snprintf(b, sizeof b, "expected stage 2m, got %s at %lld", kResName[o.res], (long long)o.t);
        msg = b;
      } else if (want_c < 3 && f[want_c] >= 0) {
        if (!same_cells(o.cnt, o.ncnt, w.cnt[f[want_c]], w.ncnt[f[want_c]])) {
          snprintf(b, sizeof b, " != c=%d ", want_c);
          msg = "counter " + tuple_repr(o.cnt, o.ncnt) + b + tuple_repr(w.cnt[f[want_c]], w.ncnt[f[want_c]]);
        }
      } else {
        for (int d = 0; d < 3; ++d)
          if (f[d] >= 0 && same_cells(o.cnt, o.ncnt, w.cnt[f[d]], w.ncnt[f[d]]))
            msg = "counter for c=3 equals an earlier one";
      }
      if (!msg.empty()) {
        if (nfails < 4) {
          snprintf(b, sizeof b, "%s(%d, %d, '", nfails ? ", " : "", c, m);
          fails += b + msg + "')";
        }
        ++nfails;
      }
    }
    char place[16];
    if (P[p].place < 0) snprintf(place, sizeof place, "None");
    else snprintf(place, sizeof place, "%d", P[p].place);
    char head[160];
    snprintf(head, sizeof head, "   halt@%s: %s stages ok to n=%d (step %lld); counters {", place,
             nfails ? "FAIL" : "PASS", kNmax, (long long)w.total[w.nstarts - 1]);
    std::string v = head;
    bool firstkey = true;
    for (int c = 0; c < 3; ++c) {
      if (f[c] < 0) continue;
      v += (firstkey ? "" : ", ") + std::to_string(c) + ": " + tuple_repr(w.cnt[f[c]], w.ncnt[f[c]]);
      firstkey = false;
    }
    v += "}; crafted fails " + std::to_string(nfails) + ": [" + fails + "]";
    verdict[p] = v;
  }

  // check.py's output (:165-173): each line with a table, then its verdicts
  {
    int p = 0;
    for (int i = 0; i < n; ++i) {
      if (!L[i].has_table) continue;
      text += L[i].text + "\n";
      while (p < np && P[p].line == i) text += verdict[p++] + "\n";
    }
  }
  if (needed) *needed = text.size() + 1;
  if (text.size() + 1 > out_len) {
    rc = E13_ERR_ARG;
  } else {
    memcpy(out, text.c_str(), text.size() + 1);
    if (overflow) rc = E13_ERR_OVERFLOW;
  }
done:
  cudaFree(d_tables);
  cudaFree(d_walk);
  cudaFree(d_runs);
  cudaFree(d_rout);
  cudaFree(d_cells);
  cudaFree(d_tape);
  return rc;
}
