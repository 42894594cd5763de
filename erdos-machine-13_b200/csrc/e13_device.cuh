// e13_device.cuh -- device-side pieces shared by the search kernels, the
// whole-table runner and the survivor checker of libe13b200.so (sm_100a).
//
// One Turing machine per lane.  A lane's tape (1364 cells, bit-packed into 43
// words) and its table (16 rows of two 16-bit cell slots) live in shared
// memory, interleaved by lane: word w of lane l sits at [w * blockDim + l], so
// every lane always hits its own bank and a warp-wide access never conflicts.
//
// Semantics follow the reference's run() (src/e13search.c:134-177) step for
// step: stage test, deadline, read, fork on a first read, halt, write + hash,
// move, window bounds, state, t++.
#pragma once
#include <stddef.h>
#include <stdint.h>

namespace e13dev {

typedef unsigned long long u64;
typedef unsigned int u32;

constexpr int kTapeCells = 1364;  // cells -64 .. 1299 (src/e13search.c:59-61)
constexpr int kTapeWords = 43;    // ceil(1364 / 32)
constexpr int kLeft = 64;
constexpr int kStages = 9;
constexpr int kCounterCells = 62; // cells < -2 hash into the counter hash hc

// Cell entry (one byte): 0..63 a move (the reference's code), plus flags.
constexpr u32 kEntHalt = 0x40;    // halt
constexpr u32 kEntUnread = 0x80;  // never read yet: the first read is an event
constexpr u32 kEntFree = 0xFF;    // free cell, no move yet (FORCED, src/e13search.c:66)
constexpr u32 kEntSpecial = 0xC0; // any of the above: leaves the fast path
// Bit 8 of a cell's 16-bit slot in a row: the cell is a read self-loop (next
// state = this state, writes the symbol it reads), so the head sweeps a run of
// that symbol; the step loop then advances over the run a word at a time.
constexpr u32 kEntSelf = 0x100;

// Node flags byte.
constexpr int kFlagAbs = 1, kFlagRel = 2, kFlagCs0 = 4, kFlagKeep = 32;

// A machine stopped at a fork (pend = the cell being read for the first time)
// or between slices (pend = -1, one child: go on).  Children still to run: the
// keep child (kFlagKeep) and the alternatives in vmask (bit v = move v).
struct __align__(16) Node {
  u64 hb;             // low 32 bits of the hash of the ones at cells >= -2 (Lane::hb)
  u64 ch[3];          // counter hash at the first stage start with c = 0, 1, 2
  u64 vmask;
  int p, st, t, deadline;  // p = head + 64
  signed char nt, stage, st0, flags;
  short p0, pend;
  unsigned char nintro, budget, job, pad1;  // job: the slot of the search this machine belongs to
  u32 pad2[3];
  unsigned short cellv[32];  // cell entries with the self-loop bit; row s = cellv[2s] | cellv[2s+1] << 16
  u32 tape[kTapeWords];
  u32 pad3;
};
static_assert(sizeof(Node) % 16 == 0, "Node must be a whole number of 16-byte chunks");
// cellv is read and written as uint4 (four rows at a time): it must start on a 16-byte boundary
static_assert(offsetof(Node, cellv) % 16 == 0, "Node::cellv must be 16-byte aligned");
static_assert(offsetof(Node, tape) % 4 == 0, "Node::tape must be word aligned");
constexpr int kNodeChunks = sizeof(Node) / 16;

// Survivor record written by the device.
struct SurvRec {
  unsigned char ent[32];
  int st0, head0, abs_ok, rel_ok, t, job, pad[2];
};

// Several searches ("jobs") can share one persistent kernel: every node, lane
// and survivor record carries its job's slot.  Per-job constants and counters:
constexpr int kMaxJobs = 16;
struct JobParam {
  int nv, sym_lo, sym_hi, pad;  // 4 * nq moves; relabel-symmetry range (-1: off)
};
constexpr int kJobCounters = 2 + kStages + 1;  // leaves, steps, deaths by stage 0..9

// Control block of one search (device memory).
struct Ctl {
  long long top;                 // nodes on the frontier stack
  long long batch;               // this launch's input: stack[top - batch .. top)
  unsigned long long cursor;     // input nodes taken
  unsigned long long nout;       // nodes written to the output buffer
  long long peak;
  unsigned long long nsurv;      // survivors found (records kept: min(nsurv, cap))
  int dump;                      // persistent: end the epoch now
  int busy;                      // persistent: warps holding work or claiming it
  int idle;                      // persistent: warps waiting for work (starved)
  int deep;                      // persistent: warps holding 2 or more stack nodes (work a dump would spread)
  int error;                     // kErr* bits
  int launches;
  // utilisation counters: warp rounds, running lanes summed over rounds,
  // pool donations and claims, idle-warp polls
  u64 rounds, lane_rounds, donations, claims, polls;
  // persistent: nodes donated by warps with deep stacks to warps without work
  // (slots [pool_head, pool_tail) are waiting; each counter on its own cache line)
  alignas(128) unsigned long long pool_head;
  alignas(128) unsigned long long pool_tail;
};
constexpr int kErrOverflow = 1, kErrOutFull = 2, kErrTimeout = 4;

// The filter's constant tables (set by the host from e13_keys()).
__constant__ u64 c_key[kTapeCells];
__constant__ u64 c_tgt[kStages + 2];
__constant__ int c_deadline[kStages + 2];  // 4 * erdos_14 stage step + 64 (src/e13search.c:159)
__constant__ int c_exc[kStages + 1];       // exceptions by stage (src/e13search.c:71)

// Shared-memory key tables of the filter, in one block of kKeySmemBytes:
// the full keys of cells < -2 (the counter hash, rebuilt from the tape at a
// stage test), then the low and the high halves of the keys of cells >= -2
// (zero below -2).  The step loop keeps only the low half of hb and reads
// only `lo`; the high half is rebuilt from the tape with `hi` where a stage
// start would be accepted (stage_check).
struct KeyTabs {
  u64 *c;
  u32 *lo, *hi;
};
constexpr int kKeySmemBytes = 64 * 8 + kTapeCells * 8;

__device__ __forceinline__ KeyTabs key_tables(unsigned char *smem) {
  KeyTabs k;
  k.c = reinterpret_cast<u64 *>(smem);
  k.lo = reinterpret_cast<u32 *>(k.c + 64);
  k.hi = k.lo + kTapeCells;
  return k;
}

// Fills the key tables (every thread of the block takes part; the caller
// synchronises before the first use).
__device__ __forceinline__ void fill_key_tables(const KeyTabs &k) {
  for (int i = threadIdx.x; i < kTapeCells; i += blockDim.x) {
    const u64 v = (i >= kCounterCells) ? c_key[i] : 0ull;
    k.lo[i] = (u32)v;
    k.hi[i] = (u32)(v >> 32);
  }
  for (int i = threadIdx.x; i < 64; i += blockDim.x) k.c[i] = (i < kCounterCells) ? c_key[i] : 0ull;
}

// Shared-memory copies of the stage tables: lanes of a warp index them by
// their own stage, which constant memory would serialise.  Every kernel that
// runs the filter fills them with load_stage_tables() before its first step.
__shared__ u64 s_tgt[kStages + 2];
__shared__ int s_deadline[kStages + 2];
__shared__ int s_exc[kStages + 1];

__device__ __forceinline__ void load_stage_tables() {
  if (threadIdx.x < kStages + 2) {
    s_tgt[threadIdx.x] = c_tgt[threadIdx.x];
    s_deadline[threadIdx.x] = c_deadline[threadIdx.x];
  }
  if (threadIdx.x < kStages + 1) s_exc[threadIdx.x] = c_exc[threadIdx.x];
}

enum { kEvRun = 0, kEvDead = 1, kEvSurv = 2, kEvStage = 3, kEvCell = 4 };

// Registers of one lane's machine.  hb and tgt are the low 32 bits of the
// reference's 64-bit hb and TGT[nt]: the step loop compares those, and a
// match goes on to the full 64-bit comparison in stage_check.
struct Lane {
  int p, st, t, deadline, tseg, job;
  u32 hb, tgt;
  int nt, stage, st0, p0, flags;
  u64 ch0, ch1, ch2;
  int nintro, budget;
};

__device__ __forceinline__ void tape_extent(int t, int &lo, int &hi) {
  // After t steps from the blank tape the head has stayed within 64 +- t, so
  // no other tape word can be nonzero.
  int a = kLeft - t, b = kLeft + t;
  a = a < 0 ? 0 : a;
  b = b > kTapeCells - 1 ? kTapeCells - 1 : b;
  lo = a >> 5;
  hi = b >> 5;
}

// Length of the run of `sym` cells starting at p in the move direction, at
// most lim (lim >= 1; cell p itself holds sym).
__device__ __forceinline__ int run_length(const u32 *__restrict__ tcol, int stride, int p, u32 sym, bool right,
                                          int lim) {
  const u32 flip = sym ? 0xFFFFFFFFu : 0u;  // after the XOR, cells holding sym are 0 bits
  int w = p >> 5, b = p & 31, k = 0;
  if (right) {
    u32 x = (tcol[w * stride] ^ flip) >> b;
    for (;;) {
      k += x ? (__ffs(x) - 1) : (32 - b);
      if (x || k >= lim || w == kTapeWords - 1) break;
      ++w;
      b = 0;
      x = tcol[w * stride] ^ flip;
    }
  } else {
    u32 x = (tcol[w * stride] ^ flip) << (31 - b);
    for (;;) {
      k += x ? __clz(x) : (b + 1);
      if (x || k >= lim || w == 0) break;
      --w;
      b = 31;
      x = tcol[w * stride] ^ flip;
    }
  }
  return k < lim ? k : lim;
}

// Runs up to n steps.  Returns kEvRun when n is used up, else the event that
// stopped it; the lane is then exactly at the reference's state for that event.
// hb and tgt are the low 32 bits of the reference's hashes (Lane); kEvStage
// means they match, and stage_check decides on the full 64 bits.  keyb holds
// the low key halves (KeyTabs::lo).
// The stage test of the current configuration has already been done on entry
// (re-running it at the same configuration changes nothing, as the reference
// notes at src/e13search.c:131-133).
//
// Run skip: on a self-loop cell the next k steps read the same symbol, write
// nothing and keep the state, so hb stays the same; when (the low half of) hb
// differs from TGT[nt] no stage test can fire inside the run.  k is clamped so
// that every skipped step would also have passed the deadline test
// (t + i <= deadline) and the window test (the head stays in 1..1362); the step
// that fails either test is then taken by the normal loop.  Steps counted and
// the death point equal single-stepping.
__device__ __forceinline__ int step_slice(int &p, int &st, int &t, const int deadline, u32 &hb, const u32 tgt,
                                          u32 *__restrict__ tcol, const u32 *__restrict__ rcol,
                                          const u32 *__restrict__ keyb, const int stride, int &n, int &cell) {
  while (n > 0) {
    if (t > deadline) return kEvDead;
    const int widx = (p >> 5) * stride;
    const u32 word = tcol[widx];
    const u32 row = rcol[st * stride];
    const u32 sym = (word >> (p & 31)) & 1u;
    const u32 e = (row >> (sym << 4)) & 0x1FFu;
    if (e & (kEntSpecial | kEntSelf)) {
      if (e & kEntSpecial) {
        cell = (st << 1) | (int)sym;
        return kEvCell;
      }
      if (hb != tgt) {
        const bool right = (e & 2u) != 0;
        int lim = deadline - t + 1;
        lim = lim < n ? lim : n;
        const int room = right ? (kTapeCells - 2) - p : p - 1;
        lim = lim < room ? lim : room;
        if (lim > 1) {
          const int k = run_length(tcol, stride, p, sym, right, lim);
          if (k > 1) {
            p += right ? k : -k;
            t += k;
            n -= k;
            continue;
          }
        }
      }
    }
    if ((e ^ sym) & 1u) {
      tcol[widx] = word ^ (1u << (p & 31));
      hb ^= keyb[p];  // low key halves; zero for cells < -2: those go to the counter hash
    }
    p += (int)(e & 2u) - 1;
    if ((unsigned)(p - 1) >= (unsigned)(kTapeCells - 2)) return kEvDead;  // head <= -64 or >= 1299
    st = (int)((e >> 2) & 15u);
    ++t;
    --n;
    if (hb == tgt) return kEvStage;
  }
  return kEvRun;
}

// One action of a running lane, the unit of the warp's lock-step loop: one
// step, one run skip (SKIP only) or one first-read event.  Every running lane
// of a warp takes exactly one action per iteration, so the warp stays
// converged except inside the rare branches, which rejoin at the end of the
// iteration.  Returns 0 (go on), kEvDead, kEvStage (the low hash halves match
// after the step: the caller runs stage_check, the reference's test at the
// start of the next step, before any further action) or kEvCell (a cell whose
// entry has kEntSpecial; *cell and *ecell say which).  Same semantics as
// step_slice(): each step follows src/e13search.c:134-177 in order.
__device__ __forceinline__ int stage_check(struct Lane &L, const u32 *tcol, const KeyTabs &K, int stride);

//
// SKIP = false takes one step per action and leaves out the run-skip
// arithmetic, which costs more than it saves while a warp's machines are
// young: their runs of a self-loop are short.
template <bool SKIP>
__device__ __forceinline__ int lane_act(Lane &L, u32 *__restrict__ tcol, const u32 *__restrict__ rcol,
                                        const KeyTabs &K, const int stride, int &cell, u32 &ecell) {
  if (L.t > L.deadline) return kEvDead;
  const int p = L.p;
  const int widx = (p >> 5) * stride;
  const u32 word = tcol[widx];
  const u32 row = rcol[L.st * stride];
  const u32 kk = K.lo[p];  // loaded with the word and the row, used only on a flip
  const u32 sym = (word >> (p & 31)) & 1u;
  const u32 e = (row >> (sym << 4)) & 0x1FFu;
  if (e & kEntSpecial) {
    cell = (L.st << 1) | (int)sym;
    ecell = e & 0xFFu;
    return kEvCell;
  }
  // k = steps of this action: 1, or on a self-loop cell (see step_slice) the
  // rest of the run of sym inside this tape word, clamped by the deadline and
  // the window.  Computed without branches so the warp does not split.
  const bool right = (e & 2u) != 0;
  const int b = p & 31;
  int k = 1;
  if (SKIP) {
    const u32 x = word ^ (0u - sym);             // cells holding sym are 0 bits
    const u32 xr = right ? x : __brev(x);        // look upwards in both directions
    const int bb = right ? b : 31 - b;
    const u32 up = xr >> bb;
    k = up ? __ffs(up) - 1 : 32 - bb;
    const int lim_t = L.deadline - L.t + 1;
    const int room = right ? (kTapeCells - 2) - p : p - 1;
    k = k < lim_t ? k : lim_t;
    k = k < room ? k : room;
    k = ((e & kEntSelf) && L.hb != L.tgt && k > 1) ? k : 1;
  }
  {  // the write, without a branch (a self-loop cell never flips)
    const u32 flip = (e ^ sym) & 1u;
    tcol[widx] = word ^ (flip << b);
    L.hb ^= kk & (0u - flip);  // the key is zero for cells < -2: those go to the counter hash
  }
  const int np = p + (right ? k : -k);
  if ((unsigned)(np - 1) >= (unsigned)(kTapeCells - 2)) return kEvDead;  // head <= -64 or >= 1299
  L.p = np;
  L.st = (int)((e >> 2) & 15u);
  L.t += k;
  if (L.hb == L.tgt) return kEvStage;  // the caller runs stage_check before the next action
  return 0;
}

// Counter hash from the tape: XOR of the keys of the ones at cells < -2
// (exactly what the reference accumulates in hc, src/e13search.c:170).
__device__ __forceinline__ u64 counter_hash(const u32 *tcol, const u64 *keyc, int stride) {
  u64 hc = 0;
  u32 w0 = tcol[0], w1 = tcol[stride] & 0x3FFFFFFFu;
  while (w0) {
    hc ^= keyc[__ffs(w0) - 1];
    w0 &= w0 - 1;
  }
  while (w1) {
    hc ^= keyc[31 + __ffs(w1)];
    w1 &= w1 - 1;
  }
  return hc;
}

// High 32 bits of the reference's hb: the XOR of the high key halves of the
// ones at cells >= -2, from the tape words a machine of t steps can have
// written (cells < -2 have zero keys in `hi`).
__device__ __forceinline__ u32 hash_hi(const u32 *tcol, const u32 *hi_keys, int stride, int t) {
  int lo, hi;
  tape_extent(t, lo, hi);
  u32 h = 0;
  for (int w = lo < 1 ? 1 : lo; w <= hi; ++w) {
    u32 x = tcol[w * stride];
    while (x) {
      h ^= hi_keys[32 * w + __ffs(x) - 1];
      x &= x - 1;
    }
  }
  return h;
}

// The stage-start test of src/e13search.c:136-161 once the low 32 bits of hb
// match TGT[nt].  The reference enters it on the full 64-bit match: the state
// and head rules come first (they need no hash), then the high halves are
// compared, and only then does the test act.  Returns 0 (go on), kEvDead or
// kEvSurv.
__device__ __forceinline__ int stage_check(Lane &L, const u32 *tcol, const KeyTabs &K, int stride) {
  const int nt = L.nt;
  if (nt > 1 && L.st != L.st0) return 0;  // the common rejection, before any load
  const int c = s_exc[nt];
  int a = L.flags & kFlagAbs, r = (L.flags >> 1) & 1;
  if (nt > 1) {
    if (L.p != L.p0) a = 0;
    if (L.p - (1 << nt) != L.p0 - 2) r = 0;
    if (!a && !r) return 0;
  }
  if (hash_hi(tcol, K.hi, stride, L.t) != (u32)(s_tgt[nt] >> 32)) return 0;  // no 64-bit match: no test
  const u64 hc = counter_hash(tcol, K.c, stride);
  const u64 chc = c == 0 ? L.ch0 : (c == 1 ? L.ch1 : L.ch2);
  if (((L.flags >> (2 + c)) & 1) && chc != hc) return kEvDead;
  if (c != 0 && (L.flags & 4) && L.ch0 == hc) return kEvDead;
  if (c != 1 && (L.flags & 8) && L.ch1 == hc) return kEvDead;
  if (c != 2 && (L.flags & 16) && L.ch2 == hc) return kEvDead;
  L.flags |= kFlagCs0 << c;
  if (c == 0) L.ch0 = hc;
  else if (c == 1) L.ch1 = hc;
  else L.ch2 = hc;
  if (nt == 1) {
    L.st0 = L.st;
    L.p0 = L.p;
  }
  L.flags = (L.flags & ~3) | a | (r << 1);
  L.stage = nt;
  if (nt == kStages) return kEvSurv;
  L.nt = nt + 1;
  L.deadline = s_deadline[nt + 1];
  L.tgt = (u32)s_tgt[nt + 1];
  return 0;
}

__device__ __forceinline__ u32 get_entry(const u32 *rcol, int stride, int cell) {
  return (rcol[(cell >> 1) * stride] >> ((cell & 1) << 4)) & 0xFFu;
}

// The 16-bit slot of a cell holding entry v, with the self-loop bit when
// run_skip is on and v is a read move that keeps the state and the symbol.
__host__ __device__ __forceinline__ u32 cell_slot(int cell, u32 v, bool run_skip) {
  const bool self = run_skip && v < 64u && (int)(v >> 2) == (cell >> 1) && (int)(v & 1u) == (cell & 1);
  return v | (self ? kEntSelf : 0u);
}

__device__ __forceinline__ void set_entry(u32 *rcol, int stride, int cell, u32 v, bool run_skip) {
  u32 *w = rcol + (cell >> 1) * stride;
  const int sh = (cell & 1) << 4;
  *w = (*w & ~(0xFFFFu << sh)) | (cell_slot(cell, v, run_skip) << sh);
}

// With no budget left, a first read of a cell that is not free can only keep
// the table's move (src/e13search.c:221-251 with budget 0: the keep child
// alone).  Clearing the unread flag of every such cell lets the step loop
// take those reads as plain steps instead of events.  Unread halts keep the
// flag (their read ends the machine), free cells keep theirs (they fork).
// The flag also marks the survivor's never-read cells ('?'), so survivors are
// given their read mask again at survival (survivor_reads).  An unread move's
// slot carries its self-loop bit already (see build_root), so clearing bit 7
// is all it takes.
static __device__ __noinline__ void clear_unread(u32 *rcol, int stride) {
#pragma unroll 1
  for (int s = 0; s < 16; ++s) {
    const u32 w = rcol[s * stride];
    // bit 7 set and bit 6 clear in a slot: an unread move (codes are < 64)
    const u32 unread_move = (w & 0x00800080u) & ~((w & 0x00400040u) << 1);
    rcol[s * stride] = w & ~unread_move;
  }
}

// Relabel symmetry (src/e13search.c:206-212): states in use after move v, or
// -1 when v names a symmetric state past the next unused one.
__device__ __forceinline__ int sym_after(int v, int nintro, int sym_lo, int sym_hi) {
  if (sym_lo < 0 || v < 0) return nintro;
  const int q = v >> 2;
  if (q < sym_lo || q > sym_hi) return nintro;
  if (q - sym_lo < nintro) return nintro;
  return (q - sym_lo == nintro) ? nintro + 1 : -1;
}

// Children of a first read of a cell with entry e (src/e13search.c:221-251):
// keep the table's move unless the cell is free; while the cell is free or
// budget remains, every other move the symmetry rule allows.
__device__ __forceinline__ void child_set(u32 e, int budget, int nintro, int nv, int sym_lo, int sym_hi, int &keep,
                                          u64 &vm) {
  const bool is_free = (e == kEntFree);
  keep = is_free ? 0 : 1;
  vm = 0;
  if (is_free || budget > 0) {
    vm = nv >= 64 ? ~0ull : ((1ull << nv) - 1ull);
    if (!is_free && !(e & kEntHalt)) vm &= ~(1ull << (e & 0x3Fu));
    if (sym_lo >= 0) {
      const int q0 = sym_lo + nintro + 1;  // first state a move may not name yet
      if (q0 <= sym_hi) {
        const int a = 4 * q0, b = 4 * (sym_hi + 1);
        const u64 below_b = b >= 64 ? ~0ull : ((1ull << b) - 1ull);
        const u64 below_a = (1ull << a) - 1ull;
        vm &= ~(below_b & ~below_a);
      }
    }
  }
}

// Position of the r-th (0-based) set bit of m (r < popc(m)).
__device__ __forceinline__ int nth_bit64(u64 m, int r) {
  u32 x = (u32)m;
  int base = 0;
  const int nlo = __popc(x);
  if (r >= nlo) {
    r -= nlo;
    x = (u32)(m >> 32);
    base = 32;
  }
  int c = __popc(x & 0xFFFFu);
  if (r >= c) { r -= c; x >>= 16; base += 16; }
  c = __popc(x & 0xFFu);
  if (r >= c) { r -= c; x >>= 8; base += 8; }
  c = __popc(x & 0xFu);
  if (r >= c) { r -= c; x >>= 4; base += 4; }
  c = __popc(x & 0x3u);
  if (r >= c) { r -= c; x >>= 2; base += 2; }
  if (r >= (int)(x & 1u)) base += 1;
  return base;
}

// Drops the first k children (keep first, then the lowest moves).
__device__ __forceinline__ void drop_children(int &keep, u64 &vm, int k) {
  if (k <= 0) return;
  if (keep) {
    keep = 0;
    --k;
  }
  if (k <= 0) return;
  if (k >= __popcll(vm)) {
    vm = 0;
    return;
  }
  const int b = nth_bit64(vm, k);
  vm &= ~((1ull << b) - 1ull);
}

}  // namespace e13dev
