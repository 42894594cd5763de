// e13_search.cu -- the TNF enumeration search on one B200 (sm_100a).
//
// Two kernels share one template:
//
//  * plain (PERSIST = false): one launch per frontier batch.  Each warp pulls
//    frontier nodes and hands their children to idle lanes; a lane runs its
//    child to the next fork, leaf or step cap.  Every fork goes back to the
//    frontier.  The host waits for each launch (the reference GPU design,
//    src/e13gpu.py:381-436, built B200-first).
//
//  * persistent (PERSIST = true): each warp runs a private depth-first search
//    over the subtrees it pulls.  A forking lane pushes its node on the warp's
//    stack and goes on with the first child in place (no copy); idle lanes take
//    the next children of the stack top at the next round.  A warp whose stack
//    is deep donates its oldest node to a device pool when the pool runs low;
//    warps without work take pool nodes.  An epoch takes the whole frontier as
//    its input and ends on a time bound (or when every warp is out of work):
//    warps then dump live lanes and stack nodes back to the frontier.  Epochs
//    are replayed from a captured CUDA graph; the host reads the control block
//    once per graph.
//
// In both, a machine whose budget is spent takes first reads of cells that
// can no longer fork as plain steps (clear_unread); survivors get their read
// mask back from a re-run of their final table.
//
// Leaves, steps and deaths per stage are exact and equal the reference's
// (src/e13search.c:214-254 explore, :357-420 run_delete).
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <string>
#include <vector>

#include "e13.h"
#include "e13_device.cuh"
#include "e13_node.cuh"

using namespace e13dev;

namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr long long kPoolNodes = 1LL << 18;  // donation pool: 256 Ki nodes (80 MiB)
constexpr long long kWholeFrontier = 1LL << 62;  // persistent batch when e13_tuning::batch is 0
constexpr long long kPoolWaitNs = 200000000;     // 200 ms: a donor publishes a claimed slot within microseconds
constexpr long long kMinEpochNs = 200000;        // 200 us: the shortest epoch a starvation dump may end
// A warp with at most kLoneLanes running machines (the tail of a search:
// a few long machines, the rest of the GPU idle) runs each of them in the
// tight single-machine loop step_slice, up to kLoneSteps steps per
// iteration: its speed is then bound by one machine's dependent chain, not
// by issue slots, and the lock-step loop's control would only lengthen it.
constexpr int kLoneLanes = 2;
constexpr int kLoneSteps = 512;

// steps a lane gets between warp-level refill rounds is Params::slice

struct Params {
  const JobParam *jobs;      // kMaxJobs entries
  unsigned long long *jobcnt;  // kMaxJobs x kJobCounters totals
  int nq;
  int slice, step_cap, wdepth, pool_low, run_skip;
  int skip_after;            // run skip only in slices of warps with a machine of at least this many steps
  long long out_cap, out_soft, surv_cap, pool_cap;
  long long epoch_ns;
  long long wait_ns;         // persistent: limit of the wait for a claimed pool slot's data
  long long min_epoch_ns;    // persistent: an epoch may end early for starvation only after this long
  Node *stack, *out, *wstack, *pool;
  int *pool_ready;
  SurvRec *surv;
  Ctl *ctl;
};

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void copy_node(Node *dst, const Node *src, int lane) {
  if (lane < kNodeChunks) reinterpret_cast<uint4 *>(dst)[lane] = reinterpret_cast<const uint4 *>(src)[lane];
}

// The cells a survivor's run read.  Unread flags cleared when the budget ran
// out (clear_unread) make some never-read cells look read, so the lane runs
// its final table again from the blank tape, in its own tape, for the t steps
// of its run: a run is fixed by its table, so this reads exactly the cells the
// search run read (the reference prints the others with '?',
// src/e13search.c:186-196).  Survivors are rare; the lane is idle afterwards,
// and its next load clears the tape words of t steps, the ones used here.
static __device__ __noinline__ u32 survivor_reads(u32 *tcol, const u32 *rcol, int stride, int t) {
  int lo, hi;
  tape_extent(t, lo, hi);
  for (int w = lo; w <= hi; ++w) tcol[w * stride] = 0;
  int p = kLeft, st = 0;
  u32 read = 0;
  for (int k = 0; k < t; ++k) {
    const int widx = (p >> 5) * stride;
    const u32 word = tcol[widx];
    const u32 sym = (word >> (p & 31)) & 1u;
    read |= 1u << (2 * st + (int)sym);
    const u32 e = (rcol[st * stride] >> (sym << 4)) & 0xFFu;
    if (e == kEntFree || (e & kEntHalt)) break;  // a survivor reads neither before its end
    tcol[widx] = word ^ (((e ^ sym) & 1u) << (p & 31));
    p += (e & 2u) ? 1 : -1;
    if (p < 1 || p > kTapeCells - 2) break;     // nor leaves the window
    st = (int)((e >> 2) & 15u);
  }
  return read;
}

// Appends a survivor record (kept only below the cap).  reads: the persistent
// kernel has the lane re-run the table for the read mask (its warp goes on
// alone, the others are not held up); the plain kernel, whose launch would
// wait for that lane, records the flags as they are and leaves the mask to
// survivor_read_masks() once the search is over.  Out of line: it is rare, and
// the step loop keeps its registers.
static __device__ __noinline__ void record_survivor(Ctl *ctl, SurvRec *surv, long long surv_cap, int st0, int p0,
                                                    int flags, int t, int job, u32 *tcol, const u32 *rcol,
                                                    int stride, bool reads) {
  const unsigned long long k = atomicAdd(&ctl->nsurv, 1ull);
  if ((long long)k >= surv_cap) return;
  SurvRec *r = surv + k;
  const u32 read = reads ? survivor_reads(tcol, rcol, stride, t) : 0u;
  for (int c = 0; c < 32; ++c) {
    const u32 e = (rcol[(c >> 1) * stride] >> ((c & 1) << 4)) & 0xFFu;
    if (!reads) r->ent[c] = (unsigned char)e;
    else r->ent[c] = (unsigned char)(e == kEntFree ? e : (((read >> c) & 1u) ? (e & 0x7Fu) : (e | kEntUnread)));
  }
  r->st0 = st0;
  r->head0 = p0 - kLeft;
  r->abs_ok = flags & 1;
  r->rel_ok = (flags >> 1) & 1;
  r->t = t;
  r->job = job;
}

enum { kStRun = 0, kStIdle = 1, kStFork = 2, kStCap = 3, kStDead = 4, kStSurv = 5 };

__device__ __forceinline__ int wrap(int s, int d) { return s >= d ? s - d : s; }

template <bool PERSIST>
__global__ void __launch_bounds__(768, 1) search_kernel(const Params P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const KeyTabs K = key_tables(smem_raw);
  u32 *tape = reinterpret_cast<u32 *>(smem_raw + kKeySmemBytes);
  const int stride = blockDim.x;
  u32 *rows = tape + kTapeWords * stride;
  // persistent: a shared-memory copy of each warp's current stack-top node, so
  // lanes taking its children read shared memory instead of HBM
  Node *mytop = reinterpret_cast<Node *>(rows + 16 * stride) + (threadIdx.x >> 5);
  __shared__ int4 s_jp[kMaxJobs];                              // per-job moves and symmetry range
  __shared__ unsigned long long s_jc[kMaxJobs][kJobCounters];  // per-job leaves, steps, deaths by stage

  fill_key_tables(K);
  if (threadIdx.x < kMaxJobs) {
    const JobParam jp = P.jobs[threadIdx.x];
    s_jp[threadIdx.x] = make_int4(jp.nv, jp.sym_lo, jp.sym_hi, 0);
  }
  for (int i = threadIdx.x; i < kMaxJobs * kJobCounters; i += stride) (&s_jc[0][0])[i] = 0ull;
  load_stage_tables();
  u32 *tcol = tape + threadIdx.x;
  u32 *rcol = rows + threadIdx.x;
  for (int w = 0; w < kTapeWords; ++w) tcol[w * stride] = 0;
  __syncthreads();

  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  const long long gwarp = ((long long)blockIdx.x * stride + threadIdx.x) >> 5;
  Ctl *ctl = P.ctl;
  const long long top0 = ctl->top;
  const long long batch = ctl->batch;
  const int tag = ctl->launches + 1;  // marks pool slots written in this launch
  const int D = P.wdepth;
  Node *wst = PERSIST ? P.wstack + gwarp * D : nullptr;
  const unsigned long long t_begin = PERSIST ? globaltimer() : 0ull;

  Lane L;
  L.t = 0;
  L.tseg = 0;
  // leaves and steps of this lane's current job, added to the block's per-job
  // counters only when the lane changes job and at the end (no atomics per leaf)
  // (deaths at stages 0 and 1, 97 % of all leaves, are counted per lane too:
  // two 16-bit halves of acc_d01, flushed before either can overflow)
  u32 acc_leaves = 0, acc_steps = 0, acc_d01 = 0;
  auto flush_counts = [&]() {
    if (acc_leaves | acc_steps) {
      atomicAdd(&s_jc[L.job][0], (unsigned long long)acc_leaves);
      atomicAdd(&s_jc[L.job][1], (unsigned long long)acc_steps);
      if (acc_d01 & 0xFFFFu) atomicAdd(&s_jc[L.job][2], (unsigned long long)(acc_d01 & 0xFFFFu));
      if (acc_d01 >> 16) atomicAdd(&s_jc[L.job][3], (unsigned long long)(acc_d01 >> 16));
      acc_leaves = 0;
      acc_steps = 0;
      acc_d01 = 0;
    }
  };
  int status = kStIdle;
  int fork_cell = 0;
  u32 fork_e = 0;
  L.job = 0;

  // warp-uniform state
  int sp = 0, wbot = 0;        // persistent: this warp's DFS stack, a ring of D slots from wbot
  bool have_cur = false;       // cursor registers hold the children left of the current node
  const Node *cur = nullptr;   // plain: the current input node
  int cur_keep = 0;
  u64 cur_vm = 0;
  bool input_done = false;
  bool busy = false;           // persistent: counted in ctl->busy
  bool top_dirty = false;      // persistent: the stack top lives only in the shared copy (its HBM slot is stale)
  bool counted_idle = false;   // persistent, lane 0: this warp is counted in ctl->idle
  bool counted_deep = false;   // persistent, lane 0: this warp is counted in ctl->deep
  const int nwarps_all = (int)(((long long)gridDim.x * stride) >> 5);
  int rounds = 0;              // slices run: a warp dumps only after one (progress every epoch)
  unsigned backoff = 256;
  unsigned long long st_lane_rounds = 0, st_polls = 0;
  unsigned st_donations = 0, st_claims = 0;

  for (;;) {
    // ---- (A) forks
    if (__any_sync(kFull, status == kStFork)) {
      int keep = 0;
      u64 vm = 0;
      if (status == kStFork) {
        const int4 jp = s_jp[L.job];
        child_set(fork_e, L.budget, L.nintro, jp.x, jp.y, jp.z, keep, vm);
      }
      if (PERSIST) {
        // the forking lane goes on with the first child in place; the rest is pushed
        int first = -2;
        if (status == kStFork) {
          if (keep) {
            first = -1;
            keep = 0;
          } else {
            first = __ffsll((long long)vm) - 1;
            vm &= vm - 1;
          }
        }
        const bool more = (status == kStFork) && (keep || vm);
        const unsigned pm = __ballot_sync(kFull, more);
        if (pm) {
          const int rank = __popc(pm & lt_mask);
          const int npush = min(__popc(pm), D - sp);
          if (npush > 0 && have_cur && sp > 0) {
            // the current top goes under the new nodes: its HBM slot gets the
            // shared copy (if that is newer) and the children still to run
            Node *t = wst + wrap(wbot + sp - 1, D);
            if (top_dirty) copy_node(t, mytop, lane);
            __syncwarp();
            if (lane == 0) {
              t->vmask = cur_vm;
              t->flags = (signed char)((t->flags & 31) | (cur_keep ? kFlagKeep : 0));
            }
          }
          __syncwarp();
          if (more) {
            Node *dst = nullptr;
            if (rank < npush - 1) {
              dst = wst + wrap(wbot + sp + rank, D);  // buried at once
            } else if (rank == npush - 1) {
              dst = mytop;  // the new top: kept in shared memory until it is buried
            } else {
              const unsigned long long k = atomicAdd(&ctl->nout, 1ull);
              if ((long long)k < P.out_cap) dst = P.out + k;
              else atomicOr(&ctl->error, kErrOutFull);
            }
            if (dst) lane_store(L, dst, tcol, rcol, stride, P.nq, fork_cell, keep, vm);
          }
          if (npush > 0) {
            top_dirty = true;
            const int src = nth_bit64((u64)pm, npush - 1);  // lane holding the last node pushed on the warp stack
            cur_keep = __shfl_sync(kFull, keep, src);
            const unsigned lo = __shfl_sync(kFull, (unsigned)vm, src);
            const unsigned hi = __shfl_sync(kFull, (unsigned)(vm >> 32), src);
            cur_vm = ((u64)hi << 32) | lo;
            sp += npush;
            have_cur = true;
          }
          __syncwarp();
        }
        if (status == kStFork) {
          if (first < 0) {
            set_entry(rcol, stride, fork_cell, fork_e & 0x7Fu, P.run_skip);
          } else {
            if (fork_e != kEntFree) {
              L.budget -= 1;
              if (L.budget == 0) clear_unread(rcol, stride);  // no first read can fork any more
            }
            L.nintro = sym_after(first, L.nintro, s_jp[L.job].y, s_jp[L.job].z);
            set_entry(rcol, stride, fork_cell, (u32)first, P.run_skip);
          }
          status = kStRun;
        }
      } else {
        if (status == kStFork) {
          const unsigned long long k = atomicAdd(&ctl->nout, 1ull);
          if ((long long)k < P.out_cap) lane_store(L, P.out + k, tcol, rcol, stride, P.nq, fork_cell, keep, vm);
          else atomicOr(&ctl->error, kErrOutFull);
          status = kStIdle;
        }
      }
    }
    if (!PERSIST && __any_sync(kFull, status == kStCap)) {
      if (status == kStCap) {
        const unsigned long long k = atomicAdd(&ctl->nout, 1ull);
        if ((long long)k < P.out_cap) lane_store(L, P.out + k, tcol, rcol, stride, P.nq, -1, 1, 0ull);
        else atomicOr(&ctl->error, kErrOutFull);
        status = kStIdle;
      }
    }

    // ---- (B) refill idle lanes: stack top, else the frontier input, else the pool
    for (;;) {
      const unsigned im = __ballot_sync(kFull, status == kStIdle);
      if (!im) break;
      if (!have_cur) {
        if (PERSIST && sp > 0) {
          // an older node is the top again: bring it into shared memory once
          copy_node(mytop, wst + wrap(wbot + sp - 1, D), lane);
          __syncwarp();
          top_dirty = false;
          cur_keep = (mytop->flags & kFlagKeep) ? 1 : 0;
          cur_vm = mytop->vmask;
          have_cur = true;
        } else {
          const Node *src = nullptr;
          bool from_pool = false;
          if (!input_done) {
            if (PERSIST && !busy) {
              if (lane == 0) atomicAdd(&ctl->busy, 1);  // before any claim, so idle warps see work in flight
              busy = true;
            }
            long long k = batch;
            // once an epoch is ending, leave the rest of the input where it is
            if (lane == 0 && !(PERSIST && *((volatile int *)&ctl->dump)))
              k = (long long)atomicAdd(&ctl->cursor, 1ull);
            k = __shfl_sync(kFull, k, 0);
            if (k >= batch) input_done = true;
            else src = P.stack + (top0 - 1 - k);
          }
          if (PERSIST && !src && (im == kFull || (rounds & 3) == 0)) {
            long long h = -1;
            int inc = 0;
            if (lane == 0 && !*((volatile int *)&ctl->dump)) {
              unsigned long long hh = *((volatile unsigned long long *)&ctl->pool_head);
              const unsigned long long tl = *((volatile unsigned long long *)&ctl->pool_tail);
              const unsigned long long lim = tl < (unsigned long long)P.pool_cap ? tl : (unsigned long long)P.pool_cap;
              if (hh < lim && !busy) {
                atomicAdd(&ctl->busy, 1);  // only when there is something to take
                inc = 1;
              }
              while (hh < lim) {
                const unsigned long long got = atomicCAS(&ctl->pool_head, hh, hh + 1);
                if (got == hh) {
                  h = (long long)hh;
                  break;
                }
                hh = got;
              }
              if (h >= 0) {
                // the donor claimed the slot before writing it; wait (bounded) for its data
                const unsigned long long t0 = globaltimer();
                while (*((volatile int *)&P.pool_ready[h]) != tag) {
                  if (globaltimer() - t0 > (unsigned long long)P.wait_ns) {
                    atomicOr(&ctl->error, kErrTimeout);
                    h = -1;
                    break;
                  }
                  __nanosleep(64);
                }
                __threadfence();
              }
            }
            h = __shfl_sync(kFull, h, 0);
            if (__shfl_sync(kFull, inc, 0)) busy = true;
            if (h >= 0) {
              src = P.pool + h;
              from_pool = true;
              ++st_claims;
            }
          }
          if (!src) break;
          if (PERSIST && counted_idle && lane == 0) {
            atomicSub(&ctl->idle, 1);
            counted_idle = false;
          }
          if (PERSIST) {
            wbot = 0;
            if (lane < kNodeChunks) {
              const uint4 v = from_pool ? __ldcg(reinterpret_cast<const uint4 *>(src) + lane)
                                        : reinterpret_cast<const uint4 *>(src)[lane];
              reinterpret_cast<uint4 *>(wst)[lane] = v;
              reinterpret_cast<uint4 *>(mytop)[lane] = v;
            }
            __syncwarp();
            sp = 1;
            top_dirty = false;
            cur_keep = (mytop->flags & kFlagKeep) ? 1 : 0;
            cur_vm = mytop->vmask;
          } else {
            cur = src;
            cur_keep = (src->flags & kFlagKeep) ? 1 : 0;
            cur_vm = src->vmask;
          }
          have_cur = true;
          backoff = 256;
        }
      }
      const Node *N = PERSIST ? mytop : cur;
      const int navail = cur_keep + __popcll(cur_vm);
      const int nidle = __popc(im);
      const int rank = __popc(im & lt_mask);
      if (status == kStIdle && rank < navail) {
        int ch = -1;
        if (!(cur_keep && rank == 0)) ch = nth_bit64(cur_vm, rank - cur_keep);
        if (N->job != L.job) flush_counts();
        lane_load(L, N, tcol, rcol, stride, P.nq);
        apply_child(L, N, ch, rcol, stride, s_jp[N->job].y, s_jp[N->job].z, P.run_skip, true);
        status = kStRun;
      }
      __syncwarp();
      if (nidle >= navail) {
        have_cur = false;
        top_dirty = false;
        if (PERSIST) --sp;
      } else {
        drop_children(cur_keep, cur_vm, nidle);
      }
    }

    // ---- (C) end of work / end of epoch
    const bool any_run = __any_sync(kFull, status == kStRun);
    const bool has_work = any_run || have_cur || (PERSIST && sp > 0);
    if (!PERSIST) {
      if (!has_work && input_done) break;
    } else {
      if (!has_work && busy) {
        if (lane == 0) atomicSub(&ctl->busy, 1);
        busy = false;
      }
      if (lane == 0 && (sp >= 2) != counted_deep) {  // (a donation below is seen next round)
        atomicAdd(&ctl->deep, counted_deep ? -1 : 1);
        counted_deep = !counted_deep;
      }
      int d = 0;
      if (!has_work || (rounds & 7) == 0) {  // the control words are in L2: read them every 8th round
        if (lane == 0) {
          d = *((volatile int *)&ctl->dump);
          if (!d && globaltimer() - t_begin > (unsigned long long)P.epoch_ns) d = 1;
          if (!d && (long long)*((volatile unsigned long long *)&ctl->nout) > P.out_soft) d = 1;
          if (d) *((volatile int *)&ctl->dump) = 1;
        }
        d = __shfl_sync(kFull, d, 0);
      }
      if (!has_work) {
        // nothing here: done when no warp holds work and the pool is empty, else wait for a donation
        int done = d;
        if (lane == 0 && !done && input_done) {
          const int b = *((volatile int *)&ctl->busy);
          const unsigned long long hh = *((volatile unsigned long long *)&ctl->pool_head);
          const unsigned long long tl = *((volatile unsigned long long *)&ctl->pool_tail);
          const unsigned long long lim = tl < (unsigned long long)P.pool_cap ? tl : (unsigned long long)P.pool_cap;
          done = (b == 0 && hh >= lim);
        }
        done = __shfl_sync(kFull, done, 0);
        if (done) break;
        // starving.  Work spreads inside an epoch only through donated nodes,
        // which a few deep warps hand out one at a time: a job whose subtrees
        // are shallow would run on a few warps for a long time.  When more
        // than half of the warps wait for work and some warp holds a stack
        // of 2 or more nodes, end the epoch (after a shortest length): the
        // dump puts every warp's stack on the frontier and the next epoch
        // deals it out over all warps.  (With no deep stack left, the work
        // is a few long-running machines that a dump would not spread.)
        if (lane == 0) {
          if (!counted_idle) {
            atomicAdd(&ctl->idle, 1);
            counted_idle = true;
          } else if (backoff >= 1024 && globaltimer() - t_begin > (unsigned long long)P.min_epoch_ns &&
                     2 * *((volatile int *)&ctl->idle) > nwarps_all && *((volatile int *)&ctl->deep) > 0) {
            *((volatile int *)&ctl->dump) = 1;
          }
        }
        ++st_polls;
        __nanosleep(backoff);
        backoff = backoff < 8192 ? 2 * backoff : 8192;
        continue;
      }
      if (d && rounds > 0) {
        // dump: live lanes as resume nodes, then this warp's stack
        if (status == kStRun) {
          acc_steps += (u32)(L.t - L.tseg);
          L.tseg = L.t;
          const unsigned long long k = atomicAdd(&ctl->nout, 1ull);
          if ((long long)k < P.out_cap) lane_store(L, P.out + k, tcol, rcol, stride, P.nq, -1, 1, 0ull);
          else atomicOr(&ctl->error, kErrOutFull);
          status = kStIdle;
        }
        __syncwarp();
        if (sp > 0) {
          unsigned long long base = 0;
          if (lane == 0) base = atomicAdd(&ctl->nout, (unsigned long long)sp);
          base = __shfl_sync(kFull, base, 0);
          for (int i = 0; i < sp; ++i) {
            const bool is_top = i == sp - 1;
            const Node *from = (is_top && top_dirty) ? mytop : wst + wrap(wbot + i, D);
            if ((long long)(base + i) < P.out_cap) copy_node(P.out + base + i, from, lane);
            else if (lane == 0) atomicOr(&ctl->error, kErrOutFull);
          }
          __syncwarp();
          if (have_cur && lane == 0 && (long long)(base + sp - 1) < P.out_cap) {
            Node *t = P.out + base + sp - 1;
            t->vmask = cur_vm;
            t->flags = (signed char)((t->flags & 31) | (cur_keep ? kFlagKeep : 0));
          }
        }
        if (busy && lane == 0) atomicSub(&ctl->busy, 1);
        break;
      }
      // donate the oldest node of a deep stack when the pool runs low
      if (sp >= 2 && (rounds & 3) == 0) {
        long long s = -1;
        if (lane == 0) {
          const unsigned long long hh = *((volatile unsigned long long *)&ctl->pool_head);
          const unsigned long long tl = *((volatile unsigned long long *)&ctl->pool_tail);
          if (tl < (unsigned long long)P.pool_cap && tl - hh < (unsigned long long)P.pool_low)
            s = (long long)atomicAdd(&ctl->pool_tail, 1ull);
        }
        s = __shfl_sync(kFull, s, 0);
        if (s >= 0 && s < P.pool_cap) {
          copy_node(P.pool + s, wst + wbot, lane);
          __threadfence();
          __syncwarp();
          if (lane == 0) atomicExch(&P.pool_ready[s], tag);
          wbot = wrap(wbot + 1, D);
          --sp;
          ++st_donations;
        }
      }
    }

    // ---- (D) run a slice: every running lane takes up to two actions per iteration
    ++rounds;
    {
      const unsigned rm = __ballot_sync(kFull, status == kStRun);
      // word-at-a-time run skips pay off only for machines that have built
      // long runs: the warp uses them in this slice when one of its machines
      // has run skip_after steps (a warp-uniform choice: no divergence)
      const bool skip_w = P.run_skip && __any_sync(kFull, status == kStRun && L.t >= P.skip_after);
      const bool lone_w = __popc(rm) <= kLoneLanes;
      st_lane_rounds += __popc(rm);
      if (rm) {
#pragma unroll 1
        for (int it = 0; it < P.slice; ++it) {
          if (status == kStRun) {
            int cell = 0;
            u32 e = 0;
            // two actions per iteration: the loop control and the event
            // dispatch below are paid once for both
            int ev;
            if (lone_w) {
              // the same steps and events as lane_act (step_slice follows
              // src/e13search.c:134-177 too); a hash match ends the iteration
              // and goes to the one stage test below
              int n = kLoneSteps;
              ev = step_slice(L.p, L.st, L.t, L.deadline, L.hb, L.tgt, tcol, rcol, K.lo, stride, n, cell);
              if (ev == kEvCell) e = get_entry(rcol, stride, cell);
            } else if (skip_w) {
              ev = lane_act<true>(L, tcol, rcol, K, stride, cell, e);
              if (!ev) ev = lane_act<true>(L, tcol, rcol, K, stride, cell, e);
            } else {
              ev = lane_act<false>(L, tcol, rcol, K, stride, cell, e);
              if (!ev) ev = lane_act<false>(L, tcol, rcol, K, stride, cell, e);
            }
            // the stage test of a hash match, once per iteration outside
            // lane_act: one copy of it in the loop instead of one per
            // inlined action (the second action waits for it)
            if (ev == kEvStage) ev = stage_check(L, tcol, K, stride);
            if (ev == kEvCell) {
              if (e == kEntHalt) {
                ev = kEvDead;
              } else if (e == kEntFree || L.budget > 0) {
                // a fork: handled by the warp at the next round (the persistent
                // kernel goes on with the first child in this lane, so its
                // steps are counted at the leaf)
                if (!PERSIST) {
                  acc_steps += (u32)(L.t - L.tseg);
                  L.tseg = L.t;
                }
                fork_cell = cell;
                fork_e = e;
                status = kStFork;
                ev = 0;
              } else {
                // first read with nothing to branch on: the cell is now fixed
                set_entry(rcol, stride, cell, e & 0x7Fu, P.run_skip);
                ev = ((e & 0x7Fu) == kEntHalt) ? kEvDead : 0;
              }
            }
            // a leaf: counted by the warp after the slice, all its leaves in
            // one converged pass (the lane would wait for the next round anyway)
            if (ev) status = (ev == kEvDead) ? kStDead : kStSurv;
          }
          // every lane comes here each iteration (the loop bounds are
          // warp-uniform): the lanes that took rare branches rejoin at the end
          // of the if-blocks above, so the next action issues once for the
          // whole warp
        }
        if (__any_sync(kFull, status >= kStDead)) {
          if (status >= kStDead) {
            acc_steps += (u32)(L.t - L.tseg);
            L.tseg = L.t;
            ++acc_leaves;
            if (acc_steps >= 0x80000000u) flush_counts();
            if (status == kStDead) {
              if (L.stage <= 1) {
                acc_d01 += L.stage ? 0x10000u : 1u;
                if (acc_d01 & 0x80008000u) flush_counts();
              } else {
                atomicAdd(&s_jc[L.job][2 + L.stage], 1ull);
              }
            } else {
              record_survivor(P.ctl, P.surv, P.surv_cap, L.st0, L.p0, L.flags, L.t, L.job, tcol, rcol, stride,
                              PERSIST);
            }
            status = kStIdle;
          }
        }
        if (!PERSIST && status == kStRun && L.t - L.tseg >= P.step_cap) {
          acc_steps += (u32)(L.t - L.tseg);
          L.tseg = L.t;
          if (acc_steps >= 0x80000000u) flush_counts();
          status = kStCap;
        }
      }
    }
  }

  // ---- totals
  flush_counts();
  if (lane == 0) {
    atomicAdd(&ctl->rounds, (unsigned long long)rounds);
    atomicAdd(&ctl->lane_rounds, st_lane_rounds);
    atomicAdd(&ctl->polls, st_polls);
    if (st_donations) atomicAdd(&ctl->donations, (unsigned long long)st_donations);
    if (st_claims) atomicAdd(&ctl->claims, (unsigned long long)st_claims);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kMaxJobs * kJobCounters; i += stride) {
    const unsigned long long v = (&s_jc[0][0])[i];
    if (v) atomicAdd(P.jobcnt + i, v);
  }
}

// Serving: moves the frontier into dst grouped by job, job k's nodes starting
// at fill[k] (the host lays the groups out so that the job with the fewest
// live nodes ends on top, where the next epoch takes its input first).  One
// warp per node.
__global__ void order_by_job(const Ctl *ctl, const Node *src, Node *dst, unsigned long long *fill, long long cap) {
  const long long top = ctl->top;
  const int lane = threadIdx.x & 31;
  const long long w0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long i = w0; i < top; i += nw) {
    unsigned long long pos = 0;
    if (lane == 0) pos = atomicAdd(&fill[src[i].job & (kMaxJobs - 1)], 1ull);
    pos = __shfl_sync(kFull, pos, 0);
    if ((long long)pos < cap) copy_node(dst + pos, src + i, lane);
  }
}

// The read masks of survivors [0, n) recorded by the plain kernel: the same
// re-run as survivor_reads(), one thread per survivor, once the search is
// over (every survivor in parallel, instead of holding up a launch each).
__global__ void survivor_read_masks(SurvRec *recs, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  SurvRec &r = recs[i];
  unsigned char ent[32];
  for (int c = 0; c < 32; ++c) ent[c] = r.ent[c];
  u32 tape[kTapeWords];
  for (int w = 0; w < kTapeWords; ++w) tape[w] = 0;
  int p = kLeft, st = 0;
  u32 read = 0;
  for (int k = 0; k < r.t; ++k) {
    const u32 sym = (tape[p >> 5] >> (p & 31)) & 1u;
    const int cell = 2 * st + (int)sym;
    read |= 1u << cell;
    const u32 e = ent[cell];
    if (e == kEntFree || (e & kEntHalt)) break;  // a survivor reads neither before its end
    tape[p >> 5] ^= ((e ^ sym) & 1u) << (p & 31);
    p += (e & 2u) ? 1 : -1;
    if (p < 1 || p > kTapeCells - 2) break;     // nor leaves the window
    st = (int)((e >> 2) & 15u);
  }
  for (int c = 0; c < 32; ++c) {
    const u32 e = ent[c];
    if (e != kEntFree) r.ent[c] = (unsigned char)(((read >> c) & 1u) ? (e & 0x7Fu) : (e | kEntUnread));
  }
}

// Live nodes of each job on the frontier stack.  Between launches every
// unfinished machine of the persistent kernel is there, so a job whose count
// is zero is finished.
__global__ void count_job_nodes(const Ctl *ctl, const Node *stack, unsigned long long *counts) {
  __shared__ unsigned int s_n[kMaxJobs];
  if (threadIdx.x < kMaxJobs) s_n[threadIdx.x] = 0;
  __syncthreads();
  const long long top = ctl->top;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < top; i += (long long)gridDim.x * blockDim.x)
    atomicAdd(&s_n[stack[i].job & (kMaxJobs - 1)], 1u);
  __syncthreads();
  if (threadIdx.x < kMaxJobs && s_n[threadIdx.x]) atomicAdd(&counts[threadIdx.x], (unsigned long long)s_n[threadIdx.x]);
}

// Between launches: the input taken from the top of the stack is gone; the
// outputs, then the pool nodes nobody took, go where it was.
__global__ void move_outputs(Ctl *ctl, Node *stack, const Node *out, const Node *pool, long long pool_cap,
                             long long cap) {
  const long long used = min((long long)ctl->cursor, ctl->batch);
  const long long base = ctl->top - used;
  const long long n = (long long)ctl->nout;
  const long long ph = (long long)ctl->pool_head;
  const long long pt = min((long long)ctl->pool_tail, pool_cap);
  const long long np = pt > ph ? pt - ph : 0;
  if (base + n + np > cap || ctl->error) return;  // finish_launch reports the overflow
  const long long chunks = n * kNodeChunks, pchunks = np * kNodeChunks;
  uint4 *dst = reinterpret_cast<uint4 *>(stack + base);
  const uint4 *src = reinterpret_cast<const uint4 *>(out);
  const uint4 *psrc = reinterpret_cast<const uint4 *>(pool + ph);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < chunks + pchunks;
       i += (long long)gridDim.x * blockDim.x)
    dst[i] = i < chunks ? src[i] : __ldcg(psrc + (i - chunks));
}

__global__ void finish_launch(Ctl *ctl, long long cap, long long batch_max, long long pool_cap) {
  const long long used = min((long long)ctl->cursor, ctl->batch);
  const long long ph = (long long)ctl->pool_head;
  const long long pt = min((long long)ctl->pool_tail, pool_cap);
  const long long np = pt > ph ? pt - ph : 0;
  long long top = ctl->top - used + (long long)ctl->nout + np;
  if (top > cap || ctl->error) {
    // the outputs did not fit (or a device wait ran out): stop here and let the host report it
    if (top > cap) ctl->error |= kErrOverflow;
    top = 0;
  }
  ctl->top = top;
  if (top > ctl->peak) ctl->peak = top;
  ctl->batch = min(top, batch_max);
  ctl->cursor = 0;
  ctl->nout = 0;
  ctl->dump = 0;
  ctl->busy = 0;
  ctl->idle = 0;
  ctl->deep = 0;
  ctl->pool_head = 0;
  ctl->pool_tail = 0;
  ctl->launches += 1;
}

// Whole-table runs (src/e13search.c:428-433): one machine per thread.
__global__ void __launch_bounds__(256) run_full_kernel(const int *tabs, int n, int nq, long long *out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const KeyTabs K = key_tables(smem_raw);
  u32 *tape = reinterpret_cast<u32 *>(smem_raw + kKeySmemBytes);
  const int stride = blockDim.x;
  u32 *rows = tape + kTapeWords * stride;
  fill_key_tables(K);
  load_stage_tables();
  __syncthreads();
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  u32 *tcol = tape + threadIdx.x;
  u32 *rcol = rows + threadIdx.x;
  for (int w = 0; w < kTapeWords; ++w) tcol[w * stride] = 0;
  const int *tab = tabs + (long long)m * E13_MAXCELLS;
  for (int s = 0; s < 16; ++s) {
    u32 e0 = kEntHalt, e1 = kEntHalt;
    if (s < nq) {
      e0 = tab[2 * s] < 0 ? kEntHalt : (u32)tab[2 * s];
      e1 = tab[2 * s + 1] < 0 ? kEntHalt : (u32)tab[2 * s + 1];
    }
    rcol[s * stride] = cell_slot(2 * s, e0, true) | (cell_slot(2 * s + 1, e1, true) << 16);
  }
  Lane L;
  L.p = kLeft; L.st = 0; L.t = 0; L.deadline = s_deadline[1]; L.hb = 0; L.tgt = (u32)s_tgt[1];
  L.nt = 1; L.stage = 0; L.st0 = -1; L.p0 = kLeft; L.flags = 3; L.ch0 = L.ch1 = L.ch2 = 0;  // head0 = 0 until stage 1
  int ev;
  for (;;) {
    int nn = 1 << 30, cell = 0;
    ev = step_slice(L.p, L.st, L.t, L.deadline, L.hb, L.tgt, tcol, rcol, K.lo, stride, nn, cell);
    if (ev == kEvStage) {
      ev = stage_check(L, tcol, K, stride);
      if (ev == 0) continue;
    }
    if (ev == kEvCell) ev = kEvDead;  // only halts are special here
    break;
  }
  long long *o = out + 7LL * m;
  o[0] = ev == kEvSurv;
  o[1] = L.stage;
  o[2] = L.st0;
  o[3] = L.p0 - kLeft;
  o[4] = L.flags & 1;
  o[5] = (L.flags >> 1) & 1;
  o[6] = L.t;
}

}  // namespace

// ------------------------------------------------------------------------
// host side

struct e13_ctx {
  int device;
  int nsm;
  cudaStream_t stream;
  cudaEvent_t ev0, ev1, k0, k1;
  bool consts_ready;
  // buffers, grown on demand
  Node *stack;
  long long stack_cap;
  Node *out;
  long long out_cap;
  Node *wstack;
  long long wstack_nodes;
  Node *pool;
  long long pool_cap;
  int *pool_ready;
  long long pool_ready_cap;
  SurvRec *surv;
  long long surv_cap;
  Ctl *ctl;
  Ctl *ctl_host;
  JobParam *d_jobs;              // kMaxJobs
  unsigned long long *d_jobcnt;  // kMaxJobs x kJobCounters
  unsigned long long *d_jobnodes;  // kMaxJobs
  unsigned long long *h_jobbuf;  // pinned: counters then node counts
  e13_stats stats;
};

static int cuda_fail(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return 0;
  fprintf(stderr, "e13: %s: %s\n", what, cudaGetErrorString(e));
  return 1;
}
#define CK(x)                                   \
  do {                                          \
    if (cuda_fail((x), #x)) return E13_ERR_CUDA; \
  } while (0)

// Host<->device copies on the context's stream, counted in its statistics
// (the bytes an end-to-end caller moves across PCIe/C2C per search).
static cudaError_t h2d(e13_ctx *c, void *dst, const void *src, size_t bytes) {
  c->stats.h2d_bytes += (int64_t)bytes;
  return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream);
}
static cudaError_t d2h(e13_ctx *c, void *dst, const void *src, size_t bytes) {
  c->stats.d2h_bytes += (int64_t)bytes;
  return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream);
}

static int ensure_consts(e13_ctx *c) {
  if (c->consts_ready) return E13_OK;
  if (upload_filter_tables() != cudaSuccess) return E13_ERR_CUDA;
  c->consts_ready = true;
  return E13_OK;
}

extern "C" int e13_ctx_create(int device, e13_ctx **out) {
  if (!out) return E13_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return E13_ERR_NO_DEVICE;
  if (device < 0 || device >= ndev) return E13_ERR_ARG;
  CK(cudaSetDevice(device));
  e13_ctx *c = (e13_ctx *)calloc(1, sizeof(e13_ctx));
  c->device = device;
  CK(cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device));
  CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  CK(cudaEventCreate(&c->ev0));
  CK(cudaEventCreate(&c->ev1));
  CK(cudaEventCreate(&c->k0));
  CK(cudaEventCreate(&c->k1));
  CK(cudaMallocHost(&c->ctl_host, sizeof(Ctl)));
  CK(cudaMalloc(&c->ctl, sizeof(Ctl)));
  CK(cudaMalloc(&c->d_jobs, sizeof(JobParam) * kMaxJobs));
  CK(cudaMalloc(&c->d_jobcnt, sizeof(unsigned long long) * kMaxJobs * kJobCounters));
  CK(cudaMalloc(&c->d_jobnodes, sizeof(unsigned long long) * kMaxJobs));
  CK(cudaMallocHost(&c->h_jobbuf, sizeof(unsigned long long) * kMaxJobs * (kJobCounters + 1)));
  *out = c;
  return E13_OK;
}

extern "C" void e13_ctx_destroy(e13_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  cudaFree(c->stack);
  cudaFree(c->out);
  cudaFree(c->wstack);
  cudaFree(c->pool);
  cudaFree(c->pool_ready);
  cudaFree(c->surv);
  cudaFree(c->ctl);
  cudaFreeHost(c->ctl_host);
  cudaFree(c->d_jobs);
  cudaFree(c->d_jobcnt);
  cudaFree(c->d_jobnodes);
  cudaFreeHost(c->h_jobbuf);
  cudaEventDestroy(c->ev0);
  cudaEventDestroy(c->ev1);
  cudaEventDestroy(c->k0);
  cudaEventDestroy(c->k1);
  cudaStreamDestroy(c->stream);
  free(c);
}

extern "C" int e13_ctx_device(const e13_ctx *c) { return c ? c->device : 0; }
extern "C" cudaStream_t e13_ctx_stream(const e13_ctx *c) { return c->stream; }
extern "C" void e13_ctx_note_run(e13_ctx *c, double ms, long long launches) {
  memset(&c->stats, 0, sizeof c->stats);
  c->stats.device_ms = ms;
  c->stats.launches = launches;
  c->stats.search_kernel_launches = launches;
}

extern "C" int e13_last_stats(const e13_ctx *c, e13_stats *out) {
  if (!c || !out) return E13_ERR_ARG;
  *out = c->stats;
  return E13_OK;
}

template <typename T>
static int grow(T **p, long long *cap, long long want) {
  if (*cap >= want) return E13_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  CK(cudaMalloc(p, sizeof(T) * (size_t)want));
  *cap = want;
  return E13_OK;
}

static void decode_survivor(const SurvRec &r, int nq, e13_survivor *s) {
  memset(s, 0, sizeof *s);
  for (int i = 0; i < E13_MAXCELLS; ++i) s->tab[i] = E13_HALT;
  uint32_t mask = 0;
  for (int i = 0; i < 2 * nq; ++i) {
    const unsigned e = r.ent[i];
    if (e == kEntFree) {
      s->tab[i] = E13_FREE;
    } else {
      if (!(e & kEntUnread)) mask |= 1u << i;
      const unsigned v = e & 0x7Fu;
      s->tab[i] = (v & kEntHalt) ? E13_HALT : (int)v;
    }
  }
  s->read_mask = mask;
  s->st0 = r.st0;
  s->head0 = r.head0;
  s->abs_ok = r.abs_ok;
  s->rel_ok = r.rel_ok;
  s->steps = r.t;
}

// Kernel parameters of a search or serve session over the context's buffers.
// dump_room: frontier nodes the warps may write when an epoch ends.
static Params make_params(const e13_ctx *c, const e13_tuning &tu, int nq, long long nwarps, long long dump_room) {
  Params P;
  memset(&P, 0, sizeof P);
  P.jobs = c->d_jobs;
  P.jobcnt = c->d_jobcnt;
  P.nq = nq;
  P.slice = tu.slice;
  P.run_skip = tu.run_skip ? 1 : 0;
  // the plain kernel's launches wait for their slowest lane, which is the
  // oldest machine: it skips in every slice
  P.skip_after = (tu.run_skip >= 2 && tu.kernel == E13_KERNEL_PERSISTENT) ? tu.run_skip : 0;
  P.step_cap = tu.step_cap;
  P.wdepth = tu.warp_stack;
  P.pool_low = (int)std::max<long long>(1, nwarps * tu.pool_low_pct / 100);
  P.pool_cap = c->pool_cap;
  P.pool = c->pool;
  P.pool_ready = c->pool_ready;
  P.out_cap = c->out_cap;
  P.out_soft = c->out_cap - dump_room - 1024;
  P.surv_cap = c->surv_cap;
  P.epoch_ns = (long long)tu.epoch_us * 1000LL;
  P.wait_ns = kPoolWaitNs;
  P.min_epoch_ns = kMinEpochNs;
  P.stack = c->stack;
  P.out = c->out;
  P.wstack = c->wstack;
  P.surv = c->surv;
  P.ctl = c->ctl;
  return P;
}

static size_t search_smem(int block) {
  return kKeySmemBytes + (size_t)(kTapeWords + 16) * block * 4 + (size_t)(block / 32) * sizeof(Node);
}

// ------------------------------------------------------------------------
// checkpoint files of one search (e13_search_resumable)
//
// <path>.<slot>.bin   the frontier stack: top nodes as they are on the device
// <path>.<slot>.meta  CkptHeader, the config string, the job's counters, the
//                     survivor records
// <path>              the slot of the last complete checkpoint ("a" or "b")

namespace {

constexpr char kCkptMagic[8] = {'E', '1', '3', 'C', 'K', 'P', 'T', '2'};  // 2: Node::hb holds the low 32 bits
constexpr long long kCkptChunk = 1LL << 16;  // nodes per host transfer (20 MiB)

struct CkptHeader {
  char magic[8];
  uint32_t node_bytes, job_counters, surv_bytes, config_len;
  int64_t top, peak, launches;
  double wall;  // seconds of the search before this checkpoint
  uint64_t nsurv, nrec;
  e13_job job;
};

double host_seconds() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

bool file_exists(const std::string &path) {
  struct stat st;
  return stat(path.c_str(), &st) == 0;
}

std::string slot_file(const e13_checkpoint *ck, int slot, const char *ext) {
  return std::string(ck->path) + (slot ? ".b" : ".a") + ext;
}

bool write_all(FILE *f, const void *p, size_t n) { return n == 0 || fwrite(p, 1, n, f) == n; }
bool read_all(FILE *f, void *p, size_t n) { return n == 0 || fread(p, 1, n, f) == n; }

// flush, fsync and close: true only if the data reached the disk
bool close_synced(FILE *f) {
  const bool ok = fflush(f) == 0 && fsync(fileno(f)) == 0;
  return fclose(f) == 0 && ok;
}

// Writes the state after the last epoch (ctl_host is current) to `slot`, then
// points the pointer file at it.
int ckpt_save(e13_ctx *c, const e13_job *job, const e13_checkpoint *ck, int slot, double wall) {
  const Ctl &h = *c->ctl_host;
  const long long top = h.top;
  FILE *f = fopen(slot_file(ck, slot, ".bin").c_str(), "wb");
  if (!f) return E13_ERR_IO;
  std::vector<Node> buf((size_t)std::min(std::max(top, 1LL), kCkptChunk));
  for (long long o = 0; o < top; o += kCkptChunk) {
    const long long n = std::min(kCkptChunk, top - o);
    if (d2h(c, buf.data(), c->stack + o, sizeof(Node) * n) !=
            cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess) {
      fclose(f);
      return E13_ERR_CUDA;
    }
    if (!write_all(f, buf.data(), sizeof(Node) * (size_t)n)) {
      fclose(f);
      return E13_ERR_IO;
    }
  }
  if (!close_synced(f)) return E13_ERR_IO;

  unsigned long long cnt[kJobCounters];
  const unsigned long long nrec = std::min<unsigned long long>(h.nsurv, (unsigned long long)c->surv_cap);
  std::vector<SurvRec> recs((size_t)nrec);
  CK(d2h(c, cnt, c->d_jobcnt, sizeof cnt));
  if (nrec) CK(d2h(c, recs.data(), c->surv, sizeof(SurvRec) * nrec));
  CK(cudaStreamSynchronize(c->stream));
  CkptHeader hd;
  memset(&hd, 0, sizeof hd);
  memcpy(hd.magic, kCkptMagic, sizeof hd.magic);
  hd.node_bytes = sizeof(Node);
  hd.job_counters = kJobCounters;
  hd.surv_bytes = sizeof(SurvRec);
  hd.config_len = (uint32_t)strlen(ck->config);
  hd.top = top;
  hd.peak = h.peak;
  hd.launches = h.launches;
  hd.wall = wall;
  hd.nsurv = h.nsurv;
  hd.nrec = nrec;
  hd.job = *job;
  f = fopen(slot_file(ck, slot, ".meta").c_str(), "wb");
  if (!f) return E13_ERR_IO;
  const bool ok = write_all(f, &hd, sizeof hd) && write_all(f, ck->config, hd.config_len) &&
                  write_all(f, cnt, sizeof cnt) && write_all(f, recs.data(), sizeof(SurvRec) * (size_t)nrec);
  if (!close_synced(f) || !ok) return E13_ERR_IO;

  // the pointer last: until the rename the previous checkpoint stays the valid one
  const std::string tmp = std::string(ck->path) + ".tmp";
  f = fopen(tmp.c_str(), "wb");
  if (!f) return E13_ERR_IO;
  const bool pok = write_all(f, slot ? "b\n" : "a\n", 2);
  if (!close_synced(f) || !pok || rename(tmp.c_str(), ck->path) != 0) return E13_ERR_IO;
  return E13_OK;
}

// Loads the slot the pointer file names onto the device (stack, control
// block, counters, survivors).  *slot = the slot read.
int ckpt_load(e13_ctx *c, const e13_job *job, const e13_checkpoint *ck, long long batch_max, long long room,
              int *slot, double *prior_wall) {
  FILE *f = fopen(ck->path, "rb");
  if (!f) return E13_ERR_CKPT;
  char name[4] = {0};
  const size_t got = fread(name, 1, 3, f);
  fclose(f);
  if (got < 1 || (name[0] != 'a' && name[0] != 'b')) return E13_ERR_CKPT;
  *slot = name[0] == 'b';

  f = fopen(slot_file(ck, *slot, ".meta").c_str(), "rb");
  if (!f) return E13_ERR_CKPT;
  CkptHeader hd;
  std::string cfg;
  unsigned long long cnt[kJobCounters];
  bool ok = read_all(f, &hd, sizeof hd) && !memcmp(hd.magic, kCkptMagic, sizeof hd.magic) &&
            hd.node_bytes == sizeof(Node) && hd.job_counters == kJobCounters && hd.surv_bytes == sizeof(SurvRec) &&
            hd.config_len == strlen(ck->config) && hd.top >= 0 && hd.nrec <= hd.nsurv;
  if (ok) {
    cfg.resize(hd.config_len);
    ok = read_all(f, &cfg[0], hd.config_len) && cfg == ck->config && !memcmp(&hd.job, job, sizeof *job) &&
         read_all(f, cnt, sizeof cnt);
  }
  std::vector<SurvRec> recs;
  if (ok) {
    recs.resize((size_t)hd.nrec);
    ok = read_all(f, recs.data(), sizeof(SurvRec) * (size_t)hd.nrec);
  }
  fclose(f);
  if (!ok) return E13_ERR_CKPT;
  if (hd.top > room) return E13_ERR_OVERFLOW;

  const std::string bin = slot_file(ck, *slot, ".bin");
  struct stat st;
  if (stat(bin.c_str(), &st) != 0 || (long long)st.st_size != hd.top * (long long)sizeof(Node)) return E13_ERR_CKPT;
  f = fopen(bin.c_str(), "rb");
  if (!f) return E13_ERR_CKPT;
  std::vector<Node> buf((size_t)std::min(std::max((long long)hd.top, 1LL), kCkptChunk));
  for (long long o = 0; o < hd.top; o += kCkptChunk) {
    const long long n = std::min(kCkptChunk, (long long)hd.top - o);
    if (!read_all(f, buf.data(), sizeof(Node) * (size_t)n)) {
      fclose(f);
      return E13_ERR_CKPT;
    }
    if (h2d(c, c->stack + o, buf.data(), sizeof(Node) * n) !=
            cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess) {
      fclose(f);
      return E13_ERR_CUDA;
    }
  }
  fclose(f);

  int rc;
  if ((rc = grow(&c->surv, &c->surv_cap, std::max<long long>((long long)hd.nrec, c->surv_cap)))) return rc;
  memset(c->ctl_host, 0, sizeof(Ctl));
  c->ctl_host->top = hd.top;
  c->ctl_host->batch = std::min<long long>(hd.top, batch_max);
  c->ctl_host->peak = std::max<long long>(hd.peak, hd.top);
  c->ctl_host->launches = (int)hd.launches;
  c->ctl_host->nsurv = hd.nsurv;
  CK(h2d(c, c->ctl, c->ctl_host, sizeof(Ctl)));
  CK(h2d(c, c->d_jobcnt, cnt, sizeof cnt));
  if (hd.nrec) CK(h2d(c, c->surv, recs.data(), sizeof(SurvRec) * hd.nrec));
  CK(cudaStreamSynchronize(c->stream));
  *prior_wall = hd.wall;
  return E13_OK;
}

void ckpt_remove(const e13_checkpoint *ck) {
  remove(ck->path);
  for (int slot = 0; slot < 2; ++slot) {
    remove(slot_file(ck, slot, ".bin").c_str());
    remove(slot_file(ck, slot, ".meta").c_str());
  }
  remove((std::string(ck->path) + ".tmp").c_str());
}

// Whether to checkpoint now: 0 no, 1 save, 2 save and stop.
struct CkptClock {
  const e13_checkpoint *ck;
  std::string stop_file;
  double t_call, last_save, last_look;
  int due(double now) {
    if (ck->stop_after_s > 0 && now - t_call >= ck->stop_after_s) return 2;
    if (now - last_look >= 1.0) {
      last_look = now;
      if (file_exists(stop_file)) return 2;
    }
    const double every = ck->interval_s > 0 ? ck->interval_s : 1800.0;
    return now - last_save >= every ? 1 : 0;
  }
};

}  // namespace

// Sharding one search (e13_search_shard): the ordering key of a frontier node,
// every field that identifies the machine and nothing uninitialised.
struct ShardKey {
  unsigned short cellv[32];
  long long t;
  int p, st, pend, flags, budget, nintro;
  u64 hb, vmask;
  bool operator<(const ShardKey &o) const { return memcmp(this, &o, sizeof *this) < 0; }
};

static ShardKey shard_key(const Node &n) {
  ShardKey k;
  memset(&k, 0, sizeof k);
  memcpy(k.cellv, n.cellv, sizeof k.cellv);
  k.t = n.t;
  k.p = n.p;
  k.st = n.st;
  k.pend = n.pend;
  k.flags = n.flags;
  k.budget = n.budget;
  k.nintro = n.nintro;
  k.hb = n.hb;
  k.vmask = n.vmask;
  return k;
}

constexpr long long kSplitPerShard = 512;  // frontier nodes per shard before the deal
constexpr int kSplitLevels = 24;           // most plain launches of the split
constexpr int kSplitSlice = 24;            // the split's slice and step cap (fixed: they shape the frontier)
constexpr int kSplitStepCap = 20000;

// One share of a search split over nshards (the reference's SPLIT frontier,
// src/e13search.c:222-235, built for the device): the plain kernel expands the
// job level by level, each launch taking the whole frontier, until it holds
// kSplitPerShard nodes per shard; the frontier is then put in an order that
// depends only on its nodes (the same on every rank) and shard s keeps nodes
// s, s + nshards, ...  What the expansion itself finished (leaves, steps,
// survivors, with their read masks) counts in shard 0 only: *cnt and *recs
// are zero / empty for the other shards.  Runs on buffers of its own (freed
// before it returns), so a serve session's frontier is left alone; `slot` is
// the job slot written into the nodes.  The expansion runs with a fixed
// slice, step cap and run skip: a lane is requeued at the first slice end
// past the step cap, so those settings shape the frontier, and with them fixed
// every shard's content depends on the job alone, whatever tuning the caller's
// search then uses (the autotuner compares shard 0 across tunings).
static int split_share(e13_ctx *c, const e13_job *job, const e13_tuning &tu, int shard, int nshards, int slot,
                       std::vector<Node> &mine, unsigned long long cnt[kJobCounters], std::vector<SurvRec> &recs,
                       long long *launches) {
  mine.clear();
  recs.clear();
  memset(cnt, 0, sizeof(unsigned long long) * kJobCounters);
  const long long nwarps = (long long)c->nsm * tu.block / 32;
  const long long fan = 4LL * job->nq + 1;
  const long long target = kSplitPerShard * nshards;
  // the last level starts below target nodes and each node has at most `fan` children
  const long long stack_n = target * fan + nwarps * 32 + 1024, out_n = stack_n, surv_n = 4096;
  Node *stack = nullptr, *out = nullptr;
  Ctl *ctl = nullptr;
  JobParam *jobs = nullptr;
  unsigned long long *jobcnt = nullptr;
  SurvRec *surv = nullptr;
  int rc = E13_OK;
  auto fail = [&](cudaError_t e, const char *what) {
    if (e != cudaSuccess && rc == E13_OK) rc = cuda_fail(e, what) ? E13_ERR_CUDA : E13_OK;
    return rc != E13_OK;
  };
  JobParam jp[kMaxJobs];
  memset(jp, 0, sizeof jp);
  jp[slot].nv = 4 * job->nq;
  jp[slot].sym_lo = job->sym_lo;
  jp[slot].sym_hi = job->sym_hi;
  Node root;
  build_root(job, slot, &root, true, true);
  Ctl h;
  memset(&h, 0, sizeof h);
  h.top = 1;
  h.batch = 1;
  h.peak = 1;
  long long top = 1;
  if (!fail(cudaMalloc(&stack, sizeof(Node) * (size_t)stack_n), "split stack") &&
      !fail(cudaMalloc(&out, sizeof(Node) * (size_t)out_n), "split outputs") &&
      !fail(cudaMalloc(&ctl, sizeof(Ctl)), "split control") &&
      !fail(cudaMalloc(&jobs, sizeof jp), "split job") &&
      !fail(cudaMalloc(&jobcnt, sizeof(unsigned long long) * kMaxJobs * kJobCounters), "split counters") &&
      !fail(cudaMalloc(&surv, sizeof(SurvRec) * (size_t)surv_n), "split survivors") &&
      !fail(h2d(c, stack, &root, sizeof root), "split root") && !fail(h2d(c, ctl, &h, sizeof h), "split ctl") &&
      !fail(h2d(c, jobs, jp, sizeof jp), "split job") &&
      !fail(cudaMemsetAsync(jobcnt, 0, sizeof(unsigned long long) * kMaxJobs * kJobCounters, c->stream), "memset")) {
    e13_tuning t = tu;
    t.kernel = E13_KERNEL_PLAIN;
    t.slice = kSplitSlice;
    t.step_cap = kSplitStepCap;
    t.run_skip = 1;
    Params S = make_params(c, t, job->nq, nwarps, nwarps * 32);
    S.jobs = jobs;
    S.jobcnt = jobcnt;
    S.stack = stack;
    S.out = out;
    S.out_cap = out_n;
    S.out_soft = out_n;
    S.surv = surv;
    S.surv_cap = surv_n;
    S.ctl = ctl;
    const size_t smem = search_smem(tu.block);
    fail(cudaFuncSetAttribute(search_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "attr");
    for (int level = 0; rc == E13_OK && level < kSplitLevels && top > 0 && top < target; ++level) {
      search_kernel<false><<<c->nsm, tu.block, smem, c->stream>>>(S);
      move_outputs<<<c->nsm * 4, 256, 0, c->stream>>>(ctl, stack, out, c->pool, 0, stack_n);
      finish_launch<<<1, 1, 0, c->stream>>>(ctl, stack_n, kWholeFrontier, 0);
      *launches += 3;
      if (fail(cudaGetLastError(), "split launch") || fail(d2h(c, &h, ctl, sizeof h), "split ctl") ||
          fail(cudaStreamSynchronize(c->stream), "split sync"))
        break;
      if (h.error) rc = E13_ERR_OVERFLOW;
      top = h.top;
    }
  }
  if (rc == E13_OK) {
    // the deal
    std::vector<Node> nodes((size_t)top);
    const long long nrec = std::min<long long>((long long)h.nsurv, surv_n);
    if (shard == 0 && nrec > 0) {
      survivor_read_masks<<<(unsigned)((nrec + 31) / 32), 32, 0, c->stream>>>(surv, nrec);
      recs.resize((size_t)nrec);
      fail(cudaGetLastError(), "split survivors");
      if (rc == E13_OK) fail(d2h(c, recs.data(), surv, sizeof(SurvRec) * (size_t)nrec), "split survivors");
    }
    if (rc == E13_OK && top > 0) fail(d2h(c, nodes.data(), stack, sizeof(Node) * (size_t)top), "split frontier");
    if (rc == E13_OK && shard == 0)
      fail(d2h(c, cnt, jobcnt + (size_t)slot * kJobCounters, sizeof(unsigned long long) * kJobCounters), "counters");
    if (rc == E13_OK) fail(cudaStreamSynchronize(c->stream), "split sync");
    if (rc == E13_OK && (long long)h.nsurv > surv_n) rc = E13_ERR_SURV_CAP;
    if (rc == E13_OK) {
      std::vector<std::pair<ShardKey, long long>> order((size_t)top);
      for (long long i = 0; i < top; ++i) order[(size_t)i] = {shard_key(nodes[(size_t)i]), i};
      std::sort(order.begin(), order.end(), [](const std::pair<ShardKey, long long> &a,
                                               const std::pair<ShardKey, long long> &b) { return a.first < b.first; });
      for (long long i = shard; i < top; i += nshards) mine.push_back(nodes[(size_t)order[(size_t)i].second]);
    }
  }
  cudaStreamSynchronize(c->stream);
  cudaFree(stack);
  cudaFree(out);
  cudaFree(ctl);
  cudaFree(jobs);
  cudaFree(jobcnt);
  cudaFree(surv);
  return rc;
}

static int search_impl(e13_ctx *c, const e13_job *job, const e13_tuning *tuning, const e13_checkpoint *ck,
                       e13_counts *counts, e13_survivor *surv, int surv_cap, int *nsurv, double *wall_s,
                       int64_t *frontier, int shard = 0, int nshards = 1) {
  const double t_call = host_seconds();
  if (!c || !job || !counts || !nsurv || (surv_cap > 0 && !surv) || surv_cap < 0) return E13_ERR_ARG;
  if (nshards < 1 || shard < 0 || shard >= nshards || (ck && nshards > 1)) return E13_ERR_ARG;
  if (job->nq < 1 || job->nq > 16) return E13_ERR_NQ;
  if (job->budget < 0) return E13_ERR_FMAX;
  for (int i = 0; i < 2 * job->nq; ++i)
    if (job->tab[i] < E13_FREE || (job->tab[i] >= 0 && (job->tab[i] >> 2) >= job->nq)) return E13_ERR_ARG;
  e13_tuning tu;
  if (e13_resolve_tuning(tuning, 0, &tu) != E13_OK) return E13_ERR_ARG;
  CK(cudaSetDevice(c->device));
  int rc = ensure_consts(c);
  if (rc) return rc;
  memset(&c->stats, 0, sizeof c->stats);

  const bool persist = tu.kernel == E13_KERNEL_PERSISTENT;
  const int blocks = c->nsm;
  const long long nwarps = (long long)blocks * tu.block / 32;
  const long long stack_nodes = tu.stack_nodes > 0 ? tu.stack_nodes : (4LL << 20);
  const long long dump_room = nwarps * (32 + (persist ? tu.warp_stack : 0));
  long long out_nodes, batch_max;
  if (persist) {
    // every epoch may take the whole frontier: an epoch then ends on its time
    // bound, not in a tail where a few warps finish the last input subtrees
    batch_max = tu.batch > 0 ? tu.batch : kWholeFrontier;
    out_nodes = 2 * dump_room + 65536;
  } else {
    batch_max = tu.batch > 0 ? tu.batch : 16384;
    out_nodes = batch_max * (4LL * job->nq + 1) + nwarps * 32 + 1024;
  }
  if ((rc = grow(&c->stack, &c->stack_cap, stack_nodes))) return rc;
  // the frontier capacity of this search: exactly what the tuning asks for,
  // else all that the context holds (a larger stack left by a serve session)
  const long long cap = tu.stack_nodes > 0 ? tu.stack_nodes : c->stack_cap;
  if ((rc = grow(&c->out, &c->out_cap, out_nodes))) return rc;
  if (persist && (rc = grow(&c->wstack, &c->wstack_nodes, nwarps * tu.warp_stack))) return rc;
  if (persist && (rc = grow(&c->pool, &c->pool_cap, kPoolNodes))) return rc;
  if (persist && (rc = grow(&c->pool_ready, &c->pool_ready_cap, kPoolNodes))) return rc;
  const long long scap = std::max<long long>(surv_cap, 1024);
  if ((rc = grow(&c->surv, &c->surv_cap, scap))) return rc;

  JobParam jp[kMaxJobs];
  memset(jp, 0, sizeof jp);
  jp[0].nv = 4 * job->nq;
  jp[0].sym_lo = job->sym_lo;
  jp[0].sym_hi = job->sym_hi;
  CK(h2d(c, c->d_jobs, jp, sizeof jp));
  CK(cudaMemsetAsync(c->d_jobcnt, 0, sizeof(unsigned long long) * kMaxJobs * kJobCounters, c->stream));
  Params P = make_params(c, tu, job->nq, nwarps, dump_room);

  const size_t smem = search_smem(tu.block);
  if (persist) CK(cudaFuncSetAttribute(search_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  else CK(cudaFuncSetAttribute(search_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));

  // the root: blank tape, every cell unread
  Node root;
  build_root(job, 0, &root, tu.run_skip != 0, true);
  memset(c->ctl_host, 0, sizeof(Ctl));
  c->ctl_host->top = 1;
  c->ctl_host->batch = 1;
  c->ctl_host->peak = 1;
  CK(h2d(c, c->stack, &root, sizeof root));
  // pool slots carry the tag of the launch that wrote them; tags restart with every search
  if (persist) CK(cudaMemsetAsync(c->pool_ready, 0, sizeof(int) * (size_t)c->pool_ready_cap, c->stream));
  CK(h2d(c, c->ctl, c->ctl_host, sizeof(Ctl)));

  // checkpoints: resume from the last complete slot, then save into the other one
  double prior_wall = 0.0;
  int slot = 0;
  bool stopped = false;
  CkptClock clk{ck, ck ? std::string(ck->path) + ".stop" : std::string(), t_call, t_call, t_call};
  if (ck) {
    if (file_exists(clk.stop_file)) remove(clk.stop_file.c_str());  // left from the last clean stop
    if (file_exists(ck->path)) {
      int loaded = 0;
      if ((rc = ckpt_load(c, job, ck, batch_max, cap - out_nodes, &loaded, &prior_wall))) return rc;
      slot = loaded ^ 1;
    }
  }
  auto checkpoint_step = [&](int &status) -> bool {  // true: leave the launch loop
    if (!ck || c->ctl_host->top == 0) return false;
    const double now = host_seconds();
    const int act = clk.due(now);
    if (!act) return false;
    const int r = ckpt_save(c, job, ck, slot, prior_wall + (now - t_call));
    if (r) {
      status = r;
      return true;
    }
    slot ^= 1;
    clk.last_save = host_seconds();
    stopped = act == 2;
    if (stopped && file_exists(clk.stop_file)) remove(clk.stop_file.c_str());  // consumed by this stop
    return stopped;
  };
  CK(cudaEventRecord(c->ev0, c->stream));

  const int move_blocks = c->nsm * 4;
  long long launches = 0, search_launches = 0;
  int err = 0;

  // sharded: the plain kernel expands the search level by level (each launch
  // takes the whole frontier) until it holds kSplitPerShard nodes per shard;
  // the frontier is then put in an order that depends only on its nodes (the
  // same on every rank) and shard s keeps nodes s, s + nshards, ...  What the
  // split itself finished (leaves, steps, survivors) counts in shard 0 only.
  bool split = false;
  if (nshards > 1) {
    split = true;
    std::vector<Node> mine;
    std::vector<SurvRec> recs;
    unsigned long long cnt[kJobCounters];
    if ((rc = split_share(c, job, tu, shard, nshards, 0, mine, cnt, recs, &launches))) return rc;
    search_launches += launches / 3;
    if ((long long)mine.size() > cap - out_nodes) return E13_ERR_OVERFLOW;
    if (!mine.empty()) CK(h2d(c, c->stack, mine.data(), sizeof(Node) * mine.size()));
    if (!recs.empty()) CK(h2d(c, c->surv, recs.data(), sizeof(SurvRec) * recs.size()));
    CK(h2d(c, c->d_jobcnt, cnt, sizeof cnt));
    c->ctl_host->top = (long long)mine.size();
    c->ctl_host->batch = std::min<long long>((long long)mine.size(), batch_max);
    c->ctl_host->peak = c->ctl_host->top;
    c->ctl_host->nsurv = recs.size();
    CK(h2d(c, c->ctl, c->ctl_host, sizeof(Ctl)));
    CK(cudaStreamSynchronize(c->stream));
  }
  if (persist) {
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    for (int e = 0; e < tu.epochs_per_graph; ++e) {
      search_kernel<true><<<blocks, tu.block, smem, c->stream>>>(P);
      move_outputs<<<move_blocks, 256, 0, c->stream>>>(c->ctl, c->stack, c->out, c->pool, c->pool_cap, cap);
      finish_launch<<<1, 1, 0, c->stream>>>(c->ctl, cap, batch_max, c->pool_cap);
    }
    CK(cudaStreamEndCapture(c->stream, &graph));
    CK(cudaGraphInstantiate(&exec, graph, 0));
    for (;;) {
      CK(cudaGraphLaunch(exec, c->stream));
      launches += 3LL * tu.epochs_per_graph;
      search_launches += tu.epochs_per_graph;
      CK(d2h(c, c->ctl_host, c->ctl, sizeof(Ctl)));
      CK(cudaStreamSynchronize(c->stream));
      if (c->ctl_host->error) {
        err = (c->ctl_host->error & kErrTimeout) ? E13_ERR_TIMEOUT : E13_ERR_OVERFLOW;
        break;
      }
      if (c->ctl_host->top == 0) break;
      if (c->ctl_host->top > cap - (long long)out_nodes) {  // the next epoch's outputs might not fit
        err = E13_ERR_OVERFLOW;
        break;
      }
      if (checkpoint_step(err)) break;
    }
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
  } else {
    for (;;) {
      search_kernel<false><<<blocks, tu.block, smem, c->stream>>>(P);
      move_outputs<<<move_blocks, 256, 0, c->stream>>>(c->ctl, c->stack, c->out, c->pool, c->pool_cap, cap);
      finish_launch<<<1, 1, 0, c->stream>>>(c->ctl, cap, batch_max, c->pool_cap);
      launches += 3;
      search_launches += 1;
      CK(cudaGetLastError());
      CK(d2h(c, c->ctl_host, c->ctl, sizeof(Ctl)));
      CK(cudaStreamSynchronize(c->stream));
      if (c->ctl_host->error) {
        err = E13_ERR_OVERFLOW;
        break;
      }
      if (c->ctl_host->top == 0) break;
      if (c->ctl_host->top > cap - (long long)out_nodes) {  // the next launch's outputs might not fit
        err = E13_ERR_OVERFLOW;
        break;
      }
      if (checkpoint_step(err)) break;
    }
  }
  CK(cudaEventRecord(c->ev1, c->stream));
  CK(cudaEventSynchronize(c->ev1));
  CK(cudaGetLastError());
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  c->stats.device_ms = ms;
  c->stats.launches = launches;
  c->stats.search_kernel_launches = search_launches;
  c->stats.epochs = c->ctl_host->launches;
  c->stats.peak_nodes = c->ctl_host->peak;
  c->stats.lane_occupancy =
      c->ctl_host->rounds ? (double)c->ctl_host->lane_rounds / (32.0 * (double)c->ctl_host->rounds) : 0.0;
  c->stats.warp_rounds = (int64_t)c->ctl_host->rounds;
  c->stats.donations = (int64_t)c->ctl_host->donations;
  c->stats.pool_claims = (int64_t)c->ctl_host->claims;
  c->stats.idle_polls = (int64_t)c->ctl_host->polls;
  if (err) return err;

  const Ctl &h = *c->ctl_host;
  CK(d2h(c, c->h_jobbuf, c->d_jobcnt, sizeof(unsigned long long) * kJobCounters));
  CK(cudaStreamSynchronize(c->stream));
  memset(counts, 0, sizeof *counts);
  counts->leaves = c->h_jobbuf[0];
  counts->steps = c->h_jobbuf[1];
  counts->survivors = h.nsurv;
  for (int j = 0; j <= E13_STAGES; ++j) counts->hist[j] = c->h_jobbuf[2 + j];
  const long long ns = (long long)h.nsurv;
  *nsurv = (int)std::min<long long>(ns, 0x7FFFFFFF);
  const long long ncopy = std::min<long long>(ns, std::min<long long>(surv_cap, c->surv_cap));
  if (ncopy > 0) {
    std::vector<SurvRec> recs((size_t)ncopy);
    if (!persist || split) {
      survivor_read_masks<<<(unsigned)((ncopy + 31) / 32), 32, 0, c->stream>>>(c->surv, ncopy);
      CK(cudaGetLastError());
    }
    CK(d2h(c, recs.data(), c->surv, sizeof(SurvRec) * (size_t)ncopy));
    CK(cudaStreamSynchronize(c->stream));
    for (long long i = 0; i < ncopy; ++i) decode_survivor(recs[(size_t)i], job->nq, &surv[i]);
  }
  if (wall_s) *wall_s = prior_wall + (host_seconds() - t_call);
  if (frontier) *frontier = stopped ? h.top : 0;
  if (stopped) return E13_STOPPED;
  if (ck) ckpt_remove(ck);
  if (ns > surv_cap || ns > c->surv_cap) return E13_ERR_SURV_CAP;
  return E13_OK;
}

extern "C" int e13_search(e13_ctx *c, const e13_job *job, const e13_tuning *tuning, e13_counts *counts,
                          e13_survivor *surv, int surv_cap, int *nsurv) {
  return search_impl(c, job, tuning, nullptr, counts, surv, surv_cap, nsurv, nullptr, nullptr);
}

extern "C" int e13_search_resumable(e13_ctx *c, const e13_job *job, const e13_tuning *tuning,
                                    const e13_checkpoint *ck, e13_counts *counts, e13_survivor *surv, int surv_cap,
                                    int *nsurv, double *wall_s, int64_t *frontier) {
  if (!ck || !ck->path || !ck->config || !ck->path[0]) return E13_ERR_ARG;
  return search_impl(c, job, tuning, ck, counts, surv, surv_cap, nsurv, wall_s, frontier);
}

extern "C" int e13_search_shard(e13_ctx *c, const e13_job *job, const e13_tuning *tuning, int shard, int nshards,
                                e13_counts *counts, e13_survivor *surv, int surv_cap, int *nsurv) {
  return search_impl(c, job, tuning, nullptr, counts, surv, surv_cap, nsurv, nullptr, nullptr, shard, nshards);
}

extern "C" int e13_run_full(e13_ctx *c, const int32_t *tabs, int n, int nq, int64_t *out) {
  if (!c || !tabs || !out || n < 0 || nq < 1 || nq > 16) return E13_ERR_ARG;
  if (n == 0) return E13_OK;
  CK(cudaSetDevice(c->device));
  int rc = ensure_consts(c);
  if (rc) return rc;
  int *d_tabs = nullptr;
  long long *d_out = nullptr;
  CK(cudaMalloc(&d_tabs, sizeof(int) * E13_MAXCELLS * (size_t)n));
  CK(cudaMalloc(&d_out, sizeof(long long) * 7 * (size_t)n));
  CK(h2d(c, d_tabs, tabs, sizeof(int) * E13_MAXCELLS * (size_t)n));
  const int bd = 256;
  const size_t smem = kKeySmemBytes + (size_t)(kTapeWords + 16) * bd * 4;
  CK(cudaFuncSetAttribute(run_full_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  run_full_kernel<<<(n + bd - 1) / bd, bd, smem, c->stream>>>(d_tabs, n, nq, d_out);
  CK(cudaGetLastError());
  CK(d2h(c, out, d_out, sizeof(long long) * 7 * (size_t)n));
  CK(cudaStreamSynchronize(c->stream));
  cudaFree(d_tabs);
  cudaFree(d_out);
  return E13_OK;
}

// One epoch of the persistent kernel in which the donation pool holds one
// claimed slot whose donor never publishes it: the warp that claims it waits
// for the slot's ready tag, gives up after wait_us, and flags kErrTimeout.
// Nothing else is on the frontier, so the epoch then ends.  The slot's data is
// never read (the claim is dropped when the wait runs out).
extern "C" int e13_selftest_pool_wait(e13_ctx *c, int32_t wait_us) {
  if (!c || wait_us < 1 || wait_us > 1000000) return E13_ERR_ARG;
  CK(cudaSetDevice(c->device));
  int rc = ensure_consts(c);
  if (rc) return rc;
  e13_tuning tu;
  e13_resolve_tuning(nullptr, 0, &tu);
  const long long nwarps = (long long)c->nsm * tu.block / 32;
  const long long dump_room = nwarps * (32 + tu.warp_stack);
  if ((rc = grow(&c->stack, &c->stack_cap, 1024))) return rc;
  if ((rc = grow(&c->out, &c->out_cap, 2 * dump_room + 65536))) return rc;
  if ((rc = grow(&c->wstack, &c->wstack_nodes, nwarps * tu.warp_stack))) return rc;
  if ((rc = grow(&c->pool, &c->pool_cap, kPoolNodes))) return rc;
  if ((rc = grow(&c->pool_ready, &c->pool_ready_cap, kPoolNodes))) return rc;
  if ((rc = grow(&c->surv, &c->surv_cap, 1024))) return rc;
  Params P = make_params(c, tu, 16, nwarps, dump_room);
  P.wait_ns = (long long)wait_us * 1000LL;
  const size_t smem = search_smem(tu.block);
  CK(cudaFuncSetAttribute(search_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  JobParam jp[kMaxJobs];
  memset(jp, 0, sizeof jp);
  CK(h2d(c, c->d_jobs, jp, sizeof jp));
  CK(cudaMemsetAsync(c->d_jobcnt, 0, sizeof(unsigned long long) * kMaxJobs * kJobCounters, c->stream));
  // ready tags 0; the launch's tag is launches + 1 = 1, so slot 0 never looks published
  CK(cudaMemsetAsync(c->pool_ready, 0, sizeof(int) * (size_t)c->pool_ready_cap, c->stream));
  memset(c->ctl_host, 0, sizeof(Ctl));
  c->ctl_host->pool_tail = 1;  // slot 0 donated (claimable), its data never written
  CK(h2d(c, c->ctl, c->ctl_host, sizeof(Ctl)));
  search_kernel<true><<<c->nsm, tu.block, smem, c->stream>>>(P);
  move_outputs<<<c->nsm * 4, 256, 0, c->stream>>>(c->ctl, c->stack, c->out, c->pool, c->pool_cap, c->stack_cap);
  finish_launch<<<1, 1, 0, c->stream>>>(c->ctl, c->stack_cap, kWholeFrontier, c->pool_cap);
  CK(cudaGetLastError());
  CK(d2h(c, c->ctl_host, c->ctl, sizeof(Ctl)));
  CK(cudaStreamSynchronize(c->stream));
  const int err = c->ctl_host->error;
  if (err & kErrTimeout) return E13_ERR_TIMEOUT;
  return err ? E13_ERR_OVERFLOW : E13_OK;
}

// ------------------------------------------------------------------------
// autotuner

// The autotuner times candidates through serve sessions (defined below).
extern "C" int e13_serve_create(e13_ctx *ctx, const e13_tuning *tuning, int64_t reserve_nodes, e13_serve **out);
extern "C" void e13_serve_destroy(e13_serve *s);
extern "C" int e13_serve_submit(e13_serve *s, const e13_job *job, int64_t id, double t_submit);
extern "C" int e13_serve_submit_shard(e13_serve *s, const e13_job *job, int64_t id, double t_submit, int shard,
                                      int nshards);
extern "C" int e13_serve_step(e13_serve *s, e13_serve_result *done, int cap, int *ndone);
extern "C" int64_t e13_serve_pending(const e13_serve *s);
extern "C" int e13_serve_stats(const e13_serve *s, double *device_ms, int64_t *epochs, int64_t *swapped_out,
                               int64_t *peak_nodes, int64_t *peak_job_nodes);

extern "C" int e13_autotune_jobs(e13_ctx *c, const e13_job *jobs, int n, int32_t proxy_shards,
                                 const e13_tuning *start, e13_tuning *best, double *best_ms) {
  if (!c || !jobs || n < 1 || n > 4096 || !best || proxy_shards < 0 || proxy_shards > 4096) return E13_ERR_ARG;
  e13_tuning cur;
  if (e13_resolve_tuning(start, 0, &cur) != E13_OK) return E13_ERR_ARG;
  cur.kernel = E13_KERNEL_PERSISTENT;
  const int nsh = proxy_shards > 1 ? proxy_shards : 1;
  // a candidate: shard 0 of nsh of every job, all in one serve session (the
  // way a workload of several jobs runs), timed over its epochs; every job's
  // counts are kept to check that the tuning changes no result
  auto run = [&](const e13_tuning &t, std::vector<e13_counts> &out, double *ms) -> int {
    e13_serve *s = nullptr;
    int rc = e13_serve_create(c, &t, 0, &s);
    if (rc) return rc;
    out.assign((size_t)n, e13_counts());
    for (int i = 0; i < n && !rc; ++i)
      rc = nsh > 1 ? e13_serve_submit_shard(s, &jobs[i], i, 0.0, 0, nsh) : e13_serve_submit(s, &jobs[i], i, 0.0);
    e13_serve_result done[kMaxJobs];
    while (!rc && e13_serve_pending(s) > 0) {
      int nd = 0;
      rc = e13_serve_step(s, done, kMaxJobs, &nd);
      for (int k = 0; k < nd && !rc; ++k) {
        if (done[k].status != E13_OK && done[k].status != E13_ERR_SURV_CAP) rc = done[k].status;
        else out[(size_t)done[k].id] = done[k].counts;
      }
    }
    if (!rc) e13_serve_stats(s, ms, nullptr, nullptr, nullptr, nullptr);
    e13_serve_destroy(s);
    return rc;
  };
  // a candidate's time is the faster of two runs: one run of the proxy
  // varies by a few per cent between repeats, as much as the axes differ
  auto timed = [&](const e13_tuning &t, std::vector<e13_counts> &out, double *ms) -> int {
    double a = 0, b = 0;
    int r = run(t, out, &a);
    if (r) return r;
    std::vector<e13_counts> again;
    if ((r = run(t, again, &b))) return r;
    if (memcmp(again.data(), out.data(), sizeof(e13_counts) * (size_t)n) != 0) return E13_ERR_CUDA;
    *ms = a < b ? a : b;
    return E13_OK;
  };
  std::vector<e13_counts> ref, got;
  double cur_ms = 0;
  int rc = run(cur, ref, &cur_ms);  // warms the buffers up
  if (rc) return rc;
  if ((rc = timed(cur, got, &cur_ms))) return rc;
  if (memcmp(got.data(), ref.data(), sizeof(e13_counts) * (size_t)n) != 0) return E13_ERR_CUDA;
  struct Axis {
    int32_t e13_tuning::*field;
    int vals[5];
    int n;
  };
  // block: lanes per CTA (one CTA per SM); slice: iterations between a
  // warp's refill rounds; warp_stack: the depth of subtree a warp keeps to
  // itself before it spills or donates; pool_low_pct: the threshold below
  // which warps with deep stacks fork work off to idle warps; run_skip: the
  // machine age (steps) from which a warp takes word-at-a-time run skips
  const Axis axes[] = {
      {&e13_tuning::run_skip, {1, 1024, 4096, 8192, 32768}, 5},
      {&e13_tuning::block, {512, 640, 768, 0, 0}, 3},
      {&e13_tuning::slice, {8, 12, 16, 24, 32}, 5},
      {&e13_tuning::warp_stack, {64, 128, 256, 512, 0}, 4},
      {&e13_tuning::pool_low_pct, {2, 5, 12, 25, 0}, 4},
  };
  for (const Axis &ax : axes) {
    e13_tuning axis_best = cur;
    double axis_ms = cur_ms;
    for (int i = 0; i < ax.n; ++i) {
      if (ax.vals[i] == cur.*(ax.field)) continue;
      e13_tuning t = cur;
      t.*(ax.field) = ax.vals[i];
      double ms = 0;
      if ((rc = timed(t, got, &ms))) return rc;
      if (memcmp(got.data(), ref.data(), sizeof(e13_counts) * (size_t)n) != 0)
        return E13_ERR_CUDA;  // results must not depend on tuning
      if (ms < axis_ms * 0.97) {  // a 3 % margin keeps timing noise from moving the choice
        axis_ms = ms;
        axis_best = t;
      }
    }
    cur = axis_best;
    cur_ms = axis_ms;
  }
  *best = cur;
  if (best_ms) *best_ms = cur_ms;
  return E13_OK;
}

extern "C" int e13_autotune(e13_ctx *c, const e13_job *job, int32_t proxy_shards, const e13_tuning *start,
                            e13_tuning *best, double *best_ms) {
  return e13_autotune_jobs(c, job, 1, proxy_shards, start, best, best_ms);
}

// ------------------------------------------------------------------------
// serving: many searches in one persistent kernel (continuous batching)

#include <chrono>
#include <deque>
#include <memory>
#include <unordered_map>

extern "C" int e13_estimate(e13_ctx *ctx, const e13_job *job, int64_t probes, uint64_t seed, e13_estimate_out *out,
                            double *per_probe);

namespace {

constexpr int64_t kAdmitProbes = 64;  // Knuth probes behind a job's frontier reservation

struct ServeJob {
  int64_t id;
  e13_job job;
  double t_submit, t_start;
  int slot;
  long long reserve;                    // frontier nodes reserved while it runs
  std::vector<e13_survivor> surv;
  // swapped out: its frontier nodes and counters, put back on re-admission
  bool swapped = false;
  std::vector<Node> saved;
  unsigned long long saved_cnt[kJobCounters];
};

double wall_seconds() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace

struct e13_serve {
  e13_ctx *c;
  e13_tuning tu;
  Params P;
  size_t smem;
  long long batch_max, out_nodes, fixed_reserve, cap, large_reserve;
  std::deque<std::unique_ptr<ServeJob>> queue;
  std::unique_ptr<ServeJob> slot_job[kMaxJobs];
  std::unordered_map<int64_t, std::vector<e13_survivor>> finished_surv;
  JobParam jp[kMaxJobs];
  unsigned long long surv_fetched;
  bool surv_overflow;
  double t0;
  double device_ms;
  long long epochs, evictions;
  long long peak_top, peak_job;  // largest frontier after an epoch, and one job's largest share of it
  // frontier order between epochs: a second stack buffer, the group starts
  Node *alt = nullptr;
  long long alt_cap = 0;
  unsigned long long *d_fill = nullptr;
  unsigned long long fill[kMaxJobs];
  bool reorder = false;
  ~e13_serve() {
    cudaFree(alt);
    cudaFree(d_fill);
  }
};

extern "C" int e13_serve_create(e13_ctx *c, const e13_tuning *tuning, int64_t reserve_nodes, e13_serve **out) {
  if (!c || !out || reserve_nodes < 0) return E13_ERR_ARG;
  *out = nullptr;
  e13_tuning tu;
  if (e13_resolve_tuning(tuning, 1, &tu) != E13_OK) return E13_ERR_ARG;
  CK(cudaSetDevice(c->device));
  int rc = ensure_consts(c);
  if (rc) return rc;
  std::unique_ptr<e13_serve> s(new e13_serve());
  s->c = c;
  s->tu = tu;
  const long long nwarps = (long long)c->nsm * tu.block / 32;
  const long long dump_room = nwarps * (32 + tu.warp_stack);
  s->batch_max = tu.batch > 0 ? tu.batch : kWholeFrontier;
  s->out_nodes = 2 * dump_room + 65536;
  s->fixed_reserve = reserve_nodes;
  // a job too big for its estimate to bound its frontier reserves what one
  // epoch's dump of every warp can leave behind
  s->large_reserve = dump_room;
  // serving keeps many frontiers resident: 16 Mi nodes (5 GB) by default
  const long long stack_nodes = tu.stack_nodes > 0 ? tu.stack_nodes : (16LL << 20);
  if ((rc = grow(&c->stack, &c->stack_cap, stack_nodes))) return rc;
  s->cap = tu.stack_nodes > 0 ? tu.stack_nodes : c->stack_cap;
  if ((rc = grow(&c->out, &c->out_cap, s->out_nodes))) return rc;
  if ((rc = grow(&c->wstack, &c->wstack_nodes, nwarps * tu.warp_stack))) return rc;
  if ((rc = grow(&c->pool, &c->pool_cap, kPoolNodes))) return rc;
  if ((rc = grow(&c->pool_ready, &c->pool_ready_cap, kPoolNodes))) return rc;
  if ((rc = grow(&c->surv, &c->surv_cap, 1LL << 20))) return rc;
  memset(s->jp, 0, sizeof s->jp);
  s->P = make_params(c, tu, 16, nwarps, dump_room);
  s->smem = search_smem(tu.block);
  CK(cudaFuncSetAttribute(search_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s->smem));
  memset(c->ctl_host, 0, sizeof(Ctl));
  CK(h2d(c, c->ctl, c->ctl_host, sizeof(Ctl)));
  CK(cudaMemsetAsync(c->pool_ready, 0, sizeof(int) * (size_t)c->pool_ready_cap, c->stream));
  CK(cudaMemsetAsync(c->d_jobcnt, 0, sizeof(unsigned long long) * kMaxJobs * kJobCounters, c->stream));
  CK(h2d(c, c->d_jobs, s->jp, sizeof s->jp));
  CK(cudaMalloc(&s->alt, sizeof(Node) * (size_t)c->stack_cap));
  s->alt_cap = c->stack_cap;
  CK(cudaMalloc(&s->d_fill, sizeof(unsigned long long) * kMaxJobs));
  CK(cudaStreamSynchronize(c->stream));
  memset(&c->stats, 0, sizeof c->stats);
  s->t0 = wall_seconds();
  *out = s.release();
  return E13_OK;
}

extern "C" void e13_serve_destroy(e13_serve *s) { delete s; }

extern "C" double e13_serve_clock(const e13_serve *s) { return s ? wall_seconds() - s->t0 : 0.0; }

extern "C" int e13_serve_submit(e13_serve *s, const e13_job *job, int64_t id, double t_submit) {
  if (!s || !job) return E13_ERR_ARG;
  if (job->nq < 1 || job->nq > 16) return E13_ERR_NQ;
  if (job->budget < 0) return E13_ERR_FMAX;
  for (int i = 0; i < 2 * job->nq; ++i)
    if (job->tab[i] < E13_FREE || (job->tab[i] >= 0 && (job->tab[i] >> 2) >= job->nq)) return E13_ERR_ARG;
  std::unique_ptr<ServeJob> j(new ServeJob());
  j->id = id;
  j->job = *job;
  j->t_submit = t_submit >= 0 ? t_submit : e13_serve_clock(s);
  j->t_start = -1;
  j->slot = -1;
  if (s->fixed_reserve > 0) {
    j->reserve = s->fixed_reserve;
  } else {
    // the frontier of a search never holds more machines than its tree has
    // nodes and leaves: a job the estimate puts below one epoch's dump
    // reserves twice its estimate, a larger one the dump bound
    e13_estimate_out est;
    const int rc = e13_estimate(s->c, job, kAdmitProbes, 0, &est, nullptr);
    if (rc) return rc;
    const double tree = est.mean[0] + est.mean[1];
    j->reserve = tree * 2.0 < (double)s->large_reserve ? std::max<long long>(64, (long long)(tree * 2.0) + 1)
                                                       : s->large_reserve;
  }
  s->queue.push_back(std::move(j));
  return E13_OK;
}

extern "C" int e13_serve_submit_shard(e13_serve *s, const e13_job *job, int64_t id, double t_submit, int shard,
                                      int nshards) {
  if (!s || !job || nshards < 1 || shard < 0 || shard >= nshards) return E13_ERR_ARG;
  if (nshards == 1) return e13_serve_submit(s, job, id, t_submit);
  int rc = e13_serve_submit(s, job, id, t_submit);  // checks the job and sizes it
  if (rc) return rc;
  std::unique_ptr<ServeJob> j = std::move(s->queue.back());
  s->queue.pop_back();
  std::vector<SurvRec> recs;
  long long launches = 0;
  CK(cudaSetDevice(s->c->device));
  if ((rc = split_share(s->c, job, s->tu, shard, nshards, 0, j->saved, j->saved_cnt, recs, &launches))) return rc;
  s->c->stats.launches += launches;
  for (const SurvRec &r : recs) {
    e13_survivor sv;
    decode_survivor(r, job->nq, &sv);
    j->surv.push_back(sv);
  }
  // it starts as a job swapped out with its share of the frontier
  j->swapped = true;
  j->reserve = std::max<long long>({64, j->reserve / nshards, 2 * (long long)j->saved.size()});
  s->queue.push_back(std::move(j));
  return E13_OK;
}

extern "C" int64_t e13_serve_pending(const e13_serve *s) {
  if (!s) return 0;
  int64_t n = (int64_t)s->queue.size();
  for (int k = 0; k < kMaxJobs; ++k) n += s->slot_job[k] ? 1 : 0;
  return n;
}

namespace {

void fill_result(e13_serve_result &r, const ServeJob &j, const unsigned long long *cnt, int status, double tdone) {
  memset(&r, 0, sizeof r);
  r.id = j.id;
  r.counts.leaves = cnt[0];
  r.counts.steps = cnt[1];
  for (int h = 0; h <= E13_STAGES; ++h) r.counts.hist[h] = cnt[2 + h];
  r.counts.survivors = (uint64_t)j.surv.size();
  r.nsurv = (int32_t)j.surv.size();
  r.status = status;
  r.t_submit = j.t_submit;
  r.t_start = j.t_start;
  r.t_done = tdone;
}

}  // namespace

// Regroups the frontier by job into s->alt, groups laid out bottom to top in
// `order` (the last one ends on top), and makes it the frontier.
static int regroup(e13_serve *s, const int *order, int n, const unsigned long long *nodes) {
  e13_ctx *c = s->c;
  unsigned long long off = 0;
  memset(s->fill, 0, sizeof s->fill);
  for (int i = 0; i < n; ++i) {
    s->fill[order[i]] = off;
    off += nodes[order[i]];
  }
  CK(h2d(c, s->d_fill, s->fill, sizeof s->fill));
  order_by_job<<<c->nsm * 4, 256, 0, c->stream>>>(c->ctl, c->stack, s->alt, s->d_fill, s->alt_cap);
  CK(cudaGetLastError());
  std::swap(c->stack, s->alt);
  s->P.stack = c->stack;
  c->stats.launches += 1;
  return E13_OK;
}

// Sets the frontier's size on the device (Ctl::top, Ctl::batch) and here.
static int set_top(e13_serve *s, long long top) {
  e13_ctx *c = s->c;
  c->ctl_host->top = top;
  c->ctl_host->batch = std::min(top, s->batch_max);
  long long tb[2] = {top, c->ctl_host->batch};
  CK(h2d(c, c->ctl, tb, sizeof tb));  // Ctl::top, Ctl::batch
  return E13_OK;
}

// Swaps jobs out of the frontier: order[0..first) leave it, order[first..n)
// stay (most live nodes first, the usual order).  The frontier is regrouped
// bottom to top as the staying jobs, then the leaving ones, whose nodes are
// then copied to host memory from above the new top (`after` nodes).  Each
// leaving job takes its counters (cnt, as of the last epoch) and goes back to
// the head of the queue, reserving at least twice the nodes it had; a slot
// already emptied (a job that failed) only has its nodes dropped.
static int swap_out(e13_serve *s, const int *order, int n, int first, const unsigned long long *nodes,
                    const unsigned long long *cnt, long long after) {
  e13_ctx *c = s->c;
  int lay[kMaxJobs], m = 0;
  for (int i = first; i < n; ++i) lay[m++] = order[i];
  for (int i = first - 1; i >= 0; --i) lay[m++] = order[i];
  int rc;
  if ((rc = regroup(s, lay, m, nodes))) return rc;
  long long pos = after;
  for (int i = first - 1; i >= 0; --i) {
    const int k = order[i];
    if (s->slot_job[k]) {
      std::unique_ptr<ServeJob> j = std::move(s->slot_job[k]);
      j->saved.resize((size_t)nodes[k]);
      if (nodes[k]) CK(d2h(c, j->saved.data(), c->stack + pos, sizeof(Node) * (size_t)nodes[k]));
      memcpy(j->saved_cnt, cnt + k * kJobCounters, sizeof j->saved_cnt);
      j->swapped = true;
      j->reserve = std::max<long long>(j->reserve, 2 * (long long)nodes[k]);
      j->slot = -1;
      s->queue.push_front(std::move(j));
      ++s->evictions;
    }
    pos += (long long)nodes[k];
  }
  CK(cudaStreamSynchronize(c->stream));
  s->reorder = false;  // the staying jobs are in order already
  return set_top(s, after);
}

extern "C" int e13_serve_preempt(e13_serve *s, int64_t id) {
  if (!s) return E13_ERR_ARG;
  for (const auto &q : s->queue)
    if (q->id == id) return E13_OK;  // queued (or swapped out already): nothing to do
  int slot = -1;
  for (int k = 0; k < kMaxJobs; ++k)
    if (s->slot_job[k] && s->slot_job[k]->id == id) slot = k;
  if (slot < 0) return E13_ERR_ARG;  // unknown or finished
  e13_ctx *c = s->c;
  CK(cudaSetDevice(c->device));
  // node counts and counters as the last epoch left them (nothing ran since)
  const unsigned long long *cnt = c->h_jobbuf, *nodes = c->h_jobbuf + kMaxJobs * kJobCounters;
  int order[kMaxJobs], n = 0;
  unsigned long long accounted = 0;
  order[n++] = slot;
  for (int k = 0; k < kMaxJobs; ++k)
    if (k != slot && s->slot_job[k] && nodes[k] > 0) order[n++] = k;
  for (int i = 0; i < n; ++i) accounted += nodes[order[i]];
  if (accounted != (unsigned long long)c->ctl_host->top) return E13_ERR_ARG;
  std::sort(order + 1, order + n, [&](int a, int b) {
    if (nodes[a] != nodes[b]) return nodes[a] > nodes[b];
    return s->slot_job[a]->t_start < s->slot_job[b]->t_start;
  });
  return swap_out(s, order, n, 1, nodes, cnt, c->ctl_host->top - (long long)nodes[slot]);
}

extern "C" int e13_serve_step(e13_serve *s, e13_serve_result *done, int cap, int *ndone) {
  if (!s || !ndone || (cap > 0 && !done) || cap < kMaxJobs) return E13_ERR_ARG;
  *ndone = 0;
  e13_ctx *c = s->c;
  CK(cudaSetDevice(c->device));
  const double now = e13_serve_clock(s);
  CK(cudaEventRecord(c->k0, c->stream));
  long long launches = 0;
  // 0. the frontier in the order the last step chose (fewest live nodes on top)
  if (s->reorder && s->alt_cap >= c->stack_cap) {
    CK(h2d(c, s->d_fill, s->fill, sizeof s->fill));
    order_by_job<<<c->nsm * 4, 256, 0, c->stream>>>(c->ctl, c->stack, s->alt, s->d_fill, s->alt_cap);
    CK(cudaGetLastError());
    std::swap(c->stack, s->alt);
    s->P.stack = c->stack;
    ++launches;
  }
  s->reorder = false;
  // 1. admission, first come first served: a free slot, the job's arrival
  //    time passed, and room for every running job's reservation plus its own
  //    (a job alone is always admitted).  A swapped-out job comes back with its
  //    frontier nodes and counters.
  int running = 0;
  long long reserved = 0;
  for (int k = 0; k < kMaxJobs; ++k)
    if (s->slot_job[k]) {
      ++running;
      reserved += s->slot_job[k]->reserve;
    }
  long long top = c->ctl_host->top;
  bool pushed = false;
  while (!s->queue.empty() && s->queue.front()->t_submit <= now) {
    int slot = -1;
    for (int k = 0; k < kMaxJobs && slot < 0; ++k)
      if (!s->slot_job[k]) slot = k;
    if (slot < 0) break;
    ServeJob &q = *s->queue.front();
    const long long start_nodes = q.swapped ? (long long)q.saved.size() : 1;
    if (running > 0 && (reserved + q.reserve + s->out_nodes > s->cap || top + start_nodes + s->out_nodes > s->cap))
      break;
    if (top + start_nodes > s->cap) break;  // cannot happen when nothing runs (the frontier is empty then)
    std::unique_ptr<ServeJob> j = std::move(s->queue.front());
    s->queue.pop_front();
    j->slot = slot;
    if (j->t_start < 0) j->t_start = now;
    s->jp[slot].nv = 4 * j->job.nq;
    s->jp[slot].sym_lo = j->job.sym_lo;
    s->jp[slot].sym_hi = j->job.sym_hi;
    if (j->swapped) {
      for (Node &nd : j->saved) nd.job = (unsigned char)slot;
      if (!j->saved.empty()) CK(h2d(c, c->stack + top, j->saved.data(), sizeof(Node) * j->saved.size()));
      CK(h2d(c, c->d_jobcnt + (size_t)slot * kJobCounters, j->saved_cnt, sizeof j->saved_cnt));
      CK(cudaStreamSynchronize(c->stream));  // the host buffer goes away next
      top += (long long)j->saved.size();
      std::vector<Node>().swap(j->saved);
      j->swapped = false;
    } else {
      Node root;
      build_root(&j->job, slot, &root, s->tu.run_skip != 0, true);
      CK(h2d(c, c->stack + top, &root, sizeof root));
      CK(cudaStreamSynchronize(c->stream));
      CK(cudaMemsetAsync(c->d_jobcnt + (size_t)slot * kJobCounters, 0, sizeof(unsigned long long) * kJobCounters,
                         c->stream));
      top += 1;
    }
    reserved += j->reserve;
    s->slot_job[slot] = std::move(j);
    ++running;
    pushed = true;
  }
  if (pushed) {
    int rc;
    if ((rc = set_top(s, top))) return rc;
    CK(h2d(c, c->d_jobs, s->jp, sizeof s->jp));
  }
  if (running == 0) return E13_OK;
  // 2. one epoch of the persistent kernel, then the live nodes of every job
  launches += 4;
  search_kernel<true><<<c->nsm, s->tu.block, s->smem, c->stream>>>(s->P);
  move_outputs<<<c->nsm * 4, 256, 0, c->stream>>>(c->ctl, c->stack, c->out, c->pool, c->pool_cap, s->cap);
  finish_launch<<<1, 1, 0, c->stream>>>(c->ctl, s->cap, s->batch_max, c->pool_cap);
  CK(cudaMemsetAsync(c->d_jobnodes, 0, sizeof(unsigned long long) * kMaxJobs, c->stream));
  count_job_nodes<<<c->nsm * 2, 256, 0, c->stream>>>(c->ctl, c->stack, c->d_jobnodes);
  CK(cudaGetLastError());
  CK(cudaEventRecord(c->k1, c->stream));
  CK(d2h(c, c->ctl_host, c->ctl, sizeof(Ctl)));
  CK(d2h(c, c->h_jobbuf, c->d_jobcnt, sizeof(unsigned long long) * kMaxJobs * kJobCounters));
  CK(d2h(c, c->h_jobbuf + kMaxJobs * kJobCounters, c->d_jobnodes, sizeof(unsigned long long) * kMaxJobs));
  CK(cudaStreamSynchronize(c->stream));
  float ms = 0;
  cudaEventElapsedTime(&ms, c->k0, c->k1);
  s->device_ms += ms;
  s->epochs += 1;
  c->stats.device_ms += ms;
  c->stats.launches += launches;
  c->stats.search_kernel_launches += 1;
  c->stats.epochs += 1;
  // 3. survivors found in this epoch go to their jobs
  const unsigned long long ns = c->ctl_host->nsurv;
  const unsigned long long avail = std::min<unsigned long long>(ns, (unsigned long long)c->surv_cap);
  if (ns > (unsigned long long)c->surv_cap) s->surv_overflow = true;
  if (avail > s->surv_fetched) {
    std::vector<SurvRec> recs((size_t)(avail - s->surv_fetched));
    CK(d2h(c, recs.data(), c->surv + s->surv_fetched, sizeof(SurvRec) * recs.size()));
    CK(cudaStreamSynchronize(c->stream));
    for (const SurvRec &r : recs) {
      ServeJob *j = (r.job >= 0 && r.job < kMaxJobs) ? s->slot_job[r.job].get() : nullptr;
      if (!j) continue;
      e13_survivor sv;
      decode_survivor(r, j->job.nq, &sv);
      j->surv.push_back(sv);
    }
    s->surv_fetched = avail;
  }
  // 4. jobs with no node left are done
  const double tdone = e13_serve_clock(s);
  const unsigned long long *cnt = c->h_jobbuf, *nodes = c->h_jobbuf + kMaxJobs * kJobCounters;
  s->peak_top = std::max<long long>(s->peak_top, c->ctl_host->top);
  for (int k = 0; k < kMaxJobs; ++k)
    if (s->slot_job[k]) s->peak_job = std::max<long long>(s->peak_job, (long long)nodes[k]);
  if (c->ctl_host->error) {
    // a device wait ran out or an epoch's outputs did not fit: finish_launch
    // dropped the frontier, so every running job ends with that status and
    // the partial counts it had; queued jobs run on a cleared control block
    const int st = (c->ctl_host->error & kErrTimeout) ? E13_ERR_TIMEOUT : E13_ERR_OVERFLOW;
    for (int k = 0; k < kMaxJobs; ++k) {
      if (!s->slot_job[k]) continue;
      ServeJob &j = *s->slot_job[k];
      fill_result(done[(*ndone)++], j, cnt + k * kJobCounters, st, tdone);
      s->finished_surv[j.id] = std::move(j.surv);
      s->slot_job[k].reset();
    }
    const int launches_so_far = c->ctl_host->launches;  // pool-slot tags must keep rising
    memset(c->ctl_host, 0, sizeof(Ctl));
    c->ctl_host->launches = launches_so_far;
    CK(h2d(c, c->ctl, c->ctl_host, sizeof(Ctl)));
    CK(cudaStreamSynchronize(c->stream));
    s->surv_fetched = 0;
    s->surv_overflow = false;
    s->reorder = false;
    return E13_OK;
  }
  for (int k = 0; k < kMaxJobs; ++k) {
    if (!s->slot_job[k] || nodes[k] != 0) continue;
    ServeJob &j = *s->slot_job[k];
    fill_result(done[(*ndone)++], j, cnt + k * kJobCounters, s->surv_overflow ? E13_ERR_SURV_CAP : E13_OK, tdone);
    s->finished_surv[j.id] = std::move(j.surv);
    s->slot_job[k].reset();
  }
  // 5. the order of the frontier for the next epoch, which takes its input
  //    from the top: the job with the most live nodes at the bottom, the one
  //    with the fewest on top (nearly finished jobs finish first); on a tie the
  //    job started later goes higher.  Only when every node is accounted for.
  int order[kMaxJobs], n = 0;
  unsigned long long accounted = 0;
  for (int k = 0; k < kMaxJobs; ++k)
    if (s->slot_job[k] && nodes[k] > 0) {
      order[n++] = k;
      accounted += nodes[k];
    }
  std::sort(order, order + n, [&](int a, int b) {
    if (nodes[a] != nodes[b]) return nodes[a] > nodes[b];
    return s->slot_job[a]->t_start < s->slot_job[b]->t_start;
  });
  const bool complete = accounted == (unsigned long long)c->ctl_host->top;
  // 6. too little room for the next epoch's outputs: swap jobs out, the one
  //    with the most live nodes first, until the rest fits.  A swapped-out
  //    job's frontier nodes and counters go to host memory and it goes back to
  //    the head of the queue; re-admitted, it goes on where it stopped (its
  //    counts stay exact).  A job that does not fit alone fails with
  //    E13_ERR_OVERFLOW.
  const long long cur_top = c->ctl_host->top;
  if (complete && n > 0 && cur_top + s->out_nodes > s->cap) {
    int first = 0;  // order[0..first) leave the frontier, order[first..n) stay
    long long after = cur_top;
    while (n - first > 1 && after + s->out_nodes > s->cap) after -= (long long)nodes[order[first++]];
    if (after + s->out_nodes > s->cap) {
      // one job left and it alone does not fit: it fails, its nodes are dropped
      const int k = order[first++];
      ServeJob &j = *s->slot_job[k];
      fill_result(done[(*ndone)++], j, cnt + k * kJobCounters, E13_ERR_OVERFLOW, tdone);
      s->finished_surv[j.id] = std::move(j.surv);
      s->slot_job[k].reset();
      after -= (long long)nodes[k];
    }
    int rc;
    if ((rc = swap_out(s, order, n, first, nodes, cnt, after))) return rc;
    n = 0;  // the frontier is in order already
  }
  if (n > 1 && complete) s->reorder = true;
  if (s->reorder) {
    unsigned long long off = 0;
    memset(s->fill, 0, sizeof s->fill);
    for (int i = 0; i < n; ++i) {
      s->fill[order[i]] = off;
      off += nodes[order[i]];
    }
  }
  // 7. idle: start the survivor buffer over
  if (e13_serve_pending(s) == 0) {
    unsigned long long zero = 0;
    CK(h2d(c, &c->ctl->nsurv, &zero, sizeof zero));
    CK(cudaStreamSynchronize(c->stream));
    s->surv_fetched = 0;
    s->surv_overflow = false;
    c->ctl_host->nsurv = 0;
  }
  return E13_OK;
}

extern "C" int e13_serve_survivors(e13_serve *s, int64_t id, e13_survivor *out, int cap, int *n) {
  if (!s || !n || (cap > 0 && !out)) return E13_ERR_ARG;
  auto it = s->finished_surv.find(id);
  if (it == s->finished_surv.end()) return E13_ERR_ARG;
  const int k = (int)std::min<size_t>(it->second.size(), (size_t)std::max(cap, 0));
  for (int i = 0; i < k; ++i) out[i] = it->second[(size_t)i];
  *n = (int)it->second.size();
  const int rc = (size_t)k < it->second.size() ? E13_ERR_SURV_CAP : E13_OK;
  s->finished_surv.erase(it);
  return rc;
}

extern "C" int e13_serve_stats(const e13_serve *s, double *device_ms, int64_t *epochs, int64_t *swapped_out,
                               int64_t *peak_nodes, int64_t *peak_job_nodes) {
  if (!s) return E13_ERR_ARG;
  if (device_ms) *device_ms = s->device_ms;
  if (epochs) *epochs = s->epochs;
  if (swapped_out) *swapped_out = s->evictions;
  if (peak_nodes) *peak_nodes = s->peak_top;
  if (peak_job_nodes) *peak_job_nodes = s->peak_job;
  return E13_OK;
}
