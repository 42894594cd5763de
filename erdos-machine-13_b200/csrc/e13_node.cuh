// e13_node.cuh -- a machine as a frontier node: moving it between a lane
// (registers + its shared-memory tape and table columns) and a Node, applying
// a child at its pending cell, the root node of a job, and the upload of the
// filter's constant tables.  Shared by the search kernels and the estimator.
#pragma once
#include <cuda_runtime.h>
#include <string.h>

#include "e13.h"
#include "e13_device.cuh"

namespace e13dev {

__device__ __forceinline__ void lane_load(Lane &L, const Node *N, u32 *tcol, u32 *rcol, int stride, int nq) {
  // the words the previous machine of this lane may have written
  int lo_old, hi_old;
  tape_extent(L.t, lo_old, hi_old);
  L.p = N->p;
  L.st = N->st;
  L.t = N->t;
  L.deadline = N->deadline;
  L.hb = (u32)N->hb;
  L.nt = N->nt;
  L.stage = N->stage;
  L.st0 = N->st0;
  L.p0 = N->p0;
  L.flags = N->flags & 31;
  L.ch0 = N->ch[0];
  L.ch1 = N->ch[1];
  L.ch2 = N->ch[2];
  L.nintro = N->nintro;
  L.budget = N->budget;
  L.job = N->job;
  L.tgt = (u32)s_tgt[L.nt];
  L.tseg = L.t;
  const uint4 *rv = reinterpret_cast<const uint4 *>(N->cellv);
  for (int k = 0; k < 4; ++k) {  // all 16 rows: states >= nq hold halts
    const uint4 v = rv[k];
    rcol[(4 * k) * stride] = v.x;
    rcol[(4 * k + 1) * stride] = v.y;
    rcol[(4 * k + 2) * stride] = v.z;
    rcol[(4 * k + 3) * stride] = v.w;
  }
  // one pass over both extents: the new machine's words are copied, the old
  // machine's other words cleared (siblings of one fork share most words)
  int lo, hi;
  tape_extent(L.t, lo, hi);
  const int a = lo < lo_old ? lo : lo_old, b = hi > hi_old ? hi : hi_old;
  for (int w = a; w <= b; ++w) tcol[w * stride] = (w >= lo && w <= hi) ? N->tape[w] : 0u;
}

__device__ __forceinline__ void lane_store(const Lane &L, Node *N, const u32 *tcol, const u32 *rcol, int stride,
                                           int nq, int pend, int keep, u64 vm) {
  N->hb = L.hb;
  N->ch[0] = L.ch0;
  N->ch[1] = L.ch1;
  N->ch[2] = L.ch2;
  N->vmask = vm;
  N->p = L.p;
  N->st = L.st;
  N->t = L.t;
  N->deadline = L.deadline;
  N->nt = (signed char)L.nt;
  N->stage = (signed char)L.stage;
  N->st0 = (signed char)L.st0;
  N->flags = (signed char)(L.flags | (keep ? kFlagKeep : 0));
  N->p0 = (short)L.p0;
  N->pend = (short)pend;
  N->nintro = (unsigned char)L.nintro;
  N->budget = (unsigned char)L.budget;
  N->job = (unsigned char)L.job;
  uint4 *rv = reinterpret_cast<uint4 *>(N->cellv);
  for (int k = 0; k < 4; ++k)
    rv[k] = make_uint4(rcol[(4 * k) * stride], rcol[(4 * k + 1) * stride], rcol[(4 * k + 2) * stride],
                       rcol[(4 * k + 3) * stride]);
  int lo, hi;
  tape_extent(L.t, lo, hi);
  for (int w = lo; w <= hi; ++w) N->tape[w] = tcol[w * stride];
}

// Applies child `ch` (-1: keep / go on, else move v) of node N to a lane that
// has just loaded N.
// clear: on the move that spends the last of the budget, clear the unread
// flags that can no longer fork (clear_unread; the search, not the estimator,
// which counts every first read as a fork).
__device__ __forceinline__ void apply_child(Lane &L, const Node *N, int ch, u32 *rcol, int stride, int sym_lo,
                                            int sym_hi, bool run_skip, bool clear = false) {
  const int pend = N->pend;
  if (pend < 0) return;
  const u32 e = N->cellv[pend] & 0xFFu;
  if (ch < 0) {
    set_entry(rcol, stride, pend, e & 0x7Fu, run_skip);  // the table's own move (or halt), now read
  } else {
    if (e != kEntFree) {
      L.budget -= 1;
      if (clear && L.budget == 0) clear_unread(rcol, stride);
    }
    L.nintro = sym_after(ch, L.nintro, sym_lo, sym_hi);
    set_entry(rcol, stride, pend, (u32)ch, run_skip);
  }
}

// ------------------------------------------------------------------------
// host side

// The root of a job: blank tape, every cell unread (free cells: kEntFree).  An
// unread move carries its self-loop bit (when run_skip is on) for the moment
// its flag is cleared.  clear: a job with no budget starts with the flags of
// its moves cleared (clear_unread).
static inline void build_root(const e13_job *job, int slot, Node *root, bool run_skip = false, bool clear = false) {
  memset(root, 0, sizeof *root);
  root->job = (unsigned char)slot;
  root->p = kLeft;
  root->deadline = 4 * 2 + 64;
  root->nt = 1;
  root->st0 = -1;
  root->p0 = kLeft;  // head0 = 0 until stage 1 sets it (src/e13search.c:123-129)
  root->flags = (signed char)(kFlagAbs | kFlagRel | kFlagKeep);
  root->pend = -1;
  root->nintro = (unsigned char)(job->sym_n0 < 0 ? 0 : job->sym_n0);
  root->budget = (unsigned char)(job->budget < 0 ? 0 : job->budget);
  for (int i = 0; i < 32; ++i) {
    unsigned char e = (unsigned char)kEntHalt;
    if (i < 2 * job->nq) {
      const int c = job->tab[i];
      if (c == E13_FREE) e = (unsigned char)kEntFree;
      else if (c < 0) e = (unsigned char)(kEntUnread | kEntHalt);
      else e = (unsigned char)(((clear && job->budget <= 0) ? 0u : kEntUnread) | (unsigned)c);
    }
    root->cellv[i] = (unsigned short)(e < 64u || (e & 0xC0u) == kEntUnread ? cell_slot(i, e & 0x3Fu, run_skip) | (e & kEntUnread) : e);
  }
}

// Uploads KEY, TGT, the stage deadlines 4 * T14S[n] + 64 and the exception
// counts (src/e13search.c:58-75, :437-444) into this translation unit's
// constant tables on the current device.  Every .cu file that runs the filter
// has its own copy of those tables, so this function is static: one shared
// (inline) copy would fill only one file's tables.
static inline cudaError_t upload_filter_tables() {
  uint64_t key[kTapeCells], tgt[E13_STAGES + 1];
  e13_keys(key, tgt);
  static const long erdos14_stage_step[E13_STAGES + 1] = {0, 2, 22, 90, 268, 944, 3434, 13450, 52068, 208864};
  static const int exc[E13_STAGES + 1] = {0, 0, 0, 1, 1, 1, 1, 1, 1, 2};
  u64 t11[E13_STAGES + 2] = {0};
  int dl[E13_STAGES + 2] = {0};
  for (int n = 0; n <= E13_STAGES; ++n) {
    t11[n] = tgt[n];
    dl[n] = (int)(4 * erdos14_stage_step[n] + 64);
  }
  t11[0] = ~0ull;  // never a target
  cudaError_t e;
  if ((e = cudaMemcpyToSymbol(c_key, key, sizeof key)) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_tgt, t11, sizeof t11)) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_deadline, dl, sizeof dl)) != cudaSuccess) return e;
  return cudaMemcpyToSymbol(c_exc, exc, sizeof exc);
}

}  // namespace e13dev
