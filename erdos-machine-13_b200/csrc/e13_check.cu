// e13_check.cu -- hash-free deep check of survivors on the device.
//
// Re-runs each machine from the blank tape to stage nmax and records, at every
// stage start, the exact set of ones left of cell -2 (the counter).  Stage
// starts are found without hashing, as src/recheck.c:61-92 does: state st0,
// head at head0 (abs) or head0 + 2^n - 2 (rel), and the ones at cells >= -2
// exactly the block -1 .. 2^n - 2.  Two variants:
//   E13_CHECK_RECHECK  recheck.c: limit t + 8*4^n + 1e5, tape +-4,000,000,
//                      stops at the first counter change (src/recheck.c:63-91)
//   E13_CHECK_DEEP     deep.c: limit t + 64*4^n + 1e5, tape -4096 .. 2^nmax+4096,
//                      off tape below -4094 or past 2^n + 2000 (src/deep.c:56-64)
//
// One machine per lane.  The tape is bit-packed; cells -4096 .. 2^nmax + 4096
// (all of deep's tape, the busy part of recheck's) sit in a shared-memory
// window interleaved by lane, the rest of recheck's +-4M cells in HBM.  The
// word under the head stays in a register; runs of a self-loop are crossed a
// word at a time.
#include <cuda_runtime.h>

#include <mutex>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "e13.h"

namespace {

typedef unsigned int u32;
typedef long long i64;

constexpr i64 kWinLeft = 4096;        // the shared-memory window starts at cell -4096
constexpr i64 kRecheckSide = 4000000;  // recheck's tape: cells -4e6 .. 4e6 (src/recheck.c:16-17)
constexpr int kSmemBudget = 200 * 1024;

struct CheckParams {
  int n, nmax, deep;
  int W;          // window words per lane: cells -4096 .. -4096 + 32W - 1
  i64 gwords;     // recheck: global tape words per machine (cells -4e6 .. 4e6)
  i64 gshift;     // global word index of window word 0
  u32 *gtapes;
  const e13_check_in *in;
  e13_check_out *out;
};

__device__ __forceinline__ int first_of_class(int n) { return n <= 2 ? 1 : (n <= 8 ? 3 : 9); }

// A lane's tape: a window of W words in shared memory (interleaved by lane,
// so a warp never has bank conflicts), the rest in HBM (recheck only).
struct Tape {
  u32 *win;
  int nl, W;
  u32 *g;
  i64 gshift;
  __device__ __forceinline__ bool in_win(i64 ww) const { return ww >= 0 && ww < W; }
  __device__ __forceinline__ u32 ld(i64 ww) const { return in_win(ww) ? win[ww * nl] : g[ww + gshift]; }
  __device__ __forceinline__ void st(i64 ww, u32 v) const {
    if (in_win(ww)) win[ww * nl] = v;
    else g[ww + gshift] = v;
  }
};

__global__ void __launch_bounds__(32) check_kernel(const CheckParams P) {
  extern __shared__ __align__(16) u32 s_win[];
  __shared__ unsigned short s_rows[16 * 32];
  const int nl = blockDim.x;
  const int m = blockIdx.x * nl + threadIdx.x;
  Tape tp;
  tp.win = s_win + threadIdx.x;
  tp.nl = nl;
  tp.W = P.W;
  tp.g = P.deep ? nullptr : P.gtapes + (i64)(m < P.n ? m : 0) * P.gwords;
  tp.gshift = P.gshift;
  if (m >= P.n) return;
  for (int w = 0; w < P.W; ++w) tp.win[w * nl] = 0;
  const e13_check_in &in = P.in[m];
  e13_check_out &o = P.out[m];
  unsigned short *rows = s_rows + threadIdx.x;  // row s at rows[s * 32]: two 8-bit cells
  // cell entry: bit 0 write, bit 1 right, bits 2..5 next, bit 6 self-loop, bit 7 not a move
  for (int s = 0; s < 16; ++s) {
    unsigned short r = 0;
    for (int a = 0; a < 2; ++a) {
      const int i = 2 * s + a;
      unsigned e = 0x80u;
      if (s < in.nq && in.kind[i] == 0) {
        e = (unsigned)(in.write[i] & 1) | (in.move[i] > 0 ? 2u : 0u) | ((unsigned)(in.next[i] & 15) << 2);
        if (in.next[i] == s && in.write[i] == a) e |= 0x40u;  // reads a, writes a, stays: sweeps a run of a
      }
      r |= (unsigned short)(e << (8 * a));
    }
    rows[s * 32] = r;
  }
  const bool deep = P.deep != 0;

  o.status = E13_CHK_OK;
  o.fail_stage = 0;
  o.stages_done = 0;
  o.fail_t = 0;
  o.fail_head = 0;
  i64 head = 0, t = 0, minhead = 0, ones = 0;
  int st = 0;
  i64 ww = kWinLeft >> 5;  // word of cell 0
  int bit = 0;
  u32 word = tp.ld(ww);
  const int st0 = in.st0;
  const i64 head0 = in.head0;
  const int rel = in.rel;

  for (int n = 1; n <= P.nmax; ++n) {
    const i64 blk = 1LL << n;
    const i64 limit = t + (deep ? 64LL : 8LL) * (1LL << (2 * n)) + 100000;
    const i64 want = rel ? head0 + blk - 2 : head0;
    int fail = 0;
    for (;;) {
      if (st == st0 && head == want && ones == blk) {
        // all of -1 .. blk-2 set?  (the cached word goes back first)
        tp.st(ww, word);
        bool ok = true;
        for (i64 c = -1; c < blk - 1 && ok;) {
          const i64 b = c + kWinLeft;
          const int sh = (int)(b & 31);
          const int take = (int)min((i64)(32 - sh), blk - 1 - c);
          const u32 mask = take == 32 ? 0xFFFFFFFFu : (((1u << take) - 1u) << sh);
          if ((tp.ld(b >> 5) & mask) != mask) ok = false;
          c += take;
        }
        if (ok) break;
      }
      if (t >= limit) { fail = E13_CHK_LIMIT; break; }
      if (deep ? (head < -4096 + 2 || head > blk + 2000) : (head <= -kRecheckSide + 2 || head >= kRecheckSide - 2)) {
        fail = E13_CHK_OFFTAPE;
        break;
      }
      const u32 s = (word >> bit) & 1u;
      const unsigned e = (rows[st * 32] >> (8 * s)) & 0xFFu;
      if (e & 0x80u) {
        const int i = 2 * st + (int)s;
        fail = in.kind[i] == 2 ? E13_CHK_FREE_READ : E13_CHK_HALT;
        o.free_state = st;
        o.free_sym = (int)s;
        break;
      }
      const bool right = (e & 2u) != 0;
      if (e & 0x40u) {
        // Run skip: the next k steps read s, write nothing, keep the state and
        // the ones count.  k stops before the step limit, before the tape ends,
        // at the window edge, and at `want` when a stage start could happen
        // there, so every test the single-step loop makes is still made.
        i64 lim = limit - t;
        if (deep) lim = min(lim, right ? blk + 2001 - head : head + 4095);
        else lim = min(lim, right ? kRecheckSide - 2 - head : head + kRecheckSide - 2);
        if (st == st0 && ones == blk) {
          const i64 dd = right ? want - head : head - want;
          if (dd > 0) lim = min(lim, dd);
        }
        if (lim > 1 && tp.in_win(ww)) {
          const u32 flip = s ? 0xFFFFFFFFu : 0u;
          i64 k = 0;
          i64 w = ww;
          if (right) {
            u32 x = (word ^ flip) >> bit;
            int b0 = bit;
            for (;;) {
              k += x ? (__ffs(x) - 1) : (32 - b0);
              if (x || k >= lim || !tp.in_win(w + 1)) break;
              ++w;
              b0 = 0;
              x = tp.ld(w) ^ flip;
            }
          } else {
            u32 x = (word ^ flip) << (31 - bit);
            int b0 = bit;
            for (;;) {
              k += x ? __clz(x) : (b0 + 1);
              if (x || k >= lim || !tp.in_win(w - 1)) break;
              --w;
              b0 = 31;
              x = tp.ld(w) ^ flip;
            }
          }
          if (k > lim) k = lim;
          if (k > 1) {
            const i64 pos = (i64)bit + (right ? k : -k);
            head += right ? k : -k;
            t += k;
            if (pos < 0 || pos > 31) {
              tp.st(ww, word);
              ww += pos >> 5;  // arithmetic shift: floor division by 32
              word = tp.ld(ww);
            }
            bit = (int)(pos & 31);
            if (head < minhead) minhead = head;
            continue;
          }
        }
      }
      const u32 wr = e & 1u;
      if (wr != s) {
        word ^= 1u << bit;
        if (head >= -2) ones += wr ? 1 : -1;
      }
      if (right) {
        ++head;
        if (++bit == 32) {
          tp.st(ww, word);
          word = tp.ld(++ww);
          bit = 0;
        }
      } else {
        --head;
        if (--bit < 0) {
          tp.st(ww, word);
          word = tp.ld(--ww);
          bit = 31;
        }
        if (head < minhead) minhead = head;
      }
      st = (int)((e >> 2) & 15u);
      ++t;
    }
    if (fail) {
      o.status = fail;
      o.fail_stage = n;
      o.fail_t = t;
      o.fail_head = head;
      return;
    }
    // stage start n: record the counter (all ones at cells <= -3)
    tp.st(ww, word);
    o.stages_done = n;
    if (n <= E13_CHECK_MAX_NMAX) {
      o.stage_t[n] = t;
      o.minhead[n] = minhead;
      int cnt = 0;
      i64 leftmost = 0;
      const i64 lowest = deep ? -4096 + 1 : minhead - 1;
      for (i64 c = -3; c >= lowest;) {
        const i64 b = c + kWinLeft;
        const int sh = (int)(b & 31);
        // bits sh down to 0 of this word hold cells c .. c - sh
        u32 x = tp.ld(b >> 5) & (sh == 31 ? 0xFFFFFFFFu : ((2u << sh) - 1u));
        const i64 wlow = c - sh;  // cell of bit 0
        while (x) {
          const int hb = 31 - __clz(x);
          const i64 cell = wlow + hb;
          if (cell < lowest) break;
          if (cnt < E13_CHECK_MAX_ONES) o.ones_cells[n][cnt] = (int)cell;
          ++cnt;
          leftmost = cell;
          x &= ~(1u << hb);
        }
        c = wlow - 1;
      }
      o.nones[n] = cnt;
      o.leftmost[n] = leftmost;
      if (!deep) {
        const int f = first_of_class(n);
        if (n != f) {
          bool same = o.nones[n] == o.nones[f];
          const int k = min(cnt, E13_CHECK_MAX_ONES);
          for (int j = 0; j < k && same; ++j) same = o.ones_cells[n][j] == o.ones_cells[f][j];
          if (!same) return;  // recheck stops at the first counter change
        }
      }
    }
  }
}

}  // namespace

struct e13_ctx;
extern "C" int e13_ctx_device(const e13_ctx *c);

extern "C" int e13_check(e13_ctx *ctx, const e13_check_in *in, int n, int nmax, int mode, e13_check_out *out) {
  if (!ctx || (n > 0 && (!in || !out)) || n < 0 || nmax < 1 || nmax > E13_CHECK_MAX_NMAX ||
      (mode != E13_CHECK_RECHECK && mode != E13_CHECK_DEEP))
    return E13_ERR_ARG;
  if (n == 0) return E13_OK;
  if (cudaSetDevice(e13_ctx_device(ctx)) != cudaSuccess) return E13_ERR_CUDA;
  const bool deep = mode == E13_CHECK_DEEP;
  // window: cells -4096 .. 2^nmax + 4096 (deep's whole tape; recheck's busy part)
  const int W = (int)((kWinLeft + (1LL << nmax) + 4096 + 31) / 32 + 2);
  int nl = (int)std::min<i64>(32, kSmemBudget / ((i64)W * 4));
  if (nl < 1) return E13_ERR_ARG;
  const size_t smem = (size_t)W * nl * 4;
  const i64 gwords = deep ? 0 : (2 * kRecheckSide + 1 + 31) / 32 + 2;
  const int chunk = deep ? n : (int)std::min<i64>(n, std::max<i64>(1, (4LL << 30) / (gwords * 4)));
  u32 *d_tapes = nullptr;
  e13_check_in *d_in = nullptr;
  e13_check_out *d_out = nullptr;
  int rc = E13_OK;
  if ((!deep && cudaMalloc(&d_tapes, (size_t)chunk * gwords * 4) != cudaSuccess) ||
      cudaMalloc(&d_in, sizeof(e13_check_in) * (size_t)chunk) != cudaSuccess ||
      cudaMalloc(&d_out, sizeof(e13_check_out) * (size_t)chunk) != cudaSuccess) {
    rc = E13_ERR_CUDA;
  }
  if (!rc && cudaFuncSetAttribute(check_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    rc = E13_ERR_CUDA;
  for (int b = 0; b < n && rc == E13_OK; b += chunk) {
    const int k = std::min(chunk, n - b);
    CheckParams P;
    P.n = k;
    P.nmax = nmax;
    P.deep = deep ? 1 : 0;
    P.W = W;
    P.gwords = gwords;
    P.gshift = (kRecheckSide - kWinLeft) / 32;
    P.gtapes = d_tapes;
    P.in = d_in;
    P.out = d_out;
    if ((!deep && cudaMemset(d_tapes, 0, (size_t)k * gwords * 4) != cudaSuccess) ||
        cudaMemset(d_out, 0, sizeof(e13_check_out) * (size_t)k) != cudaSuccess ||
        cudaMemcpy(d_in, in + b, sizeof(e13_check_in) * (size_t)k, cudaMemcpyHostToDevice) != cudaSuccess) {
      rc = E13_ERR_CUDA;
      break;
    }
    check_kernel<<<(k + nl - 1) / nl, nl, smem>>>(P);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(out + b, d_out, sizeof(e13_check_out) * (size_t)k, cudaMemcpyDeviceToHost) != cudaSuccess) {
      rc = E13_ERR_CUDA;
      break;
    }
  }
  cudaFree(d_tapes);
  cudaFree(d_in);
  cudaFree(d_out);
  return rc;
}

// ------------------------------------------------------------------------
// The same check for callers that cannot allocate device memory.
//
// All device memory this entry point uses is fixed at load time: the tapes,
// inputs and outputs of up to E13_CHECK_NOALLOC_MAX machines sit in the
// file-scope arrays below (about 16 MB; every GPU that loads the library keeps
// them until the process exits).  Host code cannot use these names as device
// addresses, so the first call on each device looks the addresses up with
// cudaGetSymbolAddress while that device is current and keeps them.

namespace {

constexpr i64 kNoAllocWords = (2 * kRecheckSide + 1 + 31) / 32 + 2;  // one recheck tape (cells -4e6 .. 4e6)

static __device__ __align__(256) u32 g_noalloc_tapes[E13_CHECK_NOALLOC_MAX * kNoAllocWords];
static __device__ __align__(256) e13_check_in g_noalloc_in[E13_CHECK_NOALLOC_MAX];
static __device__ __align__(256) e13_check_out g_noalloc_out[E13_CHECK_NOALLOC_MAX];

constexpr int kNoAllocMaxDevices = 64;
// Per device, filled once under std::call_once: the arrays' device addresses
// and a non-blocking stream of this entry point's own, so a call waits for its
// own work only (not for other streams of the device, and not for a capture
// another thread holds on the legacy default stream).
struct NoAllocDevice {
  std::once_flag once;
  int rc;
  u32 *tapes;
  e13_check_in *in;
  e13_check_out *out;
  cudaStream_t stream;
};
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];

// With `device` current.
int noalloc_device(int device, NoAllocDevice **out) {
  if (device < 0 || device >= kNoAllocMaxDevices) return E13_ERR_ARG;
  NoAllocDevice &d = g_noalloc_dev[device];
  std::call_once(d.once, [&d]() {
    d.rc = E13_OK;
    if (cudaGetSymbolAddress((void **)&d.tapes, g_noalloc_tapes) != cudaSuccess ||
        cudaGetSymbolAddress((void **)&d.in, g_noalloc_in) != cudaSuccess ||
        cudaGetSymbolAddress((void **)&d.out, g_noalloc_out) != cudaSuccess ||
        cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking) != cudaSuccess)
      d.rc = E13_ERR_CUDA;
  });
  *out = &d;
  return d.rc;
}

}  // namespace

extern "C" int e13_check_noalloc(int device, const e13_check_in *in, int n, int nmax, int mode, e13_check_out *out) {
  if ((n > 0 && (!in || !out)) || n < 0 || nmax < 1 || nmax > E13_CHECK_MAX_NMAX ||
      (mode != E13_CHECK_RECHECK && mode != E13_CHECK_DEEP))
    return E13_ERR_ARG;
  if (n > E13_CHECK_NOALLOC_MAX) return E13_ERR_NOALLOC_SIZE;
  if (n == 0) return E13_OK;
  if (cudaSetDevice(device) != cudaSuccess) return E13_ERR_CUDA;
  NoAllocDevice *a = nullptr;
  int rc = noalloc_device(device, &a);
  if (rc) return rc;
  const cudaStream_t st = a->stream;
  const bool deep = mode == E13_CHECK_DEEP;
  const int W = (int)((kWinLeft + (1LL << nmax) + 4096 + 31) / 32 + 2);
  const int nl = (int)std::min<i64>(32, kSmemBudget / ((i64)W * 4));
  if (nl < 1) return E13_ERR_NOALLOC_SIZE;
  const size_t smem = (size_t)W * nl * 4;
  if (cudaFuncSetAttribute(check_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return E13_ERR_CUDA;
  // the arrays keep the previous call's contents: clear the tapes and outputs
  if ((!deep && cudaMemsetAsync(a->tapes, 0, sizeof(u32) * (size_t)n * kNoAllocWords, st) != cudaSuccess) ||
      cudaMemsetAsync(a->out, 0, sizeof(e13_check_out) * (size_t)n, st) != cudaSuccess ||
      cudaMemcpyAsync(a->in, in, sizeof(e13_check_in) * (size_t)n, cudaMemcpyHostToDevice, st) != cudaSuccess)
    return E13_ERR_CUDA;
  CheckParams P;
  P.n = n;
  P.nmax = nmax;
  P.deep = deep ? 1 : 0;
  P.W = W;
  P.gwords = deep ? 0 : kNoAllocWords;
  P.gshift = (kRecheckSide - kWinLeft) / 32;
  P.gtapes = a->tapes;
  P.in = a->in;
  P.out = a->out;
  check_kernel<<<(n + nl - 1) / nl, nl, smem, st>>>(P);
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(out, a->out, sizeof(e13_check_out) * (size_t)n, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return E13_ERR_CUDA;
  return E13_OK;
}
