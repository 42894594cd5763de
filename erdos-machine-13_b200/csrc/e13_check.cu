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
// One machine per lane.  The tape is bit-packed in global memory (one region
// per machine); the word under the head stays in a register and goes back to
// memory only when the head leaves it.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "e13.h"

namespace {

typedef unsigned int u32;
typedef long long i64;

struct CheckParams {
  int n, nmax, mode;
  i64 side_left;    // cells left of 0 in the tape region
  i64 words;        // tape words per machine
  u32 *tapes;
  const e13_check_in *in;
  e13_check_out *out;
};

__device__ __forceinline__ int first_of_class(int n) { return n <= 2 ? 1 : (n <= 8 ? 3 : 9); }

constexpr int kCheckBlock = 32;  // one warp per block: the lanes are latency-bound, so spread them over SMs

__global__ void __launch_bounds__(kCheckBlock) check_kernel(const CheckParams P) {
  __shared__ unsigned short s_rows[16 * kCheckBlock];
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= P.n) return;
  const e13_check_in &in = P.in[m];
  e13_check_out &o = P.out[m];
  unsigned short *rows = s_rows + threadIdx.x;  // row s at rows[s * kCheckBlock]: two 8-bit cells
  // cell entry: bit 0 write, bit 1 right, bits 2..6 next, bit 7 special (kind != move)
  for (int s = 0; s < 16; ++s) {
    unsigned short r = 0;
    for (int a = 0; a < 2; ++a) {
      const int i = 2 * s + a;
      unsigned e = 0x80u;
      if (s < in.nq && in.kind[i] == 0)
        e = (unsigned)(in.write[i] & 1) | (in.move[i] > 0 ? 2u : 0u) | ((unsigned)(in.next[i] & 31) << 2);
      r |= (unsigned short)(e << (8 * a));
    }
    rows[s * kCheckBlock] = r;
  }
  u32 *tape = P.tapes + (i64)m * P.words;
  const bool deep = P.mode == E13_CHECK_DEEP;
  const i64 off = P.side_left;  // cell c is bit (c + off)

  o.status = E13_CHK_OK;
  o.fail_stage = 0;
  o.stages_done = 0;
  o.fail_t = 0;
  o.fail_head = 0;
  i64 head = 0, t = 0, minhead = 0, ones = 0;
  int st = 0;
  i64 pos = head + off;
  i64 wi = pos >> 5;
  int bit = (int)(pos & 31);
  u32 word = tape[wi];
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
        tape[wi] = word;
        bool ok = true;
        for (i64 c = -1; c < blk - 1 && ok;) {
          const i64 b = c + off;
          const int sh = (int)(b & 31);
          const int take = (int)min((i64)(32 - sh), blk - 1 - c);
          const u32 mask = take == 32 ? 0xFFFFFFFFu : (((1u << take) - 1u) << sh);
          if ((tape[b >> 5] & mask) != mask) ok = false;
          c += take;
        }
        if (ok) break;
      }
      if (t >= limit) { fail = E13_CHK_LIMIT; break; }
      if (deep ? (head < -4096 + 2 || head > blk + 2000) : (head <= -4000000LL + 2 || head >= 4000000LL - 2)) {
        fail = E13_CHK_OFFTAPE;
        break;
      }
      const u32 s = (word >> bit) & 1u;
      const unsigned e = (rows[st * kCheckBlock] >> (8 * s)) & 0xFFu;
      if (e & 0x80u) {
        const int i = 2 * st + (int)s;
        fail = in.kind[i] == 2 ? E13_CHK_FREE_READ : E13_CHK_HALT;
        o.free_state = st;
        o.free_sym = (int)s;
        break;
      }
      const u32 w = e & 1u;
      if (w != s) {
        word ^= 1u << bit;
        if (head >= -2) ones += w ? 1 : -1;
      }
      if (e & 2u) {
        ++head;
        if (++bit == 32) {
          tape[wi] = word;
          word = tape[++wi];
          bit = 0;
        }
      } else {
        --head;
        if (--bit < 0) {
          tape[wi] = word;
          word = tape[--wi];
          bit = 31;
        }
        if (head < minhead) minhead = head;
      }
      st = (int)(e >> 2);
      ++t;
    }
    if (fail) {
      o.status = fail;
      o.fail_stage = n;
      o.fail_t = t;
      o.fail_head = head;
      tape[wi] = word;
      return;
    }
    // stage start n: record the counter (all ones at cells <= -3)
    tape[wi] = word;
    o.stages_done = n;
    if (n <= E13_CHECK_MAX_NMAX) {
      o.stage_t[n] = t;
      o.minhead[n] = minhead;
      int cnt = 0;
      i64 leftmost = 0;
      const i64 lowest = deep ? -4096 + 1 : minhead - 1;
      for (i64 c = -3; c >= lowest;) {
        const i64 b = c + off;
        const int sh = (int)(b & 31);
        // bits sh down to 0 of this word hold cells c .. c - sh
        u32 x = tape[b >> 5] & (sh == 31 ? 0xFFFFFFFFu : ((2u << sh) - 1u));
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
  const i64 left = deep ? 4096 : 4000000;
  const i64 cells = deep ? 4096 + (1LL << nmax) + 4096 : 8000001;
  const i64 words = (cells + 31) / 32 + 2;
  const int chunk = (int)std::min<i64>(n, std::max<i64>(1, (4LL << 30) / (words * 4)));
  u32 *d_tapes = nullptr;
  e13_check_in *d_in = nullptr;
  e13_check_out *d_out = nullptr;
  int rc = E13_OK;
  if (cudaMalloc(&d_tapes, (size_t)chunk * words * 4) != cudaSuccess ||
      cudaMalloc(&d_in, sizeof(e13_check_in) * (size_t)chunk) != cudaSuccess ||
      cudaMalloc(&d_out, sizeof(e13_check_out) * (size_t)chunk) != cudaSuccess) {
    rc = E13_ERR_CUDA;
  }
  for (int b = 0; b < n && rc == E13_OK; b += chunk) {
    const int k = std::min(chunk, n - b);
    CheckParams P;
    P.n = k;
    P.nmax = nmax;
    P.mode = mode;
    P.side_left = left;
    P.words = words;
    P.tapes = d_tapes;
    P.in = d_in;
    P.out = d_out;
    if (cudaMemset(d_tapes, 0, (size_t)k * words * 4) != cudaSuccess ||
        cudaMemset(d_out, 0, sizeof(e13_check_out) * (size_t)k) != cudaSuccess ||
        cudaMemcpy(d_in, in + b, sizeof(e13_check_in) * (size_t)k, cudaMemcpyHostToDevice) != cudaSuccess) {
      rc = E13_ERR_CUDA;
      break;
    }
    check_kernel<<<(k + kCheckBlock - 1) / kCheckBlock, kCheckBlock>>>(P);
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
