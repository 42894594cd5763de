// e13_raw.cu -- the raw-simulator throughput set: whole tables run from the
// blank tape with no filter, at most max_steps steps each, stopping when the
// head leaves the 1364-cell window (steps (3)-(7) of src/e13search.c:163-175
// with the stage test and the deadline removed).  One machine per lane, the
// same bit-packed shared-memory tape, table rows and word-level run skip as
// the search kernels, in the same lock-step form.
#include <cuda_runtime.h>
#include <stdint.h>

#include "e13.h"
#include "e13_device.cuh"

using namespace e13dev;

namespace {

constexpr int kRawBlock = 768;

__device__ __forceinline__ u64 splitmix_at(u64 seed, u64 k) {
  // draw k (1-based) of splitmix64 started at `seed`
  u64 z = seed + k * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ void raw_load_table(u32 *rcol, int stride, const unsigned char *__restrict__ codes, u64 seed,
                                               long long m, int nq) {
  for (int s = 0; s < 16; ++s) {
    u32 r = kEntHalt | (kEntHalt << 16);
    if (s < nq) {
      u32 c0, c1;
      if (codes) {
        c0 = codes[m * 2 * nq + 2 * s];
        c1 = codes[m * 2 * nq + 2 * s + 1];
      } else {
        c0 = (u32)(splitmix_at(seed, (u64)(m * 2 * nq + 2 * s + 1)) % (u64)(4 * nq));
        c1 = (u32)(splitmix_at(seed, (u64)(m * 2 * nq + 2 * s + 2)) % (u64)(4 * nq));
      }
      if (c0 >= (u32)(4 * nq)) c0 = kEntHalt;
      if (c1 >= (u32)(4 * nq)) c1 = kEntHalt;
      r = cell_slot(2 * s, c0, true) | (cell_slot(2 * s + 1, c1, true) << 16);
    }
    rcol[s * stride] = r;
  }
}

// Each lane takes its next machine from a global counter as soon as its
// current one ends, so long runs do not hold up lanes with short ones; every
// iteration is one step (or one run skip inside a word) for every lane.
__global__ void __launch_bounds__(kRawBlock) raw_kernel(const unsigned char *__restrict__ codes, u64 seed, long long n,
                                                         int nq, long long max_steps, long long *__restrict__ out,
                                                         unsigned long long *__restrict__ total,
                                                         unsigned long long *__restrict__ next_machine) {
  extern __shared__ __align__(16) u32 raw_smem[];
  u32 *tape = raw_smem;                       // kTapeWords x kRawBlock
  u32 *rows = tape + kTapeWords * kRawBlock;  // 16 x kRawBlock
  __shared__ unsigned long long s_total;
  if (threadIdx.x == 0) s_total = 0;
  __syncthreads();
  const int stride = kRawBlock;
  u32 *tcol = tape + threadIdx.x;
  u32 *rcol = rows + threadIdx.x;
  unsigned long long my_steps = 0;
  long long m = -1;  // current machine
  int p = 0, st = 0;
  long long t = 0;
  for (;;) {
    if (m < 0) {
      m = (long long)atomicAdd(next_machine, 1ull);
      if (m < n) {
        for (int w = 0; w < kTapeWords; ++w) tcol[w * stride] = 0;
        raw_load_table(rcol, stride, codes, seed, m, nq);
        p = kLeft;
        st = 0;
        t = 0;
      }
    }
    if (!__any_sync(0xFFFFFFFFu, m < n)) break;
    int status = -1;  // -1 still running
    if (m < n) {
      if (t >= max_steps) {
        status = 0;
      } else {
        const int widx = (p >> 5) * stride;
        const u32 word = tcol[widx];
        const u32 sym = (word >> (p & 31)) & 1u;
        const u32 e = (rcol[st * stride] >> (sym << 4)) & 0x1FFu;
        if (e & kEntSpecial) {
          status = 2;
        } else {
          // k = 1, or on a self-loop cell the rest of the run inside this word
          const bool right = (e & 2u) != 0;
          const int b = p & 31;
          const u32 x = word ^ (0u - sym);
          const u32 xr = right ? x : __brev(x);
          const int bb = right ? b : 31 - b;
          const u32 up = xr >> bb;
          long long k = up ? __ffs(up) - 1 : 32 - bb;
          const long long left_steps = max_steps - t;
          const int room = right ? (kTapeCells - 2) - p : p - 1;
          k = k < left_steps ? k : left_steps;
          k = k < room ? k : room;
          k = ((e & kEntSelf) && k > 1) ? k : 1;
          if ((e ^ sym) & 1u) tcol[widx] = word ^ (1u << b);
          const int np = p + (int)(right ? k : -k);
          if ((unsigned)(np - 1) >= (unsigned)(kTapeCells - 2)) {
            status = 1;  // left the window: this step is not counted, as in run()
            p = np;
          } else {
            p = np;
            st = (int)((e >> 2) & 15u);
            t += k;
          }
        }
      }
      if (status >= 0) {
        long long ones = 0;
        for (int w = 0; w < kTapeWords; ++w) ones += __popc(tcol[w * stride]);
        if (out) {
          out[4 * m] = t;
          out[4 * m + 1] = status;
          out[4 * m + 2] = p - kLeft;
          out[4 * m + 3] = ones;
        }
        my_steps += (unsigned long long)t;
        m = -1;
      }
    }
    __syncwarp();
  }
  for (int o = 16; o > 0; o >>= 1) my_steps += __shfl_down_sync(0xFFFFFFFFu, my_steps, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(&s_total, my_steps);
  __syncthreads();
  if (threadIdx.x == 0) atomicAdd(total, s_total);
}

}  // namespace

struct e13_ctx;
extern "C" int e13_ctx_device(const e13_ctx *c);
extern "C" void e13_ctx_note_run(e13_ctx *c, double ms, long long launches);
extern "C" cudaStream_t e13_ctx_stream(const e13_ctx *c);

extern "C" int e13_raw_run(e13_ctx *ctx, const uint8_t *codes, uint64_t seed, int64_t n, int nq, int64_t max_steps,
                           int64_t *out, uint64_t *total_steps) {
  if (!ctx || n < 0 || nq < 1 || nq > 16 || max_steps < 0) return E13_ERR_ARG;
  if (n == 0) return E13_OK;
  if (cudaSetDevice(e13_ctx_device(ctx)) != cudaSuccess) return E13_ERR_CUDA;
  cudaStream_t s = e13_ctx_stream(ctx);
  unsigned char *d_codes = nullptr;
  long long *d_out = nullptr;
  unsigned long long *d_total = nullptr;  // [0] total steps, [1] next machine
  int rc = E13_OK;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  if (codes && cudaMalloc(&d_codes, (size_t)n * 2 * nq) != cudaSuccess) rc = E13_ERR_CUDA;
  if (!rc && out && cudaMalloc(&d_out, sizeof(long long) * 4 * (size_t)n) != cudaSuccess) rc = E13_ERR_CUDA;
  if (!rc && cudaMalloc(&d_total, 2 * sizeof(unsigned long long)) != cudaSuccess) rc = E13_ERR_CUDA;
  if (!rc) {
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, e13_ctx_device(ctx));
    const size_t smem = (size_t)(kTapeWords + 16) * kRawBlock * 4;
    cudaFuncSetAttribute(raw_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaEventRecord(e0, s);
    if (codes) cudaMemcpyAsync(d_codes, codes, (size_t)n * 2 * nq, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(d_total, 0, 2 * sizeof(unsigned long long), s);
    const long long need = (n + kRawBlock - 1) / kRawBlock;
    const int grid = (int)(need < (long long)nsm ? need : (long long)nsm);  // 177 KB of shared memory per CTA: one per SM
    raw_kernel<<<grid, kRawBlock, smem, s>>>(d_codes, seed, n, nq, max_steps, d_out, d_total, d_total + 1);
    if (cudaGetLastError() != cudaSuccess) rc = E13_ERR_CUDA;
    unsigned long long tot = 0;
    if (!rc && out) cudaMemcpyAsync(out, d_out, sizeof(long long) * 4 * (size_t)n, cudaMemcpyDeviceToHost, s);
    if (!rc) cudaMemcpyAsync(&tot, d_total, sizeof tot, cudaMemcpyDeviceToHost, s);
    cudaEventRecord(e1, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) rc = E13_ERR_CUDA;
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    e13_ctx_note_run(ctx, ms, 1);
    if (total_steps) *total_steps = tot;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_codes);
  cudaFree(d_out);
  cudaFree(d_total);
  return rc;
}
