// e13_estimate.cu -- the reference's Knuth size estimate of a search
// (src/e13search.c:256-313 probe, :473-510 estimate) on one B200 (sm_100a).
//
// A probe follows one random root-to-leaf path of the TNF tree.  At every
// fork all children run to their next event (fork or leaf), so the children
// that die at once are counted exactly, and the path continues into one of
// the live ones drawn at random; the weight w multiplies by the number of live
// children.  The average of the weighted counts over the probes is an
// unbiased estimate of the search's leaves, nodes, steps and survivors.
//
// One warp per probe: the lanes are the children of the current fork (a
// fork has at most 4 nq + 1 <= 65 children, so up to three passes of 32), all
// running in the lock-step form of the search kernel.  The path node lives
// in shared memory.  Probes are taken from an atomic counter.
//
// Probe p draws from its own splitmix64 stream, the one the reference gives
// its OpenMP thread p (start mix(0x5EED0000 + p + (seed << 20)), :486-491), so
// each probe's result depends only on (seed, p) and not on scheduling.  The
// per-probe results are summed on the host in probe order.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "e13.h"
#include "e13_device.cuh"
#include "e13_node.cuh"

using namespace e13dev;

namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kEstBlock = 256;

enum { kPrIdle = 0, kPrRun = 1, kPrFork = 2, kPrDead = 3, kPrSurv = 4 };

// splitmix64 (src/e13search.c:98-103): advances the state, returns the draw
__device__ __forceinline__ u64 mix_next(u64 &s) {
  u64 z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Runs every lane in kPrRun to its next event: a read of a cell that is not
// fixed yet (kPrFork: fork_cell / fork_e), or a leaf (kPrDead / kPrSurv).  Same
// per-step semantics as the search (lane_act, src/e13search.c:134-177); here
// every first read is a fork, as in run() with fixed[i] == 0.
__device__ __forceinline__ void run_to_event(Lane &L, int &status, int &fork_cell, u32 &fork_e, u32 *tcol,
                                             const u32 *rcol, const KeyTabs &K, int stride) {
  while (__any_sync(kFull, status == kPrRun)) {
    if (status == kPrRun) {
      int cell = 0;
      u32 e = 0;
      int ev = lane_act<true>(L, tcol, rcol, K, stride, cell, e);
      if (ev == kEvStage) ev = stage_check(L, tcol, K, stride);
      if (ev == kEvCell) {
        if (e == kEntHalt) {
          status = kPrDead;  // a fixed halt cell
        } else {
          status = kPrFork;
          fork_cell = cell;
          fork_e = e;
        }
      } else if (ev == kEvDead) {
        status = kPrDead;
      } else if (ev == kEvSurv) {
        status = kPrSurv;
      }
    }
    __syncwarp();
  }
}

__global__ void __launch_bounds__(kEstBlock) estimate_kernel(const Node *root, int nv, int sym_lo, int sym_hi,
                                                             long long nprobes, u64 seed, double *out,
                                                             unsigned long long *next_probe) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const KeyTabs K = key_tables(smem_raw);
  u32 *tape = reinterpret_cast<u32 *>(smem_raw + kKeySmemBytes);
  const int stride = blockDim.x;
  u32 *rows = tape + kTapeWords * stride;
  Node *node = reinterpret_cast<Node *>(rows + 16 * stride) + (threadIdx.x >> 5);  // this warp's path node
  fill_key_tables(K);
  load_stage_tables();
  u32 *tcol = tape + threadIdx.x;
  u32 *rcol = rows + threadIdx.x;
  for (int w = 0; w < kTapeWords; ++w) tcol[w * stride] = 0;
  __syncthreads();

  const int lane = threadIdx.x & 31;
  Lane L;
  L.t = 0;
  L.tseg = 0;
  L.job = 0;
  int status = kPrIdle, fork_cell = 0;
  u32 fork_e = 0;

  for (;;) {
    long long p = 0;
    if (lane == 0) p = (long long)atomicAdd(next_probe, 1ull);
    p = __shfl_sync(kFull, p, 0);
    if (p >= nprobes) break;
    u64 rng = 0x5EED0000ull + (u64)p + (seed << 20);
    rng = mix_next(rng);
    double o_leaves = 0, o_nodes = 0, o_steps = 0, o_surv = 0;  // lane 0's sums
    double w = 1.0;

    // the root runs to its first read (src/e13search.c:268-275)
    status = kPrIdle;
    if (lane == 0) {
      lane_load(L, root, tcol, rcol, stride, 0);
      status = kPrRun;
    }
    run_to_event(L, status, fork_cell, fork_e, tcol, rcol, K, stride);
    if (lane == 0) {
      o_nodes += 1.0;
      o_steps += (double)L.t;
      if (status != kPrFork) o_leaves += 1.0;
      if (status == kPrSurv) o_surv += 1.0;
      if (status == kPrFork) {
        int keep = 0;
        u64 vm = 0;
        child_set(fork_e, L.budget, L.nintro, nv, sym_lo, sym_hi, keep, vm);
        lane_store(L, node, tcol, rcol, stride, 0, fork_cell, keep, vm);
      }
    }
    bool live = __shfl_sync(kFull, status == kPrFork, 0);
    __syncwarp();

    while (live) {
      // every child of the path node (keep first, then the moves in order)
      // runs to its next event (src/e13search.c:276-298)
      const int keep = (node->flags & kFlagKeep) ? 1 : 0;
      const u64 vm = node->vmask;
      const int k = keep + __popcll(vm);
      const int last = (k - 1) >> 5;
      u32 livem[3] = {0u, 0u, 0u};
      for (int b = 0; b <= last; ++b) {
        const int c = 32 * b + lane;
        status = kPrIdle;
        int t0 = 0;
        if (c < k) {
          const int ch = (keep && c == 0) ? -1 : nth_bit64(vm, c - keep);
          lane_load(L, node, tcol, rcol, stride, 0);
          apply_child(L, node, ch, rcol, stride, sym_lo, sym_hi, true);
          t0 = L.t;
          status = kPrRun;
        }
        run_to_event(L, status, fork_cell, fork_e, tcol, rcol, K, stride);
        // weighted counts, added in child order as the reference does
        const int nb = min(32, k - 32 * b);
        for (int j = 0; j < nb; ++j) {
          const int sj = __shfl_sync(kFull, status, j);
          const int dj = __shfl_sync(kFull, L.t - t0, j);
          if (lane == 0) {
            o_nodes += w;
            o_steps += w * (double)dj;
            if (sj != kPrFork) o_leaves += w;
            if (sj == kPrSurv) o_surv += w;
          }
        }
        livem[b] = __ballot_sync(kFull, status == kPrFork);
      }
      const int n0 = __popc(livem[0]), n1 = __popc(livem[1]), nlive = n0 + n1 + __popc(livem[2]);
      if (nlive == 0) break;
      // the next path node: live child number r (src/e13search.c:299-305)
      int r = (int)(mix_next(rng) % (u64)nlive);
      int b = 0;
      if (r >= n0) {
        r -= n0;
        b = 1;
        if (r >= n1) {
          r -= n1;
          b = 2;
        }
      }
      const int c = 32 * b + (int)nth_bit64((u64)livem[b], r);
      w *= (double)nlive;
      int holder = c & 31;
      if (b != last) {
        // its lane has since run a later child: run it again in lane 0 (the
        // same start gives the same fork)
        holder = 0;
        status = kPrIdle;
        if (lane == 0) {
          const int ch = (keep && c == 0) ? -1 : nth_bit64(vm, c - keep);
          lane_load(L, node, tcol, rcol, stride, 0);
          apply_child(L, node, ch, rcol, stride, sym_lo, sym_hi, true);
          status = kPrRun;
        }
        run_to_event(L, status, fork_cell, fork_e, tcol, rcol, K, stride);
      }
      __syncwarp();  // every lane is done reading the old path node
      if (lane == holder) {
        int kp = 0;
        u64 vmn = 0;
        child_set(fork_e, L.budget, L.nintro, nv, sym_lo, sym_hi, kp, vmn);
        lane_store(L, node, tcol, rcol, stride, 0, fork_cell, kp, vmn);
      }
      __syncwarp();
      live = true;
    }
    if (lane == 0) {
      double *o = out + 4 * p;
      o[0] = o_leaves;
      o[1] = o_nodes;
      o[2] = o_steps;
      o[3] = o_surv;
    }
    __syncwarp();
  }
}

}  // namespace

extern "C" int e13_ctx_device(const e13_ctx *c);
extern "C" cudaStream_t e13_ctx_stream(const e13_ctx *c);
extern "C" void e13_ctx_note_run(e13_ctx *c, double ms, long long launches);

extern "C" int e13_estimate(e13_ctx *ctx, const e13_job *job, int64_t probes, uint64_t seed, e13_estimate_out *out,
                            double *per_probe) {
  // probe p draws from the stream that starts at mix(0x5EED0000 + p + (seed << 20)):
  // from p = 2^20 on, the streams of seed would run into those of seed + 1
  if (!ctx || !job || !out || probes < 1 || probes > E13_ESTIMATE_MAX_PROBES) return E13_ERR_ARG;
  if (job->nq < 1 || job->nq > 16) return E13_ERR_NQ;
  if (job->budget < 0) return E13_ERR_FMAX;
  for (int i = 0; i < 2 * job->nq; ++i)
    if (job->tab[i] < E13_FREE || (job->tab[i] >= 0 && (job->tab[i] >> 2) >= job->nq)) return E13_ERR_ARG;
  if (cudaSetDevice(e13_ctx_device(ctx)) != cudaSuccess) return E13_ERR_CUDA;
  cudaStream_t s = e13_ctx_stream(ctx);
  if (upload_filter_tables() != cudaSuccess) return E13_ERR_CUDA;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, e13_ctx_device(ctx));
  const size_t smem = kKeySmemBytes + (size_t)(kTapeWords + 16) * kEstBlock * 4 + (size_t)(kEstBlock / 32) * sizeof(Node);
  if (cudaFuncSetAttribute(estimate_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return E13_ERR_CUDA;

  Node root;
  build_root(job, 0, &root);
  Node *d_root = nullptr;
  double *d_out = nullptr;
  unsigned long long *d_next = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = E13_ERR_CUDA;
  std::vector<double> h((size_t)probes * 4);
  if (cudaMalloc(&d_root, sizeof(Node)) != cudaSuccess || cudaMalloc(&d_out, sizeof(double) * 4 * probes) != cudaSuccess ||
      cudaMalloc(&d_next, sizeof(unsigned long long)) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
      cudaEventCreate(&e1) != cudaSuccess)
    goto done;
  if (cudaMemcpyAsync(d_root, &root, sizeof root, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemsetAsync(d_next, 0, sizeof(unsigned long long), s) != cudaSuccess)
    goto done;
  {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, estimate_kernel, kEstBlock, smem);
    const long long want = (probes + kEstBlock / 32 - 1) / (kEstBlock / 32);
    const int grid = (int)std::min<long long>((long long)nsm * std::max(per_sm, 1), std::max(want, 1LL));
    cudaEventRecord(e0, s);
    estimate_kernel<<<grid, kEstBlock, smem, s>>>(d_root, 4 * job->nq, job->sym_lo, job->sym_hi, probes, seed, d_out,
                                                  d_next);
    cudaEventRecord(e1, s);
  }
  if (cudaGetLastError() != cudaSuccess) goto done;
  if (cudaMemcpyAsync(h.data(), d_out, sizeof(double) * 4 * probes, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    goto done;
  {
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    e13_ctx_note_run(ctx, ms, 1);
    // mean and standard error as the reference prints them (:505-509)
    double sum[4] = {0, 0, 0, 0}, sq[4] = {0, 0, 0, 0};
    for (long long p = 0; p < probes; ++p)
      for (int j = 0; j < 4; ++j) {
        const double v = h[(size_t)(4 * p + j)];
        sum[j] += v;
        sq[j] += v * v;
      }
    out->probes = probes;
    for (int j = 0; j < 4; ++j) {
      const double m = sum[j] / (double)probes, var = sq[j] / (double)probes - m * m;
      out->mean[j] = m;
      out->std_error[j] = var > 0 ? sqrt(var / (double)probes) : 0.0;
    }
    if (per_probe) memcpy(per_probe, h.data(), sizeof(double) * 4 * (size_t)probes);
    rc = E13_OK;
  }
done:
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(d_root);
  cudaFree(d_out);
  cudaFree(d_next);
  return rc;
}
