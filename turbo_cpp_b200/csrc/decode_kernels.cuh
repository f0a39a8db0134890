// decode_kernels.cuh -- the kernels of one plain-schedule decode (per half-iteration SISO
// launches, set-up, CRC24B early stop), shared by the decoder object (decoder.cu) and the
// allocation-free entry point (noalloc.cu).  Each including translation unit gets its own
// internal-linkage instances.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "decoder.hpp"
#include "siso.cuh"

namespace tcb {
namespace {

constexpr int kThreads = 64;  // threads (windows) per block of the plain SISO kernel
constexpr int kMinBlocks = 8;  // 16 warps per SM: at most 128 registers per thread

// KIND: 0 = upper SISO, 1 = lower SISO, 2 = lower SISO that also writes the posterior;
// STD: the TS 36.212 code instead of the reference's; TAPE (with GLOBAL_CKPT): the alpha
// checkpoints cover the warm-up too, plane (q - a_lo) / S of the slab for step q, and stay for
// the adjoint (a slab of (window + guard) / S + 1 planes)
template <int S, int KIND, bool GLOBAL_CKPT, bool STD = false, bool TAPE = false>
__global__ void __launch_bounds__(kThreads, kMinBlocks) siso_plain_kernel(const DevCb* __restrict__ cbs,
                                                              const int32_t* __restrict__ win_cb,
                                                              int n_win, SisoIo io,
                                                              const uint8_t* __restrict__ done,
                                                              float4* ckpt_global,
                                                              int ckpt_per_thread) {
  extern __shared__ float4 smem_ckpt[];
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_win) return;
  const int c = win_cb[g];
  if (done != nullptr && done[c]) return;
  const DevCb cb = cbs[c];
  const int w = g - cb.win0;
  if (GLOBAL_CKPT) {
    // checkpoint slab: ckpt_per_thread planes of n_win float4 pairs (windows interleaved)
    CkptStrided ck{ckpt_global, n_win, g};
    if (TAPE) {  // plane 0 is alpha at a_lo
      const int lo = w * cb.window;
      ck.p += static_cast<int64_t>(2 * (min(lo, io.guard) / S)) * n_win;
    }
    siso_window<S, KIND != 0, KIND == 2, CkptStrided, false, STD, TAPE>(cb, w, g, io, ck);
  } else {
    CkptSmem ck{smem_ckpt, static_cast<int>(blockDim.x), static_cast<int>(threadIdx.x)};
    siso_window<S, KIND != 0, KIND == 2, CkptSmem, false, STD>(cb, w, g, io, ck);
  }
}

// sys_i[i] = d0[Pi(i)]; E2 = 0 (first a-priori).  One CTA per code block: d0 is read into shared
// memory with coalesced loads, then the interleaved copy is gathered from there, so that every
// global access walks its array in order (a direct gather would read one 32-byte sector per
// 4-byte element).
constexpr int kGatherThreads = 512;
constexpr int kMaxBlockK = 6144;
__global__ void __launch_bounds__(kGatherThreads) setup_kernel(const DevCb* __restrict__ cbs,
                                                               int n_cb,
                                                               const float* __restrict__ llr,
                                                               const uint16_t* __restrict__ perm,
                                                               float* __restrict__ sys_i,
                                                               float* __restrict__ e2) {
  __shared__ float d0[kMaxBlockK];
  for (int c = blockIdx.x; c < n_cb; c += gridDim.x) {
    const DevCb cb = cbs[c];
    const float* src = llr + cb.llr;
    for (int p = threadIdx.x; p < cb.k; p += kGatherThreads) d0[p] = __ldg(src + p);
    __syncthreads();
    const uint16_t* pi = perm + cb.tab;
    for (int p = threadIdx.x; p < cb.k; p += kGatherThreads) {
      sys_i[cb.work + p] = d0[pi[p]];
      e2[cb.work + p] = 0.0f;
    }
    __syncthreads();  // d0 is reused by the next code block
  }
}

inline void launch_setup(const DevCb* cbs, int n_cb, const float* llr, const uint16_t* perm,
                         float* sys_i, float* e2, cudaStream_t st) {
  if (n_cb <= 0) return;
  const unsigned grid = static_cast<unsigned>(n_cb < (1 << 20) ? n_cb : (1 << 20));
  setup_kernel<<<grid, kGatherThreads, 0, st>>>(cbs, n_cb, llr, perm, sys_i, e2);
}

// CRC24B early stop (lte_turbo.cpp:792-804): hard decisions (>= 0 -> 1) of bits
// [filler, K) must form a codeword of the reference's CRC24B generator, i.e. the XOR of
// x^(N-1-i) mod g over the set bits i must be zero.  One warp per code block.
__global__ void crc_stop_kernel(const DevCb* __restrict__ cbs, int n_cb,
                                const float* __restrict__ post, const uint32_t* __restrict__ xpow,
                                uint8_t* __restrict__ done, uint32_t* __restrict__ iters, int it) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n_cb || done[warp]) return;
  const DevCb cb = cbs[warp];
  const int n = cb.k - cb.filler;
  const float* p = post + cb.out + cb.filler;
  uint32_t syn = 0;
  for (int i = lane; i < n; i += 32)
    if (p[i] >= 0.0f) syn ^= xpow[n - 1 - i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) syn ^= __shfl_xor_sync(0xffffffffu, syn, o);
  if (lane == 0) {
    iters[warp] = static_cast<uint32_t>(it + 1);
    if (syn == 0) done[warp] = 1;
  }
}

__global__ void init_flags_kernel(int n_cb, uint8_t* __restrict__ done, uint32_t* __restrict__ iters,
                                  uint32_t max_iterations) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_cb) {
    done[i] = 0;
    iters[i] = max_iterations;  // early stop lowers it
  }
}

__global__ void finish_kernel(int n_cb, const uint8_t* __restrict__ done, uint8_t* crc_ok,
                              int early_stop) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_cb) crc_ok[i] = early_stop ? done[i] : 0;
}

// ------------------------------------------------------------------------------------------
// Persistent schedule: one launch for all iterations, fed by a device work queue.  A task is up
// to 32 windows (one per lane) of one or more whole code blocks; a work item is one SISO
// half-iteration of one task.  Items are handed out in half-iteration order (all tasks' first
// half, then all tasks' second half, ...), so the item a warp waits for -- the same task's
// previous half -- was always handed out earlier to a running warp.  Progress per task is a
// counter released with a fence after the half's stores; a warp that waits longer than
// kWaitLimitNs (one second of the GPU global timer) sets the error flag and proceeds, so the
// kernel always terminates.  Blocks whose CRC24B passes are skipped by every later item.
// ------------------------------------------------------------------------------------------
constexpr int kPersistThreads = 64;
constexpr int kPersistMinBlocks = 6;  // 12 warps per SM: at most 168 registers per thread
constexpr int kMaxIterations = 64;
constexpr uint64_t kWaitLimitNs = 1000000000ull;  // one second

struct PersistArgs {
  const DevCb* cbs;
  const int32_t* win_cb;
  const int32_t* tasks;  // [n_tasks][32] launch-wide window index per lane, -1 = idle lane
  int n_tasks;
  int* queue;            // next work item (atomic), zero before the launch
  int* progress;         // per task: half-iterations completed, zero before the launch
  int* error;            // set when a wait gave up
  int stall_task;        // testing hook: this task's waits are never satisfied (-1: off)
  const float* llr;
  float* sys_i;
  float* e1i;
  float* e2;
  float* post;
  const uint16_t* perm;
  const uint16_t* inv;
  float* seed_up[2];
  float* seed_lo[2];
  float4* ckpt;
  int ckpt_per_window;
  int n_windows;         // windows of the launch (stride of the interleaved checkpoint slab)
  int guard;
  int max_iterations;
  int early_stop;
  uint8_t* done;
  uint32_t* iters;
  const uint32_t* xpow;
  float scale[2 * kMaxIterations];
};

__device__ __forceinline__ int load_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void store_release(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <bool STD = false>
__global__ void __launch_bounds__(kPersistThreads, kPersistMinBlocks)
    persistent_kernel(const PersistArgs p) {
  const int lane = threadIdx.x & 31;
  const int total = p.n_tasks * 2 * p.max_iterations;
  for (;;) {
    int item = 0;
    if (lane == 0) item = atomicAdd(p.queue, 1);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= total) break;
    const int h = item / p.n_tasks;  // half-iteration index
    const int t = item - h * p.n_tasks;
    const int it = h >> 1, half = h & 1;
    if (h > 0 && lane == 0) {  // wait until this task has completed half h-1
      const int need = (t == p.stall_task) ? 0x7fffffff : h;
      const uint64_t t0 = global_ns();
      while (load_acquire(p.progress + t) < need) {
        if (global_ns() - t0 > kWaitLimitNs) {
          atomicExch(p.error, 1);
          break;
        }
        __nanosleep(256);
      }
    }
    __syncwarp();
    __threadfence();  // order this lane's reads after lane 0's acquire
    const int g = p.tasks[32 * t + lane];
    const int c = g >= 0 ? p.win_cb[g] : -1;
    DevCb cb{};
    if (c >= 0) cb = p.cbs[c];
    const int w = g - cb.win0;
    const bool active = c >= 0 && __ldcg(p.done + c) == 0;
    if (__any_sync(0xffffffffu, active)) {
      const CkptStrided ck{p.ckpt, p.n_windows, g < 0 ? 0 : g};
      const bool post_now = p.early_stop || it + 1 == p.max_iterations;
      const SisoIo io =
          half == 0 ? SisoIo{p.llr, p.sys_i, p.e2, p.e1i, nullptr, p.perm, p.inv, p.seed_up[it & 1],
                             p.seed_up[(it + 1) & 1], p.scale[2 * it], p.guard}
                    : SisoIo{p.llr, p.sys_i, p.e1i, p.e2, p.post, p.perm, p.inv, p.seed_lo[it & 1],
                             p.seed_lo[(it + 1) & 1], p.scale[2 * it + 1], p.guard};
      if (active)
        // 4-step loop bodies: the one SISO copy for both halves plus the queue, CRC and wait
        // code must fit the instruction cache (measured 3166 against 2830 Mbit/s with 8-step
        // bodies at 4096 x K=6144, window 192; the plain kernels keep 8-step bodies)
        siso_window_rt<kSub, decltype(ck), true, STD, true>(cb, w, g, io, ck, half == 1,
                                                    half == 1 && post_now);
      if (half == 1 && p.early_stop) {
        // CRC24B syndrome of the hard decisions (lte_turbo.cpp:792-804): each lane XORs
        // x^(N-1-i) mod g over the set bits of its window; a block's windows sit in consecutive
        // lanes, so its first lane takes the XOR of their parts from a warp-wide XOR prefix
        // scan (no shared memory, which keeps the occupancy at the register limit).
        __threadfence();  // this lane's posterior stores, before the other lanes read them
        __syncwarp();
        uint32_t part = 0;
        if (active) {
          const int lo_p = w * cb.window, hi_p = min(lo_p + cb.window, cb.k);
          const int n = cb.k - cb.filler;
          for (int q = max(lo_p, cb.filler); q < hi_p; ++q)
            if (__ldcg(p.post + cb.out + q) >= 0.0f) part ^= p.xpow[n - 1 - (q - cb.filler)];
        }
        uint32_t pre = part;  // part[0] ^ ... ^ part[lane]
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t v = __shfl_up_sync(0xffffffffu, pre, o);
          if (lane >= o) pre ^= v;
        }
        const int last = min(lane + max(cb.nwin, 1) - 1, 31);
        const uint32_t upto_last = __shfl_sync(0xffffffffu, pre, last);
        const uint32_t before = __shfl_sync(0xffffffffu, pre, lane > 0 ? lane - 1 : 0);
        if (active && w == 0) {
          const uint32_t x = upto_last ^ (lane > 0 ? before : 0u);
          p.iters[c] = static_cast<uint32_t>(it + 1);
          if (x == 0) p.done[c] = 1;
        }
      }
    }
    __threadfence();  // every lane's stores of this half-iteration, before the release
    __syncwarp();
    if (lane == 0) store_release(p.progress + t, h + 1);
  }
}

}  // namespace
}  // namespace tcb
