// decode_kernels.cuh -- the kernels of one plain-schedule decode (per half-iteration SISO
// launches, set-up, CRC24B early stop), shared by the decoder object (decoder.cu) and the
// allocation-free entry point (noalloc.cu).  Each including translation unit gets its own
// internal-linkage instances.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "siso.cuh"

namespace tcb {
namespace {

constexpr int kThreads = 64;  // threads (windows) per block of the plain SISO kernel
constexpr int kMinBlocks = 10;  // 20 warps per SM: at most 96 registers per thread

// KIND: 0 = upper SISO, 1 = lower SISO, 2 = lower SISO that also writes the posterior
template <int S, int KIND, bool GLOBAL_CKPT>
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
    CkptGlobal ck{ckpt_global + static_cast<int64_t>(2) * ckpt_per_thread * g};
    siso_window<S, KIND != 0, KIND == 2>(cb, w, g, io, ck);
  } else {
    CkptSmem ck{smem_ckpt, static_cast<int>(blockDim.x), static_cast<int>(threadIdx.x)};
    siso_window<S, KIND != 0, KIND == 2>(cb, w, g, io, ck);
  }
}

// sys_i[i] = d0[Pi(i)]; E2 = 0 (first a-priori); one thread per (block, position).
__global__ void setup_kernel(const DevCb* __restrict__ cbs, const int64_t* __restrict__ cb_start,
                             int n_cb, int64_t total, const float* __restrict__ llr,
                             const uint16_t* __restrict__ perm, float* __restrict__ sys_i,
                             float* __restrict__ e2) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= total) return;
  // binary search of the owning block
  int lo = 0, hi = n_cb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (cb_start[mid] <= i) lo = mid; else hi = mid - 1;
  }
  const DevCb cb = cbs[lo];
  const int64_t p = i - cb_start[lo];
  sys_i[cb.work + p] = llr[cb.llr + perm[cb.tab + p]];
  e2[cb.work + p] = 0.0f;
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

}  // namespace
}  // namespace tcb
