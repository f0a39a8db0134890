// siso.cuh -- one window of one SISO half-iteration, shared by the plain (one launch per
// half-iteration) and the persistent (all iterations in one launch) decoders.
//
// A window [lo, hi) of a code block is owned by one thread, which keeps the 8 state metrics
// in registers.  Its forward recursion starts `guard` steps before the window and its backward
// recursion `guard` steps after it; a start at the block edge uses the true edge metric (state
// 0 / tail), any other start uses the seed the neighbouring window recorded at that position
// in the previous iteration (next-iteration initialisation).  This is exactly the schedule of
// or_decode_cb_windowed in the oracle; with window >= K it is the reference's full trellis
// (decode_siso_log_map, lte_turbo.cpp:410-486).
//
// Memory use per thread: the forward pass stores alpha only every S steps (checkpoints, 32 B
// each, in shared memory or a global scratch slot); the backward pass recomputes the S alphas
// of one sub-window into registers from its checkpoint and then runs beta + extrinsic over it.
#pragma once
#include <cstdint>

#include "trellis.cuh"

namespace tcb {

// Per-code-block descriptor as the kernels see it (built by the host decoder).
struct DevCb {
  int32_t k;        // block size K
  int32_t filler;   // filler bits at the block start
  int32_t tab;      // offset of this K's permutation tables (entries)
  int32_t win0;     // index of the block's first window in the launch-wide window list
  int32_t nwin;     // windows of this block
  int32_t window;   // window length used for this block
  int64_t llr;      // float offset of [d0|d1|d2] in the LLR buffer
  int64_t work;     // float offset of the block's K-long work arrays
  int64_t out;      // float offset of the block's posterior
};

struct SisoIo {
  const float* llr;       // channel LLRs, [d0|d1|d2] per block
  const float* sys_i;     // interleaved systematic LLRs (work layout)
  const float* apr;       // a-priori in: upper reads E2 (natural), lower reads E1I (interleaved)
  float* ext;             // extrinsic out: upper writes E1I[inv(p)], lower writes E2[perm(p)]
  float* post;            // lower only: posterior (natural order, output layout)
  const uint16_t* perm;   // perm[i] = Pi(i) per K, at DevCb::tab
  const uint16_t* inv;    // inv[Pi(i)] = i
  const float* seed_in;   // [window][16]: alpha seed 0..7, beta seed 8..15
  float* seed_out;
  float scale;            // extrinsic scale of this half-iteration (1.0 for the plain decoder)
  int guard;
};

__device__ __forceinline__ float4 ld4(const float* p) {
  return __ldg(reinterpret_cast<const float4*>(p));
}

// Loads 4 consecutive steps: raw sys+apr (sa), scaled a and b.
__device__ __forceinline__ void load_steps4(const float* sys, const float* apr, const float* par,
                                            int q, float* sa, float* a, float* b) {
  const float4 s = ld4(sys + q), e = ld4(apr + q), p = ld4(par + q);
  sa[0] = s.x + e.x; sa[1] = s.y + e.y; sa[2] = s.z + e.z; sa[3] = s.w + e.w;
  a[0] = kHalfLog2e * sa[0]; a[1] = kHalfLog2e * sa[1];
  a[2] = kHalfLog2e * sa[2]; a[3] = kHalfLog2e * sa[3];
  b[0] = kHalfLog2e * p.x; b[1] = kHalfLog2e * p.y; b[2] = kHalfLog2e * p.z; b[3] = kHalfLog2e * p.w;
}

// Checkpoint storage: shared memory (thread-minor float4 layout, conflict-free) or a global
// scratch slot.
struct CkptSmem {
  float4* base;  // dynamic shared memory
  int stride;    // threads per block
  int tid;
  __device__ __forceinline__ void store(int j, const float (&m)[8]) const {
    base[(2 * j) * stride + tid] = make_float4(m[0], m[1], m[2], m[3]);
    base[(2 * j + 1) * stride + tid] = make_float4(m[4], m[5], m[6], m[7]);
  }
  __device__ __forceinline__ void load(int j, float (&m)[8]) const {
    const float4 x = base[(2 * j) * stride + tid], y = base[(2 * j + 1) * stride + tid];
    m[0] = x.x; m[1] = x.y; m[2] = x.z; m[3] = x.w; m[4] = y.x; m[5] = y.y; m[6] = y.z; m[7] = y.w;
  }
};
struct CkptGlobal {
  float4* base;  // this thread's slot: 2 float4 per checkpoint
  __device__ __forceinline__ void store(int j, const float (&m)[8]) const {
    base[2 * j] = make_float4(m[0], m[1], m[2], m[3]);
    base[2 * j + 1] = make_float4(m[4], m[5], m[6], m[7]);
  }
  __device__ __forceinline__ void load(int j, float (&m)[8]) const {
    const float4 x = base[2 * j], y = base[2 * j + 1];
    m[0] = x.x; m[1] = x.y; m[2] = x.z; m[3] = x.w; m[4] = y.x; m[5] = y.y; m[6] = y.z; m[7] = y.w;
  }
};

// Tail LLRs in the reference's decoder mapping (lte_turbo.cpp:758-773).
template <bool LOWER>
__device__ __forceinline__ void tail_llrs(const float* d0, int k, float ts[3], float tp[3]) {
  const float* d1 = d0 + (k + 4);
  const float* d2 = d1 + (k + 4);
  if (!LOWER) {
    ts[0] = d0[k]; ts[1] = d0[k + 2]; ts[2] = 0.0f;
    tp[0] = d1[k]; tp[1] = d0[k + 1]; tp[2] = d1[k + 2];
  } else {
    ts[0] = d1[k + 3]; ts[1] = d2[k]; ts[2] = d2[k + 2];
    tp[0] = d2[k + 1]; tp[1] = d0[k + 3]; tp[2] = d2[k + 3];
  }
}

// Runs window w of block cb for one half-iteration.  g = launch-wide window index (seed slot).
template <int S, bool LOWER, class Ckpt>
__device__ __forceinline__ void siso_window(const DevCb& cb, int w, int g, const SisoIo& io,
                                            const Ckpt& ck) {
  static_assert(S % 4 == 0, "sub-window must be a multiple of 4 steps");
  const int K = cb.k, W = cb.window, G = io.guard;
  const int lo = w * W, hi = min(lo + W, K);
  const float* d0 = io.llr + cb.llr;
  const float* sys = LOWER ? io.sys_i + cb.work : d0;
  const float* par = d0 + (LOWER ? 2 : 1) * (K + 4);
  const float* apr = io.apr + cb.work;
  const int nsub = (hi - lo) / S;

  float sa[4], a[4], b[4];

  // ---- forward: warm-up, then alpha checkpoints every S steps ----
  float al[8];
  int a_lo = lo - G;
  if (a_lo <= 0) {
    a_lo = 0;
    alpha_start(al);
  } else {
    const float4 x = ld4(io.seed_in + 16 * g), y = ld4(io.seed_in + 16 * g + 4);
    al[0] = x.x; al[1] = x.y; al[2] = x.z; al[3] = x.w; al[4] = y.x; al[5] = y.y; al[6] = y.z; al[7] = y.w;
  }
  for (int q = a_lo; q < lo; q += 4) {
    load_steps4(sys, apr, par, q, sa, a, b);
#pragma unroll
    for (int t = 0; t < 4; ++t) alpha_step(al, a[t], b[t]);
  }
  for (int j = 0; j < nsub; ++j) {
    ck.store(j, al);
#pragma unroll
    for (int q4 = 0; q4 < S; q4 += 4) {
      load_steps4(sys, apr, par, lo + j * S + q4, sa, a, b);
#pragma unroll
      for (int t = 0; t < 4; ++t) alpha_step(al, a[t], b[t]);
    }
  }
  // seed for window w+1: alpha at hi - G
  if (w + 1 < cb.nwin && hi - G > 0) {
    float r[8];
    if (G == 0) {
#pragma unroll
      for (int s = 0; s < 8; ++s) r[s] = al[s];
    } else {
      ck.load((hi - G - lo) / S, r);
    }
    float4* o = reinterpret_cast<float4*>(io.seed_out + 16 * (g + 1));
    o[0] = make_float4(r[0], r[1], r[2], r[3]);
    o[1] = make_float4(r[4], r[5], r[6], r[7]);
  }

  // ---- backward: warm-up, then per sub-window recompute alpha + beta + extrinsic ----
  float be[8];
  int b_hi = hi + G;
  if (b_hi >= K) {
    b_hi = K;
    float ts[3], tp[3];
    tail_llrs<LOWER>(d0, K, ts, tp);
    tail_beta(be, ts, tp);
  } else {
    const float4 x = ld4(io.seed_in + 16 * g + 8), y = ld4(io.seed_in + 16 * g + 12);
    be[0] = x.x; be[1] = x.y; be[2] = x.z; be[3] = x.w; be[4] = y.x; be[5] = y.y; be[6] = y.z; be[7] = y.w;
  }
  for (int q = b_hi - 4; q >= hi; q -= 4) {
    load_steps4(sys, apr, par, q, sa, a, b);
#pragma unroll
    for (int t = 3; t >= 0; --t) beta_step(be, a[t], b[t]);
  }
  const bool rec_beta = (w > 0) && (lo + G <= hi);
  float4* bseed = rec_beta ? reinterpret_cast<float4*>(io.seed_out + 16 * (g - 1) + 8) : nullptr;
  if (rec_beta && lo + G == hi) {
    bseed[0] = make_float4(be[0], be[1], be[2], be[3]);
    bseed[1] = make_float4(be[4], be[5], be[6], be[7]);
  }
  const uint16_t* pt = (LOWER ? io.perm : io.inv) + cb.tab;
  for (int j = nsub - 1; j >= 0; --j) {
    const int base = lo + j * S;
    float SA[S], A_[S], B_[S];
#pragma unroll
    for (int q4 = 0; q4 < S; q4 += 4) load_steps4(sys, apr, par, base + q4, SA + q4, A_ + q4, B_ + q4);
    uint16_t idx[S];
#pragma unroll
    for (int q8 = 0; q8 < S; q8 += 8) {
      const uint4 v = __ldg(reinterpret_cast<const uint4*>(pt + base + q8));
      const uint32_t w4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        idx[q8 + 2 * t] = static_cast<uint16_t>(w4[t] & 0xffffu);
        idx[q8 + 2 * t + 1] = static_cast<uint16_t>(w4[t] >> 16);
      }
    }
    float Al[S][8];
    ck.load(j, Al[0]);
#pragma unroll
    for (int t = 0; t + 1 < S; ++t) {
#pragma unroll
      for (int s = 0; s < 8; ++s) Al[t + 1][s] = Al[t][s];
      alpha_step(Al[t + 1], A_[t], B_[t]);
    }
#pragma unroll
    for (int t = S - 1; t >= 0; --t) {
      const float e = io.scale * (kLn2 * extrinsic2(Al[t], be, B_[t]));
      const int n = idx[t];
      io.ext[cb.work + n] = e;
      if (LOWER) io.post[cb.out + n] = SA[t] + e;
      beta_step(be, A_[t], B_[t]);
      if (rec_beta && base + t == lo + G) {
        bseed[0] = make_float4(be[0], be[1], be[2], be[3]);
        bseed[1] = make_float4(be[4], be[5], be[6], be[7]);
      }
    }
  }
}

}  // namespace tcb
