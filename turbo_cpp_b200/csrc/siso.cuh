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
// each, in shared memory or global scratch with the windows of a launch interleaved); the
// backward pass recomputes the S alphas of one sub-window into registers from its checkpoint
// and then runs beta + extrinsic over it.  The metrics are in the deferred-log (m, s) form of
// trellis.cuh.
#pragma once
#include <cstdint>
#include <type_traits>

#include "trellis.cuh"

#ifndef TCB_LDCG
#define TCB_LDCG 0
#endif

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
// Loads of data written earlier in the same kernel (persistent schedule): an ordinary
// (coherent, L1-cacheable) global load, never the read-only non-coherent path.  The writer
// releases and the reader acquires at GPU scope before these loads, which makes them see the
// writes even when the writer ran on another SM.
__device__ __forceinline__ float4 ld4_coherent(const float* p) {
#if TCB_LDCG
  return __ldcg(reinterpret_cast<const float4*>(p));
#else
  float4 v;
  asm volatile("ld.global.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "l"(p)
               : "memory");
  return v;
#endif
}
template <bool COHERENT>
__device__ __forceinline__ float4 ld4_io(const float* p) {
  return COHERENT ? ld4_coherent(p) : ld4(p);
}

// Raw inputs of 4 consecutive steps (one float4 per stream).  The a-priori stream is written
// by the other SISO; COHERENT reads it through L2 (needed when both run in one kernel).
struct Raw4 {
  float4 s, e, p;  // systematic, a-priori, parity
};
template <bool COHERENT = false>
__device__ __forceinline__ Raw4 load_raw4(const float* sys, const float* apr, const float* par,
                                          int q) {
  return Raw4{ld4(sys + q), ld4_io<COHERENT>(apr + q), ld4(par + q)};
}
// raw -> sys+apr (sa), a = c (sys+apr), b = c par with c = log2(e)/2
__device__ __forceinline__ void scale4(const Raw4& r, float* sa, float* a, float* b) {
  sa[0] = r.s.x + r.e.x; sa[1] = r.s.y + r.e.y; sa[2] = r.s.z + r.e.z; sa[3] = r.s.w + r.e.w;
#pragma unroll
  for (int t = 0; t < 4; ++t) a[t] = kHalfLog2e * sa[t];
  b[0] = kHalfLog2e * r.p.x; b[1] = kHalfLog2e * r.p.y; b[2] = kHalfLog2e * r.p.z;
  b[3] = kHalfLog2e * r.p.w;
}

// Raw inputs of 8 consecutive steps: both halves of each 32-byte sector are requested back to
// back, so every sector crosses from L2 once.
struct Raw8 {
  Raw4 lo, hi;
};
template <bool COHERENT = false>
__device__ __forceinline__ Raw8 load_raw8(const float* sys, const float* apr, const float* par,
                                          int q) {
  return Raw8{load_raw4<COHERENT>(sys, apr, par, q), load_raw4<COHERENT>(sys, apr, par, q + 4)};
}

// Checkpoint storage, 8 floats per checkpoint as two float4.  Shared memory: thread-minor
// float4 planes (conflict-free); global scratch: a per-thread slot.
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

// Global scratch with the windows of a launch interleaved: checkpoint plane j holds one float4
// pair per window, so the 32 lanes of a warp (consecutive windows) store and load 32
// consecutive float4 -- four whole cache lines -- per instruction.
struct CkptStrided {
  float4* p;     // this window's entry of plane 0
  int stride;    // windows of the launch (float4 between planes); the host keeps the whole
                 // slab below 2^31 float4
  __device__ __forceinline__ CkptStrided(float4* base, int n_windows, int g)
      : p(base + g), stride(n_windows) {}
  __device__ __forceinline__ void store(int j, const float (&m)[8]) const {
    p[(2 * j) * stride] = make_float4(m[0], m[1], m[2], m[3]);
    p[(2 * j + 1) * stride] = make_float4(m[4], m[5], m[6], m[7]);
  }
  __device__ __forceinline__ void load(int j, float (&m)[8]) const {
    const float4 x = p[(2 * j) * stride], y = p[(2 * j + 1) * stride];
    m[0] = x.x; m[1] = x.y; m[2] = x.z; m[3] = x.w; m[4] = y.x; m[5] = y.y; m[6] = y.z; m[7] = y.w;
  }
};

// Tail LLRs in the reference's decoder mapping (lte_turbo.cpp:758-773), or (STD) in the
// inverse of TS 36.212 5.1.3.2.2's multiplexing: upper systematic x_K..x_K+2 = d0[K], d2[K],
// d1[K+1], parity z_K..z_K+2 = d1[K], d0[K+1], d2[K+1]; lower x' = d0[K+2], d2[K+2], d1[K+3],
// z' = d1[K+2], d0[K+3], d2[K+3].
template <bool STD = false>
__device__ __forceinline__ void tail_llrs(bool lower, const float* d0, int k, float ts[3],
                                          float tp[3]) {
  const float* d1 = d0 + (k + 4);
  const float* d2 = d1 + (k + 4);
  if (STD) {
    const int o = lower ? 2 : 0;
    ts[0] = d0[k + o]; ts[1] = d2[k + o]; ts[2] = d1[k + o + 1];
    tp[0] = d1[k + o]; tp[1] = d0[k + o + 1]; tp[2] = d2[k + o + 1];
    return;
  }
  if (!lower) {
    ts[0] = d0[k]; ts[1] = d0[k + 2]; ts[2] = 0.0f;
    tp[0] = d1[k]; tp[1] = d0[k + 1]; tp[2] = d1[k + 2];
  } else {
    ts[0] = d1[k + 3]; ts[1] = d2[k]; ts[2] = d2[k + 2];
    tp[0] = d2[k + 1]; tp[1] = d0[k + 3]; tp[2] = d2[k + 3];
  }
}

constexpr float kDestMaxA = 1024.0f;

// Runs window w of block cb for one half-iteration.  g = launch-wide window index (seed slot).
// lower: the SISO over interleaved order; post (lower SISO only): also write the posterior
// Ls + e1 + e2 (last iteration, early stop).  Both may be compile-time constants (the plain
// kernels, one specialisation each) or run-time values (the persistent kernel, which keeps a
// single copy of this code for both halves).  COHERENT: a-priori and seeds were written earlier
// in the same kernel (persistent schedule).  TAPE: the alpha warm-up steps also leave
// checkpoints, at negative indexes (q - lo) / S (the caller's checkpoint store is offset by the
// warm-up), so that [a_lo, hi] is covered every S steps for the adjoint.
template <int S, class Ckpt, bool COHERENT, bool STD = false, bool SMALL_LOOPS = false,
          bool TAPE = false>
__device__ __forceinline__ void siso_window_rt(const DevCb& cb, int w, int g, const SisoIo& io,
                                               const Ckpt& ck, const bool LOWER, const bool POST) {
  static_assert(S == 4, "sub-windows are one float4 group of 4 steps");
  const int K = cb.k, W = cb.window, G = io.guard;
  const int lo = w * W, hi = min(lo + W, K);
  const float* d0 = io.llr + cb.llr;
  const float* sys = LOWER ? io.sys_i + cb.work : d0;
  const float* par = d0 + (LOWER ? 2 : 1) * (K + 4);
  const float* apr = io.apr + cb.work;
  const int nsub = (hi - lo) / S;
  float sa[4], a[4], b[4];

  // ---- forward: warm-up from a_lo, then a checkpoint every 4 steps over [lo, hi) ----
  // Metrics in (m, s) form (trellis.cuh); seeds and checkpoints are log values.
  float al[8], as[8];
  ms_ones(as);
  int a_lo = lo - G;
  if (a_lo <= 0) {
    a_lo = 0;
    alpha_start(al);
  } else {
    const float4 x = ld4_io<COHERENT>(io.seed_in + 16 * g), y = ld4_io<COHERENT>(io.seed_in + 16 * g + 4);
    al[0] = x.x; al[1] = x.y; al[2] = x.z; al[3] = x.w; al[4] = y.x; al[5] = y.y; al[6] = y.z; al[7] = y.w;
  }
  float amax = 0.0f;  // largest |a| of the window (it covers [lo, hi))
  if constexpr (SMALL_LOOPS) {  // 4-step groups; the next group is requested early
    Raw4 cur = load_raw4<COHERENT>(sys, apr, par, a_lo);
    for (int q = a_lo; q < hi; q += 4) {
      Raw4 nxt = cur;
      if (q + 4 < hi) nxt = load_raw4<COHERENT>(sys, apr, par, q + 4);
      if (TAPE || q >= lo) {
        float v[8];
        ms_to_log(al, as, v);
        ck.store((q - lo) / S, v);
      }
      scale4(cur, sa, a, b);
      amax = fmaxf(amax, fmaxf(fmaxf(fabsf(a[0]), fabsf(a[1])), fmaxf(fabsf(a[2]), fabsf(a[3]))));
#pragma unroll
      for (int t = 0; t < 4; ++t) alpha_step_ms<STD>(al, as, a[t], b[t]);
      ms_renorm(al, as);
      cur = nxt;
    }
  } else {  // 8-step groups (both halves of each sector); the next group is requested early
    Raw8 cur = load_raw8<COHERENT>(sys, apr, par, a_lo);
    for (int q = a_lo; q < hi; q += 8) {
      Raw8 nxt = cur;
      if (q + 8 < hi) nxt = load_raw8<COHERENT>(sys, apr, par, q + 8);
      float v[8];
      if (TAPE || q >= lo) {
        ms_to_log(al, as, v);
        ck.store((q - lo) / S, v);
      }
      scale4(cur.lo, sa, a, b);
      amax = fmaxf(amax, fmaxf(fmaxf(fabsf(a[0]), fabsf(a[1])), fmaxf(fabsf(a[2]), fabsf(a[3]))));
#pragma unroll
      for (int t = 0; t < 4; ++t) alpha_step_ms<STD>(al, as, a[t], b[t]);
      if (TAPE || q >= lo) {
        ms_to_log(al, as, v);
        ck.store((q - lo) / S + 1, v);
      }
      scale4(cur.hi, sa, a, b);
      amax = fmaxf(amax, fmaxf(fmaxf(fabsf(a[0]), fabsf(a[1])), fmaxf(fabsf(a[2]), fabsf(a[3]))));
#pragma unroll
      for (int t = 0; t < 4; ++t) alpha_step_ms<STD>(al, as, a[t], b[t]);
      ms_renorm(al, as);
      cur = nxt;
    }
  }
  if (!STD) {  // alpha at hi, the alpha_{t+1} of the window's last step
    float v[8];
    ms_to_log(al, as, v);
    ck.store(nsub, v);
  }
  // seed for window w+1: alpha at hi - G
  if (w + 1 < cb.nwin && hi - G > 0) {
    float r[8];
    if (G == 0) {
      ms_to_log(al, as, r);
    } else {
      ck.load((hi - G - lo) / S, r);
    }
    float4* o = reinterpret_cast<float4*>(io.seed_out + 16 * (g + 1));
    o[0] = make_float4(r[0], r[1], r[2], r[3]);
    o[1] = make_float4(r[4], r[5], r[6], r[7]);
  }

  // ---- backward: warm-up from b_hi down to hi ----
  float be[8], bs[8];
  ms_ones(bs);
  int b_hi = hi + G;
  if (b_hi >= K) {
    b_hi = K;
    float ts[3], tp[3];
    tail_llrs<STD>(LOWER, d0, K, ts, tp);
    tail_beta<STD>(be, ts, tp);
  } else {
    const float4 x = ld4_io<COHERENT>(io.seed_in + 16 * g + 8), y = ld4_io<COHERENT>(io.seed_in + 16 * g + 12);
    be[0] = x.x; be[1] = x.y; be[2] = x.z; be[3] = x.w; be[4] = y.x; be[5] = y.y; be[6] = y.z; be[7] = y.w;
  }
  if (SMALL_LOOPS && b_hi > hi) {
    Raw4 cur = load_raw4<COHERENT>(sys, apr, par, b_hi - 4);
    for (int q = b_hi - 4; q >= hi; q -= 4) {
      Raw4 nxt = cur;
      if (q - 4 >= hi) nxt = load_raw4<COHERENT>(sys, apr, par, q - 4);
      scale4(cur, sa, a, b);
#pragma unroll
      for (int t = 3; t >= 0; --t) beta_step_ms<STD>(be, bs, a[t], b[t]);
      ms_renorm(be, bs);
      cur = nxt;
    }
  }
  if (!SMALL_LOOPS && b_hi > hi) {
    Raw8 cur = load_raw8<COHERENT>(sys, apr, par, b_hi - 8);
    for (int q = b_hi - 8; q >= hi; q -= 8) {
      Raw8 nxt = cur;
      if (q - 8 >= hi) nxt = load_raw8<COHERENT>(sys, apr, par, q - 8);
      scale4(cur.hi, sa, a, b);
#pragma unroll
      for (int t = 3; t >= 0; --t) beta_step_ms<STD>(be, bs, a[t], b[t]);
      scale4(cur.lo, sa, a, b);
#pragma unroll
      for (int t = 3; t >= 0; --t) beta_step_ms<STD>(be, bs, a[t], b[t]);
      ms_renorm(be, bs);
      cur = nxt;
    }
  }
  const bool rec_beta = (w > 0) && (lo + G <= hi);
  float4* bseed = rec_beta ? reinterpret_cast<float4*>(io.seed_out + 16 * (g - 1) + 8) : nullptr;
  if (rec_beta && lo + G == hi) {
    float r[8];
    ms_to_log(be, bs, r);
    bseed[0] = make_float4(r[0], r[1], r[2], r[3]);
    bseed[1] = make_float4(r[4], r[5], r[6], r[7]);
  }

  // ---- per 4-step sub-window (last to first): recompute alpha, then beta + extrinsic.  The
  // inputs, permutation indices and checkpoint of the next sub-window are requested one
  // sub-window ahead.  The reference's code takes the extrinsic from alpha_{t+1} beta_{t+1}
  // (DEST); that form subtracts Ls + La (2a) from a posterior of about that size, which costs
  // float precision when |a| is huge, so a window whose |a| exceeds kDestMaxA (base 2; ordinary
  // decoding stays below ~300 even at 6 dB) -- and the TS 36.212 code -- take the branch form.
  // The two are separate copies of the loop, each with its own register allocation. ----
  auto backward = [&](auto dest_tag) {
  constexpr bool DEST = decltype(dest_tag)::value && !STD;
  const uint16_t* pt = (LOWER ? io.perm : io.inv) + cb.tab;
  Raw4 r_n;
  uint2 i_n;
  float c_n[8];
  float an[8];  // reference code: alpha at base + S (log values), the last step's alpha_{t+1}
  if (nsub > 0) {
    const int base = lo + (nsub - 1) * S;
    r_n = load_raw4<COHERENT>(sys, apr, par, base);
    i_n = __ldg(reinterpret_cast<const uint2*>(pt + base));
    ck.load(nsub - 1, c_n);
    if constexpr (DEST) ck.load(nsub, an);
  }
  constexpr float kOnes[8] = {1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f};
  for (int j = nsub - 1; j >= 0; --j) {
    const int base = lo + j * S;
    const Raw4 r = r_n;
    const uint2 iv = i_n;
    float Al[S][8], As[S][8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      Al[0][k] = c_n[k];
      As[0][k] = 1.0f;
    }
    if (j > 0) {
      r_n = load_raw4<COHERENT>(sys, apr, par, base - S);
      i_n = __ldg(reinterpret_cast<const uint2*>(pt + base - S));
      ck.load(j - 1, c_n);
    }
    float SA[S], A_[S], B_[S];
    scale4(r, SA, A_, B_);
#pragma unroll
    for (int t = 0; t + 1 < S; ++t) {
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        Al[t + 1][k] = Al[t][k];
        As[t + 1][k] = As[t][k];
      }
      alpha_step_ms<STD>(Al[t + 1], As[t + 1], A_[t], B_[t]);
    }
    const uint32_t w2[2] = {iv.x, iv.y};
    // step t's outputs, then beta_t
    auto finish = [&](int t, float e2) {
      const float e = io.scale * (kLn2 * e2);
      const int n = static_cast<int>((w2[t >> 1] >> (16 * (t & 1))) & 0xffffu);
      io.ext[cb.work + n] = e;
      if (POST) io.post[cb.out + n] = SA[t] + e;
      beta_step_ms<STD>(be, bs, A_[t], B_[t]);
      if (rec_beta && base + t == lo + G) {
        float rr[8];
        ms_to_log(be, bs, rr);
        bseed[0] = make_float4(rr[0], rr[1], rr[2], rr[3]);
        bseed[1] = make_float4(rr[4], rr[5], rr[6], rr[7]);
      }
    };
    if constexpr (DEST) {  // posterior from alpha_{t+1} beta_{t+1} minus Ls + La
      finish(S - 1, posterior_dest_ms(an, kOnes, be, bs) - 2.0f * A_[S - 1]);
#pragma unroll
      for (int t = S - 2; t >= 0; --t)
        finish(t, posterior_dest_ms(Al[t + 1], As[t + 1], be, bs) - 2.0f * A_[t]);
    } else {  // the TS 36.212 code, and huge LLRs: from alpha_t, gamma_t and beta_{t+1}
#pragma unroll
      for (int t = S - 1; t >= 0; --t) finish(t, extrinsic_ms<STD>(Al[t], As[t], be, bs, B_[t]));
    }
    if constexpr (DEST) {
#pragma unroll
      for (int k = 0; k < 8; ++k) an[k] = Al[0][k];
    }
    ms_renorm(be, bs);
  }
  };
  if (!STD && amax <= kDestMaxA)
    backward(std::true_type{});
  else
    backward(std::false_type{});
}

template <int S, bool LOWER, bool POST, class Ckpt, bool COHERENT = false, bool STD = false,
          bool TAPE = false>
__device__ __forceinline__ void siso_window(const DevCb& cb, int w, int g, const SisoIo& io,
                                            const Ckpt& ck) {
  siso_window_rt<S, Ckpt, COHERENT, STD, false, TAPE>(cb, w, g, io, ck, LOWER, POST);
}

}  // namespace tcb
