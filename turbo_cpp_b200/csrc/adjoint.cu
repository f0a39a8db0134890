// adjoint.cu -- the hand-written adjoint of the unrolled, scaled Log-MAP iterations.
//
// Forward (taped): the plain decoder's SISO kernel, one launch per half-iteration, with the
// a-priori input and extrinsic output of every half-iteration kept in its own tape slot (slot j
// is SISO j's a-priori, slot j+1 its scaled extrinsic; slot 0 is zero), the seeds of every
// half-iteration in their own slab (SISO j reads slab j and writes slab j+2), and the alpha
// checkpoints of every half-iteration in their own slab: every 4 steps from the window's alpha
// start (seed or block start) to its end, as log values.
//
// Backward: per half-iteration, last to first, one thread per window of the forward schedule
// runs the adjoint of its window in two phases (base-2 metrics, as the forward):
//   1  backward in time from the beta start (seed or tail) to the alpha start: beta, stored
//      every 4 steps; alpha recomputed from its checkpoint 4 steps at a time; the extrinsic's
//      softmax weights give the direct alpha adjoint and d/d parity; the alpha adjoint
//      recursion (transposed softmax weights of every max*) runs through the window and on
//      through the alpha warm-up steps;
//   2  forward in time from the window start to the beta start: beta recomputed from its
//      checkpoints 4 steps at a time; the beta adjoint recursion, fed by the extrinsic's
//      direct beta adjoint, runs through the window and the beta warm-up steps to the tail.
// Per-step normalisations subtract a common value from all 8 metrics and every extrinsic is a
// difference of two log-sums over the same metrics, so they are constants of the function and
// the adjoint ignores them.  A warm-up step of one window is an output step of its neighbour, so
// each window writes its own steps' gradients and its warm-up gradients to separate arrays; a
// combine kernel (one CTA per code block) adds the three contributions of every position in a
// fixed order (the result is deterministic), adds them to d0/d1/d2 and writes the other SISO's
// a-priori adjoint, and adds the tail gradients.  d loss / d scale_j is the sum of
// d loss / d e * x over the SISO's positions (x its unscaled extrinsic), reduced per window, per
// code block and then over the blocks, each in a fixed order.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "adjoint.hpp"
#include "decode_kernels.cuh"
#include "decoder.hpp"
#include "lte_codec.hpp"

namespace tcb {
namespace {

void ok(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

constexpr int kAdjThreads = 64;

__device__ __forceinline__ float rcp(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Softmax weights of the two terms of max*(x0, x1): 2^(x0 - m), 2^(x1 - m), m = log2(2^x0 + 2^x1).
__device__ __forceinline__ void pair_weights(float x0, float x1, float& w0, float& w1) {
  const float e = ex2(-fabsf(x0 - x1));
  const float r = rcp(1.0f + e);
  const bool first = x0 >= x1;
  w0 = first ? r : e * r;
  w1 = first ? e * r : r;
}

// d(alpha_{p+1}) -> d(alpha_p): ab += J^T abn, with J the softmax weights of alpha_step at p;
// ga, gb accumulate d/da and d/db of the step's branch metrics.  (In the reference's trellis
// both predecessors of a state enter it with the same input; in the TS 36.212 one (STD) they
// differ.)
template <bool STD = false>
__device__ __forceinline__ void alpha_adjoint(const float (&al)[8], float a, float b,
                                              const float (&abn)[8], float (&ab)[8], float& ga,
                                              float& gb) {
  const float g0 = a + b, g1 = a - b;
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    const int p0 = 2 * (n & 3);
    const int u0 = pred_input<STD>(n, 0), u1 = pred_input<STD>(n, 1);
    const int par0 = pred_parity(n, 0), par1 = pred_parity(n, 1);
    float w0, w1;
    pair_weights(al[p0] + branch(u0, par0, g0, g1), al[p0 + 1] + branch(u1, par1, g0, g1), w0,
                 w1);
    const float q0 = w0 * abn[n], q1 = w1 * abn[n];
    ab[p0] += q0;
    ab[p0 + 1] += q1;
    ga += u0 == u1 ? (u0 ? (q0 + q1) : -(q0 + q1)) : (u0 ? q0 : -q0) + (u1 ? q1 : -q1);
    gb += (par0 ? q0 : -q0) + (par1 ? q1 : -q1);
  }
}

// d(beta_p) -> d(beta_{p+1}): bbn += J^T bb, J the softmax weights of beta_step at p (bn holds
// beta_{p+1}).
template <bool STD = false>
__device__ __forceinline__ void beta_adjoint(const float (&bn)[8], float a, float b,
                                             const float (&bb)[8], float (&bbn)[8], float& ga,
                                             float& gb) {
  const float g0 = a + b, g1 = a - b;
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    const int pa0 = parity<STD>(s, 0), pa1 = parity<STD>(s, 1);
    float w0, w1;
    pair_weights(bn[next_state<STD>(s, 0)] + branch(0, pa0, g0, g1),
                 bn[next_state<STD>(s, 1)] + branch(1, pa1, g0, g1), w0, w1);
    const float q0 = w0 * bb[s], q1 = w1 * bb[s];
    bbn[next_state<STD>(s, 0)] += q0;
    bbn[next_state<STD>(s, 1)] += q1;
    ga += q1 - q0;
    gb += (pa0 ? q0 : -q0) + (pa1 ? q1 : -q1);
  }
}

// Softmax weights of the two 8-way log-sums of the extrinsic (extrinsic2): w_u[s] is the weight
// of branch (s, u) in the u-side log-sum.  Returns the base-2 extrinsic when WANT_VALUE.
template <bool WANT_VALUE, bool STD = false>
__device__ __forceinline__ float ext_weights(const float (&al)[8], const float (&be)[8], float b,
                                             float (&w0)[8], float (&w1)[8]) {
  float m0[8], m1[8];
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    m0[s] = al[s] + be[next_state<STD>(s, 0)] + (parity<STD>(s, 0) ? b : -b);
    m1[s] = al[s] + be[next_state<STD>(s, 1)] + (parity<STD>(s, 1) ? b : -b);
  }
  const float x0 = fmaxf(fmaxf(fmaxf(m0[0], m0[1]), fmaxf(m0[2], m0[3])),
                         fmaxf(fmaxf(m0[4], m0[5]), fmaxf(m0[6], m0[7])));
  const float x1 = fmaxf(fmaxf(fmaxf(m1[0], m1[1]), fmaxf(m1[2], m1[3])),
                         fmaxf(fmaxf(m1[4], m1[5]), fmaxf(m1[6], m1[7])));
  float s0 = 0.0f, s1 = 0.0f;
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    w0[s] = ex2(m0[s] - x0);
    w1[s] = ex2(m1[s] - x1);
    s0 += w0[s];
    s1 += w1[s];
  }
  const float r0 = rcp(s0), r1 = rcp(s1);
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    w0[s] *= r0;
    w1[s] *= r1;
  }
  return WANT_VALUE ? (x1 - x0) + (lg2(s1) - lg2(s0)) : 0.0f;
}

// The reference code's extrinsic in the destination form of the forward decoder (trellis.cuh
// posterior_dest_ms): F = log-sum over the states entered with input 1 of alpha_{t+1} +
// beta_{t+1} minus the same over input 0, and the extrinsic is F - 2a.  w[n] = dF/d alpha_{t+1}(n)
// = dF/d beta_{t+1}(n): the softmax weight of state n within its side, positive for input 1,
// negative for input 0 (8 ex2 + 2 rcp instead of 16 ex2 + 2 rcp for the branch form).  alpha may
// be in (m, s) form (sa, log values when all 1); beta in log values.  Returns F when WANT_VALUE.
template <bool WANT_VALUE>
__device__ __forceinline__ float dest_weights(const float (&ma)[8], const float (&sa)[8],
                                              const float (&mb)[8], float (&w)[8]) {
  float v[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) v[n] = ma[n] + mb[n];
  const float x1 = fmaxf(max3(v[1], v[2], v[4]), v[7]);
  const float x0 = fmaxf(max3(v[0], v[3], v[5]), v[6]);
  float s1 = 0.0f, s0 = 0.0f;
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    const bool one = pred_input<false>(n, 0);
    w[n] = sa[n] * ex2(v[n] - (one ? x1 : x0));
    if (one) s1 += w[n]; else s0 += w[n];
  }
  const float r1 = rcp(s1), r0 = rcp(s0);
#pragma unroll
  for (int n = 0; n < 8; ++n) w[n] *= pred_input<false>(n, 0) ? r1 : -r0;
  return WANT_VALUE ? (x1 - x0) + (lg2(s1) - lg2(s0)) : 0.0f;
}

struct AdjIo {
  const float* llr;       // channel LLRs, [d0|d1|d2] per block
  const float* sys_i;     // interleaved systematic LLRs (work layout)
  const float* apr;       // the a-priori this SISO read in the forward pass (work layout)
  const float* ge;        // d loss / d (scaled extrinsic of this SISO), work layout, this SISO's
                          // order (the lower SISO's: interleaved)
  const float* seeds;     // [launch window][16]: the seeds this SISO used
  float4* alpha_ckpt;     // the taped alpha checkpoints of this SISO: ckpt_slots planes of n_win
                          // float4 pairs, plane m = alpha at a_lo + 4m
  float* own_sa;          // [work]: d loss / d(Ls+La) of the window's own steps (SISO order),
                          // phase 1's part; phase 2's part follows at own_sa + 2 * work
  float* own_par;         // [work]: d loss / d Lp (likewise)
  int64_t work;
  float* guard_g;         // [launch window][4][guard]: alpha warm-up sa, par; beta warm-up sa, par
  float* tail_g;          // [launch window][8]: d/d ts[0..2], d/d tp[0..2] (tail-started windows)
  float* scale_part;      // [launch window]: sum of ge * x over the window
  float4* ckpt;           // beta checkpoints: ckpt_slots planes of n_win float4 pairs
  int ckpt_slots;         // checkpoints of each kind per window
  float scale;
  int guard;
};

__device__ __forceinline__ void load8(const float* p, float (&m)[8]) {
  const float4 x = ld4(p), y = ld4(p + 4);
  m[0] = x.x; m[1] = x.y; m[2] = x.z; m[3] = x.w; m[4] = y.x; m[5] = y.y; m[6] = y.z; m[7] = y.w;
}

// d loss / d e of 4 consecutive positions of this SISO
__device__ __forceinline__ void load_ge(const AdjIo& io, const DevCb& cb, int q, float (&ge)[4]) {
  const float4 v = ld4(io.ge + cb.work + q);
  ge[0] = v.x; ge[1] = v.y; ge[2] = v.z; ge[3] = v.w;
}

// PHASES: 1 or 2, as separate launches (phase 2 reads what phase 1 stored in global memory): each
// holds less live state, so that 6 blocks per SM (168 registers) fit where a single kernel held
// 4 (234 registers).
constexpr int kAdjMinBlocks = 6;
template <bool LOWER, int PHASES, bool STD = false>
__global__ void __launch_bounds__(kAdjThreads, kAdjMinBlocks) siso_adjoint_kernel(const DevCb* __restrict__ cbs,
                                                                  const int32_t* __restrict__ win_cb,
                                                                  int n_win, AdjIo io) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_win) return;
  const DevCb cb = cbs[win_cb[g]];
  const int w = g - cb.win0;
  const int K = cb.k, W = cb.window, G = io.guard;
  const int lo = w * W, hi = min(lo + W, K);
  int a_lo = lo - G, b_hi = hi + G;
  const bool start = a_lo <= 0, tail = b_hi >= K;
  if (start) a_lo = 0;
  if (tail) b_hi = K;
  const float* d0 = io.llr + cb.llr;
  const float* sys = LOWER ? io.sys_i + cb.work : d0;
  const float* par = d0 + (LOWER ? 2 : 1) * (K + 4);
  const float* apr = io.apr + cb.work;
  // alpha (taped) and beta checkpoints, each a slab of planes with the launch's windows
  // interleaved
  const CkptStrided cka{io.alpha_ckpt, n_win, g};
  const CkptStrided ckb{io.ckpt, n_win, g};
  float sa[4], a[4], b[4];
  float* ag = io.guard_g + static_cast<int64_t>(4 * g) * G;
  const float xs = kLn2 * io.scale;  // d e / d(base-2 extrinsic)

  if (PHASES & 1) {
  // ---- phase 1: backward in time ----
  float be[8];
  if (tail) {
    float ts[3], tp[3];
    tail_llrs<STD>(LOWER, d0, K, ts, tp);
    tail_beta<STD>(be, ts, tp);
  } else {
    load8(io.seeds + 16 * g + 8, be);
  }
  {  // beta warm-up in (m, s) form: checkpoints (log values) at lo + 4m
    float bs[8];
    ms_ones(bs);
    for (int P = b_hi; P > hi; P -= 4) {
      float v[8];
      ms_to_log(be, bs, v);
      ckb.store((P - lo) >> 2, v);
      scale4(load_raw4(sys, apr, par, P - 4), sa, a, b);
#pragma unroll
      for (int t = 3; t >= 0; --t) beta_step_ms<STD>(be, bs, a[t], b[t]);
      ms_renorm(be, bs);
    }
    float v[8];
    ms_to_log(be, bs, v);
#pragma unroll
    for (int k = 0; k < 8; ++k) be[k] = v[k];
  }
  float ab[8];
#pragma unroll
  for (int s = 0; s < 8; ++s) ab[s] = 0.0f;
  float spart = 0.0f;
  float an[8];  // reference code: alpha at P (log values), the last step's alpha_{t+1}
  if (!STD) cka.load((hi - a_lo) >> 2, an);
  constexpr float kOnes[8] = {1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f};
  for (int P = hi; P > lo; P -= 4) {  // the window's own steps
    ckb.store((P - lo) >> 2, be);
    const int q = P - 4;
    scale4(load_raw4(sys, apr, par, q), sa, a, b);
    float ge[4];
    load_ge(io, cb, q, ge);
    float Al[4][8];
    cka.load((q - a_lo) >> 2, Al[0]);
#pragma unroll
    for (int t = 0; t < 3; ++t) {
#pragma unroll
      for (int s = 0; s < 8; ++s) Al[t + 1][s] = Al[t][s];
      alpha_step<STD>(Al[t + 1], a[t], b[t]);
    }
    float gsa[4], gpar[4];
#pragma unroll
    for (int t = 3; t >= 0; --t) {
      const float G2 = xs * ge[t];
      float nab[8], ga = 0.0f, gb = 0.0f;
      if constexpr (!STD) {  // destination form: direct adjoint on alpha_{t+1}, -2 on a_t
        float w[8];
        const float F = dest_weights<true>(t == 3 ? an : Al[t < 3 ? t + 1 : t], kOnes, be, w);
        spart += ge[t] * (kLn2 * (F - 2.0f * a[t]));
#pragma unroll
        for (int s = 0; s < 8; ++s) {
          ab[s] += G2 * w[s];
          nab[s] = 0.0f;
        }
        ga = -2.0f * G2;
      } else {
        float w0[8], w1[8];
        const float d2 = ext_weights<true, STD>(Al[t], be, b[t], w0, w1);
        spart += ge[t] * (kLn2 * d2);
#pragma unroll
        for (int s = 0; s < 8; ++s) {
          nab[s] = G2 * (w1[s] - w0[s]);
          gb += G2 * ((parity<STD>(s, 1) ? w1[s] : -w1[s]) - (parity<STD>(s, 0) ? w0[s] : -w0[s]));
        }
      }
      alpha_adjoint<STD>(Al[t], a[t], b[t], ab, nab, ga, gb);
#pragma unroll
      for (int s = 0; s < 8; ++s) ab[s] = nab[s];
      beta_step<STD>(be, a[t], b[t]);
      gsa[t] = kHalfLog2e * ga;
      gpar[t] = kHalfLog2e * gb;
    }
    *reinterpret_cast<float4*>(io.own_sa + cb.work + q) = make_float4(gsa[0], gsa[1], gsa[2], gsa[3]);
    *reinterpret_cast<float4*>(io.own_par + cb.work + q) = make_float4(gpar[0], gpar[1], gpar[2], gpar[3]);
    if (!STD) {
#pragma unroll
      for (int s = 0; s < 8; ++s) an[s] = Al[0][s];
    }
  }
  for (int P = lo; P > a_lo; P -= 4) {  // alpha warm-up steps
    const int q = P - 4;
    scale4(load_raw4(sys, apr, par, q), sa, a, b);
    float Al[4][8];
    cka.load((q - a_lo) >> 2, Al[0]);
#pragma unroll
    for (int t = 0; t < 3; ++t) {
#pragma unroll
      for (int s = 0; s < 8; ++s) Al[t + 1][s] = Al[t][s];
      alpha_step<STD>(Al[t + 1], a[t], b[t]);
    }
    float gsa[4], gpar[4];
#pragma unroll
    for (int t = 3; t >= 0; --t) {
      float nab[8], ga = 0.0f, gb = 0.0f;
#pragma unroll
      for (int s = 0; s < 8; ++s) nab[s] = 0.0f;
      alpha_adjoint<STD>(Al[t], a[t], b[t], ab, nab, ga, gb);
#pragma unroll
      for (int s = 0; s < 8; ++s) ab[s] = nab[s];
      gsa[t] = kHalfLog2e * ga;
      gpar[t] = kHalfLog2e * gb;
    }
    const int j = q - (lo - G);  // index within the G warm-up steps before lo
    *reinterpret_cast<float4*>(ag + j) = make_float4(gsa[0], gsa[1], gsa[2], gsa[3]);
    *reinterpret_cast<float4*>(ag + G + j) = make_float4(gpar[0], gpar[1], gpar[2], gpar[3]);
  }
  io.scale_part[g] = spart;
  }

  if (PHASES & 2) {
  // ---- phase 2: forward in time ----
  float bb[8], al[8], as[8];  // alpha in (m, s) form, advanced over the window's own steps
#pragma unroll
  for (int s = 0; s < 8; ++s) bb[s] = 0.0f;
  ms_ones(as);
  cka.load((lo - a_lo) >> 2, al);
  float* bg = ag + 2 * G;
  for (int P = lo; P < b_hi; P += 4) {
    scale4(load_raw4(sys, apr, par, P), sa, a, b);
    float Bt[4][8];  // Bt[t] = beta at P + t + 1
    ckb.load((P + 4 - lo) >> 2, Bt[3]);
#pragma unroll
    for (int t = 3; t > 0; --t) {
#pragma unroll
      for (int s = 0; s < 8; ++s) Bt[t - 1][s] = Bt[t][s];
      beta_step<STD>(Bt[t - 1], a[t], b[t]);
    }
    const bool own = P < hi;
    float ge[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if (own) load_ge(io, cb, P, ge);
    float gsa[4], gpar[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      float nbb[8], ga = 0.0f, gb = 0.0f;
#pragma unroll
      for (int s = 0; s < 8; ++s) nbb[s] = 0.0f;
      beta_adjoint<STD>(Bt[t], a[t], b[t], bb, nbb, ga, gb);
      if (own) {
        const float G2 = xs * ge[t];
        if constexpr (!STD) {  // destination form: direct adjoint on beta_{t+1}
          alpha_step_ms<STD>(al, as, a[t], b[t]);  // alpha_{t+1}
          float w[8];
          dest_weights<false>(al, as, Bt[t], w);
#pragma unroll
          for (int s = 0; s < 8; ++s) nbb[s] += G2 * w[s];
        } else {
          float w0[8], w1[8];
          float lal[8];
          ms_to_log(al, as, lal);
          ext_weights<false, STD>(lal, Bt[t], b[t], w0, w1);
#pragma unroll
          for (int s = 0; s < 8; ++s) {
            nbb[next_state<STD>(s, 0)] -= G2 * w0[s];
            nbb[next_state<STD>(s, 1)] += G2 * w1[s];
          }
          alpha_step_ms<STD>(al, as, a[t], b[t]);
        }
      }
#pragma unroll
      for (int s = 0; s < 8; ++s) bb[s] = nbb[s];
      gsa[t] = kHalfLog2e * ga;
      gpar[t] = kHalfLog2e * gb;
    }
    ms_renorm(al, as);
    if (own) {
      *reinterpret_cast<float4*>(io.own_sa + 2 * io.work + cb.work + P) = make_float4(gsa[0], gsa[1], gsa[2], gsa[3]);
      *reinterpret_cast<float4*>(io.own_par + 2 * io.work + cb.work + P) = make_float4(gpar[0], gpar[1], gpar[2], gpar[3]);
    } else {
      const int j = P - hi;
      *reinterpret_cast<float4*>(bg + j) = make_float4(gsa[0], gsa[1], gsa[2], gsa[3]);
      *reinterpret_cast<float4*>(bg + G + j) = make_float4(gpar[0], gpar[1], gpar[2], gpar[3]);
    }
  }
  if (tail) {  // beta at K = the termination metrics (tail_beta): d/d tail LLRs
    float gt[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int s0 = 0; s0 < 8; ++s0) {
      int s = s0;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const int u = termination_input<STD>(s);
        const int p = parity<STD>(s, u);
        gt[i] += u ? bb[s0] : -bb[s0];
        gt[3 + i] += p ? bb[s0] : -bb[s0];
        s = next_state<STD>(s, u);
      }
    }
    float* o = io.tail_g + 8 * g;
#pragma unroll
    for (int i = 0; i < 6; ++i) o[i] = kHalfLog2e * gt[i];
  }
  }
}

struct CombineIo {
  const DevCb* cbs;
  int n_cb;
  int guard;
  const float* own_sa;     // phase 1's own-step gradients; phase 2's at + 2 * work
  const float* own_par;
  int64_t work;
  const float* guard_g;
  const float* tail_g;
  const uint16_t* perm;    // interleaved position i is natural position perm[i]
  const uint16_t* inv;     // natural position q is interleaved position inv[q]
  const float* grad_post;  // posterior layout
  const float* win_part;   // [launch window]: this SISO's sum of ge * x per window
  float* grad_llr;         // LLR layout
  float* ge_out;           // upper: d/d e2 of the previous iteration (interleaved order, as the
                           // lower SISO reads it); lower: d/d e1 (natural order)
  double* cb_part;         // [code block]: the block's windows' win_part, summed in window order
};

constexpr int kMaxK = 6144;  // largest QPP block size
constexpr int kCombineThreads = 256;
constexpr int kCombineBatch = 1;  // measured best of 1, 2, 4 (registers against loads in flight)

__device__ __forceinline__ float4 add4(float4 x, float4 y) {
  return make_float4(x.x + y.x, x.y + y.y, x.z + y.z, x.w + y.w);
}
__device__ __forceinline__ float4 ldg4(const float* p) {
  return __ldg(reinterpret_cast<const float4*>(p));
}

// d loss / d(Ls+La) and d loss / d Lp at SISO positions p..p+3 (p a multiple of 4, so all four
// lie in one window and on the same side of every guard boundary, which are multiples of 8):
// their own window's gradient (phase 1's part plus phase 2's), then the alpha warm-up gradient
// of window w+1, then the beta warm-up gradient of window w-1 (a fixed order, so the result is
// deterministic).
__device__ __forceinline__ void position_grads4(const CombineIo& c, const DevCb& cb, int p,
                                                float4& sa, float4& par) {
  const int W = cb.window, G = c.guard;
  const int w = p / W, lo = w * W;
  const int64_t o = cb.work + p;
  sa = add4(ldg4(c.own_sa + o), ldg4(c.own_sa + 2 * c.work + o));
  par = add4(ldg4(c.own_par + o), ldg4(c.own_par + 2 * c.work + o));
  if (w + 1 < cb.nwin && p >= lo + W - G) {
    const float* ag = c.guard_g + static_cast<int64_t>(4 * (cb.win0 + w + 1)) * G;
    const int j = p - (lo + W - G);
    sa = add4(sa, ldg4(ag + j));
    par = add4(par, ldg4(ag + G + j));
  }
  if (w > 0 && p < lo + G) {
    const float* bg = c.guard_g + static_cast<int64_t>(4 * (cb.win0 + w - 1)) * G + 2 * G;
    const int j = p - lo;
    sa = add4(sa, ldg4(bg + j));
    par = add4(par, ldg4(bg + G + j));
  }
}

// Tail LLRs: the tail-started windows' gradients summed in window order.
template <bool LOWER, bool STD>
__device__ __forceinline__ void combine_tail(const CombineIo& c, const DevCb& cb, float* g0) {
  const int W = cb.window, G = c.guard, K = cb.k;
  float* g1 = g0 + (K + 4);
  float* g2 = g1 + (K + 4);
  float gt[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  for (int v = 0; v < cb.nwin; ++v) {
    if (min((v + 1) * W, K) + G < K) continue;
    const float* t = c.tail_g + 8 * (cb.win0 + v);
    for (int k = 0; k < 6; ++k) gt[k] += t[k];
  }
  if (STD) {  // 36.212: ts = {d0[K+o], d2[K+o], d1[K+o+1]}, tp = {d1[K+o], d0[K+o+1], d2[K+o+1]}
    const int o = LOWER ? 2 : 0;
    g0[K + o] += gt[0];
    g2[K + o] += gt[1];
    g1[K + o + 1] += gt[2];
    g1[K + o] += gt[3];
    g0[K + o + 1] += gt[4];
    g2[K + o + 1] += gt[5];
  } else if (!LOWER) {  // ts = {d0[K], d0[K+2], 0}, tp = {d1[K], d0[K+1], d1[K+2]}
    g0[K] += gt[0];
    g0[K + 2] += gt[1];
    g1[K] += gt[3];
    g0[K + 1] += gt[4];
    g1[K + 2] += gt[5];
  } else {  // ts = {d1[K+3], d2[K], d2[K+2]}, tp = {d2[K+1], d0[K+3], d2[K+3]}
    g1[K + 3] += gt[0];
    g2[K] += gt[1];
    g2[K + 2] += gt[2];
    g2[K + 1] += gt[3];
    g0[K + 3] += gt[4];
    g2[K + 3] += gt[5];
  }
}

// One block per code block.  Adds the SISO's gradients to d0/d1 (upper, natural order) or to
// d2 (lower, SISO order) and d0 (lower: gathered through the inverse permutation), and writes the
// adjoint of the a-priori, the other SISO's scaled extrinsic, in that SISO's order (upper: the
// lower SISO's interleaved order, gathered through the permutation; lower: natural order, plus
// d loss / d posterior for the last lower SISO, whose extrinsic also enters the posterior).  The
// gradients are staged in shared memory by this SISO's position, so that every global access
// walks an order of its own.  Also adds the tail gradients and sums the block's per-window scale
// parts in a fixed order.
template <bool LOWER, bool LAST, bool STD = false>
__global__ void __launch_bounds__(kCombineThreads) adj_combine_kernel(CombineIo c) {
  __shared__ __align__(16) float sa_s[kMaxK];
  __shared__ double red[kCombineThreads];
  for (int i = blockIdx.x; i < c.n_cb; i += gridDim.x) {
    const DevCb cb = c.cbs[i];
    const int K = cb.k;
    float* g0 = c.grad_llr + cb.llr;
    // 4 consecutive positions per thread (float4; offsets are multiples of 4), kCombineBatch
    // groups per pass, all loads before the stores
    float4* s4 = reinterpret_cast<float4*>(sa_s);
    float* gp = g0 + (LOWER ? 2 : 1) * (K + 4);  // parity: d1 (upper) or d2 (lower)
    for (int p0 = 4 * threadIdx.x; p0 < K; p0 += 4 * kCombineThreads * kCombineBatch) {
      float4 sa[kCombineBatch], par[kCombineBatch], g[kCombineBatch], h[kCombineBatch];
#pragma unroll
      for (int k = 0; k < kCombineBatch; ++k) {
        const int p = p0 + 4 * k * kCombineThreads;
        if (p < K) {
          position_grads4(c, cb, p, sa[k], par[k]);
          if (!LOWER) g[k] = *reinterpret_cast<const float4*>(g0 + p);
          h[k] = *reinterpret_cast<const float4*>(gp + p);
        }
      }
#pragma unroll
      for (int k = 0; k < kCombineBatch; ++k) {
        const int p = p0 + 4 * k * kCombineThreads;
        if (p < K) {
          if (!LOWER) *reinterpret_cast<float4*>(g0 + p) = add4(g[k], sa[k]);
          s4[p >> 2] = sa[k];
          *reinterpret_cast<float4*>(gp + p) = add4(h[k], par[k]);
        }
      }
    }
    if (threadIdx.x == 0) combine_tail<LOWER, STD>(c, cb, g0);
    double s = 0.0;
    for (int v = threadIdx.x; v < cb.nwin; v += kCombineThreads) s += c.win_part[cb.win0 + v];
    red[threadIdx.x] = s;
    __syncthreads();
    if (!LOWER) {
      const uint16_t* perm = c.perm + cb.tab;
      for (int i = 4 * threadIdx.x; i < K; i += 4 * kCombineThreads) {
        const uint2 v = __ldg(reinterpret_cast<const uint2*>(perm + i));
        *reinterpret_cast<float4*>(c.ge_out + cb.work + i) =
            make_float4(sa_s[v.x & 0xffffu], sa_s[v.x >> 16], sa_s[v.y & 0xffffu], sa_s[v.y >> 16]);
      }
    } else {
      const uint16_t* inv = c.inv + cb.tab;
      for (int q0 = 4 * threadIdx.x; q0 < K; q0 += 4 * kCombineThreads * kCombineBatch) {
        float4 v[kCombineBatch], g[kCombineBatch];
        float gq[kCombineBatch][4];
#pragma unroll
        for (int k = 0; k < kCombineBatch; ++k) {
          const int q = q0 + 4 * k * kCombineThreads;
          if (q < K) {
            const uint2 iv = __ldg(reinterpret_cast<const uint2*>(inv + q));
            v[k] = make_float4(sa_s[iv.x & 0xffffu], sa_s[iv.x >> 16], sa_s[iv.y & 0xffffu],
                               sa_s[iv.y >> 16]);
            g[k] = *reinterpret_cast<const float4*>(g0 + q);
#pragma unroll
            for (int e = 0; e < 4; ++e) gq[k][e] = LAST ? c.grad_post[cb.out + q + e] : 0.0f;
          }
        }
#pragma unroll
        for (int k = 0; k < kCombineBatch; ++k) {
          const int q = q0 + 4 * k * kCombineThreads;
          if (q < K) {
            *reinterpret_cast<float4*>(g0 + q) = add4(g[k], v[k]);
            *reinterpret_cast<float4*>(c.ge_out + cb.work + q) =
                make_float4(v[k].x + gq[k][0], v[k].y + gq[k][1], v[k].z + gq[k][2],
                            v[k].w + gq[k][3]);
          }
        }
      }
    }
    for (int o = kCombineThreads / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) c.cb_part[i] = red[0];
    __syncthreads();  // sa_s and red are reused by the next code block
  }
}

// grad_llr: d0 gets d loss / d posterior (posterior = Ls + e1 + e2); ge2 = d loss / d e2 of the
// last iteration, in the lower SISO's (interleaved) order.  grad_llr was zeroed before.  One CTA
// per code block: the block's d loss / d posterior is staged in shared memory and gathered
// through the permutation from there, so that every global access walks its array in order.
__global__ void __launch_bounds__(kCombineThreads) adj_init_kernel(
    const DevCb* __restrict__ cbs, int n_cb, const float* __restrict__ grad_post,
    const uint16_t* __restrict__ perm, float* __restrict__ grad_llr, float* __restrict__ ge2) {
  __shared__ float gp[kMaxK];
  for (int i = blockIdx.x; i < n_cb; i += gridDim.x) {
    const DevCb cb = cbs[i];
    for (int p = threadIdx.x; p < cb.k; p += kCombineThreads) {
      const float v = grad_post[cb.out + p];
      gp[p] = v;
      grad_llr[cb.llr + p] = v;
    }
    __syncthreads();
    const uint16_t* pi = perm + cb.tab;
    for (int p = threadIdx.x; p < cb.k; p += kCombineThreads) ge2[cb.work + p] = gp[pi[p]];
    __syncthreads();  // gp is reused by the next code block
  }
}

// grad_scales[j] = sum over code blocks of cb_part[j][block], in a fixed order (one block per j).
__global__ void adj_scale_reduce_kernel(const double* __restrict__ cb_part, int n_cb,
                                        float* __restrict__ grad_scales) {
  __shared__ double acc[256];
  const int j = blockIdx.x;
  double s = 0.0;
  for (int i = threadIdx.x; i < n_cb; i += blockDim.x) s += cb_part[static_cast<int64_t>(j) * n_cb + i];
  acc[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) acc[threadIdx.x] += acc[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) grad_scales[j] = static_cast<float>(acc[0]);
}

template <class T>
T* reserve(DeviceBuffer& b, size_t count) {
  b.reserve(count * sizeof(T));
  return static_cast<T*>(b.ptr);
}

}  // namespace

Adjoint::~Adjoint() {
  for (DeviceBuffer* b : {&d_cbs_, &d_wincb_, &d_sysi_, &d_tape_, &d_seeds_, &d_tapeckpt_, &d_ckpt_,
                          &d_own_, &d_guard_, &d_tail_, &d_part_, &d_cbpart_, &d_ge2_, &d_ga1_})
    b->release();
}

uint64_t Adjoint::forward(const AdjointRequest& rq) {
  std::lock_guard<std::mutex> lock(mu_);
  ok(cudaSetDevice(dec_.device()), "cudaSetDevice");
  cudaStream_t st = static_cast<cudaStream_t>(rq.stream);
  have_tape_ = false;
  const size_t n = rq.n_cb;
  if (n == 0) throw InvalidArgument("no code blocks");
  if (rq.iterations == 0 || rq.iterations > 64) throw InvalidArgument("iterations must be 1..64");
  if (reinterpret_cast<uintptr_t>(rq.llr) % 16 != 0)
    throw InvalidArgument("the LLR buffer must be 16-byte aligned");
  const int guard = rq.guard < 0 ? kAdjGuard : rq.guard;
  const int window_req = rq.window > 0 ? rq.window : kAdjWindow;
  if (guard % kGroup != 0) throw InvalidArgument("guard must be a multiple of 8");
  if (window_req % kGroup != 0) throw InvalidArgument("window must be a multiple of 8");

  std::vector<DevCb> cbs_(n);
  std::vector<int32_t> wincb;
  int64_t work = 0;
  int max_window = 0;
  for (size_t i = 0; i < n; ++i) {
    const int32_t k = rq.cbs[i].k;
    DevCb& d = cbs_[i];
    d.tab = dec_.table_offset(k);
    if (rq.cbs[i].filler < 0 || rq.cbs[i].filler >= k) throw InvalidArgument("invalid filler count");
    if (rq.cbs[i].llr_offset < 0 || rq.cbs[i].llr_offset % 4 != 0 ||
        static_cast<size_t>(rq.cbs[i].llr_offset) + 3 * static_cast<size_t>(k + 4) > rq.llr_len)
      throw InvalidArgument("invalid LLR offset (must be a multiple of 4 and in range)");
    if (rq.cbs[i].out_offset < 0 ||
        static_cast<size_t>(rq.cbs[i].out_offset) + static_cast<size_t>(k) > rq.post_len)
      throw InvalidArgument("invalid posterior offset");
    d.k = k;
    d.filler = rq.cbs[i].filler;
    d.window = std::min<int32_t>(window_req, k);
    if (guard > d.window && d.window < k) throw InvalidArgument("guard must not exceed the window");
    d.nwin = (k + d.window - 1) / d.window;
    d.win0 = static_cast<int32_t>(wincb.size());
    d.llr = rq.cbs[i].llr_offset;
    d.work = work;
    d.out = rq.cbs[i].out_offset;
    work += k;
    max_window = std::max(max_window, d.window);
    for (int w = 0; w < d.nwin; ++w) wincb.push_back(static_cast<int32_t>(i));
  }
  const int n_win = static_cast<int>(wincb.size());
  const uint32_t I = rq.iterations;
  n_cb_ = n;
  llr_len_ = rq.llr_len;
  post_len_ = rq.post_len;
  work_ = work;
  n_win_ = n_win;
  guard_ = guard;
  iterations_ = I;
  llr_ = rq.llr;
  std3gpp_ = rq.std3gpp;
  scales_.assign(2 * I, 1.0f);
  if (rq.scales) std::copy(rq.scales, rq.scales + 2 * I, scales_.begin());
  ckpt_bwd_ = (max_window + guard) / 4 + 1;

  DevCb* dcbs = reserve<DevCb>(d_cbs_, n);
  int32_t* dwin = reserve<int32_t>(d_wincb_, n_win);
  float* sysi = reserve<float>(d_sysi_, work);
  float* tape = reserve<float>(d_tape_, static_cast<size_t>(2 * I + 1) * work);
  const size_t slab = static_cast<size_t>(n_win) * 16;
  float* seeds = reserve<float>(d_seeds_, (2 * I + 2) * slab);
  // alpha checkpoints of every half-iteration, a slab each
  const size_t aslab = ckpt_slab(n_win, 2 * static_cast<size_t>(ckpt_bwd_));
  float4* actp = reserve<float4>(d_tapeckpt_, 2 * I * aslab);
  ok(cudaMemcpyAsync(dcbs, cbs_.data(), n * sizeof(DevCb), cudaMemcpyHostToDevice, st), "copy descriptors");
  ok(cudaMemcpyAsync(dwin, wincb.data(), n_win * sizeof(int32_t), cudaMemcpyHostToDevice, st), "copy descriptors");
  ok(cudaMemsetAsync(seeds, 0, 2 * slab * sizeof(float), st), "zero seeds");
  const uint16_t* dperm = dec_.perm_table();
  const uint16_t* dinv = dec_.inv_table();
  // sys_i and tape slot 0 (the first a-priori, zero)
  launch_setup(dcbs, static_cast<int>(n), rq.llr, dperm, sysi, tape, st);
  ok(cudaGetLastError(), "setup launch");
  launches_ += 1;
  const int blocks = (n_win + kThreads - 1) / kThreads;
  for (uint32_t j = 0; j < 2 * I; ++j) {
    const bool lower = j & 1;
    SisoIo io{rq.llr, sysi, tape + j * work, tape + (j + 1) * work,
              (j + 1 == 2 * I) ? rq.posterior : nullptr, dperm, dinv, seeds + j * slab,
              seeds + (j + 2) * slab, scales_[j], guard};
    float4* ck = actp + j * aslab;
    if (rq.std3gpp) {
      if (!lower)
        siso_plain_kernel<kSub, 0, true, true, true><<<blocks, kThreads, 0, st>>>(dcbs, dwin, n_win, io, nullptr, ck, ckpt_bwd_);
      else if (j + 1 < 2 * I)
        siso_plain_kernel<kSub, 1, true, true, true><<<blocks, kThreads, 0, st>>>(dcbs, dwin, n_win, io, nullptr, ck, ckpt_bwd_);
      else
        siso_plain_kernel<kSub, 2, true, true, true><<<blocks, kThreads, 0, st>>>(dcbs, dwin, n_win, io, nullptr, ck, ckpt_bwd_);
    } else {
      if (!lower)
        siso_plain_kernel<kSub, 0, true, false, true><<<blocks, kThreads, 0, st>>>(dcbs, dwin, n_win, io, nullptr, ck, ckpt_bwd_);
      else if (j + 1 < 2 * I)
        siso_plain_kernel<kSub, 1, true, false, true><<<blocks, kThreads, 0, st>>>(dcbs, dwin, n_win, io, nullptr, ck, ckpt_bwd_);
      else
        siso_plain_kernel<kSub, 2, true, false, true><<<blocks, kThreads, 0, st>>>(dcbs, dwin, n_win, io, nullptr, ck, ckpt_bwd_);
    }
    ok(cudaGetLastError(), "SISO launch");
    launches_ += 1;
  }
  have_tape_ = true;
  return ++tape_id_;
}

void Adjoint::backward(uint64_t tape_id, const float* grad_post, float* grad_llr,
                       float* grad_scales, void* stream) {
  std::lock_guard<std::mutex> lock(mu_);
  if (!have_tape_ || tape_id != tape_id_)
    throw InvalidArgument("the tape of this forward pass was replaced by a later forward pass");
  ok(cudaSetDevice(dec_.device()), "cudaSetDevice");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (reinterpret_cast<uintptr_t>(grad_llr) % 16 != 0)
    throw InvalidArgument("grad_llr must be 16-byte aligned");
  const int64_t work = work_;
  const int n_win = n_win_, G = guard_;
  const uint32_t I = iterations_;
  const size_t slab = static_cast<size_t>(n_win) * 16;
  float* own = reserve<float>(d_own_, 4 * static_cast<size_t>(work));
  float* guard_g = reserve<float>(d_guard_, static_cast<size_t>(n_win) * 4 * std::max(G, 4));
  float* tail_g = reserve<float>(d_tail_, static_cast<size_t>(n_win) * 8);
  float* part = reserve<float>(d_part_, static_cast<size_t>(n_win));
  double* cb_part = reserve<double>(d_cbpart_, static_cast<size_t>(2 * I) * n_cb_);
  float* ge2 = reserve<float>(d_ge2_, work);
  float* ga1 = reserve<float>(d_ga1_, work);
  float4* ckpt = reserve<float4>(d_ckpt_, ckpt_slab(n_win, 2 * static_cast<size_t>(ckpt_bwd_)));
  const size_t aslab = ckpt_slab(n_win, 2 * static_cast<size_t>(ckpt_bwd_));
  float4* actp = static_cast<float4*>(d_tapeckpt_.ptr);
  const DevCb* dcbs = static_cast<const DevCb*>(d_cbs_.ptr);
  const int32_t* dwin = static_cast<const int32_t*>(d_wincb_.ptr);
  const float* sysi = static_cast<const float*>(d_sysi_.ptr);
  const float* tape = static_cast<const float*>(d_tape_.ptr);
  const float* seeds = static_cast<const float*>(d_seeds_.ptr);
  const uint16_t* dperm = dec_.perm_table();
  const uint16_t* dinv = dec_.inv_table();
  const int n = static_cast<int>(n_cb_);
  const unsigned cb_blocks = static_cast<unsigned>(std::min(n, 1 << 20));

  ok(cudaMemsetAsync(grad_llr, 0, llr_len_ * sizeof(float), st), "zero grad_llr");
  adj_init_kernel<<<cb_blocks, kCombineThreads, 0, st>>>(dcbs, n, grad_post, dperm, grad_llr, ge2);
  ok(cudaGetLastError(), "adjoint init launch");
  launches_ += 1;
  const int blocks = (n_win + kAdjThreads - 1) / kAdjThreads;
  for (int j = static_cast<int>(2 * I) - 1; j >= 0; --j) {
    const bool lower = j & 1;
    const bool last = j + 2 >= static_cast<int>(2 * I);  // a SISO of the last iteration
    AdjIo io{llr_, sysi, tape + j * work, lower ? ge2 : ga1, seeds + j * slab,
             actp + j * aslab, own,
             own + work, work, guard_g, tail_g, part, ckpt, ckpt_bwd_,
             scales_[j], G};
    if (std3gpp_) {
      if (lower) {
        siso_adjoint_kernel<true, 1, true><<<blocks, kAdjThreads, 0, st>>>(dcbs, dwin, n_win, io);
        siso_adjoint_kernel<true, 2, true><<<blocks, kAdjThreads, 0, st>>>(dcbs, dwin, n_win, io);
      } else {
        siso_adjoint_kernel<false, 1, true><<<blocks, kAdjThreads, 0, st>>>(dcbs, dwin, n_win, io);
        siso_adjoint_kernel<false, 2, true><<<blocks, kAdjThreads, 0, st>>>(dcbs, dwin, n_win, io);
      }
    } else if (lower) {
      siso_adjoint_kernel<true, 1><<<blocks, kAdjThreads, 0, st>>>(dcbs, dwin, n_win, io);
      siso_adjoint_kernel<true, 2><<<blocks, kAdjThreads, 0, st>>>(dcbs, dwin, n_win, io);
    } else {
      siso_adjoint_kernel<false, 1><<<blocks, kAdjThreads, 0, st>>>(dcbs, dwin, n_win, io);
      siso_adjoint_kernel<false, 2><<<blocks, kAdjThreads, 0, st>>>(dcbs, dwin, n_win, io);
    }
    ok(cudaGetLastError(), "SISO adjoint launch");
    CombineIo c{dcbs, n, G, own, own + work, work, guard_g, tail_g, dperm, dinv, grad_post, part, grad_llr,
                lower ? ga1 : ge2, cb_part + static_cast<int64_t>(j) * n};
    if (std3gpp_) {
      if (lower && last)
        adj_combine_kernel<true, true, true><<<cb_blocks, kCombineThreads, 0, st>>>(c);
      else if (lower)
        adj_combine_kernel<true, false, true><<<cb_blocks, kCombineThreads, 0, st>>>(c);
      else
        adj_combine_kernel<false, false, true><<<cb_blocks, kCombineThreads, 0, st>>>(c);
    } else if (lower && last) {
      adj_combine_kernel<true, true><<<cb_blocks, kCombineThreads, 0, st>>>(c);
    } else if (lower) {
      adj_combine_kernel<true, false><<<cb_blocks, kCombineThreads, 0, st>>>(c);
    } else {
      adj_combine_kernel<false, false><<<cb_blocks, kCombineThreads, 0, st>>>(c);
    }
    ok(cudaGetLastError(), "adjoint combine launch");
    launches_ += 3;
  }
  adj_scale_reduce_kernel<<<2 * I, 256, 0, st>>>(cb_part, n, grad_scales);
  ok(cudaGetLastError(), "scale reduce launch");
  launches_ += 1;
}

}  // namespace tcb
