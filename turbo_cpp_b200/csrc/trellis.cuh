// trellis.cuh -- device-side exact Log-MAP arithmetic for the LTE constituent code.
//
// Metrics are kept in the base-2 log domain (natural-log metric * log2(e)), so that the
// Jacobian logarithm max*(x, y) = max(x, y) + log2(1 + 2^-|x-y|) costs one ex2 and one lg2
// (the MUFU instructions ex2.approx / lg2.approx) and no scaling multiplies.  The branch metric
// of the reference, 0.5 * (+-(Ls+La) +- Lp) (lte_turbo.cpp:437-438), becomes +-a +-b with
// a = 0.5*log2(e)*(Ls+La) and b = 0.5*log2(e)*Lp.
//
// Trellis (lte_turbo.cpp:333-341): state = (s2 s1 s0), s2 the newest register, feedback
// fb = u^s1^s2, parity fb^s0^s2, next state (fb s2 s1).  Hence next state n = (n2 n1 n0) is
// reached from the two predecessors 2*(n&3) + x, x in {0,1}, with input u = n2^n1^n0 and
// parities n2^n1^x.  The TS 36.212 code (template flag STD; not the reference's convention)
// feeds back the two oldest registers, fb = u^s0^s1 (g0 = 1 + D^2 + D^3); its parity is the
// same fb^s0^s2 and its next state the same (fb s2 s1), so only the inputs change: predecessor
// x reaches n with u = n2^n0^x.  All state/branch indexing below is resolved at compile time.
#pragma once
#include <cstdint>



namespace tcb {

constexpr float kLog2e = 1.4426950408889634f;
constexpr float kLn2 = 0.6931471805599453f;
constexpr float kHalfLog2e = 0.5f * kLog2e;
// Stand-in for -infinity: finite, so that max*(-inf, -inf) stays well defined
// (d = 0 instead of NaN) while 2^(kNegBig - m) underflows to exactly 0.
constexpr float kNegBig = -1.0e30f;

__device__ __forceinline__ float ex2(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float lg2(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Three-input maximum (one sm_100 instruction) and the maximum of 8 values in four.
__device__ __forceinline__ float max3(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ float max8(const float (&v)[8]) {
  return fmaxf(max3(v[0], v[1], v[2]), max3(v[3], v[4], max3(v[5], v[6], v[7])));
}

// Jacobian logarithm in base 2: log2(2^x + 2^y).
__device__ __forceinline__ float max_star(float x, float y) {
  const float m = fmaxf(x, y);
  const float d = fabsf(x - y);
  return m + lg2(1.0f + ex2(-d));
}

template <bool STD = false>
__host__ __device__ constexpr int feedback(int s, int u) {
  return STD ? (u ^ (s & 1) ^ ((s >> 1) & 1)) : (u ^ ((s >> 1) & 1) ^ ((s >> 2) & 1));
}
template <bool STD = false>
__host__ __device__ constexpr int next_state(int s, int u) {
  return (feedback<STD>(s, u) << 2) | (((s >> 2) & 1) << 1) | ((s >> 1) & 1);
}
template <bool STD = false>
__host__ __device__ constexpr int parity(int s, int u) {
  return feedback<STD>(s, u) ^ (s & 1) ^ ((s >> 2) & 1);
}
// the termination input of state s: the one that makes the feedback 0
template <bool STD = false>
__host__ __device__ constexpr int termination_input(int s) {
  return STD ? ((s & 1) ^ ((s >> 1) & 1)) : (((s >> 1) & 1) ^ ((s >> 2) & 1));
}
// input and parity of the branch from predecessor 2*(n&3) + x into next state n
template <bool STD = false>
__host__ __device__ constexpr int pred_input(int n, int x) {
  return STD ? (((n >> 2) & 1) ^ (n & 1) ^ x) : (((n >> 2) & 1) ^ ((n >> 1) & 1) ^ (n & 1));
}
__host__ __device__ constexpr int pred_parity(int n, int x) {
  return ((n >> 2) & 1) ^ ((n >> 1) & 1) ^ x;
}
// branch metric +-a +-b for input u and parity p: g0 = a+b, g1 = a-b
__device__ __forceinline__ float branch(int u, int p, float g0, float g1) {
  return u ? (p ? g0 : g1) : (p ? -g1 : -g0);
}

// alpha_{t+1} from alpha_t (in place); normalised so that state 0 is 0.
template <bool STD = false>
__device__ __forceinline__ void alpha_step(float (&al)[8], float a, float b) {
  const float g0 = a + b, g1 = a - b;
  float an[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    const int p0 = 2 * (n & 3);
    an[n] = max_star(al[p0] + branch(pred_input<STD>(n, 0), pred_parity(n, 0), g0, g1),
                     al[p0 + 1] + branch(pred_input<STD>(n, 1), pred_parity(n, 1), g0, g1));
  }
  const float r = an[0];
  al[0] = 0.0f;  // an[0] - an[0]
#pragma unroll
  for (int s = 1; s < 8; ++s) al[s] = an[s] - r;
}

// beta_t from beta_{t+1} (in place); normalised so that state 0 is 0.
template <bool STD = false>
__device__ __forceinline__ void beta_step(float (&be)[8], float a, float b) {
  const float g0 = a + b, g1 = a - b;
  float bn[8];
#pragma unroll
  for (int s = 0; s < 8; ++s)
    bn[s] = max_star(be[next_state<STD>(s, 0)] + branch(0, parity<STD>(s, 0), g0, g1),
                     be[next_state<STD>(s, 1)] + branch(1, parity<STD>(s, 1), g0, g1));
  const float r = bn[0];
  be[0] = 0.0f;  // bn[0] - bn[0]
#pragma unroll
  for (int s = 1; s < 8; ++s) be[s] = bn[s] - r;
}

// Extrinsic LLR (base-2) of one step: log-sum over the u=1 branches minus log-sum over the
// u=0 branches of alpha_t + beta_{t+1} +- b.  The +-a part is common to each side and is the
// (Ls+La) term the reference subtracts again (lte_turbo.cpp:483), so it is left out.
// Each 8-way log-sum is max + lg2(sum 2^(m - max)): 8 ex2 + 1 lg2 instead of 7 pairwise max*.
template <bool STD = false>
__device__ __forceinline__ float extrinsic2(const float (&al)[8], const float (&be)[8], float b) {
  float m0[8], m1[8];
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    m0[s] = al[s] + be[next_state<STD>(s, 0)] + (parity<STD>(s, 0) ? b : -b);
    m1[s] = al[s] + be[next_state<STD>(s, 1)] + (parity<STD>(s, 1) ? b : -b);
  }
  float x0 = fmaxf(fmaxf(fmaxf(m0[0], m0[1]), fmaxf(m0[2], m0[3])),
                   fmaxf(fmaxf(m0[4], m0[5]), fmaxf(m0[6], m0[7])));
  float x1 = fmaxf(fmaxf(fmaxf(m1[0], m1[1]), fmaxf(m1[2], m1[3])),
                   fmaxf(fmaxf(m1[4], m1[5]), fmaxf(m1[6], m1[7])));
  float s0 = 0.0f, s1 = 0.0f;
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    s0 += ex2(m0[s] - x0);
    s1 += ex2(m1[s] - x1);
  }
  return (x1 - x0) + (lg2(s1) - lg2(s0));
}

// beta at the block end from the three termination steps (lte_turbo.cpp:343-378): from each
// state the tail input is the one that zeroes the feedback, which drives every state to 0 in
// three steps.  ts/tp are the tail systematic / parity LLRs of this SISO.
template <bool STD = false>
__device__ __forceinline__ void tail_beta(float (&be)[8], const float ts[3], const float tp[3]) {
#pragma unroll
  for (int s0 = 0; s0 < 8; ++s0) {
    int s = s0;
    float m = 0.0f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const int u = termination_input<STD>(s);
      const int p = parity<STD>(s, u);
      m += (u ? ts[i] : -ts[i]) + (p ? tp[i] : -tp[i]);
      s = next_state<STD>(s, u);
    }
    be[s0] = m * kHalfLog2e;
  }
  const float r = be[0];
#pragma unroll
  for (int s = 1; s < 8; ++s) be[s] -= r;
  be[0] = 0.0f;
}

__device__ __forceinline__ void alpha_start(float (&al)[8]) {
  al[0] = 0.0f;
#pragma unroll
  for (int s = 1; s < 8; ++s) al[s] = kNegBig;
}

// ------------------------------------------------------------------------------------------
// Deferred-logarithm form of the recursions.  A state metric is a pair (m, s) standing for the
// base-2 log value m + log2(s), s >= 1.  The Jacobian logarithm of two branches x = (mx, sx),
// y = (my, sy) is then exact without a logarithm:
//     log2(sx 2^mx + sy 2^my) = max(mx, my) + log2(s_hi + s_lo 2^-|mx - my|),
// where s_hi belongs to the larger m and s_lo to the other: one ex2 and one FMA per state and
// step instead of an ex2 and an lg2.  s grows by at most a factor of two per step and is folded
// back into m (its binary exponent, integer operations only) every few steps; the log values
// m + lg2(s) are formed only where metrics leave the thread (seeds, checkpoints).  The values
// are the same Jacobian logarithms as max_star's, up to float rounding.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void ms_join(float x, float y, float sx, float sy, float& m, float& s) {
  const float d = x - y;
  const float t = ex2(-fabsf(d));
  const bool c = d >= 0.0f;
  s = fmaf(c ? sy : sx, t, c ? sx : sy);
  m = fmaxf(x, y);
}

// alpha_{t+1} from alpha_t in (m, s) form, normalised by the largest incoming metric, as the
// reference normalises by the largest metric (lte_turbo.cpp:392-402): the likely states stay
// near 0, where float rounding is finest.  The normalisation goes through the branch metrics
// (a - r, -a - r with r = max(m), sm_100's three-input max.f32: 10 instructions instead of a
// 14-instruction normalisation of the outputs); every value is shift-invariant.  (Normalising
// to state 0 instead puts the likely states at state 0's offset, which on LLRs in the
// thousands was measured to cost their precision.)
template <bool STD = false>
__device__ __forceinline__ void alpha_step_ms(float (&m)[8], float (&s)[8], float a, float b) {
  const float r = max8(m);
  const float ap = a - r, am = -a - r;
  float mn[8], sn[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    const int p0 = 2 * (n & 3);
    const float bx = (pred_input<STD>(n, 0) ? ap : am) + (pred_parity(n, 0) ? b : -b);
    const float by = (pred_input<STD>(n, 1) ? ap : am) + (pred_parity(n, 1) ? b : -b);
    ms_join(m[p0] + bx, m[p0 + 1] + by, s[p0], s[p0 + 1], mn[n], sn[n]);
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    m[k] = mn[k];
    s[k] = sn[k];
  }
}

// beta_t from beta_{t+1} in (m, s) form, normalised through the branch metrics as alpha_step_ms.
template <bool STD = false>
__device__ __forceinline__ void beta_step_ms(float (&m)[8], float (&s)[8], float a, float b) {
  const float r = max8(m);
  const float ap = a - r, am = -a - r;
  float mn[8], sn[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int n0 = next_state<STD>(k, 0), n1 = next_state<STD>(k, 1);
    ms_join(m[n0] + (am + (parity<STD>(k, 0) ? b : -b)),
            m[n1] + (ap + (parity<STD>(k, 1) ? b : -b)), s[n0], s[n1], mn[k], sn[k]);
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    m[k] = mn[k];
    s[k] = sn[k];
  }
}

// Folds the binary exponent of each s (s >= 1) into its m, leaving s in [1, 2).
__device__ __forceinline__ void ms_renorm(float (&m)[8], float (&s)[8]) {
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int bits = __float_as_int(s[k]);
    const int e = (bits >> 23) - 127;
    s[k] = __int_as_float(bits - (e << 23));
    m[k] += static_cast<float>(e);
  }
}

// (m, s) -> log values m + lg2(s), normalised by their largest value.
__device__ __forceinline__ void ms_to_log(const float (&m)[8], const float (&s)[8], float (&v)[8]) {
  float r[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) r[k] = m[k] + lg2(s[k]);
  const float x = max8(r);
#pragma unroll
  for (int k = 0; k < 8; ++k) v[k] = r[k] - x;
}

__device__ __forceinline__ void ms_ones(float (&s)[8]) {
#pragma unroll
  for (int k = 0; k < 8; ++k) s[k] = 1.0f;
}

// Posterior LLR (base 2) of step t of the reference's code from alpha_{t+1} and beta_{t+1} in
// (m, s) form.  In that trellis the input of a branch is fixed by the state it enters
// (u = n2^n1^n0, pred_input), so the log-sum over the u-branches of alpha_t + gamma_t +
// beta_{t+1} equals the log-sum over the states n with that input of alpha_{t+1}(n) +
// beta_{t+1}(n): two 4-way log-sums, each max + lg2(sum s_a s_b 2^(m - max)).  Any common shift
// of alpha_{t+1} or beta_{t+1} cancels.  The extrinsic is this minus (Ls + La), as the reference
// computes it (lte_turbo.cpp:483).  Not for the TS 36.212 code (its input depends on the
// predecessor as well).
__device__ __forceinline__ float posterior_dest_ms(const float (&ma)[8], const float (&sa)[8],
                                                   const float (&mb)[8], const float (&sb)[8]) {
  float v[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) v[n] = ma[n] + mb[n];
  // states entered with input 1: {1, 2, 4, 7}; with input 0: {0, 3, 5, 6}
  const float x1 = fmaxf(max3(v[1], v[2], v[4]), v[7]);
  const float x0 = fmaxf(max3(v[0], v[3], v[5]), v[6]);
  float s1 = 0.0f, s0 = 0.0f;
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    const float w = sa[n] * sb[n];
    if (pred_input<false>(n, 0)) s1 = fmaf(w, ex2(v[n] - x1), s1);
    else s0 = fmaf(w, ex2(v[n] - x0), s0);
  }
  return (x1 - x0) + (lg2(s1) - lg2(s0));
}

// Extrinsic LLR (base 2) of one step from alpha_t and beta_{t+1} in (m, s) form: the same
// two 8-way log-sums as extrinsic2, each max + lg2(sum s_a s_b 2^(m - max)).
template <bool STD = false>
__device__ __forceinline__ float extrinsic_ms(const float (&ma)[8], const float (&sa)[8],
                                              const float (&mb)[8], const float (&sb)[8],
                                              float b) {
  float m0[8], m1[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    m0[k] = ma[k] + mb[next_state<STD>(k, 0)] + (parity<STD>(k, 0) ? b : -b);
    m1[k] = ma[k] + mb[next_state<STD>(k, 1)] + (parity<STD>(k, 1) ? b : -b);
  }
  const float x0 = max8(m0), x1 = max8(m1);
  float s0 = 0.0f, s1 = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    s0 = fmaf(sa[k] * sb[next_state<STD>(k, 0)], ex2(m0[k] - x0), s0);
    s1 = fmaf(sa[k] * sb[next_state<STD>(k, 1)], ex2(m1[k] - x1), s1);
  }
  return (x1 - x0) + (lg2(s1) - lg2(s0));
}

}  // namespace tcb
