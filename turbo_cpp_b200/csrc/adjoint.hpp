// adjoint.hpp -- the differentiable decoder: a taped forward pass over the unrolled iterations
// with per-half-iteration extrinsic scales, and its hand-written adjoint (adjoint.cu).
//
// The differentiated function is the windowed schedule of the plain decoder (window W, guard G,
// next-iteration-initialisation seeds), no early stop, with the extrinsic of SISO j (j = 2*it
// upper, 2*it+1 lower) multiplied by scales[j] before it becomes the other SISO's a-priori and
// before it enters the posterior Ls + e1 + e2.  The seeds are constants of the function (the
// gradient stops at them); with W >= K there are none and the function is the reference's
// full-trellis decoder (turbo_decode_code_block_cpu, lte_turbo.cpp:736-813) with the scales
// inserted.  The oracle's or_adj_vjp is the same function in FP64.
#pragma once
#include <cstddef>
#include <cstdint>
#include <mutex>
#include <vector>

#include "decoder.hpp"

namespace tcb {

constexpr int kAdjWindow = 64;  // default window of the differentiable schedule
constexpr int kAdjGuard = 32;   // default guard

struct AdjointRequest {
  size_t n_cb = 0;
  const CodeBlockDesc* cbs = nullptr;  // host
  size_t llr_len = 0;
  const float* llr = nullptr;          // device; must stay unchanged until the backward pass
  size_t post_len = 0;
  float* posterior = nullptr;          // device
  uint32_t iterations = 6;
  const float* scales = nullptr;       // host, 2 per iteration; null = all 1
  int window = 0;                      // 0: kAdjWindow
  int guard = -1;                      // <0: kAdjGuard
  void* stream = nullptr;              // cudaStream_t (NULL = legacy default stream)
  bool std3gpp = false;                // the TS 36.212 code instead of the reference's
};

class Adjoint {
 public:
  explicit Adjoint(Decoder& dec) : dec_(dec) {}
  ~Adjoint();
  Adjoint(const Adjoint&) = delete;
  Adjoint& operator=(const Adjoint&) = delete;

  // Decodes and records the tape; returns the tape id that backward() must be given.
  uint64_t forward(const AdjointRequest& rq);
  // d loss / d llr and d loss / d scales of the last forward pass from d loss / d posterior.
  // grad_posterior: post_len floats in the posterior's layout; grad_llr: llr_len floats in the
  // LLR layout (positions outside every block are 0); grad_scales: 2*iterations floats.  All
  // device pointers, ordered on `stream`.
  void backward(uint64_t tape, const float* grad_posterior, float* grad_llr, float* grad_scales,
                void* stream);
  uint64_t launches() const { return launches_; }

 private:
  Decoder& dec_;
  std::mutex mu_;
  uint64_t tape_id_ = 0;
  bool have_tape_ = false;
  uint64_t launches_ = 0;
  // layout of the taped forward pass
  size_t n_cb_ = 0, llr_len_ = 0, post_len_ = 0;
  int64_t work_ = 0;
  int n_win_ = 0, guard_ = 0, ckpt_bwd_ = 0;
  uint32_t iterations_ = 0;
  bool std3gpp_ = false;
  std::vector<float> scales_;
  const float* llr_ = nullptr;
  DeviceBuffer d_cbs_, d_wincb_, d_sysi_, d_tape_, d_seeds_, d_tapeckpt_, d_ckpt_;
  DeviceBuffer d_own_, d_guard_, d_tail_, d_part_, d_cbpart_, d_ge2_, d_ga1_;
};

}  // namespace tcb
