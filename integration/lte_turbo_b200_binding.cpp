// lte_turbo_b200_binding.cpp -- the file a maintainer of Wiseung/Turbo_CPP adds to the
// reference's CUDA build in place of src/lte_turbo_cuda.cu.  It implements the three GPU impls
// that src/lte_turbo.cpp:15-42 forward-declares under TURBO_CPP_HAS_CUDA over the C ABI of
// libturbo_b200.so (include/turbo_b200.h), so that the reference's public
// turbo_decode_code_block_gpu_stage1/2 (lte_turbo.cpp:815-889) and decode_transport_block
// with DecoderBackend::GpuStage1Exact / GpuStage2Windowed (:891-980) decode on a B200.
//
// Compile with the reference's include/ and this repository's include/ on the include path,
// C++20, TURBO_CPP_HAS_CUDA=1, and link libturbo_b200.so.  oracle/build_reference_suite.sh does
// exactly that with the unmodified src/lte_turbo.cpp and the reference's tests/test_main.cpp.
//
// Mapping: Stage 1 ("exact", lte_turbo_cuda.cu:1391-1498) and the tile8 experiment
// (:1500-1690) -> the full trellis (window = K); Stage 2 ("windowed", :1719-1899) -> the
// default windowed schedule.  Status codes become the reference's exception types
// (std::invalid_argument, std::out_of_range, std::runtime_error).
#include <algorithm>
#include <cstdint>
#include <span>
#include <stdexcept>
#include <string>
#include <vector>

#include "turbo_b200.h"
#include "turbo_cpp/lte_turbo.h"

namespace turbo_cpp {
namespace {

// One decoder per process; tc_decode serialises concurrent calls on it, so the reference's
// std::async fan-out over code blocks (lte_turbo.cpp:941-951) stays safe.
tc_decoder* decoder() {
  static tc_decoder* d = [] {
    tc_decoder* p = nullptr;
    if (tc_decoder_create(0, &p) != TC_OK) throw std::runtime_error(tc_last_error());
    return p;
  }();
  return d;
}

void raise(int rc) {
  if (rc == TC_OK) return;
  if (rc == TC_ERR_INVALID_ARGUMENT) throw std::invalid_argument(tc_last_error());
  if (rc == TC_ERR_OUT_OF_RANGE) throw std::out_of_range(tc_last_error());
  throw std::runtime_error(tc_last_error());
}

std::vector<float> decode(const CodeBlockDescriptor& d, std::span<const float> d0,
                          std::span<const float> d1, std::span<const float> d2,
                          std::uint32_t iters, bool early, bool* crc_ok, std::uint32_t* used,
                          bool full_trellis) {
  if (d0.size() != d.d_r || d1.size() != d.d_r || d2.size() != d.d_r)
    throw std::invalid_argument("invalid LLR sizes for turbo decode");
  std::vector<float> llr(3 * d.d_r), post(d.k_r);
  std::copy(d0.begin(), d0.end(), llr.begin());
  std::copy(d1.begin(), d1.end(), llr.begin() + static_cast<std::ptrdiff_t>(d.d_r));
  std::copy(d2.begin(), d2.end(), llr.begin() + static_cast<std::ptrdiff_t>(2 * d.d_r));
  tc_code_block cb{static_cast<int32_t>(d.k_r), static_cast<int32_t>(d.filler_count), 0, 0};
  tc_decode_options o;
  tc_decode_options_init(&o);
  o.max_iterations = iters;
  o.early_stop = early ? 1 : 0;
  o.window = full_trellis ? static_cast<int32_t>(d.k_r) : 0;  // 0: the default windows
  std::uint8_t ok = 0;
  std::uint32_t it = 0;
  raise(tc_decode(decoder(), 1, &cb, llr.size(), llr.data(), post.size(), post.data(), &ok, &it,
                  &o));
  if (crc_ok) *crc_ok = ok != 0;
  if (used) *used = it;
  return post;
}

}  // namespace

std::vector<float> turbo_decode_code_block_gpu_stage1_cuda_impl(
    const CodeBlockDescriptor& d, std::span<const float> d0, std::span<const float> d1,
    std::span<const float> d2, std::uint32_t it, bool es, bool* ok, std::uint32_t* used) {
  return decode(d, d0, d1, d2, it, es, ok, used, true);
}

std::vector<float> turbo_decode_code_block_gpu_stage2_cuda_impl(
    const CodeBlockDescriptor& d, std::span<const float> d0, std::span<const float> d1,
    std::span<const float> d2, std::uint32_t it, bool es, bool* ok, std::uint32_t* used) {
  return decode(d, d0, d1, d2, it, es, ok, used, false);
}

std::vector<float> turbo_decode_code_block_gpu_stage1_tile8_experimental_cuda_impl(
    const CodeBlockDescriptor& d, std::span<const float> d0, std::span<const float> d1,
    std::span<const float> d2, std::uint32_t it, bool es, bool* ok, std::uint32_t* used) {
  return decode(d, d0, d1, d2, it, es, ok, used, true);
}

}  // namespace turbo_cpp
