// turbo_b200.hpp -- the reference's C++ API (namespace turbo_cpp, include/turbo_cpp/lte_turbo.h)
// over the C ABI of libturbo_b200.so, header-only, C++20.
//
// A program written against turbo_cpp switches by including this header, using namespace
// turbo_b200 instead of turbo_cpp and linking libturbo_b200.so: the types, function names,
// argument meaning and exception classes are the reference's (std::invalid_argument,
// std::out_of_range, std::runtime_error).  Differences:
//  * there is no CPU decoder: turbo_decode_code_block_cpu is not provided and
//    DecoderBackend::CpuReference is refused (std::invalid_argument);
//  * every GPU backend decodes with the exact Log-MAP of the reference's CPU decoder
//    (GpuStage1Exact / tile8: full trellis; GpuStage2Windowed and GpuB200*: the windowed
//    schedule with a 96-step guard, within 1e-3 of the full trellis), honours early stop, and
//    decode_transport_block decodes all code blocks of a transport block in one GPU call;
//  * DecoderBackend has two more values (GpuB200Plain, GpuB200Persistent: the two batched
//    schedules), and decode_code_blocks decodes any number of code blocks at once.
// The GPU is device 0 unless set_device() is called before the first decode.
#pragma once

#include <array>
#include <cstddef>
#include <cstdint>
#include <mutex>
#include <optional>
#include <span>
#include <stdexcept>
#include <string>
#include <vector>

#include "turbo_b200.h"

namespace turbo_b200 {

// ---- types (lte_turbo.h:13-92) ----
enum class LteChannelType { UL_SCH, DL_SCH, PCH, MCH };

enum class DecoderBackend {
  CpuReference,
  GpuStage1Exact,
  GpuStage2Windowed,
  GpuB200Plain,
  GpuB200Persistent,
};

struct LteTurboCodecParams {
  LteChannelType channel_type = LteChannelType::DL_SCH;
  std::size_t transport_block_bits = 0;
  std::size_t g_total = 0;
  std::uint32_t rv = 0;
  std::uint32_t num_layers = 1;
  std::uint32_t mod_order = 2;
  std::size_t n_soft = 0;
  std::uint32_t max_iterations = 8;
  bool enable_early_stop = false;
  // new: TC_CONVENTION_REFERENCE (the reference's code) or TC_CONVENTION_3GPP (TS 36.212)
  std::uint32_t convention = TC_CONVENTION_REFERENCE;
};

struct CodeBlockDescriptor {
  std::size_t block_index = 0;
  std::size_t k_r = 0;
  std::size_t d_r = 0;
  std::size_t e_r = 0;
  std::size_t filler_count = 0;
  std::size_t qpp_index = 0;
};

struct EncodedCodeBlock {
  CodeBlockDescriptor descriptor;
  std::vector<std::uint8_t> cb_bits;
  std::vector<std::uint8_t> systematic;
  std::vector<std::uint8_t> parity0;
  std::vector<std::uint8_t> parity1;
  std::array<std::uint8_t, 3> upper_tail_systematic{};
  std::array<std::uint8_t, 3> upper_tail_parity{};
  std::array<std::uint8_t, 3> lower_tail_systematic{};
  std::array<std::uint8_t, 3> lower_tail_parity{};
  std::vector<std::uint8_t> rate_matched_bits;
};

struct EncodedTransportBlock {
  LteTurboCodecParams params;
  std::vector<std::uint8_t> tb_bits_with_crc;
  std::vector<EncodedCodeBlock> code_blocks;
  std::vector<std::uint8_t> transport_bits;
};

struct DecodedTransportBlock {
  std::vector<std::uint8_t> tb_bits;
  std::vector<bool> code_block_crc_ok;
  bool transport_block_crc_ok = false;
  std::uint32_t iterations_used = 0;
  std::optional<std::vector<float>> posterior_llr;
};

struct QppEntry {
  std::size_t k = 0;
  std::size_t f1 = 0;
  std::size_t f2 = 0;
};

struct SegmentationResult {
  std::size_t c = 0;
  std::size_t c_plus = 0;
  std::size_t c_minus = 0;
  std::size_t k_plus = 0;
  std::size_t k_minus = 0;
  std::size_t filler_bits = 0;
  std::size_t l = 0;
  std::vector<std::vector<std::uint8_t>> code_blocks;
};

namespace detail {

// C ABI status -> the reference's exception classes
inline void check(int rc) {
  if (rc == TC_OK) return;
  const std::string msg = tc_last_error();
  if (rc == TC_ERR_INVALID_ARGUMENT) throw std::invalid_argument(msg);
  if (rc == TC_ERR_OUT_OF_RANGE) throw std::out_of_range(msg);
  throw std::runtime_error(std::string(tc_status_name(rc)) + ": " + msg);
}

inline int& device_index() {
  static int device = 0;
  return device;
}

// one decoder per process (its calls are serialised inside the library)
inline tc_decoder* decoder() {
  struct Holder {
    tc_decoder* h = nullptr;
    ~Holder() {
      if (h) tc_decoder_destroy(h);
    }
  };
  static std::mutex mu;
  static Holder holder;
  std::lock_guard<std::mutex> lock(mu);
  if (!holder.h) check(tc_decoder_create(device_index(), &holder.h));
  return holder.h;
}

inline std::vector<std::uint8_t> crc_append(int kind, std::span<const std::uint8_t> bits,
                                            std::size_t len, std::uint32_t conv) {
  std::vector<std::uint8_t> out(bits.size() + len);
  check(tc_crc_append_conv(static_cast<int>(conv), kind, bits.data(), bits.size(), out.data()));
  return out;
}

inline bool crc_check(int kind, std::span<const std::uint8_t> bits, std::uint32_t conv) {
  int ok = 0;
  check(tc_crc_check_conv(static_cast<int>(conv), kind, bits.data(), bits.size(), &ok));
  return ok != 0;
}

}  // namespace detail

// Selects the GPU of the decode functions; call it before the first decode.
inline void set_device(int device) { detail::device_index() = device; }

// ---- QPP interleaver (lte_turbo.h:94-95, 108-109) ----
inline std::span<const QppEntry> qpp_interleaver_table() {
  static const std::vector<QppEntry> table = [] {
    std::vector<QppEntry> t(static_cast<std::size_t>(tc_qpp_table_size()));
    for (std::size_t i = 0; i < t.size(); ++i) {
      int32_t k = 0, f1 = 0, f2 = 0;
      detail::check(tc_qpp_entry(static_cast<int>(i), &k, &f1, &f2));
      t[i] = QppEntry{static_cast<std::size_t>(k), static_cast<std::size_t>(f1),
                      static_cast<std::size_t>(f2)};
    }
    return t;
  }();
  return table;
}

inline const QppEntry& qpp_entry_for_k(std::size_t k) {
  int32_t index = 0;
  detail::check(tc_qpp_index(static_cast<int32_t>(k), &index));
  return qpp_interleaver_table()[static_cast<std::size_t>(index)];
}

inline std::vector<std::size_t> qpp_permutation(std::size_t k) {
  std::vector<int32_t> p(k);
  detail::check(tc_qpp_permutation(static_cast<int32_t>(k), p.data()));
  return std::vector<std::size_t>(p.begin(), p.end());
}

inline std::vector<std::size_t> qpp_inverse_permutation(std::size_t k) {
  std::vector<int32_t> p(k);
  detail::check(tc_qpp_inverse_permutation(static_cast<int32_t>(k), p.data()));
  return std::vector<std::size_t>(p.begin(), p.end());
}

// ---- CRC (lte_turbo.h:97-104); conv (new): TC_CONVENTION_3GPP for the TS 36.212 generators ----
constexpr std::uint32_t kRef = TC_CONVENTION_REFERENCE;
inline std::vector<std::uint8_t> append_crc24a(std::span<const std::uint8_t> b, std::uint32_t conv = kRef) { return detail::crc_append(TC_CRC24A, b, 24, conv); }
inline std::vector<std::uint8_t> append_crc24b(std::span<const std::uint8_t> b, std::uint32_t conv = kRef) { return detail::crc_append(TC_CRC24B, b, 24, conv); }
inline std::vector<std::uint8_t> append_crc16(std::span<const std::uint8_t> b, std::uint32_t conv = kRef) { return detail::crc_append(TC_CRC16, b, 16, conv); }
inline std::vector<std::uint8_t> append_crc8(std::span<const std::uint8_t> b, std::uint32_t conv = kRef) { return detail::crc_append(TC_CRC8, b, 8, conv); }
inline bool check_crc24a(std::span<const std::uint8_t> b, std::uint32_t conv = kRef) { return detail::crc_check(TC_CRC24A, b, conv); }
inline bool check_crc24b(std::span<const std::uint8_t> b, std::uint32_t conv = kRef) { return detail::crc_check(TC_CRC24B, b, conv); }
inline bool check_crc16(std::span<const std::uint8_t> b, std::uint32_t conv = kRef) { return detail::crc_check(TC_CRC16, b, conv); }
inline bool check_crc8(std::span<const std::uint8_t> b, std::uint32_t conv = kRef) { return detail::crc_check(TC_CRC8, b, conv); }

// ---- segmentation (lte_turbo.h:106): the K- blocks first, then the K+ blocks ----
inline SegmentationResult segment_transport_block(std::span<const std::uint8_t> bits_with_crc,
                                                  std::uint32_t conv = kRef) {
  tc_segmentation info{};
  const int c = static_cast<int>(conv);
  detail::check(tc_segment_transport_block_conv(c, bits_with_crc.data(), bits_with_crc.size(),
                                                &info, nullptr, 0));
  std::vector<std::uint8_t> all(info.c_plus * info.k_plus + info.c_minus * info.k_minus);
  detail::check(tc_segment_transport_block_conv(c, bits_with_crc.data(), bits_with_crc.size(),
                                                &info, all.data(), all.size()));
  SegmentationResult out{info.c, info.c_plus, info.c_minus, info.k_plus, info.k_minus,
                         info.filler_bits, info.l, {}};
  std::size_t pos = 0;
  for (std::size_t r = 0; r < info.c; ++r) {
    const std::size_t kr = r < info.c_minus ? info.k_minus : info.k_plus;
    out.code_blocks.emplace_back(all.begin() + static_cast<std::ptrdiff_t>(pos),
                                 all.begin() + static_cast<std::ptrdiff_t>(pos + kr));
    pos += kr;
  }
  return out;
}

// ---- encoder and rate matching (lte_turbo.h:111-118) ----
// The tail bits, reference code: each encoder's termination input is s1^s2 (feedback 0), so its
// third input is always 0 and its third parity equals its second input; the multiplexed streams
// (d0, d1, d2 tails) carry the rest.  TS 36.212 code: the twelve tail bits are all in the
// streams (5.1.3.2.2), x_K..x_K+2 = d0[K], d2[K], d1[K+1] and z_K..z_K+2 = d1[K], d0[K+1],
// d2[K+1] for the upper encoder, the same two positions on for the lower one.
inline EncodedCodeBlock turbo_encode_code_block(const CodeBlockDescriptor& descriptor,
                                                std::span<const std::uint8_t> cb_bits,
                                                std::uint32_t conv = kRef) {
  if (cb_bits.size() != descriptor.k_r) throw std::invalid_argument("code block length mismatch");
  const std::size_t k = descriptor.k_r;
  std::vector<std::uint8_t> d(3 * (k + 4));
  detail::check(tc_turbo_encode_conv(static_cast<int>(conv), static_cast<int32_t>(k),
                                     static_cast<int32_t>(descriptor.filler_count), cb_bits.data(),
                                     d.data()));
  EncodedCodeBlock out;
  out.descriptor = descriptor;
  out.descriptor.d_r = k + 4;
  out.cb_bits.assign(cb_bits.begin(), cb_bits.end());
  const auto at = [&](std::size_t s) { return d.begin() + static_cast<std::ptrdiff_t>(s * (k + 4)); };
  out.systematic.assign(at(0), at(1));
  out.parity0.assign(at(1), at(2));
  out.parity1.assign(at(2), at(3));
  const std::uint8_t* d0 = d.data();
  const std::uint8_t* d1 = d0 + (k + 4);
  const std::uint8_t* d2 = d1 + (k + 4);
  if (conv == TC_CONVENTION_3GPP) {
    out.upper_tail_systematic = {d0[k], d2[k], d1[k + 1]};
    out.upper_tail_parity = {d1[k], d0[k + 1], d2[k + 1]};
    out.lower_tail_systematic = {d0[k + 2], d2[k + 2], d1[k + 3]};
    out.lower_tail_parity = {d1[k + 2], d0[k + 3], d2[k + 3]};
    return out;
  }
  out.upper_tail_systematic = {d0[k], d0[k + 2], 0};
  out.upper_tail_parity = {d1[k], d0[k + 1], d0[k + 3]};
  out.lower_tail_systematic = {d1[k + 3], d2[k + 1], d2[k + 3]};
  out.lower_tail_parity = {d2[k], d2[k + 2], d2[k + 1]};
  return out;
}

inline EncodedTransportBlock encode_transport_block(const LteTurboCodecParams& params,
                                                    std::span<const std::uint8_t> transport_bits) {
  if (params.transport_block_bits != transport_bits.size())
    throw std::invalid_argument("transport block size does not match params");
  EncodedTransportBlock out;
  out.params = params;
  out.transport_bits.assign(transport_bits.begin(), transport_bits.end());
  out.tb_bits_with_crc = append_crc24a(transport_bits, params.convention);
  const SegmentationResult seg = segment_transport_block(out.tb_bits_with_crc, params.convention);
  for (std::size_t r = 0; r < seg.code_blocks.size(); ++r) {
    const auto& bits = seg.code_blocks[r];
    CodeBlockDescriptor desc;
    desc.block_index = r;
    desc.k_r = bits.size();
    desc.d_r = bits.size() + 4;
    detail::check(tc_compute_e(r, params.g_total, seg.c, params.num_layers, params.mod_order,
                               &desc.e_r));
    desc.filler_count = r == 0 ? seg.filler_bits : 0;
    int32_t qi = 0;
    detail::check(tc_qpp_index(static_cast<int32_t>(desc.k_r), &qi));
    desc.qpp_index = static_cast<std::size_t>(qi);
    EncodedCodeBlock enc = turbo_encode_code_block(desc, bits, params.convention);
    std::vector<std::uint8_t> d012(enc.systematic);
    d012.insert(d012.end(), enc.parity0.begin(), enc.parity0.end());
    d012.insert(d012.end(), enc.parity1.begin(), enc.parity1.end());
    enc.rate_matched_bits.resize(desc.e_r);
    detail::check(tc_rate_match(static_cast<int32_t>(desc.k_r), static_cast<int32_t>(desc.filler_count),
                                d012.data(), desc.e_r, params.rv, enc.rate_matched_bits.data()));
    out.code_blocks.push_back(std::move(enc));
  }
  return out;
}

// hard bits -> [d0|d1|d2] LLRs of +-8 per received bit (lte_turbo.h:116-118)
inline std::vector<float> derate_match_code_block(const LteTurboCodecParams& params,
                                                  const CodeBlockDescriptor& descriptor,
                                                  std::span<const std::uint8_t> rate_matched_bits) {
  std::vector<float> out(3 * (descriptor.k_r + 4));
  detail::check(tc_derate_match_bits(static_cast<int32_t>(descriptor.k_r),
                                     static_cast<int32_t>(descriptor.filler_count),
                                     rate_matched_bits.data(), rate_matched_bits.size(), params.rv,
                                     out.data()));
  return out;
}

// ---- GPU decoding ----
// Any number of code blocks in one call: ks[i] / fillers[i], their [d0|d1|d2] LLRs back to back
// in `llr`; returns the K posterior LLRs per block back to back.
inline std::vector<float> decode_code_blocks(std::span<const std::size_t> ks,
                                             std::span<const std::size_t> fillers,
                                             std::span<const float> llr,
                                             std::uint32_t max_iterations, bool enable_early_stop,
                                             DecoderBackend backend,
                                             std::vector<bool>* crc_ok = nullptr,
                                             std::vector<std::uint32_t>* iterations_used = nullptr,
                                             std::uint32_t conv = kRef) {
  if (backend == DecoderBackend::CpuReference)
    throw std::invalid_argument("CPU decoding is not part of turbo_b200; use a GPU backend");
  if (fillers.size() != ks.size()) throw std::invalid_argument("one filler count per block");
  std::vector<tc_code_block> cbs(ks.size());
  int64_t lo = 0, po = 0;
  for (std::size_t i = 0; i < ks.size(); ++i) {
    cbs[i] = tc_code_block{static_cast<int32_t>(ks[i]), static_cast<int32_t>(fillers[i]), lo, po};
    lo += 3 * static_cast<int64_t>(ks[i] + 4);
    po += static_cast<int64_t>(ks[i]);
  }
  if (static_cast<std::size_t>(lo) != llr.size())
    throw std::invalid_argument("invalid LLR sizes for turbo decode");
  tc_decode_options o;
  detail::check(tc_decode_options_init(&o));
  o.max_iterations = max_iterations;
  o.early_stop = enable_early_stop ? 1u : 0u;
  o.window = backend == DecoderBackend::GpuStage1Exact ? 6144 : 0;
  o.schedule = backend == DecoderBackend::GpuB200Persistent ? TC_SCHEDULE_PERSISTENT
                                                            : TC_SCHEDULE_PLAIN;
  o.convention = conv;
  std::vector<float> post(static_cast<std::size_t>(po));
  std::vector<std::uint8_t> ok(ks.size());
  std::vector<std::uint32_t> used(ks.size());
  detail::check(tc_decode(detail::decoder(), ks.size(), cbs.data(), llr.size(), llr.data(),
                          post.size(), post.data(), ok.data(), used.data(), &o));
  if (crc_ok) crc_ok->assign(ok.begin(), ok.end());
  if (iterations_used) *iterations_used = used;
  return post;
}

namespace detail {
inline std::vector<float> decode_one(const CodeBlockDescriptor& descriptor,
                                     std::span<const float> d0, std::span<const float> d1,
                                     std::span<const float> d2, std::uint32_t max_iterations,
                                     bool enable_early_stop, bool* crc_ok,
                                     std::uint32_t* iterations_used, DecoderBackend backend) {
  const std::size_t d = descriptor.k_r + 4;
  if (d0.size() != d || d1.size() != d || d2.size() != d)
    throw std::invalid_argument("invalid LLR sizes for turbo decode");
  std::vector<float> llr(d0.begin(), d0.end());
  llr.insert(llr.end(), d1.begin(), d1.end());
  llr.insert(llr.end(), d2.begin(), d2.end());
  const std::size_t k[1] = {descriptor.k_r}, f[1] = {descriptor.filler_count};
  std::vector<bool> ok;
  std::vector<std::uint32_t> used;
  auto post = decode_code_blocks(k, f, llr, max_iterations, enable_early_stop, backend, &ok, &used);
  if (crc_ok) *crc_ok = ok[0];
  if (iterations_used) *iterations_used = used[0];
  return post;
}
}  // namespace detail

// turbo_decode_code_block_gpu_stage1/2 and the tile8 variant (lte_turbo.h:129-155): Stage 1
// and tile8 decode the full trellis, Stage 2 the windowed schedule.
inline std::vector<float> turbo_decode_code_block_gpu_stage1(
    const CodeBlockDescriptor& descriptor, std::span<const float> d0_llr,
    std::span<const float> d1_llr, std::span<const float> d2_llr, std::uint32_t max_iterations,
    bool enable_early_stop, bool* crc_ok = nullptr, std::uint32_t* iterations_used = nullptr) {
  return detail::decode_one(descriptor, d0_llr, d1_llr, d2_llr, max_iterations, enable_early_stop,
                            crc_ok, iterations_used, DecoderBackend::GpuStage1Exact);
}

inline std::vector<float> turbo_decode_code_block_gpu_stage2(
    const CodeBlockDescriptor& descriptor, std::span<const float> d0_llr,
    std::span<const float> d1_llr, std::span<const float> d2_llr, std::uint32_t max_iterations,
    bool enable_early_stop, bool* crc_ok = nullptr, std::uint32_t* iterations_used = nullptr) {
  return detail::decode_one(descriptor, d0_llr, d1_llr, d2_llr, max_iterations, enable_early_stop,
                            crc_ok, iterations_used, DecoderBackend::GpuStage2Windowed);
}

inline std::vector<float> turbo_decode_code_block_gpu_stage1_tile8_experimental(
    const CodeBlockDescriptor& descriptor, std::span<const float> d0_llr,
    std::span<const float> d1_llr, std::span<const float> d2_llr, std::uint32_t max_iterations,
    bool enable_early_stop, bool* crc_ok = nullptr, std::uint32_t* iterations_used = nullptr) {
  return turbo_decode_code_block_gpu_stage1(descriptor, d0_llr, d1_llr, d2_llr, max_iterations,
                                            enable_early_stop, crc_ok, iterations_used);
}

// decode_transport_block (lte_turbo.h:157-159): all code blocks in one GPU call, then hard
// decisions (>= 0 -> 1), the first block's filler dropped, CRC24B checked and stripped when
// C > 1, blocks concatenated, CRC24A checked; iterations_used is the largest of the blocks.
inline DecodedTransportBlock decode_transport_block(const LteTurboCodecParams& params,
                                                    const EncodedTransportBlock& encoded,
                                                    DecoderBackend backend) {
  std::vector<std::size_t> ks, fillers;
  std::vector<float> llr;
  for (const auto& b : encoded.code_blocks) {
    ks.push_back(b.descriptor.k_r);
    fillers.push_back(b.descriptor.filler_count);
    const auto l = derate_match_code_block(params, b.descriptor, b.rate_matched_bits);
    llr.insert(llr.end(), l.begin(), l.end());
  }
  std::vector<std::uint32_t> used;
  DecodedTransportBlock out;
  out.posterior_llr =
      decode_code_blocks(ks, fillers, llr, params.max_iterations, params.enable_early_stop,
                         backend, nullptr, &used, params.convention);
  std::vector<std::uint8_t> tb;
  std::size_t pos = 0;
  for (std::size_t i = 0; i < ks.size(); ++i) {
    out.iterations_used = std::max(out.iterations_used, used[i]);
    std::vector<std::uint8_t> hard;
    for (std::size_t j = fillers[i]; j < ks[i]; ++j)
      hard.push_back((*out.posterior_llr)[pos + j] >= 0.0f ? 1u : 0u);
    pos += ks[i];
    bool ok = true;
    if (ks.size() > 1) {
      ok = check_crc24b(hard, params.convention);
      hard.resize(hard.size() - 24);
    }
    tb.insert(tb.end(), hard.begin(), hard.end());
    out.code_block_crc_ok.push_back(ok);
  }
  out.transport_block_crc_ok = check_crc24a(tb, params.convention);
  out.tb_bits.assign(tb.begin(), tb.end() - 24);
  return out;
}

inline std::string to_string(LteChannelType channel_type) {
  switch (channel_type) {
    case LteChannelType::UL_SCH: return "UL_SCH";
    case LteChannelType::DL_SCH: return "DL_SCH";
    case LteChannelType::PCH: return "PCH";
    case LteChannelType::MCH: return "MCH";
  }
  throw std::invalid_argument("unknown LTE channel type");
}

}  // namespace turbo_b200
