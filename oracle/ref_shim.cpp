// ref_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// extern "C" wrappers around the Wiseung/Turbo_CPP public C++ API
// (include/turbo_cpp/lte_turbo.h).  oracle/Makefile compiles this file together with the
// reference's own src/lte_turbo.cpp (CPU-only, TURBO_CPP_HAS_CUDA=0) into
// oracle/_ref/libturbo_ref.so.  Tests use it to pin the C restatement (turbo_oracle.c) and to
// generate golden fixtures; bench.py times ref_decode_batch as the reference CPU baseline.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <exception>
#include <span>
#include <thread>
#include <vector>

#include "turbo_cpp/lte_turbo.h"

using namespace turbo_cpp;

namespace {

std::vector<std::uint8_t> (*const kAppend[4])(std::span<const std::uint8_t>) = {
    append_crc24a, append_crc24b, append_crc16, append_crc8};
bool (*const kCheck[4])(std::span<const std::uint8_t>) = {check_crc24a, check_crc24b,
                                                           check_crc16, check_crc8};

CodeBlockDescriptor make_desc(std::int32_t k, std::int32_t filler) {
  CodeBlockDescriptor d;
  d.k_r = static_cast<std::size_t>(k);
  d.d_r = d.k_r + 4;
  d.filler_count = static_cast<std::size_t>(filler);
  const auto& q = qpp_entry_for_k(d.k_r);
  d.qpp_index = static_cast<std::size_t>(&q - qpp_interleaver_table().data());
  return d;
}

LteTurboCodecParams make_params(std::size_t tbs, std::size_t g_total, std::uint32_t rv,
                                std::uint32_t nl, std::uint32_t qm, std::uint32_t iters,
                                int early) {
  LteTurboCodecParams p;
  p.transport_block_bits = tbs;
  p.g_total = g_total;
  p.rv = rv;
  p.num_layers = nl;
  p.mod_order = qm;
  p.max_iterations = iters;
  p.enable_early_stop = early != 0;
  return p;
}

}  // namespace

extern "C" {

int ref_qpp_count() { return static_cast<int>(qpp_interleaver_table().size()); }

void ref_qpp_entry(int i, std::int32_t* k, std::int32_t* f1, std::int32_t* f2) {
  const auto& e = qpp_interleaver_table()[static_cast<std::size_t>(i)];
  *k = static_cast<std::int32_t>(e.k);
  *f1 = static_cast<std::int32_t>(e.f1);
  *f2 = static_cast<std::int32_t>(e.f2);
}

int ref_qpp_perm(std::int32_t k, std::int32_t* perm) {
  try {
    const auto p = qpp_permutation(static_cast<std::size_t>(k));
    for (std::size_t i = 0; i < p.size(); ++i) perm[i] = static_cast<std::int32_t>(p[i]);
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

void ref_crc_append(int kind, const std::uint8_t* bits, std::size_t n, std::uint8_t* out) {
  const auto v = kAppend[kind](std::span<const std::uint8_t>(bits, n));
  std::memcpy(out, v.data(), v.size());
}

int ref_crc_check(int kind, const std::uint8_t* bits, std::size_t n) {
  return kCheck[kind](std::span<const std::uint8_t>(bits, n)) ? 1 : 0;
}

// info[7] = {c, c_plus, c_minus, k_plus, k_minus, filler, l}
int ref_segment(const std::uint8_t* bits, std::size_t b, std::int64_t* info,
                std::uint8_t* cb_out) {
  try {
    const auto s = segment_transport_block(std::span<const std::uint8_t>(bits, b));
    const std::size_t v[7] = {s.c, s.c_plus, s.c_minus, s.k_plus, s.k_minus, s.filler_bits, s.l};
    for (int i = 0; i < 7; ++i) info[i] = static_cast<std::int64_t>(v[i]);
    if (cb_out) {
      std::size_t pos = 0;
      for (const auto& blk : s.code_blocks) {
        std::memcpy(cb_out + pos, blk.data(), blk.size());
        pos += blk.size();
      }
    }
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

int ref_turbo_encode(std::int32_t k, std::int32_t filler, const std::uint8_t* cb,
                     std::uint8_t* d0, std::uint8_t* d1, std::uint8_t* d2) {
  try {
    const auto e = turbo_encode_code_block(make_desc(k, filler),
                                           std::span<const std::uint8_t>(cb, k));
    std::memcpy(d0, e.systematic.data(), e.systematic.size());
    std::memcpy(d1, e.parity0.data(), e.parity0.size());
    std::memcpy(d2, e.parity1.data(), e.parity1.size());
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

// The reference encoder's tail arrays (EncodedCodeBlock upper/lower tail systematic/parity,
// lte_turbo.cpp:655-685) in that order, 3 bytes each.
int ref_turbo_encode_tails(std::int32_t k, std::int32_t filler, const std::uint8_t* cb,
                           std::uint8_t* tails) {
  try {
    const auto e = turbo_encode_code_block(make_desc(k, filler),
                                           std::span<const std::uint8_t>(cb, k));
    for (int i = 0; i < 3; ++i) {
      tails[i] = e.upper_tail_systematic[i];
      tails[3 + i] = e.upper_tail_parity[i];
      tails[6 + i] = e.lower_tail_systematic[i];
      tails[9 + i] = e.lower_tail_parity[i];
    }
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

// Full transport-block encode.  Per code block r: cb_k[r], cb_filler[r], cb_e[r]; the rate
// matched bits of all blocks back to back in rm_out (capacity rm_cap).
int ref_encode_tb(std::size_t tbs, std::size_t g_total, std::uint32_t rv, std::uint32_t nl,
                  std::uint32_t qm, const std::uint8_t* bits, std::int32_t* n_cb,
                  std::int32_t* cb_k, std::int32_t* cb_filler, std::int64_t* cb_e,
                  std::int32_t cb_cap, std::uint8_t* rm_out, std::size_t rm_cap) {
  try {
    const auto p = make_params(tbs, g_total, rv, nl, qm, 8, 0);
    const auto enc = encode_transport_block(p, std::span<const std::uint8_t>(bits, tbs));
    if (static_cast<std::int32_t>(enc.code_blocks.size()) > cb_cap) return -2;
    *n_cb = static_cast<std::int32_t>(enc.code_blocks.size());
    std::size_t pos = 0;
    for (std::size_t r = 0; r < enc.code_blocks.size(); ++r) {
      const auto& b = enc.code_blocks[r];
      cb_k[r] = static_cast<std::int32_t>(b.descriptor.k_r);
      cb_filler[r] = static_cast<std::int32_t>(b.descriptor.filler_count);
      cb_e[r] = static_cast<std::int64_t>(b.descriptor.e_r);
      if (pos + b.rate_matched_bits.size() > rm_cap) return -3;
      std::memcpy(rm_out + pos, b.rate_matched_bits.data(), b.rate_matched_bits.size());
      pos += b.rate_matched_bits.size();
    }
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

int ref_derate_bits(std::int32_t k, std::int32_t filler, std::uint32_t rv,
                    const std::uint8_t* e_bits, std::size_t e, float* out) {
  try {
    auto p = make_params(0, 0, rv, 1, 2, 8, 0);
    auto d = make_desc(k, filler);
    d.e_r = e;
    const auto v = derate_match_code_block(p, d, std::span<const std::uint8_t>(e_bits, e));
    std::memcpy(out, v.data(), v.size() * sizeof(float));
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

int ref_decode_cb(std::int32_t k, std::int32_t filler, const float* llr,
                  std::int32_t max_iterations, int early_stop, float* posterior, int* crc_ok,
                  std::int32_t* iterations_used) {
  try {
    const auto d = make_desc(k, filler);
    const std::size_t dr = d.d_r;
    bool ok = false;
    std::uint32_t used = 0;
    const auto post = turbo_decode_code_block_cpu(
        d, std::span<const float>(llr, dr), std::span<const float>(llr + dr, dr),
        std::span<const float>(llr + 2 * dr, dr), static_cast<std::uint32_t>(max_iterations),
        early_stop != 0, &ok, &used);
    std::memcpy(posterior, post.data(), post.size() * sizeof(float));
    if (crc_ok) *crc_ok = ok ? 1 : 0;
    if (iterations_used) *iterations_used = static_cast<std::int32_t>(used);
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

// Many independent code blocks, one per task, on `threads` std::threads (0 = all cores).
// Each call of turbo_decode_code_block_cpu stays single threaded, as in the reference.
int ref_decode_batch(std::int32_t n, const std::int32_t* k, const std::int32_t* filler,
                     const std::int64_t* llr_off, const float* llr, const std::int64_t* out_off,
                     float* posterior, std::int32_t max_iterations, int early_stop,
                     int* crc_ok, std::int32_t* iterations_used, int threads) {
  if (threads <= 0) threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
  threads = std::min(threads, std::max(n, 1));
  std::atomic<std::int32_t> next{0};
  std::atomic<int> failed{0};
  auto work = [&] {
    for (;;) {
      const std::int32_t i = next.fetch_add(1);
      if (i >= n) return;
      int ok = 0;
      std::int32_t used = 0;
      if (ref_decode_cb(k[i], filler[i], llr + llr_off[i], max_iterations, early_stop,
                        posterior + out_off[i], &ok, &used) != 0)
        failed.store(1);
      if (crc_ok) crc_ok[i] = ok;
      if (iterations_used) iterations_used[i] = used;
    }
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) pool.emplace_back(work);
  for (auto& t : pool) t.join();
  return failed.load() ? -1 : 0;
}

// decode_transport_block(params, encode_transport_block(params, bits), CpuReference):
// tb_out receives TBS bits, cb_crc_ok per block, posterior (sum K) and flags.
int ref_roundtrip_tb(std::size_t tbs, std::size_t g_total, std::uint32_t rv, std::uint32_t nl,
                     std::uint32_t qm, std::uint32_t iters, int early, const std::uint8_t* bits,
                     std::uint8_t* tb_out, int* tb_crc_ok, std::int32_t* iterations_used,
                     float* posterior, std::size_t post_cap) {
  try {
    const auto p = make_params(tbs, g_total, rv, nl, qm, iters, early);
    const auto enc = encode_transport_block(p, std::span<const std::uint8_t>(bits, tbs));
    const auto dec = decode_transport_block(p, enc, DecoderBackend::CpuReference);
    std::memcpy(tb_out, dec.tb_bits.data(), dec.tb_bits.size());
    *tb_crc_ok = dec.transport_block_crc_ok ? 1 : 0;
    *iterations_used = static_cast<std::int32_t>(dec.iterations_used);
    if (posterior) {
      if (dec.posterior_llr->size() > post_cap) return -2;
      std::memcpy(posterior, dec.posterior_llr->data(), dec.posterior_llr->size() * sizeof(float));
    }
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

}  // extern "C"
