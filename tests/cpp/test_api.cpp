// The reference's own test cases (tests/test_main.cpp of Wiseung/Turbo_CPP: CRC, QPP table,
// segmentation, transport-block round trips through every GPU backend) run against the C++ API
// of this library (include/turbo_b200.hpp), plus checks of what that API adds.  The CPU
// decoder of the reference, which those cases compare the GPU posteriors with, is the oracle
// (oracle/turbo_oracle.c, bitwise equal to it).  Parity bar: |gpu - cpu| <= 1e-3 max(|cpu|, 1),
// and on the reference's own noise-free round trips (±8 LLRs) a tighter 2e-5 max(|cpu|, 1):
// the same exact Log-MAP in other float arithmetic agrees there to ~1.5e-6 (a few ulps of
// posteriors up to ~640; the reference's own Stage-1 check asks 2e-5 absolute, about one ulp).
//
//   test_api cpu   -- codec cases only (no GPU)
//   test_api gpu   -- codec and decoder cases
// An optional second argument is the reference library (oracle/_ref/libturbo_ref.so) used to
// check the encoder's tail arrays.
#include <dlfcn.h>

#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "turbo_b200.hpp"

extern "C" void or_decode_cb(int32_t k, int32_t filler, const float* llr, int32_t max_iterations,
                             int32_t early_stop, float* posterior, int32_t* crc_ok,
                             int32_t* iterations_used);
extern "C" void or_std_decode_cb_windowed(int32_t k, int32_t filler, const float* llr,
                                          int32_t max_iterations, int32_t early_stop,
                                          int32_t window, int32_t guard, float* posterior,
                                          int32_t* crc_ok, int32_t* iterations_used);

namespace tb = turbo_b200;

namespace {

int g_checks = 0;

void expect(bool cond, const std::string& what) {
  ++g_checks;
  if (!cond) throw std::runtime_error(what);
}

template <class E, class F>
void expect_throw(F&& f, const std::string& what) {
  ++g_checks;
  try {
    f();
  } catch (const E&) {
    return;
  }
  throw std::runtime_error("expected exception: " + what);
}

std::vector<std::uint8_t> pattern(std::size_t n, std::size_t a, std::size_t c) {
  std::vector<std::uint8_t> v(n);
  for (std::size_t i = 0; i < n; ++i) v[i] = static_cast<std::uint8_t>((i * a + c) & 1u);
  return v;
}

void crc_cases() {
  const std::vector<std::uint8_t> bits = {1, 0, 1, 1, 0, 1, 0, 0, 1, 1, 0, 1};
  const auto a = tb::append_crc24a(bits), b = tb::append_crc24b(bits), c = tb::append_crc16(bits),
             d = tb::append_crc8(bits);
  expect(a.size() == 36 && b.size() == 36 && c.size() == 28 && d.size() == 20, "CRC lengths");
  expect(tb::check_crc24a(a) && tb::check_crc24b(b) && tb::check_crc16(c) && tb::check_crc8(d),
         "CRC round trips");
  auto bad = a;
  bad[3] ^= 1u;
  expect(!tb::check_crc24a(bad), "CRC24A detects a flipped bit");
  expect(std::equal(bits.begin(), bits.end(), a.begin()), "CRC keeps the payload");
}

void qpp_cases() {
  const auto t = tb::qpp_interleaver_table();
  expect(t.size() == 188, "QPP table size");
  expect(t.front().k == 40 && t.front().f1 == 3 && t.front().f2 == 10, "QPP first entry");
  expect(t.back().k == 6144 && t.back().f1 == 263 && t.back().f2 == 480, "QPP last entry");
  expect(tb::qpp_entry_for_k(1024).f1 == 31 && tb::qpp_entry_for_k(1024).f2 == 64, "QPP K=1024");
  expect_throw<std::out_of_range>([] { tb::qpp_entry_for_k(44); }, "unsupported K");
  const auto p = tb::qpp_permutation(6144), q = tb::qpp_inverse_permutation(6144);
  bool inv = true;
  for (std::size_t i = 0; i < p.size(); ++i) inv &= q[p[i]] == i;
  expect(inv, "QPP inverse permutation");
}

void segmentation_cases() {
  const auto s40 = tb::segment_transport_block(std::vector<std::uint8_t>(40, 1u));
  expect(s40.c == 1 && s40.code_blocks.front().size() == 40, "B=40 stays one block");
  const auto s = tb::segment_transport_block(std::vector<std::uint8_t>(6145, 0u));
  expect(s.c > 1 && s.filler_bits > 0, "B=6145 segments with filler");
  std::size_t total = 0;
  for (const auto& b : s.code_blocks) total += b.size();
  expect(total == s.c_plus * s.k_plus + s.c_minus * s.k_minus, "segment sizes");
  expect(total == 6145 + 24 * s.c + s.filler_bits - (s.c > 1 ? 0 : 24), "segment bit count");
}

void encoder_cases(const char* ref_lib) {
  using TailsFn = int (*)(int32_t, int32_t, const std::uint8_t*, std::uint8_t*);
  TailsFn ref_tails = nullptr;
  if (ref_lib) {
    void* h = dlopen(ref_lib, RTLD_NOW | RTLD_LOCAL);
    if (h) ref_tails = reinterpret_cast<TailsFn>(dlsym(h, "ref_turbo_encode_tails"));
  }
  std::mt19937 rng(7);
  const auto table = tb::qpp_interleaver_table();
  for (int rep = 0; rep < 40; ++rep) {
    const std::size_t k = table[rng() % table.size()].k;
    const std::size_t f = (rep % 3 == 0) ? 8 : 0;
    std::vector<std::uint8_t> bits(k);
    for (auto& x : bits) x = static_cast<std::uint8_t>(rng() & 1u);
    for (std::size_t i = 0; i < f; ++i) bits[i] = 0;
    tb::CodeBlockDescriptor d;
    d.k_r = k;
    d.filler_count = f;
    const auto e = tb::turbo_encode_code_block(d, bits);
    expect(e.systematic.size() == k + 4 && e.parity0.size() == k + 4 && e.parity1.size() == k + 4 &&
               e.descriptor.d_r == k + 4,
           "encoded stream sizes");
    // the multiplexed tails carry the tail arrays (lte_turbo.cpp:664-677)
    expect(e.systematic[k] == e.upper_tail_systematic[0] && e.systematic[k + 1] == e.upper_tail_parity[1] &&
               e.systematic[k + 2] == e.upper_tail_systematic[1] && e.systematic[k + 3] == e.upper_tail_parity[2] &&
               e.parity0[k + 3] == e.lower_tail_systematic[0] && e.parity1[k] == e.lower_tail_parity[0],
           "tail multiplexing");
    if (ref_tails) {
      std::uint8_t t[12];
      expect(ref_tails(static_cast<int32_t>(k), static_cast<int32_t>(f), bits.data(), t) == 0,
             "reference encoder");
      for (int i = 0; i < 3; ++i)
        expect(t[i] == e.upper_tail_systematic[i] && t[3 + i] == e.upper_tail_parity[i] &&
                   t[6 + i] == e.lower_tail_systematic[i] && t[9 + i] == e.lower_tail_parity[i],
               "tail arrays equal the reference encoder's");
    }
  }
  tb::CodeBlockDescriptor d;
  d.k_r = 40;
  expect_throw<std::invalid_argument>([&] { tb::turbo_encode_code_block(d, std::vector<std::uint8_t>(39)); },
                                      "code block length mismatch");
  tb::LteTurboCodecParams p;
  p.transport_block_bits = 41;
  expect_throw<std::invalid_argument>([&] { tb::encode_transport_block(p, std::vector<std::uint8_t>(40)); },
                                      "TBS mismatch");
  // reference roundtrip_small: de-rate-matched systematic LLR signs follow the encoded bits
  p.transport_block_bits = 40;
  p.g_total = 3 * (64 + 4);
  p.max_iterations = 6;
  const auto enc = tb::encode_transport_block(p, pattern(40, 7, 3));
  const auto& blk = enc.code_blocks.front();
  const auto llr = tb::derate_match_code_block(p, blk.descriptor, blk.rate_matched_bits);
  bool same = true;
  for (std::size_t i = 0; i < blk.descriptor.k_r; ++i)
    same &= (blk.systematic[i] ? 1 : -1) == (llr[i] >= 0.0f ? 1 : -1);
  expect(same, "systematic LLR signs after de-rate matching");
  expect(tb::to_string(tb::LteChannelType::DL_SCH) == "DL_SCH", "channel type name");
}

// The TS 36.212 code (TC_CONVENTION_3GPP, an addition of this API): the published check values
// of the 36.212 CRCs on ASCII "123456789", and the encoder's tail arrays against a constituent
// encoder written here from g0 = 1 + D^2 + D^3, g1 = 1 + D + D^3.
void std3gpp_codec_cases() {
  std::vector<std::uint8_t> msg;
  for (char ch : std::string("123456789"))
    for (int b = 7; b >= 0; --b) msg.push_back(static_cast<std::uint8_t>((ch >> b) & 1));
  const auto last = [](const std::vector<std::uint8_t>& v, std::size_t n) {
    std::uint32_t r = 0;
    for (std::size_t i = v.size() - n; i < v.size(); ++i) r = (r << 1) | v[i];
    return r;
  };
  const std::uint32_t c3 = TC_CONVENTION_3GPP;
  expect(last(tb::append_crc24a(msg, c3), 24) == 0xCDE703u, "36.212 CRC24A check value");
  expect(last(tb::append_crc24b(msg, c3), 24) == 0x23EF52u, "36.212 CRC24B check value");
  expect(last(tb::append_crc16(msg, c3), 16) == 0x31C3u, "36.212 CRC16 check value");
  expect(last(tb::append_crc8(msg, c3), 8) == 0xEAu, "36.212 CRC8 check value");
  expect(tb::check_crc24a(tb::append_crc24a(msg, c3), c3) && !tb::check_crc24a(tb::append_crc24a(msg, c3)),
         "36.212 CRC24A is not the reference's");
  for (std::size_t k : {40u, 1056u, 6144u}) {
    const auto bits = pattern(k, 13, 1);
    tb::CodeBlockDescriptor d;
    d.k_r = k;
    const auto enc = tb::turbo_encode_code_block(d, bits, c3);
    const auto perm = tb::qpp_permutation(k);
    for (int lower = 0; lower < 2; ++lower) {
      int r1 = 0, r2 = 0, r3 = 0;  // delayed by D, D^2, D^3
      bool parity_ok = true;
      for (std::size_t i = 0; i < k; ++i) {
        const int u = lower ? bits[perm[i]] : bits[i];
        const int a = u ^ r2 ^ r3;
        const int z = a ^ r1 ^ r3;
        parity_ok &= z == (lower ? enc.parity1[i] : enc.parity0[i]);
        r3 = r2; r2 = r1; r1 = a;
      }
      std::array<std::uint8_t, 3> xs{}, zs{};
      for (int t = 0; t < 3; ++t) {
        xs[t] = static_cast<std::uint8_t>(r2 ^ r3);
        zs[t] = static_cast<std::uint8_t>(r1 ^ r3);  // register input 0
        r3 = r2; r2 = r1; r1 = 0;
      }
      const std::string tag = "36.212 encoder K=" + std::to_string(k) + (lower ? " lower" : " upper");
      expect(parity_ok, tag + ": parity");
      expect(xs == (lower ? enc.lower_tail_systematic : enc.upper_tail_systematic), tag + ": tail x");
      expect(zs == (lower ? enc.lower_tail_parity : enc.upper_tail_parity), tag + ": tail z");
    }
  }
}

double rel_err(const std::vector<float>& got, const std::vector<float>& ref) {
  double worst = 0.0;
  for (std::size_t i = 0; i < ref.size(); ++i)
    worst = std::max(worst, std::fabs(double(got[i]) - ref[i]) / std::max(1.0, std::fabs(double(ref[i]))));
  return worst;
}

// The reference's round-trip cases (test_main.cpp) through every GPU backend, with the CPU
// decoder's posterior as the reference.
void roundtrip_case(std::size_t tbs, std::size_t a, std::size_t c, bool g_from_blocks,
                    std::size_t g_total) {
  tb::LteTurboCodecParams p;
  p.transport_block_bits = tbs;
  p.max_iterations = 6;
  const auto bits = pattern(tbs, a, c);
  if (g_from_blocks) {
    g_total = 0;
    for (const auto& b : tb::segment_transport_block(tb::append_crc24a(bits)).code_blocks)
      g_total += 3 * (b.size() + 4);
  }
  p.g_total = g_total;
  const auto enc = tb::encode_transport_block(p, bits);
  // CPU decoder (oracle) posterior per block
  std::vector<float> cpu;
  for (const auto& b : enc.code_blocks) {
    const auto llr = tb::derate_match_code_block(p, b.descriptor, b.rate_matched_bits);
    std::vector<float> post(b.descriptor.k_r);
    int32_t ok = 0, it = 0;
    or_decode_cb(static_cast<int32_t>(b.descriptor.k_r), static_cast<int32_t>(b.descriptor.filler_count),
                 llr.data(), 6, 0, post.data(), &ok, &it);
    cpu.insert(cpu.end(), post.begin(), post.end());
  }
  for (auto be : {tb::DecoderBackend::GpuStage1Exact, tb::DecoderBackend::GpuStage2Windowed,
                  tb::DecoderBackend::GpuB200Plain, tb::DecoderBackend::GpuB200Persistent}) {
    const auto dec = tb::decode_transport_block(p, enc, be);
    const std::string tag = "TBS " + std::to_string(tbs) + " backend " + std::to_string(int(be));
    expect(dec.tb_bits == bits, tag + ": round trip");
    expect(dec.transport_block_crc_ok, tag + ": TB CRC");
    expect(dec.posterior_llr && dec.posterior_llr->size() == cpu.size(), tag + ": posterior size");
    bool finite = true;
    for (float v : *dec.posterior_llr) finite &= std::isfinite(v);
    expect(finite, tag + ": finite posterior");
    const double err = rel_err(*dec.posterior_llr, cpu);
    expect(err <= 2e-5, tag + ": posterior vs CPU decoder " + std::to_string(err));
    for (bool ok : dec.code_block_crc_ok) expect(ok, tag + ": code block CRC");
  }
  // tile8 entry point: hard decisions equal the encoded block
  const auto& blk = enc.code_blocks.front();
  const auto llr = tb::derate_match_code_block(p, blk.descriptor, blk.rate_matched_bits);
  const std::size_t d = blk.descriptor.k_r + 4;
  bool crc = false;
  std::uint32_t it = 0;
  const auto post = tb::turbo_decode_code_block_gpu_stage1_tile8_experimental(
      blk.descriptor, std::span<const float>(llr.data(), d), std::span<const float>(llr.data() + d, d),
      std::span<const float>(llr.data() + 2 * d, d), 6, false, &crc, &it);
  bool hard = post.size() == blk.cb_bits.size();
  for (std::size_t i = 0; hard && i < post.size(); ++i) hard &= (post[i] >= 0.0f) == (blk.cb_bits[i] != 0);
  expect(hard && it == 6, "tile8 hard decisions");
}

// A transport block of the 36.212 code through the GPU backends, checked against the oracle's 36.212
// restatement on the full trellis.
void std3gpp_roundtrip_case(std::size_t tbs) {
  tb::LteTurboCodecParams p;
  p.transport_block_bits = tbs;
  p.max_iterations = 6;
  p.convention = TC_CONVENTION_3GPP;
  const auto bits = pattern(tbs, 23, 7);
  p.g_total = 0;
  for (const auto& b :
       tb::segment_transport_block(tb::append_crc24a(bits, p.convention), p.convention).code_blocks)
    p.g_total += 3 * (b.size() + 4);
  const auto enc = tb::encode_transport_block(p, bits);
  std::vector<float> cpu;
  for (const auto& b : enc.code_blocks) {
    const auto llr = tb::derate_match_code_block(p, b.descriptor, b.rate_matched_bits);
    std::vector<float> post(b.descriptor.k_r);
    int32_t ok = 0, it = 0;
    or_std_decode_cb_windowed(static_cast<int32_t>(b.descriptor.k_r),
                              static_cast<int32_t>(b.descriptor.filler_count), llr.data(), 6, 0, 0,
                              0, post.data(), &ok, &it);
    cpu.insert(cpu.end(), post.begin(), post.end());
  }
  for (auto be : {tb::DecoderBackend::GpuStage1Exact, tb::DecoderBackend::GpuB200Persistent}) {
    const auto dec = tb::decode_transport_block(p, enc, be);
    const std::string tag = "36.212 TBS " + std::to_string(tbs) + " backend " + std::to_string(int(be));
    expect(dec.tb_bits == bits && dec.transport_block_crc_ok, tag + ": round trip");
    for (bool ok : dec.code_block_crc_ok) expect(ok, tag + ": code block CRC");
    if (be == tb::DecoderBackend::GpuStage1Exact) {
      const double err = rel_err(*dec.posterior_llr, cpu);
      expect(err <= 1e-3, tag + ": posterior vs the oracle " + std::to_string(err));
    }
  }
}

void decoder_cases() {
  std3gpp_roundtrip_case(1000);
  std3gpp_roundtrip_case(12000);
  roundtrip_case(40, 7, 3, false, 3 * (64 + 4));
  roundtrip_case(512, 11, 5, false, 3 * (536 + 4));
  roundtrip_case(6112, 19, 11, true, 0);
  roundtrip_case(12000, 17, 9, true, 0);
  tb::LteTurboCodecParams p;
  p.transport_block_bits = 40;
  p.g_total = 3 * 68;
  const auto enc = tb::encode_transport_block(p, pattern(40, 7, 3));
  expect_throw<std::invalid_argument>(
      [&] { tb::decode_transport_block(p, enc, tb::DecoderBackend::CpuReference); },
      "no CPU decoder");
  tb::CodeBlockDescriptor d;
  d.k_r = 40;
  std::vector<float> s(43);
  expect_throw<std::invalid_argument>(
      [&] { tb::turbo_decode_code_block_gpu_stage2(d, s, s, s, 8, false); }, "LLR sizes");
}

}  // namespace

int main(int argc, char** argv) {
  const std::string mode = argc > 1 ? argv[1] : "cpu";
  try {
    crc_cases();
    qpp_cases();
    segmentation_cases();
    encoder_cases(argc > 2 ? argv[2] : nullptr);
    std3gpp_codec_cases();
    if (mode == "gpu") decoder_cases();
    std::printf("All %d checks passed (%s)\n", g_checks, mode.c_str());
    return 0;
  } catch (const std::exception& ex) {
    std::fprintf(stderr, "Test failure: %s\n", ex.what());
    return 1;
  }
}
