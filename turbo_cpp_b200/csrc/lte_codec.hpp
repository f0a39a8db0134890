// lte_codec.hpp -- host side of the LTE turbo codec chain: QPP tables, CRC, code-block
// segmentation, turbo encoding, rate matching and de-rate matching.  Bit-exact with the
// reference CPU chain (Wiseung/Turbo_CPP src/lte_turbo.cpp), including its deviations from
// TS 36.212 (see the notes on each function).
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

namespace tcb {

// ---- QPP interleaver (lte_turbo.cpp:54-102, 157-161, 498-506, 606-622) ----
struct QppEntry {
  int32_t k, f1, f2;
};
constexpr int kQppCount = 188;
QppEntry qpp_entry(int index);
int qpp_index(int32_t k);  // -1 if K is not an LTE turbo block size
std::vector<int32_t> qpp_permutation(int32_t k);          // Pi(i) = (f1 i + f2 i^2) mod K
std::vector<int32_t> qpp_inverse_permutation(int32_t k);

// ---- code conventions ----
// Reference: the conventions of the reference (its CRC coefficient arrays, RSC feedback
// u^s1^s2, its tail multiplexing) -- the default everywhere, and what parity is checked against.
// Std3gpp: TS 36.212 (CRC generators gCRC24A/24B/16/8 of 5.1.1, RSC feedback g0 = 1+D^2+D^3 and
// the tail multiplexing of 5.1.3.2.2).  Segmentation and rate matching do not depend on it.
enum class Convention : int { Reference = 0, Std3gpp = 1 };

// ---- CRC (lte_turbo.cpp:104-155, 508-538) ----
// Reference generators are the reference's coefficient arrays (g[j] multiplies D^(L-1-j),
// leading D^L implicit); they are not all the TS 36.212 polynomials.
enum class CrcKind : int { Crc24A = 0, Crc24B = 1, Crc16 = 2, Crc8 = 3 };
int crc_length(CrcKind kind);
uint32_t crc_generator_mask(CrcKind kind, Convention conv = Convention::Reference);
uint32_t crc_remainder(CrcKind kind, const uint8_t* bits, size_t n,
                       Convention conv = Convention::Reference);  // M(D) D^L mod g(D)
void crc_append(CrcKind kind, const uint8_t* bits, size_t n, uint8_t* out,
                Convention conv = Convention::Reference);  // out: n+L bits
bool crc_check(CrcKind kind, const uint8_t* bits, size_t n,
               Convention conv = Convention::Reference);

// ---- code-block segmentation (lte_turbo.cpp:540-604) ----
struct Segmentation {
  size_t c = 0, c_plus = 0, c_minus = 0, k_plus = 0, k_minus = 0, filler = 0, l = 0;
  int32_t block_k(size_t r) const { return static_cast<int32_t>(r < c_minus ? k_minus : k_plus); }
  size_t total_bits() const { return c_plus * k_plus + c_minus * k_minus; }
};
Segmentation segment_sizes(size_t b);  // throws InvalidArgument / std::runtime_error
// Writes the C code blocks back to back (filler zeros first in block 0, CRC24B per block when
// C > 1).
void segment_bits(const uint8_t* bits_with_crc, size_t b, const Segmentation& s, uint8_t* out,
                  Convention conv = Convention::Reference);

// ---- turbo encoder (lte_turbo.cpp:333-353, 624-688) ----
// d012 = [d0 | d1 | d2], each K+4 bits; filler positions of d0/d1 are 0; tails multiplexed as
// the reference does (lte_turbo.cpp:664-677), or as TS 36.212 5.1.3.2.2 with Std3gpp.
void turbo_encode(int32_t k, int32_t filler, const uint8_t* cb_bits, uint8_t* d012,
                  Convention conv = Convention::Reference);

// ---- rate matching (lte_turbo.cpp:167-325) ----
size_t compute_e(size_t r, size_t g_total, size_t c, size_t num_layers, size_t mod_order);

class RateMatchLayout {
 public:
  RateMatchLayout(int32_t d, int32_t filler);
  int32_t d() const { return d_; }
  int32_t kpi() const { return kpi_; }
  int32_t ncb() const { return 3 * kpi_; }
  int32_t k0(uint32_t rv) const;
  // circular-buffer position -> index into the concatenated [d0|d1|d2] stream, -1 for <NULL>
  int32_t source(int32_t pos) const { return src_[pos]; }

 private:
  int32_t d_, rows_, kpi_;
  std::vector<int32_t> src_;
};

void rate_match(int32_t k, int32_t filler, const uint8_t* d012, size_t e, uint32_t rv,
                uint8_t* out);
// hard bits -> +-8.0 per bit, repetitions summed, <NULL>/filler positions 0
// (derate_match_streams, lte_turbo.cpp:280-325)
void derate_match_bits(int32_t k, int32_t filler, const uint8_t* e_bits, size_t e, uint32_t rv,
                       float* d012);
// the same bit-selection walk over soft LLRs (e_llr[j] added where bit j would be +-8)
void derate_match_llr(int32_t k, int32_t filler, const float* e_llr, size_t e, uint32_t rv,
                      float* d012);

// ---- seeded channel for test data (not part of the reference) ----
// bits[i] = uniform {0,1}; counter-based, reproducible from (seed, i).
void random_bits(uint64_t seed, uint64_t first, size_t n, uint8_t* bits);
// BPSK (bit 1 -> +1) over AWGN with noise variance sigma2; llr = 2 y / sigma2.
void awgn_llr(uint64_t seed, uint64_t first, const uint8_t* bits, size_t n, double sigma2,
              float* llr);

// Seeded code blocks for tests and benchmarks: per block i, uniform info bits (filler zeros
// first; the last 24 bits a CRC24B of the rest when crc24b), turbo encoding, BPSK over AWGN at
// ebn0_db[i] with rate K/(3(K+4)), LLR = 2y/sigma^2, filler LLRs of d0/d1 set to 0 (erasures).
// Block i's LLRs start at 3 * sum_{j<i}(K_j + 4), its bits at sum_{j<i} K_j.  Reproducible
// from (seed, i) whatever the thread count.
void awgn_code_blocks(uint64_t seed, size_t n, const int32_t* k, const int32_t* filler,
                      const float* ebn0_db, bool crc24b, uint8_t* bits, float* llr, int threads);

}  // namespace tcb
