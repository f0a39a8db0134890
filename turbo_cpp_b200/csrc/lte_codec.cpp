// lte_codec.cpp -- host codec chain, bit-exact with the reference CPU chain.
#include "lte_codec.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <stdexcept>
#include <thread>

#include "decoder.hpp"

namespace tcb {

// ------------------------------------------------------------------------------------------
// QPP: TS 36.212 Table 5.1.3-3 (the table of lte_turbo.cpp:54-102).  The 188 block sizes are
// 40..512 step 8, 528..1024 step 16, 1056..2048 step 32 and 2112..6144 step 64; f1/f2 listed.
// ------------------------------------------------------------------------------------------
namespace {
constexpr uint16_t kF1[kQppCount] = {
    3,   7,   19,  7,   7,   11,  5,   11,  7,   41,  103, 15,  9,   17,  9,   21,  101, 21,
    57,  23,  13,  27,  11,  27,  85,  29,  33,  15,  17,  33,  103, 19,  19,  37,  19,  21,
    21,  115, 193, 21,  133, 81,  45,  23,  243, 151, 155, 25,  51,  47,  91,  29,  29,  247,
    29,  89,  91,  157, 55,  31,  17,  35,  227, 65,  19,  37,  41,  39,  185, 43,  21,  155,
    79,  139, 23,  217, 25,  17,  127, 25,  239, 17,  137, 215, 29,  15,  147, 29,  59,  65,
    55,  31,  17,  171, 67,  35,  19,  39,  19,  199, 21,  211, 21,  43,  149, 45,  49,  71,
    13,  17,  25,  183, 55,  127, 27,  29,  29,  57,  45,  31,  59,  185, 113, 31,  17,  171,
    209, 253, 367, 265, 181, 39,  27,  127, 143, 43,  29,  45,  157, 47,  13,  111, 443, 51,
    51,  451, 257, 57,  313, 271, 179, 331, 363, 375, 127, 31,  33,  43,  33,  477, 35,  233,
    357, 337, 37,  71,  71,  37,  39,  127, 39,  39,  31,  113, 41,  251, 43,  21,  43,  45,
    45,  161, 89,  323, 47,  23,  47,  263};
constexpr uint16_t kF2[kQppCount] = {
    10,  12,  42,  16,  18,  20,  22,  24,  26,  84,  90,  32,  34,  108, 38,  120, 84,  44,
    46,  48,  50,  52,  36,  56,  58,  60,  62,  32,  198, 68,  210, 36,  74,  76,  78,  120,
    82,  84,  86,  44,  90,  46,  94,  48,  98,  40,  102, 52,  106, 72,  110, 168, 114, 58,
    118, 180, 122, 62,  84,  64,  66,  68,  420, 96,  74,  76,  234, 80,  82,  252, 86,  44,
    120, 92,  94,  48,  98,  80,  102, 52,  106, 48,  110, 112, 114, 58,  118, 60,  122, 124,
    84,  64,  66,  204, 140, 72,  74,  76,  78,  240, 82,  252, 86,  88,  60,  92,  846, 48,
    28,  80,  102, 104, 954, 96,  110, 112, 114, 116, 354, 120, 610, 124, 420, 64,  66,  136,
    420, 216, 444, 456, 468, 80,  164, 504, 172, 88,  300, 92,  188, 96,  28,  240, 204, 104,
    212, 192, 220, 336, 228, 232, 236, 120, 244, 248, 168, 64,  130, 264, 134, 408, 138, 280,
    142, 480, 146, 444, 120, 152, 462, 234, 158, 80,  96,  902, 166, 336, 170, 86,  174, 176,
    178, 120, 182, 184, 186, 94,  190, 480};

int32_t k_of(int i) {
  if (i < 60) return 40 + 8 * i;
  if (i < 92) return 528 + 16 * (i - 60);
  if (i < 124) return 1056 + 32 * (i - 92);
  return 2112 + 64 * (i - 124);
}
}  // namespace

QppEntry qpp_entry(int index) {
  if (index < 0 || index >= kQppCount) throw OutOfRange("QPP index out of range");
  return QppEntry{k_of(index), kF1[index], kF2[index]};
}

int qpp_index(int32_t k) {
  // invert k_of() arithmetically (every region is an arithmetic progression)
  int i = -1;
  if (k >= 40 && k <= 512 && k % 8 == 0) i = (k - 40) / 8;
  else if (k >= 528 && k <= 1024 && k % 16 == 0) i = 60 + (k - 528) / 16;
  else if (k >= 1056 && k <= 2048 && k % 32 == 0) i = 92 + (k - 1056) / 32;
  else if (k >= 2112 && k <= 6144 && k % 64 == 0) i = 124 + (k - 2112) / 64;
  return i;
}

std::vector<int32_t> qpp_permutation(int32_t k) {
  const int i = qpp_index(k);
  if (i < 0) throw OutOfRange("unsupported QPP block size");
  const uint64_t f1 = kF1[i], f2 = kF2[i], kk = static_cast<uint64_t>(k);
  std::vector<int32_t> p(k);
  // incremental form: Pi(x+1) = Pi(x) + (f1 + f2 (2x+1)) mod K
  uint64_t pi = 0, step = (f1 + f2) % kk;
  for (int32_t x = 0; x < k; ++x) {
    p[x] = static_cast<int32_t>(pi);
    pi = (pi + step) % kk;
    step = (step + 2 * f2) % kk;
  }
  return p;
}

std::vector<int32_t> qpp_inverse_permutation(int32_t k) {
  const auto p = qpp_permutation(k);
  std::vector<int32_t> inv(k);
  for (int32_t i = 0; i < k; ++i) inv[p[i]] = i;
  return inv;
}

// ------------------------------------------------------------------------------------------
// CRC as an L-bit shift register (equivalent to the reference's long division on bit arrays)
// ------------------------------------------------------------------------------------------
namespace {
struct CrcSpec {
  int len;
  std::array<uint8_t, 24> g;  // reference coefficient arrays (lte_turbo.cpp:104-116)
};
constexpr CrcSpec kCrc[4] = {
    {24, {1, 1, 0, 0, 0, 0, 0, 1, 1, 0, 0, 1, 1, 0, 0, 1, 1, 0, 1, 1, 1, 1, 1, 1}},
    {24, {1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 0, 0, 0, 1, 1}},
    {16, {1, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 1}},
    {8, {1, 1, 0, 1, 1, 0, 0, 1}},
};
const CrcSpec& spec(CrcKind k) {
  const int i = static_cast<int>(k);
  if (i < 0 || i > 3) throw InvalidArgument("unknown CRC kind");
  return kCrc[i];
}
}  // namespace

int crc_length(CrcKind kind) { return spec(kind).len; }

// TS 36.212 5.1.1: gCRC24A, gCRC24B, gCRC16, gCRC8 without the leading D^L (bit j = D^j)
constexpr uint32_t kStdCrcMask[4] = {0x864CFBu, 0x800063u, 0x1021u, 0x9Bu};

uint32_t crc_generator_mask(CrcKind kind, Convention conv) {
  const CrcSpec& s = spec(kind);
  if (conv == Convention::Std3gpp) return kStdCrcMask[static_cast<int>(kind)];
  uint32_t m = 0;
  for (int j = 0; j < s.len; ++j)
    if (s.g[j]) m |= 1u << (s.len - 1 - j);
  return m;
}

uint32_t crc_remainder(CrcKind kind, const uint8_t* bits, size_t n, Convention conv) {
  const int L = spec(kind).len;
  const uint32_t g = crc_generator_mask(kind, conv), top = 1u << (L - 1),
                 mask = (L == 32) ? 0xffffffffu : ((1u << L) - 1u);
  uint32_t r = 0;
  for (size_t i = 0; i < n; ++i) {
    const uint32_t fb = ((r & top) ? 1u : 0u) ^ (bits[i] & 1u);
    r = (r << 1) & mask;
    if (fb) r ^= g;
  }
  return r;
}

void crc_append(CrcKind kind, const uint8_t* bits, size_t n, uint8_t* out, Convention conv) {
  const int L = crc_length(kind);
  const uint32_t r = crc_remainder(kind, bits, n, conv);
  if (out != bits) std::copy(bits, bits + n, out);
  for (int j = 0; j < L; ++j) out[n + j] = static_cast<uint8_t>((r >> (L - 1 - j)) & 1u);
}

bool crc_check(CrcKind kind, const uint8_t* bits, size_t n, Convention conv) {
  const size_t L = static_cast<size_t>(crc_length(kind));
  if (n < L) return false;
  const uint32_t r = crc_remainder(kind, bits, n - L, conv);
  for (size_t j = 0; j < L; ++j)
    if (((r >> (L - 1 - j)) & 1u) != (bits[n - L + j] & 1u)) return false;
  return true;
}

// ------------------------------------------------------------------------------------------
// Segmentation (lte_turbo.cpp:540-604)
// ------------------------------------------------------------------------------------------
Segmentation segment_sizes(size_t b) {
  if (b == 0) throw InvalidArgument("transport block cannot be empty");
  Segmentation s;
  size_t bp = b;
  if (b <= 6144) {
    s.c = 1;
  } else {
    s.l = 24;
    s.c = (b + (6144 - 24) - 1) / (6144 - 24);
    bp = b + s.c * s.l;
  }
  int up = -1;
  for (int i = 0; i < kQppCount; ++i)
    if (s.c * static_cast<size_t>(k_of(i)) >= bp) {
      up = i;
      break;
    }
  if (up < 0) throw std::runtime_error("failed to select K+");
  s.k_plus = static_cast<size_t>(k_of(up));
  if (s.c == 1) {
    s.c_plus = 1;
  } else {
    if (up == 0) throw std::runtime_error("failed to select K-");
    s.k_minus = static_cast<size_t>(k_of(up - 1));
    s.c_minus = (s.c * s.k_plus - bp) / (s.k_plus - s.k_minus);
    s.c_plus = s.c - s.c_minus;
  }
  s.filler = s.c_plus * s.k_plus + s.c_minus * s.k_minus - bp;
  return s;
}

void segment_bits(const uint8_t* bits, size_t b, const Segmentation& s, uint8_t* out,
                  Convention conv) {
  size_t cursor = 0;
  for (size_t r = 0; r < s.c; ++r) {
    const size_t kr = static_cast<size_t>(s.block_k(r));
    std::fill(out, out + kr, uint8_t{0});
    const size_t off = (r == 0) ? s.filler : 0;
    const size_t payload = kr - off - s.l;
    if (cursor + payload > b) throw InvalidArgument("segmentation does not match B");
    std::copy(bits + cursor, bits + cursor + payload, out + off);
    cursor += payload;
    if (s.l == 24) crc_append(CrcKind::Crc24B, out + off, payload, out + off, conv);
    out += kr;
  }
}

// ------------------------------------------------------------------------------------------
// Turbo encoder
// ------------------------------------------------------------------------------------------
namespace {
// one RSC step: the reference's feedback u^s1^s2 (lte_turbo.cpp:337) or TS 36.212's u^s0^s1
// (g0 = 1 + D^2 + D^3); parity fb^s0^s2 (g1 = 1 + D + D^3) and next state (fb s2 s1) in both
inline void rsc(uint8_t& state, uint8_t u, uint8_t& parity, bool std3gpp) {
  const uint8_t s0 = state & 1u, s1 = (state >> 1) & 1u, s2 = (state >> 2) & 1u;
  const uint8_t fb = std3gpp ? (u ^ s0 ^ s1) : (u ^ s1 ^ s2);
  parity = fb ^ s0 ^ s2;
  state = static_cast<uint8_t>((fb << 2) | (s2 << 1) | s1);
}
inline uint8_t termination_input(uint8_t state, bool std3gpp) {  // the input that zeroes fb
  return std3gpp ? ((state & 1u) ^ ((state >> 1) & 1u))
                 : (((state >> 1) & 1u) ^ ((state >> 2) & 1u));
}
}  // namespace

void turbo_encode(int32_t k, int32_t filler, const uint8_t* cb, uint8_t* d012, Convention conv) {
  const bool std3gpp = conv == Convention::Std3gpp;
  const auto perm = qpp_permutation(k);
  uint8_t* d0 = d012;
  uint8_t* d1 = d012 + (k + 4);
  uint8_t* d2 = d012 + 2 * (k + 4);
  uint8_t su = 0, sl = 0, p = 0;
  for (int32_t i = 0; i < k; ++i) {
    rsc(su, cb[i] & 1u, p, std3gpp);
    d0[i] = (i < filler) ? 0 : (cb[i] & 1u);
    d1[i] = (i < filler) ? 0 : p;
    rsc(sl, cb[perm[i]] & 1u, p, std3gpp);
    d2[i] = p;
  }
  uint8_t us[3], up[3], ls[3], lp[3];
  for (int i = 0; i < 3; ++i) {
    us[i] = termination_input(su, std3gpp);
    rsc(su, us[i], up[i], std3gpp);
    ls[i] = termination_input(sl, std3gpp);
    rsc(sl, ls[i], lp[i], std3gpp);
  }
  if (!std3gpp) {  // the reference's multiplexing (lte_turbo.cpp:664-677)
    d0[k] = us[0]; d0[k + 1] = up[1]; d0[k + 2] = us[1]; d0[k + 3] = up[2];
    d1[k] = up[0]; d1[k + 1] = us[1]; d1[k + 2] = up[2]; d1[k + 3] = ls[0];
    d2[k] = lp[0]; d2[k + 1] = ls[1]; d2[k + 2] = lp[1]; d2[k + 3] = ls[2];
  } else {  // TS 36.212 5.1.3.2.2: x_K z_K+1 x'_K z'_K+1 / z_K x_K+2 z'_K x'_K+2 / x_K+1 z_K+2 x'_K+1 z'_K+2
    d0[k] = us[0]; d0[k + 1] = up[1]; d0[k + 2] = ls[0]; d0[k + 3] = lp[1];
    d1[k] = up[0]; d1[k + 1] = us[2]; d1[k + 2] = lp[0]; d1[k + 3] = ls[2];
    d2[k] = us[1]; d2[k + 1] = up[2]; d2[k + 2] = ls[1]; d2[k + 3] = lp[2];
  }
}

// ------------------------------------------------------------------------------------------
// Rate matching
// ------------------------------------------------------------------------------------------
size_t compute_e(size_t r, size_t g_total, size_t c, size_t num_layers, size_t mod_order) {
  if (c == 0) throw InvalidArgument("code block count must be positive");
  if (num_layers == 0 || mod_order == 0)
    throw InvalidArgument("num_layers and mod_order must be positive");
  const size_t nlqm = num_layers * mod_order;
  if (g_total % nlqm != 0) throw InvalidArgument("g_total must be divisible by num_layers * mod_order");
  const size_t gp = g_total / nlqm, gamma = gp % c;
  return (r + gamma + 1 <= c) ? nlqm * (gp / c) : nlqm * ((gp + c - 1) / c);
}

namespace {
constexpr uint8_t kColPerm[32] = {0, 16, 8, 24, 4, 20, 12, 28, 2, 18, 10, 26, 6, 22, 14, 30,
                                  1, 17, 9, 25, 5, 21, 13, 29, 3, 19, 11, 27, 7, 23, 15, 31};
}

RateMatchLayout::RateMatchLayout(int32_t d, int32_t filler) : d_(d) {
  if (d <= 0) throw InvalidArgument("invalid stream length");
  rows_ = (d + 31) / 32;
  kpi_ = rows_ * 32;
  const int32_t dummy = kpi_ - d;
  src_.assign(3 * static_cast<size_t>(kpi_), -1);
  // d0 and d1: row-wise write with <NULL> padding and filler, columns permuted, read
  // column-wise (lte_turbo.cpp:195-219); d2: pi(k) = (P[k/R] + 32 (k mod R) + 1) mod K_pi
  // (lte_turbo.cpp:221-236).  Interlacing into the circular buffer per lte_turbo.cpp:256-262.
  int32_t pos = 0;
  for (int c = 0; c < 32; ++c)
    for (int32_t r = 0; r < rows_; ++r, ++pos) {
      const int32_t y = r * 32 + kColPerm[c] - dummy;  // index into the stream
      const int32_t v = (y < 0 || y < filler) ? -1 : y;
      src_[pos] = v;                                      // systematic
      src_[kpi_ + 2 * pos] = (v < 0) ? -1 : d + v;        // parity 1
    }
  for (int32_t k = 0; k < kpi_; ++k) {
    const int32_t y = (kColPerm[k / rows_] + 32 * (k % rows_) + 1) % kpi_ - dummy;
    src_[kpi_ + 2 * k + 1] = (y < 0) ? -1 : 2 * d + y;   // parity 2 (filler not nulled)
  }
}

int32_t RateMatchLayout::k0(uint32_t rv) const {
  const int32_t n = ncb();
  return rows_ * (2 * ((n + 8 * rows_ - 1) / (8 * rows_)) * static_cast<int32_t>(rv) + 2);
}

void rate_match(int32_t k, int32_t filler, const uint8_t* d012, size_t e, uint32_t rv,
                uint8_t* out) {
  const RateMatchLayout L(k + 4, filler);
  const int32_t n = L.ncb();
  int64_t j = L.k0(rv) % n;
  for (size_t o = 0; o < e;) {
    const int32_t s = L.source(static_cast<int32_t>(j));
    if (s >= 0) out[o++] = d012[s];
    if (++j == n) j = 0;
  }
}

namespace {
template <class Value>
void derate(int32_t k, int32_t filler, size_t e, uint32_t rv, float* d012, Value value) {
  const RateMatchLayout L(k + 4, filler);
  const int32_t n = L.ncb();
  // the circular buffer is walked as in the encoder; every <NULL>-free position receives the
  // sum of the values landing on it, which is then moved to its stream slot
  std::fill(d012, d012 + 3 * static_cast<size_t>(k + 4), 0.0f);
  std::vector<float> circ(static_cast<size_t>(n), 0.0f);
  int64_t j = L.k0(rv) % n;
  for (size_t o = 0; o < e;) {
    if (L.source(static_cast<int32_t>(j)) >= 0) circ[j] += value(o++);
    if (++j == n) j = 0;
  }
  for (int32_t p = 0; p < n; ++p) {
    const int32_t s = L.source(p);
    if (s >= 0) d012[s] += circ[p];
  }
}
}  // namespace

void derate_match_bits(int32_t k, int32_t filler, const uint8_t* e_bits, size_t e, uint32_t rv,
                       float* d012) {
  derate(k, filler, e, rv, d012, [e_bits](size_t o) { return e_bits[o] ? 8.0f : -8.0f; });
}

void derate_match_llr(int32_t k, int32_t filler, const float* e_llr, size_t e, uint32_t rv,
                      float* d012) {
  derate(k, filler, e, rv, d012, [e_llr](size_t o) { return e_llr[o]; });
}

// ------------------------------------------------------------------------------------------
// Seeded channel: SplitMix64 finaliser over (seed, index) counters; Box-Muller for normals.
// ------------------------------------------------------------------------------------------
namespace {
inline uint64_t mix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}
inline double unit(uint64_t x) { return (static_cast<double>(x >> 11) + 0.5) * 0x1.0p-53; }
}  // namespace

void random_bits(uint64_t seed, uint64_t first, size_t n, uint8_t* bits) {
  const uint64_t key = mix64(seed ^ 0x6a09e667f3bcc909ull);
  for (size_t i = 0; i < n; ++i) bits[i] = static_cast<uint8_t>(mix64(key + first + i) >> 63);
}

void awgn_llr(uint64_t seed, uint64_t first, const uint8_t* bits, size_t n, double sigma2,
              float* llr) {
  const uint64_t key = mix64(seed ^ 0xbb67ae8584caa73bull);
  const double sigma = std::sqrt(sigma2), scale = 2.0 / sigma2;
  for (size_t i = 0; i < n; ++i) {
    const uint64_t c = first + i;
    // one Box-Muller draw per sample from two counter-derived uniforms
    const double u1 = unit(mix64(key + 2 * c)), u2 = unit(mix64(key + 2 * c + 1));
    const double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    const double y = (bits[i] ? 1.0 : -1.0) + sigma * z;
    llr[i] = static_cast<float>(scale * y);
  }
}

void awgn_code_blocks(uint64_t seed, size_t n, const int32_t* k, const int32_t* filler,
                      const float* ebn0_db, bool crc24b, uint8_t* bits, float* llr, int threads) {
  std::vector<size_t> bit_off(n + 1, 0), llr_off(n + 1, 0);
  for (size_t i = 0; i < n; ++i) {
    if (qpp_index(k[i]) < 0) throw OutOfRange("unsupported QPP block size");
    if (filler[i] < 0 || filler[i] >= k[i] || (crc24b && filler[i] + 24 >= k[i]))
      throw InvalidArgument("invalid filler count");
    bit_off[i + 1] = bit_off[i] + static_cast<size_t>(k[i]);
    llr_off[i + 1] = llr_off[i] + 3 * static_cast<size_t>(k[i] + 4);
  }
  auto one = [&](size_t i) {
    const int32_t K = k[i], F = filler[i];
    const uint64_t s = mix64(seed + 0x51ed270b27ull * (i + 1));
    uint8_t* b = bits + bit_off[i];
    random_bits(s, 0, static_cast<size_t>(K), b);
    std::fill(b, b + F, uint8_t{0});
    if (crc24b) crc_append(CrcKind::Crc24B, b + F, static_cast<size_t>(K - F - 24), b + F);
    std::vector<uint8_t> d(3 * static_cast<size_t>(K + 4));
    turbo_encode(K, F, b, d.data());
    const double rate = static_cast<double>(K) / (3.0 * (K + 4));
    const double sigma2 = 1.0 / (2.0 * rate * std::pow(10.0, ebn0_db[i] / 10.0));
    float* x = llr + llr_off[i];
    awgn_llr(s ^ 0x2545f4914f6cdd1dull, 0, d.data(), d.size(), sigma2, x);
    std::fill(x, x + F, 0.0f);
    std::fill(x + (K + 4), x + (K + 4) + F, 0.0f);
  };
  if (threads <= 0) threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
  threads = static_cast<int>(std::min<size_t>(static_cast<size_t>(threads), std::max<size_t>(n, 1)));
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&, t] {
      for (size_t i = static_cast<size_t>(t); i < n; i += static_cast<size_t>(threads)) one(i);
    });
  for (auto& th : pool) th.join();
}

}  // namespace tcb
