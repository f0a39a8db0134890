// generate.cu -- test-vector generation on the device: seeded information bits with CRC24B,
// the turbo encoder, the rate matcher and the BPSK/AWGN channel.  The bits, encoded streams and
// rate-matched bits are bit-identical to the host codec (lte_codec.cpp: random_bits,
// crc_append, turbo_encode, rate_match, i.e. the reference's turbo_encode_code_block
// lte_turbo.cpp:624-688 and puncture_and_collect :250-278); the channel uses the same
// counter-based draws as the host's awgn_llr, so the LLRs equal the host's up to the last bit
// of CUDA's double log/cos against the host C library's.
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "circular_buffer.cuh"
#include "decoder.hpp"
#include "lte_codec.hpp"

namespace tcb {
namespace {

void ok(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

// SplitMix64 finaliser (the host generator's mixing function)
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}
uint64_t host_mix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

struct GenBlock {
  int32_t k, filler;
  int64_t bits;     // offset of the K information bits
  int64_t llr;      // offset of the 3(K+4) LLRs (or encoded bits)
  uint64_t seed;    // per-block stream seed
  double sigma, scale;  // channel: noise deviation, LLR scale 2 / sigma^2
};

constexpr int kGenThreads = 256;

// One CTA per block: bits[i] = top bit of mix64(key + i), the filler zeroed, and with crc24b
// the last 24 bits replaced by the CRC24B of bits [filler, K-24): the remainder is the XOR of
// x^(n-1-i) mod g over the set payload bits i (n = K - filler, table xpow), whose coefficient
// of x^(23-j) is CRC bit j -- the codeword the decoder's syndrome check accepts.
__global__ void __launch_bounds__(kGenThreads) gen_bits_kernel(const GenBlock* __restrict__ blocks,
                                                              int crc24b,
                                                              const uint32_t* __restrict__ xpow,
                                                              uint8_t* __restrict__ bits) {
  __shared__ uint32_t part[kGenThreads / 32];
  const GenBlock b = blocks[blockIdx.x];
  const uint64_t key = mix64(b.seed ^ 0x6a09e667f3bcc909ull);
  const int n = b.k - b.filler;
  const int pay_end = crc24b ? b.k - 24 : b.k;
  uint8_t* out = bits + b.bits;
  uint32_t r = 0;
  for (int i = threadIdx.x; i < b.k; i += blockDim.x) {
    uint8_t v = static_cast<uint8_t>(mix64(key + static_cast<uint64_t>(i)) >> 63);
    if (i < b.filler) v = 0;
    if (i < pay_end) {
      out[i] = v;
      if (crc24b && v) r ^= xpow[n - 1 - (i - b.filler)];
    }
  }
  if (!crc24b) return;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) r ^= __shfl_xor_sync(0xffffffffu, r, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = r;
  __syncthreads();
  if (threadIdx.x < 24) {
    uint32_t x = 0;
    for (int w = 0; w < kGenThreads / 32; ++w) x ^= part[w];
    out[b.k - 24 + threadIdx.x] = static_cast<uint8_t>((x >> (23 - threadIdx.x)) & 1u);
  }
}

__device__ __forceinline__ uint8_t rsc_step(uint8_t& s, uint8_t u) {
  const uint8_t s0 = s & 1u, s1 = (s >> 1) & 1u, s2 = (s >> 2) & 1u;
  const uint8_t fb = u ^ s1 ^ s2;  // the reference's feedback u^s1^s2 (lte_turbo.cpp:337)
  s = static_cast<uint8_t>((fb << 2) | (s2 << 1) | s1);
  return fb ^ s0 ^ s2;
}

// Two threads per block (even lane: upper encoder over natural order; odd lane: lower encoder
// over QPP order); the tail multiplexing of lte_turbo.cpp:664-677 combines both encoders'
// termination bits, exchanged between the lane pair.
__global__ void encode_kernel(const GenBlock* __restrict__ blocks, int n_blocks,
                              const uint16_t* __restrict__ perm, const int32_t* __restrict__ tab,
                              const uint8_t* __restrict__ bits, uint8_t* __restrict__ d012) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = t >> 1;
  const bool lower = t & 1;
  const bool active = c < n_blocks;
  GenBlock b{};
  if (active) b = blocks[c];
  const int K = b.k;
  const uint8_t* cb = bits + b.bits;
  uint8_t* d0 = d012 + b.llr;
  uint8_t* d1 = d0 + (K + 4);
  uint8_t* d2 = d1 + (K + 4);
  uint8_t s = 0;
  if (active) {
    if (!lower) {
      for (int i = 0; i < K; ++i) {
        const uint8_t u = cb[i] & 1u;
        const uint8_t p = rsc_step(s, u);
        d0[i] = i < b.filler ? 0 : u;
        d1[i] = i < b.filler ? 0 : p;
      }
    } else {
      const uint16_t* pm = perm + tab[c];
      for (int i = 0; i < K; ++i) d2[i] = rsc_step(s, cb[pm[i]] & 1u);
    }
  }
  uint8_t ts[3], tp[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    ts[i] = ((s >> 1) & 1u) ^ ((s >> 2) & 1u);  // the input that zeroes the feedback
    tp[i] = rsc_step(s, ts[i]);
  }
  // pack (ts, tp) and swap with the partner lane
  const uint32_t mine = ts[0] | ts[1] << 1 | ts[2] << 2 | tp[0] << 3 | tp[1] << 4 | tp[2] << 5;
  const uint32_t other = __shfl_xor_sync(0xffffffffu, mine, 1);
  if (!active || lower) return;
  const uint8_t ls[3] = {static_cast<uint8_t>(other & 1u), static_cast<uint8_t>((other >> 1) & 1u),
                         static_cast<uint8_t>((other >> 2) & 1u)};
  const uint8_t lp[3] = {static_cast<uint8_t>((other >> 3) & 1u), static_cast<uint8_t>((other >> 4) & 1u),
                         static_cast<uint8_t>((other >> 5) & 1u)};
  d0[K] = ts[0]; d0[K + 1] = tp[1]; d0[K + 2] = ts[1]; d0[K + 3] = tp[2];
  d1[K] = tp[0]; d1[K + 1] = ts[1]; d1[K + 2] = tp[2]; d1[K + 3] = ls[0];
  d2[K] = lp[0]; d2[K + 1] = ls[1]; d2[K + 2] = lp[1]; d2[K + 3] = ls[2];
}

// BPSK over AWGN: one Box-Muller draw per encoded bit from two counter-derived uniforms (the
// host's awgn_llr), LLR = 2 y / sigma^2; filler positions of d0 and d1 get 0.
__global__ void __launch_bounds__(kGenThreads) awgn_kernel(const GenBlock* __restrict__ blocks,
                                                          const uint8_t* __restrict__ d012,
                                                          float* __restrict__ llr) {
  const GenBlock b = blocks[blockIdx.x];
  const uint64_t key = mix64((b.seed ^ 0x2545f4914f6cdd1dull) ^ 0xbb67ae8584caa73bull);
  const int n = 3 * (b.k + 4);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const uint64_t c = static_cast<uint64_t>(i);
    // every product and sum rounded on its own (no contraction into FMA), as on the host
    const double u1 = __dmul_rn(__dadd_rn(static_cast<double>(mix64(key + 2 * c) >> 11), 0.5), 0x1.0p-53);
    const double u2 = __dmul_rn(__dadd_rn(static_cast<double>(mix64(key + 2 * c + 1) >> 11), 0.5), 0x1.0p-53);
    const double z = __dmul_rn(sqrt(__dmul_rn(-2.0, log(u1))), cos(__dmul_rn(6.283185307179586, u2)));
    const double y = __dadd_rn(d012[b.llr + i] ? 1.0 : -1.0, __dmul_rn(b.sigma, z));
    const int lane_pos = i % (b.k + 4);
    const bool filler = i < 2 * (b.k + 4) && lane_pos < b.filler;
    llr[b.llr + i] = filler ? 0.0f : __double2float_rn(__dmul_rn(b.scale, y));
  }
}

constexpr int kRmGenThreads = kCircThreads;

struct RmGen {
  int32_t k, filler, e, rv;
  int64_t e_off, d_off;
};

// One CTA per block: output bit kk is the stream bit at the kk-th <NULL>-free position of the
// circular walk from k0 (wrapping), i.e. the valid position of rank (rank(k0) + kk) mod Nv.
__global__ void __launch_bounds__(kRmGenThreads) rate_match_kernel(const RmGen* __restrict__ blocks,
                                                                  const uint8_t* __restrict__ d012,
                                                                  uint8_t* __restrict__ e_bits) {
  __shared__ int warp_sum[kRmGenThreads / 32];
  __shared__ int s_rank_k0, s_total;
  const RmGen b = blocks[blockIdx.x];
  CircularScan cs(b.k, b.filler);
  cs.scan(warp_sum, &s_total);
  cs.rank_of(cs.k0(b.rv), &s_rank_k0);
  __syncthreads();
  const int nv = s_total, r0 = s_rank_k0;
  const uint8_t* src_bits = d012 + b.d_off;
  uint8_t* out = e_bits + b.e_off;
  int rank = cs.before;
  CircularWalk wk = cs.walk(cs.p0);
  for (int p = cs.p0; p < cs.p1; ++p) {
    const int src = wk.next();
    if (src < 0) continue;
    int kk = rank - r0;
    if (kk < 0) kk += nv;
    const uint8_t v = src_bits[src];
    for (; kk < b.e; kk += nv) out[kk] = v;
    ++rank;
  }
}

template <class T>
T* reserve(DeviceBuffer& b, size_t count) {
  b.reserve(count * sizeof(T));
  return static_cast<T*>(b.ptr);
}

}  // namespace

void Decoder::awgn_code_blocks_device(uint64_t seed, size_t n, const int32_t* k,
                                      const int32_t* filler, const float* ebn0_db, bool crc24b,
                                      uint8_t* bits, float* llr, void* stream) {
  std::lock_guard<std::mutex> lock(mu_);
  ok(cudaSetDevice(device_), "cudaSetDevice");
  if (n == 0) return;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::vector<GenBlock> v(n);
  std::vector<int32_t> tab(n);
  int64_t boff = 0, loff = 0;
  for (size_t i = 0; i < n; ++i) {
    if (qpp_index(k[i]) < 0) throw OutOfRange("unsupported QPP block size");
    if (filler[i] < 0 || filler[i] >= k[i] || (crc24b && filler[i] + 24 >= k[i]))
      throw InvalidArgument("invalid filler count");
    GenBlock& g = v[i];
    g.k = k[i];
    g.filler = filler[i];
    g.bits = boff;
    g.llr = loff;
    g.seed = host_mix64(seed + 0x51ed270b27ull * (i + 1));
    // the host generator's channel parameters, computed the same way
    const double rate = static_cast<double>(k[i]) / (3.0 * (k[i] + 4));
    const double sigma2 = 1.0 / (2.0 * rate * std::pow(10.0, ebn0_db[i] / 10.0));
    g.sigma = std::sqrt(sigma2);
    g.scale = 2.0 / sigma2;
    tab[i] = table_offset(k[i]);
    boff += k[i];
    loff += 3 * static_cast<int64_t>(k[i] + 4);
  }
  order_after_previous(stream);
  GenBlock* dv = reserve<GenBlock>(d_gen_, n);
  int32_t* dt = reserve<int32_t>(d_gentab_, n);
  uint8_t* enc = reserve<uint8_t>(d_genenc_, static_cast<size_t>(loff));
  upload(dv, v.data(), n * sizeof(GenBlock), stream);
  upload(dt, tab.data(), n * sizeof(int32_t), stream);
  gen_bits_kernel<<<static_cast<unsigned>(n), kGenThreads, 0, st>>>(
      dv, crc24b ? 1 : 0, static_cast<const uint32_t*>(d_xpow_.ptr), bits);
  ok(cudaGetLastError(), "bit generation launch");
  encode_kernel<<<static_cast<unsigned>((2 * n + 63) / 64), 64, 0, st>>>(
      dv, static_cast<int>(n), perm_table(), dt, bits, enc);
  ok(cudaGetLastError(), "encoder launch");
  awgn_kernel<<<static_cast<unsigned>(n), kGenThreads, 0, st>>>(dv, enc, llr);
  ok(cudaGetLastError(), "channel launch");
  timing_.launches += 3;
  mark_done(stream);
}

void Decoder::turbo_encode_device(size_t n, const int32_t* k, const int32_t* filler,
                                  const uint8_t* bits, uint8_t* d012, void* stream) {
  std::lock_guard<std::mutex> lock(mu_);
  ok(cudaSetDevice(device_), "cudaSetDevice");
  if (n == 0) return;
  std::vector<GenBlock> v(n);
  std::vector<int32_t> tab(n);
  int64_t boff = 0, loff = 0;
  for (size_t i = 0; i < n; ++i) {
    if (qpp_index(k[i]) < 0) throw OutOfRange("unsupported QPP block size");
    if (filler[i] < 0 || filler[i] >= k[i]) throw InvalidArgument("invalid filler count");
    v[i] = GenBlock{k[i], filler[i], boff, loff, 0, 0.0, 0.0};
    tab[i] = table_offset(k[i]);
    boff += k[i];
    loff += 3 * static_cast<int64_t>(k[i] + 4);
  }
  order_after_previous(stream);
  GenBlock* dv = reserve<GenBlock>(d_gen_, n);
  int32_t* dt = reserve<int32_t>(d_gentab_, n);
  upload(dv, v.data(), n * sizeof(GenBlock), stream);
  upload(dt, tab.data(), n * sizeof(int32_t), stream);
  encode_kernel<<<static_cast<unsigned>((2 * n + 63) / 64), 64, 0, static_cast<cudaStream_t>(stream)>>>(
      dv, static_cast<int>(n), perm_table(), dt, bits, d012);
  ok(cudaGetLastError(), "encoder launch");
  timing_.launches += 1;
  mark_done(stream);
}

void Decoder::rate_match_device(size_t n, const RmBlockDesc* blocks, const uint8_t* d012,
                                size_t d012_len, uint8_t* e_bits, size_t e_len, void* stream) {
  std::lock_guard<std::mutex> lock(mu_);
  ok(cudaSetDevice(device_), "cudaSetDevice");
  if (n == 0) return;
  std::vector<RmGen> v(n);
  for (size_t i = 0; i < n; ++i) {
    const RmBlockDesc& b = blocks[i];
    if (qpp_index(b.k) < 0) throw OutOfRange("unsupported QPP block size");
    if (b.filler < 0 || b.filler >= b.k || b.rv > 3 || b.e < 0)
      throw InvalidArgument("invalid filler count, rv or E");
    if (b.e_offset < 0 || static_cast<size_t>(b.e_offset) + static_cast<size_t>(b.e) > e_len)
      throw InvalidArgument("rate-matched bits out of range");
    if (b.llr_offset < 0 ||
        static_cast<size_t>(b.llr_offset) + 3 * static_cast<size_t>(b.k + 4) > d012_len)
      throw InvalidArgument("encoded bits out of range");
    v[i] = RmGen{b.k, b.filler, b.e, static_cast<int32_t>(b.rv), b.e_offset, b.llr_offset};
  }
  order_after_previous(stream);
  RmGen* dv = reserve<RmGen>(d_genrm_, n);
  upload(dv, v.data(), n * sizeof(RmGen), stream);
  rate_match_kernel<<<static_cast<unsigned>(n), kRmGenThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      dv, d012, e_bits);
  ok(cudaGetLastError(), "rate matching launch");
  timing_.launches += 1;
  mark_done(stream);
}

}  // namespace tcb
