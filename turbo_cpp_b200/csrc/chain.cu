// chain.cu -- the decode side of the transport-block chain on the device: LLR-domain de-rate
// matching, batched turbo decoding (decoder.cu), hard decisions, filler and CRC24B strip,
// transport-block reassembly and CRC24A.  Batched over many transport blocks per call; the
// reference does the same per transport block on the host (decode_transport_block,
// lte_turbo.cpp:891-980, de-rate matching lte_turbo.cpp:280-325).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "decoder.hpp"
#include "lte_codec.hpp"
#include "circular_buffer.cuh"
#include "siso.cuh"

namespace tcb {
namespace {

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

struct DevRm {
  int32_t k, filler, e, rv;
  int64_t e_off;  // first rate-matched LLR of the block
  int64_t out;    // float offset of [d0|d1|d2] (3(K+4) floats)
};

constexpr int kRmThreads = 1024;
// largest circular buffer (K = 6144: 3 x 32 x 193 positions), floats
constexpr int kMaxNcb = 3 * 32 * ((6144 + 4 + 31) / 32);

// circular-buffer positions (floats of shared memory) of the largest block in `v`
inline int max_ncb(const std::vector<DevRm>& v) {
  int m = 0;
  for (const DevRm& b : v) m = std::max(m, 3 * 32 * ((b.k + 4 + 31) / 32));
  return m;
}

// acc[(r0 + kk) mod nv] += x[kk] for kk in [0, e), one round of nv LLRs at a time (each rank at
// most once per round), so that every rank sums its LLRs in increasing kk -- the reference's
// summation order.  Each thread requests kRmBatch LLRs before adding any (coalesced loads, kept in
// flight together); consecutive kk hit consecutive shared-memory banks.  Ends with a barrier.
constexpr int kRmBatch = 4;
__device__ __forceinline__ void accumulate_rounds(float* acc, const float* __restrict__ x, int e,
                                                  int nv, int r0) {
  for (int base = 0; base < e; base += nv) {
    const int n = min(nv, e - base);
    for (int j0 = threadIdx.x; j0 < n; j0 += kRmThreads * kRmBatch) {
      float v[kRmBatch];
#pragma unroll
      for (int u = 0; u < kRmBatch; ++u) {
        const int j = j0 + u * kRmThreads;
        v[u] = j < n ? __ldg(x + base + j) : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < kRmBatch; ++u) {
        const int j = j0 + u * kRmThreads;
        if (j < n) {
          int r = r0 + j;
          if (r >= nv) r -= nv;
          acc[r] += v[u];
        }
      }
    }
    __syncthreads();
  }
}

// One CTA per code block.  The rate-matched LLR kk lands on the valid circular-buffer position of
// rank (rank(k0) + kk) mod Nv: the LLRs are summed per rank in shared memory (coalesced reads,
// increasing kk from 0.0f, the reference's order, so the result is bit-identical to
// derate_match_streams with LLR values), then every [d0|d1|d2] element takes the sum of its
// position's rank (closed form, CircularRank; coalesced stores); the filler elements of d0 and
// d1 (<NULL> in the buffer) are 0.  Dynamic shared memory: Ncb floats of the largest block.
__global__ void __launch_bounds__(kRmThreads) derate_llr_kernel(const DevRm* __restrict__ blocks,
                                                                const float* __restrict__ e_llr,
                                                                float* __restrict__ d012) {
  extern __shared__ float acc[];
  __shared__ int tables[kRankTableInts];
  const DevRm b = blocks[blockIdx.x];
  CircularRank cr(b.k, b.filler, tables);
  cr.setup();
  for (int j = threadIdx.x; j < cr.ncb; j += kRmThreads) acc[j] = 0.0f;
  __syncthreads();
  accumulate_rounds(acc, e_llr + b.e_off, b.e, cr.valid(), cr.rank(cr.k0(b.rv)));
  float* out = d012 + b.out;
  for (int i = threadIdx.x; i < 3 * cr.d; i += kRmThreads) {
    const int r = cr.rank_of_element(i);
    out[i] = r >= 0 ? acc[r] : 0.0f;
  }
}

// HARQ soft combining: one CTA per code block, whose transmissions (up to kMaxHarqTx, each with
// its own rv, E and rate-matched LLRs) are consecutive in `tx`.  The ranks of the valid
// circular-buffer positions depend only on K and the filler count; each transmission's LLRs are
// summed per rank in increasing kk from 0.0f (its de-rate-matched value, as derate_llr_kernel)
// and added to the total in transmission order -- bit-identical to de-rate matching each
// transmission alone and adding the results in that order.  Dynamic shared memory: 2 Ncb floats
// of the largest block.
constexpr int kMaxHarqTx = 8;

__global__ void __launch_bounds__(kRmThreads) derate_combine_kernel(
    const DevRm* __restrict__ tx, const int32_t* __restrict__ group_first,
    const float* __restrict__ e_llr, float* __restrict__ d012) {
  extern __shared__ float acc[];  // [0, Ncb): the total; [Ncb, 2 Ncb): one transmission
  __shared__ int tables[kRankTableInts];
  const int t0 = group_first[blockIdx.x], nt = group_first[blockIdx.x + 1] - t0;
  const DevRm b = tx[t0];
  CircularRank cr(b.k, b.filler, tables);
  cr.setup();
  float* part = acc + cr.ncb;
  for (int j = threadIdx.x; j < cr.ncb; j += kRmThreads) acc[j] = 0.0f;
  __syncthreads();
  const int nv = cr.valid();
  for (int t = 0; t < nt; ++t) {
    const DevRm x = tx[t0 + t];
    for (int j = threadIdx.x; j < nv; j += kRmThreads) part[j] = 0.0f;
    __syncthreads();
    accumulate_rounds(part, e_llr + x.e_off, x.e, nv, cr.rank(cr.k0(x.rv)));
    for (int j = threadIdx.x; j < nv; j += kRmThreads) acc[j] += part[j];
    __syncthreads();
  }
  float* out = d012 + b.out;
  for (int i = threadIdx.x; i < 3 * cr.d; i += kRmThreads) {
    const int r = cr.rank_of_element(i);
    out[i] = r >= 0 ? acc[r] : 0.0f;
  }
}

struct DevTb {
  int32_t first_cb, n_cb;
  int64_t tbs;       // transport block size without CRC24A
  int64_t bits_out;  // offset of the block's TBS output bits
};

// Per code block of a transport-block call: its transport block and where its kept bits start in
// that block's TBS + CRC24A stream (the sum of the kept bits of the blocks before it).
struct DevTbCb {
  int32_t tb;
  int32_t pos;
};

constexpr int kFinishThreads = 256;

// Finish, part 1 (lte_turbo.cpp:958-979), one CTA per code block: hard decisions (>= 0 -> 1)
// of bits [filler, K), the CRC24B syndrome over them (checked when C > 1), the kept bits (the
// CRC24B dropped when C > 1) written at their place in the transport block's output, and this
// block's share of the transport block's CRC24A syndrome.  A CRC is a syndrome: the XOR of
// x^(N-1-j) mod g over the set bits j of the N-bit codeword, so the shares of a transport
// block's code blocks XOR to its syndrome.
__global__ void __launch_bounds__(kFinishThreads) tb_finish_cb_kernel(
    const DevTb* __restrict__ tbs, const DevTbCb* __restrict__ tbcb, const DevCb* __restrict__ cbs,
    const float* __restrict__ post, const uint32_t* __restrict__ xpow_a,
    const uint32_t* __restrict__ xpow_b, uint8_t* __restrict__ bits, uint8_t* __restrict__ cb_ok,
    uint32_t* __restrict__ syn_a_part) {
  __shared__ uint32_t red[2][kFinishThreads / 32];
  const int c = blockIdx.x;
  const DevTbCb m = tbcb[c];
  if (m.tb < 0) {  // in no transport block
    if (threadIdx.x == 0) {
      cb_ok[c] = 0;
      syn_a_part[c] = 0;
    }
    return;
  }
  const DevTb t = tbs[m.tb];
  const DevCb cb = cbs[c];
  const int64_t n_a = t.tbs + 24;             // TB codeword length with CRC24A
  const int n_b = cb.k - cb.filler;           // CRC24B codeword length
  const int keep = n_b - (t.n_cb > 1 ? 24 : 0);
  uint32_t syn_b = 0, syn_a = 0;
  for (int i = threadIdx.x; i < n_b; i += kFinishThreads) {
    const uint8_t bit = post[cb.out + cb.filler + i] >= 0.0f ? 1 : 0;
    if (bit) syn_b ^= xpow_b[n_b - 1 - i];
    if (i < keep) {
      const int64_t j = m.pos + i;
      if (bit && j < n_a) syn_a ^= xpow_a[n_a - 1 - j];
      if (j < t.tbs) bits[t.bits_out + j] = bit;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    syn_b ^= __shfl_xor_sync(0xffffffffu, syn_b, o);
    syn_a ^= __shfl_xor_sync(0xffffffffu, syn_a, o);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][wid] = syn_b;
    red[1][wid] = syn_a;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t b = 0, a = 0;
    for (int w = 0; w < kFinishThreads / 32; ++w) {
      b ^= red[0][w];
      a ^= red[1][w];
    }
    cb_ok[c] = (t.n_cb == 1) ? 1 : (b == 0);
    syn_a_part[c] = a;
  }
}

// Finish, part 2, one thread per transport block: the XOR of its code blocks' CRC24A shares,
// and whether the kept bits add up to TBS + 24.
__global__ void tb_finish_tb_kernel(const DevTb* __restrict__ tbs, int n_tb,
                                    const DevTbCb* __restrict__ tbcb, const DevCb* __restrict__ cbs,
                                    const uint32_t* __restrict__ syn_a_part,
                                    uint8_t* __restrict__ tb_ok) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_tb) return;
  const DevTb d = tbs[t];
  uint32_t a = 0;
  for (int r = 0; r < d.n_cb; ++r) a ^= syn_a_part[d.first_cb + r];
  const int last = d.first_cb + d.n_cb - 1;
  const DevCb cb = cbs[last];
  const int64_t kept_end = tbcb[last].pos + cb.k - cb.filler - (d.n_cb > 1 ? 24 : 0);
  tb_ok[t] = (kept_end == d.tbs + 24) && a == 0;
}

std::vector<uint32_t> xpow_table(CrcKind kind, size_t n, Convention conv) {
  std::vector<uint32_t> t(n);
  const uint32_t g = crc_generator_mask(kind, conv);
  uint32_t r = 1;
  for (size_t j = 0; j < n; ++j) {
    t[j] = r;
    r <<= 1;
    if (r & (1u << 24)) r ^= (1u << 24) | g;
  }
  return t;
}

}  // namespace

// The de-rate kernels' shared memory above the default 48 KB: Ncb floats of the largest block
// (two buffers for HARQ combining).
void configure_chain_kernels() {
  check(cudaFuncSetAttribute(derate_llr_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kMaxNcb * static_cast<int>(sizeof(float))),
        "de-rate smem attr");
  check(cudaFuncSetAttribute(derate_combine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             2 * kMaxNcb * static_cast<int>(sizeof(float))),
        "combine smem attr");
}

// d012 = de-rate-matched LLRs of every block ([d0|d1|d2] each, at blocks[i].llr_offset).
void Decoder::derate_device(size_t n, const RmBlockDesc* blocks, const float* e_llr, size_t e_len,
                            float* d012, size_t llr_len, void* stream) {
  std::vector<DevRm> v(n);
  for (size_t i = 0; i < n; ++i) {
    const RmBlockDesc& b = blocks[i];
    if (qpp_index(b.k) < 0) throw OutOfRange("unsupported QPP block size");
    if (b.filler < 0 || b.filler >= b.k || b.rv > 3 || b.e < 0)
      throw InvalidArgument("invalid filler count, rv or E");
    if (b.e_offset < 0 || static_cast<size_t>(b.e_offset) + static_cast<size_t>(b.e) > e_len)
      throw InvalidArgument("rate-matched LLRs out of range");
    if (b.llr_offset < 0 || b.llr_offset % 4 != 0 ||
        static_cast<size_t>(b.llr_offset) + 3 * static_cast<size_t>(b.k + 4) > llr_len)
      throw InvalidArgument("invalid LLR offset (must be a multiple of 4 and in range)");
    v[i] = DevRm{b.k, b.filler, b.e, static_cast<int32_t>(b.rv), b.e_offset, b.llr_offset};
  }
  if (n == 0) return;
  DevRm* d = grow<DevRm>(d_rm_, n);
  upload(d, v.data(), n * sizeof(DevRm), stream);
  derate_llr_kernel<<<static_cast<unsigned>(n), kRmThreads, max_ncb(v) * sizeof(float),
                      static_cast<cudaStream_t>(stream)>>>(d, e_llr, d012);
  check(cudaGetLastError(), "de-rate launch");
  timing_.launches += 1;
}

// HARQ combining: transmissions of one code block are consecutive entries with the same
// llr_offset (and K, filler); each group's [d0|d1|d2] becomes the sum of its transmissions'
// de-rate-matched LLRs.
void Decoder::derate_combine_llr(size_t n, const RmBlockDesc* tx, const float* e_llr, size_t e_len,
                                 float* d012, size_t llr_len, void* stream) {
  std::lock_guard<std::mutex> lock(mu_);
  check(cudaSetDevice(device_), "cudaSetDevice");
  std::vector<DevRm> v(n);
  std::vector<int32_t> first;
  for (size_t i = 0; i < n; ++i) {
    const RmBlockDesc& b = tx[i];
    if (qpp_index(b.k) < 0) throw OutOfRange("unsupported QPP block size");
    if (b.filler < 0 || b.filler >= b.k || b.rv > 3 || b.e < 0)
      throw InvalidArgument("invalid filler count, rv or E");
    if (b.e_offset < 0 || static_cast<size_t>(b.e_offset) + static_cast<size_t>(b.e) > e_len)
      throw InvalidArgument("rate-matched LLRs out of range");
    if (b.llr_offset < 0 || b.llr_offset % 4 != 0 ||
        static_cast<size_t>(b.llr_offset) + 3 * static_cast<size_t>(b.k + 4) > llr_len)
      throw InvalidArgument("invalid LLR offset (must be a multiple of 4 and in range)");
    const bool same = i > 0 && b.llr_offset == tx[i - 1].llr_offset;
    if (same && (b.k != tx[i - 1].k || b.filler != tx[i - 1].filler))
      throw InvalidArgument("transmissions of one code block must agree on K and filler");
    if (!same) first.push_back(static_cast<int32_t>(i));
    else if (static_cast<int>(i) - first.back() >= kMaxHarqTx)
      throw InvalidArgument("at most 8 transmissions per code block");
    v[i] = DevRm{b.k, b.filler, b.e, static_cast<int32_t>(b.rv), b.e_offset, b.llr_offset};
  }
  if (n == 0) return;
  const size_t groups = first.size();
  first.push_back(static_cast<int32_t>(n));
  order_after_previous(stream);
  DevRm* d = grow<DevRm>(d_rm_, n);
  int32_t* g = grow<int32_t>(d_rmgroup_, groups + 1);
  upload(d, v.data(), n * sizeof(DevRm), stream);
  upload(g, first.data(), (groups + 1) * sizeof(int32_t), stream);
  derate_combine_kernel<<<static_cast<unsigned>(groups), kRmThreads,
                          2 * max_ncb(v) * sizeof(float), static_cast<cudaStream_t>(stream)>>>(
      d, g, e_llr, d012);
  check(cudaGetLastError(), "combine launch");
  timing_.launches += 1;
  mark_done(stream);
}

void Decoder::derate_match_llr(size_t n, const RmBlockDesc* blocks, const float* e_llr,
                               size_t e_len, float* d012, size_t llr_len, void* stream) {
  std::lock_guard<std::mutex> lock(mu_);
  check(cudaSetDevice(device_), "cudaSetDevice");
  order_after_previous(stream);
  derate_device(n, blocks, e_llr, e_len, d012, llr_len, stream);
  mark_done(stream);
}

// TC_MEM_HOST_ASYNC: the whole call goes to one of the worker decoders (own device buffers
// and stream, used in turn) and is not waited for, so that one call's copies overlap earlier
// calls' decoding; sync() waits for the workers.  Descriptor uploads read host vectors of this
// call, which cudaMemcpyAsync stages before it returns.
void Decoder::decode_transport_blocks(const TbRequest& q) {
  if (q.host_async && !q.device_memory) {
    std::lock_guard<std::mutex> lock(mu_);
    check(cudaSetDevice(device_), "cudaSetDevice");
    while (workers_.size() < kAsyncWorkers) workers_.push_back(std::make_unique<Decoder>(device_));
    Decoder& w = *workers_[next_worker_];
    next_worker_ = (next_worker_ + 1) % workers_.size();
    w.tuning_ = tuning_;  // SCHEDULE_AUTO resolves on the worker: give it this decoder's table
    TbRequest r = q;
    r.host_async = false;
    r.stream = nullptr;  // the worker's own stream
    const uint64_t launches_before = w.timing_.launches;
    // (no ordering across workers here: consecutive transport-block calls overlap each other's
    // de-rate matching, finish kernel and host work, measured faster than one at a time)
    w.transport_blocks(r, false);
    timing_.launches += w.timing_.launches - launches_before;
    return;
  }
  transport_blocks(q, true);
}

void Decoder::transport_blocks(const TbRequest& q, bool wait, void* after, void* done) {
  std::lock_guard<std::mutex> lock(mu_);
  check(cudaSetDevice(device_), "cudaSetDevice");
  cudaStream_t st = static_cast<cudaStream_t>(q.device_memory ? q.stream
                                                              : (q.stream ? q.stream : stream_));
  order_after_previous(st);
  // ---- validate the transport blocks and lay out their code blocks ----
  std::vector<DevTb> tbs(q.n_tb);
  std::vector<RmBlockDesc> rm(q.n_cb);
  std::vector<CodeBlockDesc> cbs(q.n_cb);
  int64_t llr_len = 0, post_len = 0, bits_len = 0;
  for (size_t i = 0; i < q.n_cb; ++i) {
    rm[i] = q.cbs[i];
    rm[i].llr_offset = llr_len;
    cbs[i] = CodeBlockDesc{q.cbs[i].k, q.cbs[i].filler, llr_len, post_len};
    llr_len += 3 * static_cast<int64_t>(q.cbs[i].k + 4);
    post_len += q.cbs[i].k;
  }
  for (size_t t = 0; t < q.n_tb; ++t) {
    const TbDesc& d = q.tbs[t];
    if (d.n_cb < 1 || d.first_cb < 0 || static_cast<size_t>(d.first_cb) + d.n_cb > q.n_cb || d.tbs < 1)
      throw InvalidArgument("invalid transport block descriptor");
    int64_t payload = 0;
    for (int r = 0; r < d.n_cb; ++r) {
      const auto& c = q.cbs[d.first_cb + r];
      payload += c.k - c.filler - (d.n_cb > 1 ? 24 : 0);
    }
    if (payload != d.tbs + 24)
      throw InvalidArgument("code blocks do not add up to TBS + 24 (segmentation mismatch)");
    if (d.bits_offset < 0 || static_cast<size_t>(d.bits_offset + d.tbs) > q.bits_len)
      throw InvalidArgument("transport block bits out of range");
    tbs[t] = DevTb{d.first_cb, d.n_cb, d.tbs, d.bits_offset};
    bits_len = std::max<int64_t>(bits_len, d.bits_offset + d.tbs);
  }
  // per code block: its transport block and the start of its kept bits in that block's stream
  // (a block that belongs to no transport block keeps tb = -1: decoded, then left out)
  std::vector<DevTbCb> tbcb(q.n_cb, DevTbCb{-1, 0});
  for (size_t t = 0; t < q.n_tb; ++t) {
    int64_t pos = 0;
    for (int r = 0; r < tbs[t].n_cb; ++r) {
      const auto& c = q.cbs[tbs[t].first_cb + r];
      if (tbcb[tbs[t].first_cb + r].tb >= 0)
        throw InvalidArgument("a code block belongs to two transport blocks");
      tbcb[tbs[t].first_cb + r] = DevTbCb{static_cast<int32_t>(t), static_cast<int32_t>(pos)};
      pos += c.k - c.filler - (tbs[t].n_cb > 1 ? 24 : 0);
    }
  }

  if (q.n_tb == 0) return;
  // ---- device buffers ----
  const float* e_llr = q.e_llr;
  if (!q.device_memory) {
    float* de = grow<float>(d_e_llr_, q.e_len);
    check(cudaMemcpyAsync(de, q.e_llr, q.e_len * sizeof(float), cudaMemcpyHostToDevice, st),
          "copy rate-matched LLRs in");
    e_llr = de;
  }
  if (after) check(cudaStreamWaitEvent(st, static_cast<cudaEvent_t>(after), 0), "cudaStreamWaitEvent");
  float* d012 = grow<float>(d_d012_, static_cast<size_t>(llr_len));
  float* post = grow<float>(d_tbpost_, static_cast<size_t>(post_len));
  uint8_t* bits = q.device_memory ? q.bits : grow<uint8_t>(d_tbbits_, q.bits_len);
  uint8_t* tb_ok = q.device_memory && q.tb_crc_ok ? q.tb_crc_ok : grow<uint8_t>(d_tbok_, q.n_tb);
  uint8_t* cb_ok = q.device_memory && q.cb_crc_ok ? q.cb_crc_ok : grow<uint8_t>(d_cbok_, q.n_cb);
  uint32_t* iters = q.device_memory && q.iterations_used ? q.iterations_used
                                                         : grow<uint32_t>(d_tbiters_, q.n_cb);
  DevTb* dtb = grow<DevTb>(d_tb_, q.n_tb);
  DevTbCb* dtbcb = grow<DevTbCb>(d_tbcb_, q.n_cb);
  uint32_t* dsyn = grow<uint32_t>(d_synpart_, q.n_cb);
  const bool std3gpp = q.decode.std3gpp;
  DeviceBuffer& xpow_a = std3gpp ? d_xpow_a_std_ : d_xpow_a_;  // x^j mod g_CRC24A
  if (xpow_a.bytes == 0) {
    const auto xa = xpow_table(CrcKind::Crc24A, 6144 * 17,  // > largest TB + CRC24A
                               std3gpp ? Convention::Std3gpp : Convention::Reference);
    xpow_a.reserve(xa.size() * 4);
    check(cudaMemcpy(xpow_a.ptr, xa.data(), xa.size() * 4, cudaMemcpyHostToDevice), "upload crc");
  }
  for (size_t t = 0; t < q.n_tb; ++t)
    if (tbs[t].tbs + 24 > static_cast<int64_t>(xpow_a.bytes / 4))
      throw CapacityExceeded("transport block larger than 104424 bits");
  // ---- de-rate matching, decoding, transport-block finish ----
  DecodeRequest rq = q.decode;
  rq.n_cb = q.n_cb;
  rq.cbs = cbs.data();
  rq.llr_len = static_cast<size_t>(llr_len);
  rq.llr = d012;
  rq.post_len = static_cast<size_t>(post_len);
  rq.posterior = post;
  rq.crc_ok = nullptr;
  rq.iterations_used = iters;
  rq.device_memory = true;
  rq.stream = st;
  rq.graph = false;
  if (rq.auto_schedule) rq = resolve_locked(rq);  // the tuning table's schedule and window
  auto body = [&] {
    derate_device(q.n_cb, rm.data(), e_llr, q.e_len, d012, static_cast<size_t>(llr_len), st);
    if (rq.persistent) decode_persistent(rq); else decode_plain(rq);
    // decode_* chained its own completion event; the finish kernel follows on the same stream
    upload(dtb, tbs.data(), q.n_tb * sizeof(DevTb), st);
    upload(dtbcb, tbcb.data(), q.n_cb * sizeof(DevTbCb), st);
    const DevCb* dcbs = static_cast<const DevCb*>(d_cbs_.ptr);
    tb_finish_cb_kernel<<<static_cast<unsigned>(q.n_cb), kFinishThreads, 0, st>>>(
        dtb, dtbcb, dcbs, post, static_cast<const uint32_t*>(xpow_a.ptr),
        static_cast<const uint32_t*>(std3gpp ? d_xpow_std_.ptr : d_xpow_.ptr), bits, cb_ok, dsyn);
    tb_finish_tb_kernel<<<static_cast<unsigned>((q.n_tb + 255) / 256), 256, 0, st>>>(
        dtb, static_cast<int>(q.n_tb), dtbcb, dcbs, dsyn, tb_ok);
    check(cudaGetLastError(), "finish launch");
    timing_.launches += 2;
    if (q.device_memory && q.posterior)
      check(cudaMemcpyAsync(q.posterior, post, static_cast<size_t>(post_len) * 4,
                            cudaMemcpyDeviceToDevice, st), "copy");
  };
  if (q.decode.graph && q.device_memory) {
    // capture once per key (every descriptor, buffer address and option baked into the
    // launches), then replay: one graph launch per call
    std::string key = "tb";
    auto put = [&key](const void* p, size_t n) { key.append(static_cast<const char*>(p), n); };
    const uintptr_t ptrs[6] = {reinterpret_cast<uintptr_t>(e_llr), reinterpret_cast<uintptr_t>(bits),
                               reinterpret_cast<uintptr_t>(tb_ok), reinterpret_cast<uintptr_t>(cb_ok),
                               reinterpret_cast<uintptr_t>(iters),
                               reinterpret_cast<uintptr_t>(q.posterior)};
    const int64_t opts[9] = {static_cast<int64_t>(q.n_tb), static_cast<int64_t>(q.n_cb),
                             static_cast<int64_t>(q.e_len), static_cast<int64_t>(q.bits_len),
                             rq.max_iterations, rq.early_stop, rq.window, rq.guard,
                             (rq.std3gpp ? 4 : 0) | (rq.persistent ? 2 : 0) | (rq.smem_checkpoints ? 1 : 0)};
    put(ptrs, sizeof ptrs);
    put(opts, sizeof opts);
    put(rm.data(), q.n_cb * sizeof(RmBlockDesc));
    put(tbs.data(), q.n_tb * sizeof(DevTb));
    if (rq.scales) put(rq.scales, 2 * rq.max_iterations * sizeof(float));
    launch_graph(graph_for(key, st, body), st);
    return;
  }
  body();
  if (done) check(cudaEventRecord(static_cast<cudaEvent_t>(done), st), "cudaEventRecord");
  if (!q.device_memory) {
    check(cudaMemcpyAsync(q.bits, bits, static_cast<size_t>(bits_len), cudaMemcpyDeviceToHost, st),
          "copy bits out");
    if (q.tb_crc_ok) check(cudaMemcpyAsync(q.tb_crc_ok, tb_ok, q.n_tb, cudaMemcpyDeviceToHost, st), "copy");
    if (q.cb_crc_ok) check(cudaMemcpyAsync(q.cb_crc_ok, cb_ok, q.n_cb, cudaMemcpyDeviceToHost, st), "copy");
    if (q.iterations_used)
      check(cudaMemcpyAsync(q.iterations_used, iters, q.n_cb * 4, cudaMemcpyDeviceToHost, st), "copy");
    if (q.posterior)
      check(cudaMemcpyAsync(q.posterior, post, static_cast<size_t>(post_len) * 4,
                            cudaMemcpyDeviceToHost, st), "copy");
  }
  mark_done(st);
  if (!q.device_memory && wait) {
    check(cudaStreamSynchronize(st), "sync");
    if (rq.persistent) take_error();
  }
}

}  // namespace tcb
