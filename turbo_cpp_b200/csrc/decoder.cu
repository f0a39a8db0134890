// decoder.cu -- the plain (host-driven) GPU turbo decoder and its device buffers.
//
// One tc_decode call decodes any number of code blocks of any LTE sizes.  Per full iteration
// the host enqueues two launches (upper SISO over natural order, lower SISO over QPP order) and,
// with early stop, one CRC24B launch; every thread owns one window of one code block.  This is
// the replacement of the reference's Stage 1/2 host loops (lte_turbo_cuda.cu:1391-1540,
// 1719-1899), batched over code blocks and correct for every K.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "decoder.hpp"
#include "lte_codec.hpp"
#include "decode_kernels.cuh"

namespace tcb {

namespace {

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess)
    throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
T* grow(DeviceBuffer& b, size_t count) {
  b.reserve(count * sizeof(T));
  return static_cast<T*>(b.ptr);
}

}  // namespace

// ------------------------------------------------------------------------------------------
void DeviceBuffer::reserve(size_t need) {
  if (need <= bytes) return;
  release();
  size_t n = std::max<size_t>(need, 256);
  n = n + n / 4;  // headroom for slightly larger later calls
  cudaError_t e = cudaMalloc(&ptr, n);
  if (e != cudaSuccess) {
    ptr = nullptr;
    bytes = 0;
    throw CudaError(std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  bytes = n;
}

void DeviceBuffer::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
}

Decoder::Decoder(int device) : device_(device) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    throw NoDevice("no CUDA device is visible");
  if (device < 0 || device >= count) throw InvalidArgument("device index out of range");
  check(cudaSetDevice(device_), "cudaSetDevice");
  cudaStream_t own = nullptr;
  check(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking), "cudaStreamCreate");
  stream_ = own;
  cudaDeviceProp prop{};
  check(cudaGetDeviceProperties(&prop, device_), "cudaGetDeviceProperties");
  sm_count_ = prop.multiProcessorCount;
  smem_optin_ = static_cast<int>(prop.sharedMemPerBlockOptin);

  // QPP permutation tables for all 188 block sizes, uint16 per position.
  std::vector<uint16_t> perm, inv;
  tab_offset_.resize(kQppCount);
  for (int i = 0; i < kQppCount; ++i) {
    const QppEntry e = qpp_entry(i);
    tab_offset_[i] = static_cast<int32_t>(perm.size());
    const auto p = qpp_permutation(e.k);
    std::vector<uint16_t> iv(e.k);
    for (int32_t j = 0; j < e.k; ++j) {
      perm.push_back(static_cast<uint16_t>(p[j]));
      iv[p[j]] = static_cast<uint16_t>(j);
    }
    inv.insert(inv.end(), iv.begin(), iv.end());
  }
  // x^j mod g_CRC24B for j < 6144
  std::vector<uint32_t> xpow(6144);
  const uint32_t g = crc_generator_mask(CrcKind::Crc24B);
  uint32_t r = 1;
  for (int j = 0; j < 6144; ++j) {
    xpow[j] = r;
    r <<= 1;
    if (r & (1u << 24)) r ^= (1u << 24) | g;
  }
  d_perm_.reserve(perm.size() * 2);
  d_inv_.reserve(inv.size() * 2);
  d_xpow_.reserve(xpow.size() * 4);
  check(cudaMemcpy(d_perm_.ptr, perm.data(), perm.size() * 2, cudaMemcpyHostToDevice), "upload perm");
  check(cudaMemcpy(d_inv_.ptr, inv.data(), inv.size() * 2, cudaMemcpyHostToDevice), "upload inv");
  check(cudaMemcpy(d_xpow_.ptr, xpow.data(), xpow.size() * 4, cudaMemcpyHostToDevice), "upload crc");
  d_err_.reserve(sizeof(int));
  check(cudaMemset(d_err_.ptr, 0, sizeof(int)), "zero error word");

  const int smem = smem_optin_;
  check(cudaFuncSetAttribute(siso_plain_kernel<kSub, 0, false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "smem attr");
  check(cudaFuncSetAttribute(siso_plain_kernel<kSub, 1, false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "smem attr");
  check(cudaFuncSetAttribute(siso_plain_kernel<kSub, 2, false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "smem attr");
  for (const void* f : {reinterpret_cast<const void*>(siso_plain_kernel<kSub, 0, true>),
                        reinterpret_cast<const void*>(siso_plain_kernel<kSub, 1, true>),
                        reinterpret_cast<const void*>(siso_plain_kernel<kSub, 2, true>)})
    check(cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 0),
          "carveout attr");
  check(cudaFuncSetAttribute(persistent_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 0),
        "carveout attr");
  check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&persist_blocks_per_sm_, persistent_kernel,
                                                      kPersistThreads, 0),
        "occupancy");
}

Decoder::~Decoder() {
  cudaSetDevice(device_);
  if (last_event_) cudaEventDestroy(static_cast<cudaEvent_t>(last_event_));
  d_err_.release();
  for (auto& e : events_) {
    if (e.start) cudaEventDestroy(static_cast<cudaEvent_t>(e.start));
    if (e.stop) cudaEventDestroy(static_cast<cudaEvent_t>(e.stop));
  }
  if (stream_) cudaStreamDestroy(static_cast<cudaStream_t>(stream_));
  for (DeviceBuffer* b : {&d_perm_, &d_inv_, &d_xpow_, &d_cbs_, &d_wincb_, &d_start_, &d_llr_,
                          &d_sysi_, &d_e1i_, &d_e2_, &d_post_, &d_seed_, &d_done_, &d_iters_,
                          &d_crc_, &d_ckpt_})
    b->release();
}

void Decoder::order_after_previous(void* stream) {
  if (last_event_)
    check(cudaStreamWaitEvent(static_cast<cudaStream_t>(stream),
                              static_cast<cudaEvent_t>(last_event_), 0), "cudaStreamWaitEvent");
}

void Decoder::mark_done(void* stream) {
  if (!last_event_) {
    cudaEvent_t e;
    check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    last_event_ = e;
  }
  check(cudaEventRecord(static_cast<cudaEvent_t>(last_event_), static_cast<cudaStream_t>(stream)),
        "cudaEventRecord");
}

void Decoder::take_error() {
  int err = 0;
  check(cudaMemcpy(&err, d_err_.ptr, sizeof(int), cudaMemcpyDeviceToHost), "read error word");
  if (err != 0) {
    check(cudaMemset(d_err_.ptr, 0, sizeof(int)), "clear error word");
    throw DeviceTimeout("a persistent-schedule wait gave up (device queue stalled)");
  }
}

void Decoder::sync() {
  std::lock_guard<std::mutex> lock(mu_);
  check(cudaSetDevice(device_), "cudaSetDevice");
  if (last_event_)
    check(cudaEventSynchronize(static_cast<cudaEvent_t>(last_event_)), "cudaEventSynchronize");
  take_error();
}

void Decoder::set_timing(bool on) {
  std::lock_guard<std::mutex> lock(mu_);
  timing_on_ = on;
}

void Decoder::record_start(void* stream) {
  if (!timing_on_) return;
  if (events_used_ == events_.size()) {
    EventPair p;
    cudaEvent_t a, b;
    check(cudaEventCreate(&a), "cudaEventCreate");
    check(cudaEventCreate(&b), "cudaEventCreate");
    p.start = a;
    p.stop = b;
    events_.push_back(p);
  }
  check(cudaEventRecord(static_cast<cudaEvent_t>(events_[events_used_].start),
                        static_cast<cudaStream_t>(stream)), "cudaEventRecord");
}

void Decoder::record_stop(void* stream, uint64_t steps) {
  if (!timing_on_) return;
  EventPair& p = events_[events_used_++];
  p.steps = steps;
  check(cudaEventRecord(static_cast<cudaEvent_t>(p.stop), static_cast<cudaStream_t>(stream)),
        "cudaEventRecord");
}

Timing Decoder::timing(bool reset) {
  std::lock_guard<std::mutex> lock(mu_);
  check(cudaSetDevice(device_), "cudaSetDevice");
  for (size_t i = 0; i < events_used_; ++i) {
    float ms = 0.0f;
    check(cudaEventSynchronize(static_cast<cudaEvent_t>(events_[i].stop)), "cudaEventSynchronize");
    check(cudaEventElapsedTime(&ms, static_cast<cudaEvent_t>(events_[i].start),
                               static_cast<cudaEvent_t>(events_[i].stop)), "cudaEventElapsedTime");
    timing_.siso_ms += ms;
    timing_.siso_launches += 1;
    timing_.trellis_steps += events_[i].steps;
  }
  events_used_ = 0;
  const Timing t = timing_;
  if (reset) timing_ = Timing{};
  return t;
}

int Decoder::pick_window(int32_t k, int32_t requested) const {
  if (requested > 0) return std::min<int32_t>(requested, k);
  return std::min<int32_t>(kDefaultWindow, k);
}

void Decoder::decode(const DecodeRequest& rq) {
  if (rq.persistent) {
    decode_persistent(rq);
    return;
  }
  std::lock_guard<std::mutex> lock(mu_);
  check(cudaSetDevice(device_), "cudaSetDevice");
  // device memory: the caller's stream as given (NULL = legacy default stream, as in CUDA);
  // host memory: the caller's stream if given, else the decoder's own stream
  cudaStream_t st = static_cast<cudaStream_t>(rq.device_memory ? rq.stream
                                                               : (rq.stream ? rq.stream : stream_));
  const size_t n = rq.n_cb;
  if (n == 0) return;

  // ---- validate and lay out ----
  if (reinterpret_cast<uintptr_t>(rq.llr) % 16 != 0)
    throw InvalidArgument("the LLR buffer must be 16-byte aligned");
  order_after_previous(st);
  const int guard = rq.guard < 0 ? kDefaultGuard : rq.guard;
  if (guard % kGroup != 0) throw InvalidArgument("guard must be a multiple of 8");
  std::vector<DevCb> cbs(n);
  std::vector<int64_t> start(n);
  std::vector<int32_t> wincb;
  int64_t work = 0;
  int max_ckpt = 0;
  for (size_t i = 0; i < n; ++i) {
    const int32_t k = rq.cbs[i].k;
    const int qi = qpp_index(k);
    if (qi < 0) throw OutOfRange("unsupported QPP block size");
    if (rq.cbs[i].filler < 0 || rq.cbs[i].filler >= k) throw InvalidArgument("invalid filler count");
    if (rq.cbs[i].llr_offset < 0 || rq.cbs[i].llr_offset % 4 != 0 ||
        static_cast<size_t>(rq.cbs[i].llr_offset) + 3 * static_cast<size_t>(k + 4) > rq.llr_len)
      throw InvalidArgument("invalid LLR offset (must be a multiple of 4 and in range)");
    if (rq.cbs[i].out_offset < 0 ||
        static_cast<size_t>(rq.cbs[i].out_offset) + static_cast<size_t>(k) > rq.post_len)
      throw InvalidArgument("invalid posterior offset");
    DevCb& d = cbs[i];
    d.k = k;
    d.filler = rq.cbs[i].filler;
    d.tab = tab_offset_[qi];
    d.window = pick_window(k, rq.window);
    if (d.window % kGroup != 0) throw InvalidArgument("window must be a multiple of 8");
    if (guard > d.window && d.window < k) throw InvalidArgument("guard must not exceed the window");
    d.nwin = (k + d.window - 1) / d.window;
    d.win0 = static_cast<int32_t>(wincb.size());
    d.llr = rq.cbs[i].llr_offset;
    d.work = work;
    d.out = rq.cbs[i].out_offset;
    start[i] = work;
    work += k;
    max_ckpt = std::max(max_ckpt, d.window / kSub);
    for (int w = 0; w < d.nwin; ++w) wincb.push_back(static_cast<int32_t>(i));
  }
  const int n_win = static_cast<int>(wincb.size());
  // Checkpoints live in a global scratch slot per window: 8 B of traffic per output step, and
  // leaving shared memory unused gives the L1 cache the whole 256 KB for the input streams.
  const size_t ckpt_bytes = static_cast<size_t>(kThreads) * max_ckpt * 2 * sizeof(float4);
  const bool global_ckpt = rq.smem_checkpoints ? ckpt_bytes > static_cast<size_t>(smem_optin_)
                                               : true;

  // ---- device buffers ----
  DevCb* dcbs = grow<DevCb>(d_cbs_, n);
  int32_t* dwin = grow<int32_t>(d_wincb_, n_win);
  int64_t* dstart = grow<int64_t>(d_start_, n);
  float* sysi = grow<float>(d_sysi_, work);
  float* e1i = grow<float>(d_e1i_, work);
  float* e2 = grow<float>(d_e2_, work);
  float* seeds = grow<float>(d_seed_, static_cast<size_t>(n_win) * 16 * 4);
  uint8_t* done = grow<uint8_t>(d_done_, n);
  uint32_t* iters = (rq.device_memory && rq.iterations_used) ? rq.iterations_used
                                                              : grow<uint32_t>(d_iters_, n);
  uint8_t* crc = (rq.device_memory && rq.crc_ok) ? rq.crc_ok : grow<uint8_t>(d_crc_, n);
  const float* llr = rq.llr;
  float* post = rq.posterior;
  if (!rq.device_memory) {
    float* dl = grow<float>(d_llr_, rq.llr_len);
    check(cudaMemcpyAsync(dl, rq.llr, rq.llr_len * sizeof(float), cudaMemcpyHostToDevice, st),
          "copy LLRs in");
    llr = dl;
    post = grow<float>(d_post_, rq.post_len);
    // positions outside every block's range come back as 0
    check(cudaMemsetAsync(post, 0, rq.post_len * sizeof(float), st), "zero posterior");
  }
  float4* ckpt = nullptr;
  if (global_ckpt) ckpt = grow<float4>(d_ckpt_, static_cast<size_t>(n_win) * 2 * max_ckpt);

  check(cudaMemcpyAsync(dcbs, cbs.data(), n * sizeof(DevCb), cudaMemcpyHostToDevice, st), "copy cbs");
  check(cudaMemcpyAsync(dwin, wincb.data(), n_win * sizeof(int32_t), cudaMemcpyHostToDevice, st),
        "copy windows");
  check(cudaMemcpyAsync(dstart, start.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice, st),
        "copy starts");
  check(cudaMemsetAsync(seeds, 0, static_cast<size_t>(n_win) * 16 * 4 * sizeof(float), st), "zero seeds");
  init_flags_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(
      static_cast<int>(n), done, iters, rq.max_iterations);
  check(cudaGetLastError(), "init launch");

  const uint16_t* dperm = static_cast<const uint16_t*>(d_perm_.ptr);
  const uint16_t* dinv = static_cast<const uint16_t*>(d_inv_.ptr);
  timing_.launches += 3;  // init, setup, finish
  setup_kernel<<<static_cast<unsigned>((work + 255) / 256), 256, 0, st>>>(
      dcbs, dstart, static_cast<int>(n), work, llr, dperm, sysi, e2);
  check(cudaGetLastError(), "setup launch");

  const int blocks = (n_win + kThreads - 1) / kThreads;
  const size_t smem = global_ckpt ? 0 : ckpt_bytes;
  const size_t seed_slab = static_cast<size_t>(n_win) * 16;
  float* seed_up[2] = {seeds, seeds + seed_slab};
  float* seed_lo[2] = {seeds + 2 * seed_slab, seeds + 3 * seed_slab};
  for (uint32_t it = 0; it < rq.max_iterations; ++it) {
    const float s_up = rq.scales ? rq.scales[2 * it] : 1.0f;
    const float s_lo = rq.scales ? rq.scales[2 * it + 1] : 1.0f;
    SisoIo up{llr, sysi, e2, e1i, nullptr, dperm, dinv, seed_up[it & 1], seed_up[(it + 1) & 1],
              s_up, guard};
    SisoIo lo{llr, sysi, e1i, e2, post, dperm, dinv, seed_lo[it & 1], seed_lo[(it + 1) & 1],
              s_lo, guard};
    const uint8_t* dn = rq.early_stop ? done : nullptr;
    // the posterior is needed after the last iteration and, with early stop, after each one
    const bool post_now = rq.early_stop || it + 1 == rq.max_iterations;
    for (int half = 0; half < 2; ++half) {
      const SisoIo& io = half ? lo : up;
      const int kind = half == 0 ? 0 : (post_now ? 2 : 1);
      record_start(st);
      if (global_ckpt) {
        if (kind == 0) siso_plain_kernel<kSub, 0, true><<<blocks, kThreads, 0, st>>>(dcbs, dwin, n_win, io, dn, ckpt, max_ckpt);
        else if (kind == 1) siso_plain_kernel<kSub, 1, true><<<blocks, kThreads, 0, st>>>(dcbs, dwin, n_win, io, dn, ckpt, max_ckpt);
        else siso_plain_kernel<kSub, 2, true><<<blocks, kThreads, 0, st>>>(dcbs, dwin, n_win, io, dn, ckpt, max_ckpt);
      } else {
        if (kind == 0) siso_plain_kernel<kSub, 0, false><<<blocks, kThreads, smem, st>>>(dcbs, dwin, n_win, io, dn, nullptr, 0);
        else if (kind == 1) siso_plain_kernel<kSub, 1, false><<<blocks, kThreads, smem, st>>>(dcbs, dwin, n_win, io, dn, nullptr, 0);
        else siso_plain_kernel<kSub, 2, false><<<blocks, kThreads, smem, st>>>(dcbs, dwin, n_win, io, dn, nullptr, 0);
      }
      check(cudaGetLastError(), "SISO launch");
      record_stop(st, static_cast<uint64_t>(work));
      timing_.launches += 1;
    }
    if (rq.early_stop) {
      crc_stop_kernel<<<static_cast<unsigned>((n * 32 + 255) / 256), 256, 0, st>>>(
          dcbs, static_cast<int>(n), post, static_cast<const uint32_t*>(d_xpow_.ptr), done, iters,
          static_cast<int>(it));
      check(cudaGetLastError(), "CRC launch");
      timing_.launches += 1;
    }
  }
  finish_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(static_cast<int>(n), done, crc,
                                                                         rq.early_stop ? 1 : 0);
  check(cudaGetLastError(), "finish launch");
  if (!rq.device_memory) {
    check(cudaMemcpyAsync(rq.posterior, post, rq.post_len * sizeof(float), cudaMemcpyDeviceToHost, st),
          "copy posterior out");
    if (rq.crc_ok) check(cudaMemcpyAsync(rq.crc_ok, crc, n, cudaMemcpyDeviceToHost, st), "copy crc out");
    if (rq.iterations_used)
      check(cudaMemcpyAsync(rq.iterations_used, iters, n * 4, cudaMemcpyDeviceToHost, st), "copy iters out");
  }
  mark_done(st);
  if (!rq.device_memory) check(cudaStreamSynchronize(st), "sync");
}

// ------------------------------------------------------------------------------------------
// Persistent schedule: warp tasks of whole code blocks, one launch for all iterations.
// ------------------------------------------------------------------------------------------
void Decoder::decode_persistent(const DecodeRequest& rq) {
  std::lock_guard<std::mutex> lock(mu_);
  check(cudaSetDevice(device_), "cudaSetDevice");
  cudaStream_t st = static_cast<cudaStream_t>(rq.device_memory ? rq.stream
                                                               : (rq.stream ? rq.stream : stream_));
  const size_t n = rq.n_cb;
  if (n == 0) return;
  if (reinterpret_cast<uintptr_t>(rq.llr) % 16 != 0)
    throw InvalidArgument("the LLR buffer must be 16-byte aligned");
  order_after_previous(st);
  if (rq.max_iterations > static_cast<uint32_t>(kMaxIterations))
    throw InvalidArgument("max_iterations above 64");
  const int guard = rq.guard < 0 ? kDefaultGuard : rq.guard;
  if (guard % kGroup != 0) throw InvalidArgument("guard must be a multiple of 8");
  const int target = rq.window > 0 ? rq.window : kPersistWindow;

  // ---- per block: at most 32 windows of >= `target` steps (a multiple of 8, >= guard) ----
  std::vector<DevCb> cbs(n);
  std::vector<int64_t> start(n);
  int64_t work = 0;
  int max_ckpt = 0;
  for (size_t i = 0; i < n; ++i) {
    const int32_t k = rq.cbs[i].k;
    const int qi = qpp_index(k);
    if (qi < 0) throw OutOfRange("unsupported QPP block size");
    if (rq.cbs[i].filler < 0 || rq.cbs[i].filler >= k) throw InvalidArgument("invalid filler count");
    if (rq.cbs[i].llr_offset < 0 || rq.cbs[i].llr_offset % 4 != 0 ||
        static_cast<size_t>(rq.cbs[i].llr_offset) + 3 * static_cast<size_t>(k + 4) > rq.llr_len)
      throw InvalidArgument("invalid LLR offset (must be a multiple of 4 and in range)");
    if (rq.cbs[i].out_offset < 0 ||
        static_cast<size_t>(rq.cbs[i].out_offset) + static_cast<size_t>(k) > rq.post_len)
      throw InvalidArgument("invalid posterior offset");
    DevCb& d = cbs[i];
    d.k = k;
    d.filler = rq.cbs[i].filler;
    d.tab = tab_offset_[qi];
    int nwin = std::max(1, std::min(32, k / std::max(target, 8)));
    int wlen = ((k + nwin - 1) / nwin + kGroup - 1) / kGroup * kGroup;
    if (nwin > 1 && wlen < guard) {  // windows may not be shorter than the guard
      nwin = std::max(1, k / guard);
      wlen = ((k + nwin - 1) / nwin + kGroup - 1) / kGroup * kGroup;
    }
    d.window = std::min<int32_t>(wlen, k);
    d.nwin = (k + d.window - 1) / d.window;
    d.llr = rq.cbs[i].llr_offset;
    d.work = work;
    d.out = rq.cbs[i].out_offset;
    start[i] = work;
    work += k;
    max_ckpt = std::max(max_ckpt, d.window / kSub);
  }
  // ---- tasks: blocks sorted by size, largest first, packed first-fit into 32 lanes ----
  std::vector<int32_t> order(n);
  for (size_t i = 0; i < n; ++i) order[i] = static_cast<int32_t>(i);
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
    return cbs[a].nwin != cbs[b].nwin ? cbs[a].nwin > cbs[b].nwin : cbs[a].k > cbs[b].k;
  });
  std::vector<int32_t> wincb, tasks;
  int lanes_used = 32;
  for (const int32_t i : order) {
    DevCb& d = cbs[i];
    if (lanes_used + d.nwin > 32) {  // open a new task
      tasks.insert(tasks.end(), 32, -1);
      lanes_used = 0;
    }
    d.win0 = static_cast<int32_t>(wincb.size());
    for (int w = 0; w < d.nwin; ++w) {
      tasks[tasks.size() - 32 + lanes_used + w] = static_cast<int32_t>(wincb.size());
      wincb.push_back(i);
    }
    lanes_used += d.nwin;
  }
  const int n_tasks = static_cast<int>(tasks.size() / 32);
  const int n_win = static_cast<int>(wincb.size());

  // ---- device buffers ----
  DevCb* dcbs = grow<DevCb>(d_cbs_, n);
  int32_t* dwin = grow<int32_t>(d_wincb_, n_win);
  int64_t* dstart = grow<int64_t>(d_start_, n);
  int32_t* dtasks = grow<int32_t>(d_tasks_, tasks.size());
  int* dqueue = grow<int>(d_queue_, 2 + static_cast<size_t>(n_tasks));  // queue, error, progress
  float* sysi = grow<float>(d_sysi_, work);
  float* e1i = grow<float>(d_e1i_, work);
  float* e2 = grow<float>(d_e2_, work);
  float* seeds = grow<float>(d_seed_, static_cast<size_t>(n_win) * 16 * 4);
  float4* ckpt = grow<float4>(d_ckpt_, static_cast<size_t>(n_win) * 2 * max_ckpt);
  uint8_t* done = grow<uint8_t>(d_done_, n);
  uint32_t* iters = (rq.device_memory && rq.iterations_used) ? rq.iterations_used
                                                              : grow<uint32_t>(d_iters_, n);
  uint8_t* crc = (rq.device_memory && rq.crc_ok) ? rq.crc_ok : grow<uint8_t>(d_crc_, n);
  const float* llr = rq.llr;
  float* post = rq.posterior;
  if (!rq.device_memory) {
    float* dl = grow<float>(d_llr_, rq.llr_len);
    check(cudaMemcpyAsync(dl, rq.llr, rq.llr_len * sizeof(float), cudaMemcpyHostToDevice, st),
          "copy LLRs in");
    llr = dl;
    post = grow<float>(d_post_, rq.post_len);
    check(cudaMemsetAsync(post, 0, rq.post_len * sizeof(float), st), "zero posterior");
  }
  check(cudaMemcpyAsync(dcbs, cbs.data(), n * sizeof(DevCb), cudaMemcpyHostToDevice, st), "copy cbs");
  check(cudaMemcpyAsync(dwin, wincb.data(), n_win * sizeof(int32_t), cudaMemcpyHostToDevice, st),
        "copy windows");
  check(cudaMemcpyAsync(dstart, start.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice, st),
        "copy starts");
  check(cudaMemcpyAsync(dtasks, tasks.data(), tasks.size() * sizeof(int32_t),
                        cudaMemcpyHostToDevice, st), "copy tasks");
  check(cudaMemsetAsync(dqueue, 0, (2 + static_cast<size_t>(n_tasks)) * sizeof(int), st),
        "zero queue");
  check(cudaMemsetAsync(seeds, 0, static_cast<size_t>(n_win) * 16 * 4 * sizeof(float), st),
        "zero seeds");
  init_flags_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(
      static_cast<int>(n), done, iters, rq.max_iterations);
  setup_kernel<<<static_cast<unsigned>((work + 255) / 256), 256, 0, st>>>(
      dcbs, dstart, static_cast<int>(n), work, llr, static_cast<const uint16_t*>(d_perm_.ptr),
      sysi, e2);
  check(cudaGetLastError(), "set-up launch");

  PersistArgs a{};
  a.cbs = dcbs;
  a.win_cb = dwin;
  a.tasks = dtasks;
  a.n_tasks = n_tasks;
  a.queue = dqueue;
  a.error = static_cast<int*>(d_err_.ptr);
  a.progress = dqueue + 2;
  a.llr = llr;
  a.sys_i = sysi;
  a.e1i = e1i;
  a.e2 = e2;
  a.post = post;
  a.perm = static_cast<const uint16_t*>(d_perm_.ptr);
  a.inv = static_cast<const uint16_t*>(d_inv_.ptr);
  const size_t slab = static_cast<size_t>(n_win) * 16;
  a.seed_up[0] = seeds;
  a.seed_up[1] = seeds + slab;
  a.seed_lo[0] = seeds + 2 * slab;
  a.seed_lo[1] = seeds + 3 * slab;
  a.ckpt = ckpt;
  a.ckpt_per_window = max_ckpt;
  a.guard = guard;
  a.max_iterations = static_cast<int>(rq.max_iterations);
  a.early_stop = rq.early_stop ? 1 : 0;
  a.done = done;
  a.iters = iters;
  a.xpow = static_cast<const uint32_t*>(d_xpow_.ptr);
  for (int i = 0; i < 2 * kMaxIterations; ++i)
    a.scale[i] = (rq.scales && i < 2 * static_cast<int>(rq.max_iterations)) ? rq.scales[i] : 1.0f;
  const int grid = std::max(1, sm_count_ * std::max(persist_blocks_per_sm_, 1));
  record_start(st);
  persistent_kernel<<<grid, kPersistThreads, 0, st>>>(a);
  check(cudaGetLastError(), "persistent launch");
  record_stop(st, static_cast<uint64_t>(work) * 2 * rq.max_iterations);
  finish_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(static_cast<int>(n), done,
                                                                         crc, rq.early_stop ? 1 : 0);
  check(cudaGetLastError(), "finish launch");
  timing_.launches += 4;
  if (!rq.device_memory) {
    check(cudaMemcpyAsync(rq.posterior, post, rq.post_len * sizeof(float), cudaMemcpyDeviceToHost, st),
          "copy posterior out");
    if (rq.crc_ok) check(cudaMemcpyAsync(rq.crc_ok, crc, n, cudaMemcpyDeviceToHost, st), "copy crc out");
    if (rq.iterations_used)
      check(cudaMemcpyAsync(rq.iterations_used, iters, n * 4, cudaMemcpyDeviceToHost, st),
            "copy iters out");
    mark_done(st);
    check(cudaStreamSynchronize(st), "sync");
    take_error();
  } else {
    mark_done(st);
  }
}

}  // namespace tcb
