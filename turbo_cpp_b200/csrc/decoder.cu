// decoder.cu -- the plain (host-driven) GPU turbo decoder and its device buffers.
//
// One tc_decode call decodes any number of code blocks of any LTE sizes.  Per full iteration
// the host enqueues two launches (upper SISO over natural order, lower SISO over QPP order) and,
// with early stop, one CRC24B launch; every thread owns one window of one code block.  This is
// the replacement of the reference's Stage 1/2 host loops (lte_turbo_cuda.cu:1391-1540,
// 1719-1899), batched over code blocks and correct for every K.
#include <cuda_runtime.h>

#include <functional>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
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

}  // namespace

void Decoder::upload(void* dst, const void* src, size_t bytes, void* stream) {
  if (bytes == 0) return;
  const size_t padded = (bytes + 255) & ~size_t{255};
  upload_bytes_ += padded;
  if (capturing_ != nullptr) {  // the graph reads its own pinned copy at every replay
    GraphEntry& g = *capturing_;
    if (g.arena_used + padded > g.arena_bytes)
      throw CudaError("graph descriptor arena too small");
    char* pinned = static_cast<char*>(g.arena) + g.arena_used;
    g.arena_used += padded;
    std::memcpy(pinned, src, bytes);
    src = pinned;
  }
  check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, static_cast<cudaStream_t>(stream)),
        "copy descriptors");
}

void Decoder::drop_graph(GraphEntry& e) {
  if (e.exec) cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(e.exec));
  if (e.arena) cudaFreeHost(e.arena);
  e.exec = nullptr;
  e.arena = nullptr;
}

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
  {  // the same for TS 36.212's CRC24B
    const uint32_t gs = crc_generator_mask(CrcKind::Crc24B, Convention::Std3gpp);
    uint32_t q = 1;
    for (int j = 0; j < 6144; ++j) {
      xpow[j] = q;
      q <<= 1;
      if (q & (1u << 24)) q ^= (1u << 24) | gs;
    }
    d_xpow_std_.reserve(xpow.size() * 4);
    check(cudaMemcpy(d_xpow_std_.ptr, xpow.data(), xpow.size() * 4, cudaMemcpyHostToDevice),
          "upload crc");
  }
  d_err_.reserve(sizeof(int));
  check(cudaMemset(d_err_.ptr, 0, sizeof(int)), "zero error word");

  const int smem = smem_optin_;
  for (const void* f : {reinterpret_cast<const void*>(siso_plain_kernel<kSub, 0, false>),
                        reinterpret_cast<const void*>(siso_plain_kernel<kSub, 1, false>),
                        reinterpret_cast<const void*>(siso_plain_kernel<kSub, 2, false>),
                        reinterpret_cast<const void*>(siso_plain_kernel<kSub, 0, false, true>),
                        reinterpret_cast<const void*>(siso_plain_kernel<kSub, 1, false, true>),
                        reinterpret_cast<const void*>(siso_plain_kernel<kSub, 2, false, true>)})
    check(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "smem attr");
  for (const void* f : {reinterpret_cast<const void*>(siso_plain_kernel<kSub, 0, true>),
                        reinterpret_cast<const void*>(siso_plain_kernel<kSub, 1, true>),
                        reinterpret_cast<const void*>(siso_plain_kernel<kSub, 2, true>),
                        reinterpret_cast<const void*>(siso_plain_kernel<kSub, 0, true, true>),
                        reinterpret_cast<const void*>(siso_plain_kernel<kSub, 1, true, true>),
                        reinterpret_cast<const void*>(siso_plain_kernel<kSub, 2, true, true>),
                        reinterpret_cast<const void*>(persistent_kernel<false>),
                        reinterpret_cast<const void*>(persistent_kernel<true>)})
    check(cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 0),
          "carveout attr");
  configure_chain_kernels();
  int per_sm_std = 0;
  check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_std, persistent_kernel<true>,
                                                      kPersistThreads, 0),
        "occupancy");
  check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&persist_blocks_per_sm_, persistent_kernel<false>,
                                                      kPersistThreads, 0),
        "occupancy");
  persist_blocks_per_sm_ = std::min(persist_blocks_per_sm_, per_sm_std);
}

Decoder::~Decoder() {
  cudaSetDevice(device_);
  for (auto& g : graphs_) drop_graph(g);
  if (last_event_) cudaEventDestroy(static_cast<cudaEvent_t>(last_event_));
  if (compute_done_) cudaEventDestroy(static_cast<cudaEvent_t>(compute_done_));
  d_err_.release();
  for (auto& e : events_) {
    if (e.start) cudaEventDestroy(static_cast<cudaEvent_t>(e.start));
    if (e.stop) cudaEventDestroy(static_cast<cudaEvent_t>(e.stop));
  }
  workers_.clear();  // each waits for its own work (cudaFree) and releases its buffers
  if (stream_) cudaStreamDestroy(static_cast<cudaStream_t>(stream_));
  for (DeviceBuffer* b : {&d_perm_, &d_inv_, &d_xpow_, &d_xpow_std_, &d_xpow_a_std_, &d_cbs_, &d_wincb_, &d_llr_,
                          &d_sysi_, &d_e1i_, &d_e2_, &d_post_, &d_seed_, &d_done_, &d_iters_,
                          &d_crc_, &d_ckpt_, &d_tasks_, &d_queue_, &d_rm_, &d_e_llr_, &d_d012_,
                          &d_tbpost_, &d_tbbits_, &d_tbok_, &d_cbok_, &d_tbiters_, &d_tb_, &d_tbcb_, &d_synpart_,
                          &d_xpow_a_, &d_rmgroup_, &d_gen_, &d_gentab_, &d_genenc_, &d_genrm_})
    b->release();
}

void Decoder::order_after_previous(void* stream) {
  if (capturing_ != nullptr) return;  // a replayed graph is ordered at its launch
  if (last_event_)
    check(cudaStreamWaitEvent(static_cast<cudaStream_t>(stream),
                              static_cast<cudaEvent_t>(last_event_), 0), "cudaStreamWaitEvent");
}

void Decoder::mark_done(void* stream) {
  if (capturing_ != nullptr) return;
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
  for (auto& w : workers_) w->sync();  // asynchronous host-memory calls (and their timeouts)
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

int32_t Decoder::table_offset(int32_t k) const {
  const int qi = qpp_index(k);
  if (qi < 0) throw OutOfRange("unsupported QPP block size");
  return tab_offset_[qi];
}

int Decoder::pick_window(int32_t k, int32_t requested) const {
  if (requested > 0) return std::min<int32_t>(requested, k);
  return std::min<int32_t>(kDefaultWindow, k);
}

void Decoder::decode(const DecodeRequest& rq_in) {
  const DecodeRequest rq = rq_in.auto_schedule ? resolve(rq_in) : rq_in;
  if (rq.graph && rq.device_memory && rq.n_cb > 0) {
    decode_graph(rq);
    return;
  }
  std::lock_guard<std::mutex> lock(mu_);
  if (rq.host_async) {
    decode_host_async(rq);
    return;
  }
  if (rq.persistent)
    decode_persistent(rq);
  else
    decode_plain(rq);
}

// ------------------------------------------------------------------------------------------
// Autotuner
// ------------------------------------------------------------------------------------------
std::string Decoder::signature(const DecodeRequest& rq) {
  double sum_k = 0.0;
  for (size_t i = 0; i < rq.n_cb; ++i) sum_k += rq.cbs[i].k;
  const int mean_k = rq.n_cb ? static_cast<int>(std::lround(sum_k / rq.n_cb / 512.0)) * 512 : 0;
  const int n_log2 = rq.n_cb ? static_cast<int>(std::lround(std::log2(static_cast<double>(rq.n_cb)))) : 0;
  std::ostringstream o;
  o << "es=" << (rq.early_stop ? 1 : 0) << ",it=" << rq.max_iterations << ",n~2^" << n_log2
    << ",meanK~" << mean_k << ",guard=" << rq.guard << (rq.std3gpp ? ",std3gpp" : "");
  return o.str();
}

DecodeRequest Decoder::resolve(const DecodeRequest& rq) {
  std::lock_guard<std::mutex> lock(mu_);
  return resolve_locked(rq);
}

DecodeRequest Decoder::resolve_locked(const DecodeRequest& rq) const {
  DecodeRequest r = rq;
  r.auto_schedule = false;
  const std::string sig = signature(rq);
  for (const auto& kv : tuning_)
    if (kv.first == sig) {
      r.persistent = kv.second.persistent;
      if (rq.window == 0) r.window = kv.second.window;
      return r;
    }
  return r;  // untuned: plain schedule, default window
}

Decoder::TuneChoice Decoder::autotune(const DecodeRequest& rq_in) {
  if (!rq_in.device_memory) throw InvalidArgument("autotuning needs device-memory buffers");
  if (rq_in.n_cb == 0) throw InvalidArgument("nothing to tune");
  struct Cand {
    bool persistent;
    int window;
  };
  std::vector<Cand> cands = {{false, 128}, {false, 144}, {false, 160}, {false, 168},
                             {false, 176}, {false, 192}, {false, 224}, {false, 256},
                             {true, 192},  {true, 256},  {true, 320}};
  const int guard = rq_in.guard < 0 ? kDefaultGuard : rq_in.guard;
  // Plain-schedule windows that fill whole waves: the smallest window (a multiple of 8, at
  // least the guard) whose windows over all blocks fit in j resident waves of the SISO kernel
  // (SMs x blocks per SM x threads per block), for j = 1 .. 4.  A launch with a partly filled
  // last wave idles SMs for the length of a window (measured at 4096 x K=6144: window 136 = two
  // full waves 2606 Mbit/s, window 128 = 2.07 waves 2457 Mbit/s); one wave of long windows
  // spends the least on the guard warm-ups.
  const int64_t wave = static_cast<int64_t>(sm_count_) * kMinBlocks * kThreads;
  for (int j = 1; j <= 4; ++j) {
    for (int w = std::max(guard, kGroup); w <= 1024; w += kGroup) {
      int64_t windows = 0;
      for (size_t i = 0; i < rq_in.n_cb; ++i) windows += (rq_in.cbs[i].k + w - 1) / w;
      if (windows <= j * wave) {
        bool have = false;
        for (const Cand& c : cands) have |= !c.persistent && c.window == w;
        if (!have) cands.push_back(Cand{false, w});
        break;
      }
    }
  }
  cudaStream_t st = static_cast<cudaStream_t>(rq_in.stream);
  cudaEvent_t a, b;
  check(cudaEventCreate(&a), "cudaEventCreate");
  check(cudaEventCreate(&b), "cudaEventCreate");
  TuneChoice best;
  best.ms = 1e30;
  try {
    for (const Cand& c : cands) {
      if (c.window < guard) continue;
      DecodeRequest r = rq_in;
      r.auto_schedule = false;
      r.graph = false;
      r.persistent = c.persistent;
      r.window = c.window;
      decode(r);  // warm-up (sizes the workspace)
      check(cudaEventRecord(a, st), "cudaEventRecord");
      decode(r);
      decode(r);
      check(cudaEventRecord(b, st), "cudaEventRecord");
      check(cudaEventSynchronize(b), "cudaEventSynchronize");
      float ms = 0.0f;
      check(cudaEventElapsedTime(&ms, a, b), "cudaEventElapsedTime");
      if (ms / 2 < best.ms) best = TuneChoice{c.persistent, c.window, ms / 2.0};
    }
  } catch (...) {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    throw;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  const std::string sig = signature(rq_in);
  std::lock_guard<std::mutex> lock(mu_);
  for (auto& kv : tuning_)
    if (kv.first == sig) {
      kv.second = best;
      return best;
    }
  tuning_.emplace_back(sig, best);
  return best;
}

void Decoder::save_tuning(const std::string& path) {
  std::lock_guard<std::mutex> lock(mu_);
  std::ofstream f(path);
  if (!f) throw InvalidArgument("cannot open the tuning file for writing");
  f << "# turbo_cpp_b200 autotuning table: signature schedule window ms\n";
  for (const auto& kv : tuning_)
    f << kv.first << ' ' << (kv.second.persistent ? "persistent" : "plain") << ' '
      << kv.second.window << ' ' << kv.second.ms << '\n';
}

void Decoder::load_tuning(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw InvalidArgument("cannot open the tuning file");
  std::vector<std::pair<std::string, TuneChoice>> t;
  std::string line;
  while (std::getline(f, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream in(line);
    std::string sig, sched;
    TuneChoice c;
    if (!(in >> sig >> sched >> c.window >> c.ms) || (sched != "plain" && sched != "persistent") ||
        c.window <= 0 || c.window % kGroup != 0)
      throw InvalidArgument("malformed tuning file line: " + line);
    c.persistent = sched == "persistent";
    t.emplace_back(sig, c);
  }
  std::lock_guard<std::mutex> lock(mu_);
  tuning_ = std::move(t);
}

// Capture-once / replay: the key covers everything baked into the captured launches (block
// descriptors, buffer addresses, options, scales); a workspace reallocation invalidates it.
// Called with mu_ held.  `body` enqueues the launches on `st`; on a miss it runs once eagerly
// (sizing the workspace and the descriptor uploads, so that capturing allocates nothing) and
// once under capture.  Returns the entry to launch.
Decoder::GraphEntry* Decoder::graph_for(const std::string& key, void* stream,
                                        const std::function<void()>& body) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (st == nullptr || st == cudaStreamLegacy)
    throw InvalidArgument("graph: the legacy default stream cannot be captured; pass a created stream");
  for (auto it = graphs_.begin(); it != graphs_.end(); ++it)
    if (it->key == key) {
      if (it->generation == generation_) {
        graphs_.splice(graphs_.begin(), graphs_, it);  // most recently used first
        return &graphs_.front();
      }
      drop_graph(*it);
      graphs_.erase(it);
      break;
    }
  upload_bytes_ = 0;
  body();  // the dry run
  graphs_.emplace_front();
  GraphEntry& e = graphs_.front();
  e.key = key;
  e.arena_bytes = upload_bytes_;
  check(cudaMallocHost(&e.arena, std::max<size_t>(e.arena_bytes, 256)), "cudaMallocHost");
  const uint64_t launches_before = timing_.launches;
  const bool timing_was = timing_on_;
  timing_on_ = false;
  capturing_ = &e;
  cudaGraph_t g = nullptr;
  // any failure from here on removes the half-made entry, so that no later call replays it
  cudaGraphExec_t exec = nullptr;
  try {
    check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    try {
      body();
    } catch (...) {
      cudaStreamEndCapture(st, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    check(cudaStreamEndCapture(st, &g), "cudaStreamEndCapture");
    const cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    check(ie, "cudaGraphInstantiate");
  } catch (...) {
    capturing_ = nullptr;
    timing_on_ = timing_was;
    timing_.launches = launches_before;
    drop_graph(e);
    graphs_.pop_front();
    throw;
  }
  capturing_ = nullptr;
  timing_on_ = timing_was;
  e.exec = exec;
  e.generation = generation_;
  e.launches = timing_.launches - launches_before;
  timing_.launches = launches_before;
  while (graphs_.size() > 16) {  // keep the most recent 16
    drop_graph(graphs_.back());
    graphs_.pop_back();
  }
  return &graphs_.front();
}

void Decoder::launch_graph(GraphEntry* e, void* stream) {
  order_after_previous(stream);
  check(cudaGraphLaunch(static_cast<cudaGraphExec_t>(e->exec), static_cast<cudaStream_t>(stream)),
        "cudaGraphLaunch");
  mark_done(stream);
  timing_.launches += e->launches;
}

void Decoder::decode_graph(const DecodeRequest& rq) {
  std::lock_guard<std::mutex> lock(mu_);
  check(cudaSetDevice(device_), "cudaSetDevice");
  std::string key = "cb";
  auto put = [&key](const void* p, size_t n) { key.append(static_cast<const char*>(p), n); };
  const uintptr_t ptrs[4] = {reinterpret_cast<uintptr_t>(rq.llr),
                             reinterpret_cast<uintptr_t>(rq.posterior),
                             reinterpret_cast<uintptr_t>(rq.crc_ok),
                             reinterpret_cast<uintptr_t>(rq.iterations_used)};
  const int64_t opts[8] = {static_cast<int64_t>(rq.n_cb), static_cast<int64_t>(rq.llr_len),
                           static_cast<int64_t>(rq.post_len), rq.max_iterations, rq.early_stop,
                           rq.window, rq.guard,
                           (rq.std3gpp ? 4 : 0) | (rq.persistent ? 2 : 0) | (rq.smem_checkpoints ? 1 : 0)};
  put(ptrs, sizeof ptrs);
  put(opts, sizeof opts);
  put(rq.cbs, rq.n_cb * sizeof(CodeBlockDesc));
  if (rq.scales) put(rq.scales, 2 * rq.max_iterations * sizeof(float));
  DecodeRequest eager = rq;
  eager.graph = false;
  GraphEntry* e = graph_for(key, rq.stream, [&] {
    if (eager.persistent) decode_persistent(eager); else decode_plain(eager);
  });
  launch_graph(e, rq.stream);
}

namespace {
// one plain-schedule SISO launch: kind 0 upper, 1 lower, 2 lower + posterior
template <bool STD>
void launch_plain(int kind, bool global_ckpt, int blocks, size_t smem, cudaStream_t st,
                  const DevCb* dcbs, const int32_t* dwin, int n_win, const SisoIo& io,
                  const uint8_t* dn, float4* ckpt, int max_ckpt) {
  if (global_ckpt) {
    if (kind == 0) siso_plain_kernel<kSub, 0, true, STD><<<blocks, kThreads, 0, st>>>(dcbs, dwin, n_win, io, dn, ckpt, max_ckpt);
    else if (kind == 1) siso_plain_kernel<kSub, 1, true, STD><<<blocks, kThreads, 0, st>>>(dcbs, dwin, n_win, io, dn, ckpt, max_ckpt);
    else siso_plain_kernel<kSub, 2, true, STD><<<blocks, kThreads, 0, st>>>(dcbs, dwin, n_win, io, dn, ckpt, max_ckpt);
  } else {
    if (kind == 0) siso_plain_kernel<kSub, 0, false, STD><<<blocks, kThreads, smem, st>>>(dcbs, dwin, n_win, io, dn, nullptr, 0);
    else if (kind == 1) siso_plain_kernel<kSub, 1, false, STD><<<blocks, kThreads, smem, st>>>(dcbs, dwin, n_win, io, dn, nullptr, 0);
    else siso_plain_kernel<kSub, 2, false, STD><<<blocks, kThreads, smem, st>>>(dcbs, dwin, n_win, io, dn, nullptr, 0);
  }
}
}  // namespace

void Decoder::decode_plain(const DecodeRequest& rq) {
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
    work += k;
    max_ckpt = std::max(max_ckpt, d.window / kSub + 1);
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
  if (global_ckpt) ckpt = grow<float4>(d_ckpt_, ckpt_slab(n_win, 2 * static_cast<size_t>(max_ckpt)));

  upload(dcbs, cbs.data(), n * sizeof(DevCb), st);
  upload(dwin, wincb.data(), n_win * sizeof(int32_t), st);
  check(cudaMemsetAsync(seeds, 0, static_cast<size_t>(n_win) * 16 * 4 * sizeof(float), st), "zero seeds");
  init_flags_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(
      static_cast<int>(n), done, iters, rq.max_iterations);
  check(cudaGetLastError(), "init launch");

  const uint16_t* dperm = static_cast<const uint16_t*>(d_perm_.ptr);
  const uint16_t* dinv = static_cast<const uint16_t*>(d_inv_.ptr);
  timing_.launches += 3;  // init, setup, finish
  launch_setup(dcbs, static_cast<int>(n), llr, dperm, sysi, e2, st);
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
      if (rq.std3gpp)
        launch_plain<true>(kind, global_ckpt, blocks, smem, st, dcbs, dwin, n_win, io, dn, ckpt, max_ckpt);
      else
        launch_plain<false>(kind, global_ckpt, blocks, smem, st, dcbs, dwin, n_win, io, dn, ckpt, max_ckpt);
      check(cudaGetLastError(), "SISO launch");
      record_stop(st, static_cast<uint64_t>(work));
      timing_.launches += 1;
    }
    if (rq.early_stop) {
      crc_stop_kernel<<<static_cast<unsigned>((n * 32 + 255) / 256), 256, 0, st>>>(
          dcbs, static_cast<int>(n), post,
          static_cast<const uint32_t*>(rq.std3gpp ? d_xpow_std_.ptr : d_xpow_.ptr), done, iters,
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
// Asynchronous host-memory calls
// ------------------------------------------------------------------------------------------
void* Decoder::compute_event() {
  if (!compute_done_) {
    cudaEvent_t e;
    check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    compute_done_ = e;
  }
  return compute_done_;
}

void Decoder::decode_host_async(const DecodeRequest& rq) {
  if (rq.n_cb == 0) return;
  check(cudaSetDevice(device_), "cudaSetDevice");
  while (workers_.size() < kAsyncWorkers) workers_.push_back(std::make_unique<Decoder>(device_));
  Decoder& w = *workers_[next_worker_];
  next_worker_ = (next_worker_ + 1) % workers_.size();
  std::lock_guard<std::mutex> wl(w.mu_);
  const uint64_t launches_before = w.timing_.launches;
  cudaStream_t ws = static_cast<cudaStream_t>(w.stream_);
  // this worker's previous call is ordered before on its own stream; a buffer that has to grow
  // is freed with cudaFree, which waits for the device
  float* dl = w.grow<float>(w.d_llr_, rq.llr_len);
  float* dp = w.grow<float>(w.d_post_, rq.post_len);
  uint8_t* dc = w.grow<uint8_t>(w.d_crc_, rq.n_cb);
  uint32_t* di = w.grow<uint32_t>(w.d_iters_, rq.n_cb);
  check(cudaMemcpyAsync(dl, rq.llr, rq.llr_len * sizeof(float), cudaMemcpyHostToDevice, ws),
        "copy LLRs in");
  // positions outside every block's range come back as 0, as in synchronous host calls
  check(cudaMemsetAsync(dp, 0, rq.post_len * sizeof(float), ws), "zero posterior");
  DecodeRequest r = rq;
  r.llr = dl;
  r.posterior = dp;
  r.crc_ok = dc;
  r.iterations_used = di;
  r.device_memory = true;
  r.host_async = false;
  r.graph = false;
  r.auto_schedule = false;
  r.stream = ws;
  // the decode follows the previous call's decode (another worker); the copy-in above does not
  if (last_compute_)
    check(cudaStreamWaitEvent(ws, static_cast<cudaEvent_t>(last_compute_), 0), "cudaStreamWaitEvent");
  if (r.persistent) w.decode_persistent(r); else w.decode_plain(r);
  check(cudaEventRecord(static_cast<cudaEvent_t>(w.compute_event()), ws), "cudaEventRecord");
  last_compute_ = w.compute_done_;
  check(cudaMemcpyAsync(rq.posterior, dp, rq.post_len * sizeof(float), cudaMemcpyDeviceToHost, ws),
        "copy posterior out");
  if (rq.crc_ok)
    check(cudaMemcpyAsync(rq.crc_ok, dc, rq.n_cb, cudaMemcpyDeviceToHost, ws), "copy crc out");
  if (rq.iterations_used)
    check(cudaMemcpyAsync(rq.iterations_used, di, rq.n_cb * sizeof(uint32_t),
                          cudaMemcpyDeviceToHost, ws), "copy iters out");
  w.mark_done(ws);
  timing_.launches += w.timing_.launches - launches_before;
}

// ------------------------------------------------------------------------------------------
// Persistent schedule: warp tasks of whole code blocks, one launch for all iterations.
// ------------------------------------------------------------------------------------------
void Decoder::decode_persistent(const DecodeRequest& rq) {
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
    work += k;
    max_ckpt = std::max(max_ckpt, d.window / kSub + 1);
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
  int32_t* dtasks = grow<int32_t>(d_tasks_, tasks.size());
  int* dqueue = grow<int>(d_queue_, 2 + static_cast<size_t>(n_tasks));  // queue, error, progress
  float* sysi = grow<float>(d_sysi_, work);
  float* e1i = grow<float>(d_e1i_, work);
  float* e2 = grow<float>(d_e2_, work);
  float* seeds = grow<float>(d_seed_, static_cast<size_t>(n_win) * 16 * 4);
  float4* ckpt = grow<float4>(d_ckpt_, ckpt_slab(n_win, 2 * static_cast<size_t>(max_ckpt)));
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
  upload(dcbs, cbs.data(), n * sizeof(DevCb), st);
  upload(dwin, wincb.data(), n_win * sizeof(int32_t), st);
  upload(dtasks, tasks.data(), tasks.size() * sizeof(int32_t), st);
  check(cudaMemsetAsync(dqueue, 0, (2 + static_cast<size_t>(n_tasks)) * sizeof(int), st),
        "zero queue");
  check(cudaMemsetAsync(seeds, 0, static_cast<size_t>(n_win) * 16 * 4 * sizeof(float), st),
        "zero seeds");
  init_flags_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(
      static_cast<int>(n), done, iters, rq.max_iterations);
  launch_setup(dcbs, static_cast<int>(n), llr, static_cast<const uint16_t*>(d_perm_.ptr), sysi,
               e2, st);
  check(cudaGetLastError(), "set-up launch");

  PersistArgs a{};
  a.cbs = dcbs;
  a.win_cb = dwin;
  a.tasks = dtasks;
  a.n_tasks = n_tasks;
  a.queue = dqueue;
  a.error = static_cast<int*>(d_err_.ptr);
  a.stall_task = stall_task_;
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
  a.n_windows = n_win;
  a.guard = guard;
  a.max_iterations = static_cast<int>(rq.max_iterations);
  a.early_stop = rq.early_stop ? 1 : 0;
  a.done = done;
  a.iters = iters;
  a.xpow = static_cast<const uint32_t*>(rq.std3gpp ? d_xpow_std_.ptr : d_xpow_.ptr);
  for (int i = 0; i < 2 * kMaxIterations; ++i)
    a.scale[i] = (rq.scales && i < 2 * static_cast<int>(rq.max_iterations)) ? rq.scales[i] : 1.0f;
  const int grid = std::max(1, sm_count_ * std::max(persist_blocks_per_sm_, 1));
  record_start(st);
  if (rq.std3gpp)
    persistent_kernel<true><<<grid, kPersistThreads, 0, st>>>(a);
  else
    persistent_kernel<false><<<grid, kPersistThreads, 0, st>>>(a);
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
