// decoder.hpp -- host-side objects of the GPU decoder (no CUDA types in the interface).
#pragma once
#include <cstddef>
#include <cstdint>
#include <functional>
#include <list>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

namespace tcb {

// Error classes; the C ABI maps each to a status code, the C++ API rethrows the reference's
// exception types (std::invalid_argument, std::out_of_range, std::runtime_error).
struct InvalidArgument : std::invalid_argument {
  using std::invalid_argument::invalid_argument;
};
struct OutOfRange : std::out_of_range {
  using std::out_of_range::out_of_range;
};
struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct NoDevice : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct DeviceTimeout : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct CapacityExceeded : std::length_error {
  using std::length_error::length_error;
};

constexpr int kSub = 4;              // alpha checkpoint interval (steps)
constexpr int kGroup = 8;            // load granularity: windows and guards are multiples of 8
constexpr int kDefaultWindow = 128;  // window length (steps)
constexpr int kDefaultGuard = 96;    // warm-up steps on each side of a window
constexpr int kPersistWindow = 192;  // target window of the persistent schedule (<= 32 per block)
constexpr size_t kAsyncWorkers = 3;  // TC_MEM_HOST_ASYNC workspaces: call i+2's copy-in needs no wait for call i

struct CodeBlockDesc {
  int32_t k;
  int32_t filler;
  int64_t llr_offset;  // floats; [d0|d1|d2], 3*(K+4) floats, multiple of 4
  int64_t out_offset;  // floats; K posterior LLRs
};

struct DecodeRequest {
  size_t n_cb = 0;
  const CodeBlockDesc* cbs = nullptr;  // host memory
  size_t llr_len = 0;
  const float* llr = nullptr;
  size_t post_len = 0;
  float* posterior = nullptr;
  uint8_t* crc_ok = nullptr;
  uint32_t* iterations_used = nullptr;
  uint32_t max_iterations = 8;
  bool early_stop = false;
  int window = 0;   // 0: default
  int guard = -1;   // <0: default
  bool device_memory = false;  // llr/posterior/crc_ok/iterations_used are device pointers
  bool host_async = false;     // host pointers; enqueue copies + decode and return (see sync())
  bool smem_checkpoints = false;  // alpha checkpoints in shared memory instead of global scratch
  bool persistent = false;  // persistent warp-task schedule instead of per-half-iteration launches
  bool graph = false;       // device memory: capture the launch sequence once, replay it after
  bool auto_schedule = false;  // take schedule and window from the autotuning table
  const float* scales = nullptr;  // host; 2 per iteration (upper, lower); null = all 1
  bool std3gpp = false;  // the TS 36.212 code (trellis, tail mapping, CRC24B) instead of the reference's
  void* stream = nullptr;
};

// One code block of the transport-block chain: its rate-matched LLRs (E of them at e_offset)
// and where its de-rate-matched [d0|d1|d2] go (llr_offset, multiple of 4 floats).
struct RmBlockDesc {
  int32_t k;
  int32_t filler;
  int32_t e;
  uint32_t rv;
  int64_t e_offset;
  int64_t llr_offset;
};

// One transport block: its code blocks are [first_cb, first_cb + n_cb); its TBS decoded bits
// go to bits_offset.
struct TbDesc {
  int64_t tbs;
  int32_t first_cb;
  int32_t n_cb;
  int64_t bits_offset;
};

struct TbRequest {
  size_t n_tb = 0;
  const TbDesc* tbs = nullptr;        // host
  size_t n_cb = 0;
  const RmBlockDesc* cbs = nullptr;   // host; llr_offset ignored (laid out internally)
  size_t e_len = 0;
  const float* e_llr = nullptr;
  size_t bits_len = 0;
  uint8_t* bits = nullptr;            // one byte per decoded bit
  uint8_t* tb_crc_ok = nullptr;       // n_tb
  uint8_t* cb_crc_ok = nullptr;       // n_cb
  uint32_t* iterations_used = nullptr;  // n_cb
  float* posterior = nullptr;         // optional: sum K, blocks back to back
  bool device_memory = false;
  bool host_async = false;            // host pointers; enqueued on a worker, valid after sync()
  void* stream = nullptr;
  DecodeRequest decode;               // iterations, early stop, schedule, window, guard, scales
};

struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  void reserve(size_t need);  // grows (discarding contents) when too small
  void release();
};

// Kernel accounting: every launch is counted; with timing on, each SISO launch is bracketed by
// CUDA events on the launching stream and the elapsed times are summed on request.
struct Timing {
  uint64_t launches = 0;       // kernels launched by this decoder
  uint64_t siso_launches = 0;  // SISO half-iteration launches timed
  double siso_ms = 0.0;        // summed device time of the timed SISO launches
  uint64_t trellis_steps = 0;  // output trellis steps of the timed SISO launches
};

class Decoder {
 public:
  explicit Decoder(int device);
  ~Decoder();
  Decoder(const Decoder&) = delete;
  Decoder& operator=(const Decoder&) = delete;

  void decode(const DecodeRequest& rq);  // plain or persistent schedule
  int device() const { return device_; }
  void set_timing(bool on);
  void sync();  // waits for this decoder's enqueued work; reports a persistent wait timeout
  void inject_stall(int task) { stall_task_ = task; }  // testing hook (-1: off)

  // Autotuning: times candidate (schedule, window) pairs on a device-memory request and keeps
  // the fastest for requests with the same signature.
  struct TuneChoice {
    bool persistent = false;
    int window = 0;
    double ms = 0.0;
  };
  TuneChoice autotune(const DecodeRequest& rq);
  void save_tuning(const std::string& path);
  void load_tuning(const std::string& path);
  static std::string signature(const DecodeRequest& rq);
  Timing timing(bool reset);  // waits for the recorded events

  // transport-block chain on the device (chain.cu)
  void derate_match_llr(size_t n, const RmBlockDesc* blocks, const float* e_llr, size_t e_len,
                        float* d012, size_t llr_len, void* stream);
  void decode_transport_blocks(const TbRequest& q);
  // test-vector generation on the device (generate.cu): the host generator's seeded bits
  // (+ CRC24B), encoder and channel; the encoder and the rate matcher alone
  void awgn_code_blocks_device(uint64_t seed, size_t n, const int32_t* k, const int32_t* filler,
                               const float* ebn0_db, bool crc24b, uint8_t* bits, float* llr,
                               void* stream);
  void turbo_encode_device(size_t n, const int32_t* k, const int32_t* filler, const uint8_t* bits,
                           uint8_t* d012, void* stream);
  void rate_match_device(size_t n, const RmBlockDesc* blocks, const uint8_t* d012,
                         size_t d012_len, uint8_t* e_bits, size_t e_len, void* stream);
  // HARQ soft combining of several transmissions (redundancy versions) per code block
  void derate_combine_llr(size_t n, const RmBlockDesc* tx, const float* e_llr, size_t e_len,
                          float* d012, size_t llr_len, void* stream);
  int sm_count() const { return sm_count_; }

  // QPP tables on the device (uint16 per position; all 188 sizes back to back) and the offset
  // of block size k's table in them (throws OutOfRange for a size outside the table)
  const uint16_t* perm_table() const { return static_cast<const uint16_t*>(d_perm_.ptr); }
  const uint16_t* inv_table() const { return static_cast<const uint16_t*>(d_inv_.ptr); }
  int32_t table_offset(int32_t k) const;

 private:
  int pick_window(int32_t k, int32_t requested) const;
  void decode_persistent(const DecodeRequest& rq);
  void decode_plain(const DecodeRequest& rq);
  // Asynchronous host-memory calls rotate over kAsyncWorkers worker decoders, each with its own
  // device buffers and stream: a call enqueues copy-in, decode and copy-out on the next worker
  // and returns, so that its copies run while the previous calls decode.  sync() waits for them.
  // wait: synchronise host-memory calls; after/done (cudaEvent_t, may be null): the chain's
  // device work waits for `after` once its inputs are copied in and records `done` before its
  // outputs are copied out
  void transport_blocks(const TbRequest& q, bool wait, void* after = nullptr,
                        void* done = nullptr);
  void decode_host_async(const DecodeRequest& rq);
  std::vector<std::unique_ptr<Decoder>> workers_;
  size_t next_worker_ = 0;
  void decode_graph(const DecodeRequest& rq);
  // host -> device copy of launch descriptors; while capturing, from graph-owned pinned memory
  void upload(void* dst, const void* src, size_t bytes, void* stream);
  template <class T>
  T* grow(DeviceBuffer& b, size_t count) {
    void* before = b.ptr;
    b.reserve(count * sizeof(T));
    if (b.ptr != before) ++generation_;  // cached graphs hold the old addresses
    return static_cast<T*>(b.ptr);
  }
  void derate_device(size_t n, const RmBlockDesc* blocks, const float* e_llr, size_t e_len,
                     float* d012, size_t llr_len, void* stream);

  // CUDA graphs of previously seen device-memory requests (same shapes, pointers, options)
  struct GraphEntry {
    std::string key;
    uint64_t generation = 0;
    void* exec = nullptr;                 // cudaGraphExec_t
    void* arena = nullptr;                // pinned host copies of the descriptors
    size_t arena_bytes = 0, arena_used = 0;
    uint64_t launches = 0;
  };
  std::list<GraphEntry> graphs_;
  std::vector<std::pair<std::string, TuneChoice>> tuning_;
  DecodeRequest resolve(const DecodeRequest& rq);  // applies the tuning table to an auto request
  DecodeRequest resolve_locked(const DecodeRequest& rq) const;  // the same, mu_ already held
  // the cached graph of `key`, captured from `body` on a miss (mu_ held), and its launch
  GraphEntry* graph_for(const std::string& key, void* stream, const std::function<void()>& body);
  void launch_graph(GraphEntry* e, void* stream);
  GraphEntry* capturing_ = nullptr;       // entry being captured (uploads go to its staging)
  uint64_t generation_ = 0;               // bumped whenever a workspace buffer moves
  size_t upload_bytes_ = 0;               // descriptor bytes uploaded (sizes a graph's arena)
  void drop_graph(GraphEntry& e);
  void record_start(void* stream);
  void record_stop(void* stream, uint64_t steps);

  struct EventPair {
    void* start = nullptr;
    void* stop = nullptr;
    uint64_t steps = 0;
  };
  bool timing_on_ = false;
  Timing timing_;
  std::vector<EventPair> events_;   // pool
  size_t events_used_ = 0;

  std::mutex mu_;
  int device_ = 0;
  int sm_count_ = 0;
  int smem_optin_ = 0;
  void* stream_ = nullptr;  // cudaStream_t
  std::vector<int32_t> tab_offset_;
  DeviceBuffer d_perm_, d_inv_, d_xpow_, d_xpow_std_;  // x^j mod g_CRC24B: reference, TS 36.212
  DeviceBuffer d_cbs_, d_wincb_, d_llr_, d_sysi_, d_e1i_, d_e2_, d_post_, d_seed_,
      d_done_, d_iters_, d_crc_, d_ckpt_, d_tasks_, d_queue_;
  DeviceBuffer d_rmgroup_, d_gen_, d_gentab_, d_genenc_, d_genrm_, d_xpow_a_std_;
  DeviceBuffer d_tbcb_, d_synpart_;
  DeviceBuffer d_rm_, d_e_llr_, d_d012_, d_tbpost_, d_tbbits_, d_tbok_, d_cbok_, d_tbiters_, d_tb_,
      d_xpow_a_;
  int persist_blocks_per_sm_ = 0;
  DeviceBuffer d_err_;          // sticky: set by a persistent-schedule wait that gave up
  int stall_task_ = -1;
  void* last_event_ = nullptr;  // completion of the previous decode (orders workspace reuse)
  // Host-async calls: the decode of each call waits for the previous call's decode (on another
  // worker), so that decodes run one at a time on the whole GPU while copies overlap them.
  void* compute_done_ = nullptr;  // worker: end of its latest call's device compute
  void* last_compute_ = nullptr;  // caller: the latest worker's compute_done_ event
  void* compute_event();          // this decoder's compute_done_ (created on first use)
  void order_after_previous(void* stream);
  void mark_done(void* stream);
  void take_error();  // throws DeviceTimeout (and clears the flag) if it is set; host-synchronous
};

// The kernels index a checkpoint slab (windows interleaved, siso.cuh CkptStrided) with 32-bit
// plane offsets: a call whose slab would reach 2^31 float4 (32 GB) is refused.
// Kernel attributes of the transport-block chain (chain.cu); the decoder sets them on its device.
void configure_chain_kernels();

inline size_t ckpt_slab(size_t n_win, size_t planes) {
  const size_t n = n_win * planes;
  if (n >= (size_t{1} << 31))
    throw CapacityExceeded("too many windows in one call for the checkpoint slab");
  return n;
}

// Plain-schedule decode on the current device with all scratch in a fixed array of the library
// image (noalloc.cu); device pointers in rq, ordered on rq.stream; never allocates.  Writes the
// scratch bytes the request needs to *bytes_needed when given, and throws CapacityExceeded when
// they exceed the array.
void decode_noalloc(const DecodeRequest& rq, size_t* bytes_needed);

}  // namespace tcb
