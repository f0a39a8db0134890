// noalloc.cu -- tc_decode_noalloc: the plain-schedule decode with every piece of device
// scratch taken from fixed-size arrays that live in the library image, so that the call never
// allocates device memory.
//
// Who needs this: callers that may not call cudaMalloc or cudaFree -- a real-time receiver
// thread that cannot afford the device-wide synchronisation and unbounded latency that
// cudaMalloc/cudaFree may incur, a host program whose device memory is entirely owned by
// another allocator (a framework's caching pool) that forbids raw allocations, or a plug-in
// that is handed input and output buffers and nothing else.  They pass device inputs and
// outputs; everything else comes from g_scratch below.
//
// Limits and sharing: g_scratch holds kNoAllocScratchBytes (32 MiB) on every GPU that loads the
// library, for as long as the library stays loaded.  A call whose working set does not fit is
// rejected with TC_ERR_CAPACITY before anything is launched.  All calls on a device share the
// same array and the array keeps whatever the previous call left in it; each call therefore
// clears what must start at zero itself (next-iteration seeds, a-priori LLRs, stop flags).  Two
// calls whose work overlaps on the GPU (different streams, or different host threads without
// ordering) race on the shared array and corrupt each other's results.
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "../../include/turbo_b200.h"
#include "decode_kernels.cuh"
#include "decoder.hpp"
#include "lte_codec.hpp"

namespace tcb {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t{32} << 20;
constexpr int kQppTotalEntries = 355248;  // sum of the 188 block sizes
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kNoAllocScratchBytes];
static __device__ __align__(256) uint16_t g_perm[kQppTotalEntries];
static __device__ __align__(256) uint16_t g_inv[kQppTotalEntries];
static __device__ __align__(256) uint32_t g_xpow[6144];

// Device addresses of the arrays above.  In host code g_scratch etc. name host-side stand-ins,
// not device memory, so the real addresses are looked up once per device (with that device
// current) and only these pointers are ever passed to kernels.
struct DeviceState {
  bool ready = false;
  unsigned char* scratch = nullptr;
  uint16_t* perm = nullptr;
  uint16_t* inv = nullptr;
  uint32_t* xpow = nullptr;
  std::vector<int32_t> tab_offset;
};
std::mutex g_setup_mu;
DeviceState g_state[kMaxDevices];

void ok(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

// First call on a device: symbol addresses and the constant tables (QPP permutations and
// x^j mod g_CRC24B).  This uses synchronous copies, so the first call on each device must not
// be made while a stream is being captured.  Later calls re-read one symbol address (a cheap
// lookup) and redo the set-up when the module was loaded again at another address.  A device
// reset that reloads the module at the same address is not detected: the tables are then gone,
// which the header states as a limit.
const DeviceState& setup(int device) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (device < 0 || device >= kMaxDevices) throw InvalidArgument("device ordinal out of range");
  DeviceState& d = g_state[device];
  if (d.ready) {
    uint16_t* perm = nullptr;
    ok(cudaGetSymbolAddress(reinterpret_cast<void**>(&perm), g_perm), "table address");
    if (perm == d.perm) return d;
    d.ready = false;
  }
  ok(cudaGetSymbolAddress(reinterpret_cast<void**>(&d.scratch), g_scratch), "scratch address");
  ok(cudaGetSymbolAddress(reinterpret_cast<void**>(&d.perm), g_perm), "table address");
  ok(cudaGetSymbolAddress(reinterpret_cast<void**>(&d.inv), g_inv), "table address");
  ok(cudaGetSymbolAddress(reinterpret_cast<void**>(&d.xpow), g_xpow), "table address");
  std::vector<uint16_t> perm, inv;
  perm.reserve(kQppTotalEntries);
  inv.reserve(kQppTotalEntries);
  d.tab_offset.assign(kQppCount, 0);
  for (int i = 0; i < kQppCount; ++i) {
    const QppEntry e = qpp_entry(i);
    d.tab_offset[i] = static_cast<int32_t>(perm.size());
    const auto p = qpp_permutation(e.k);
    std::vector<uint16_t> iv(e.k);
    for (int32_t j = 0; j < e.k; ++j) {
      perm.push_back(static_cast<uint16_t>(p[j]));
      iv[p[j]] = static_cast<uint16_t>(j);
    }
    inv.insert(inv.end(), iv.begin(), iv.end());
  }
  if (perm.size() != static_cast<size_t>(kQppTotalEntries))
    throw std::runtime_error("QPP table size mismatch");
  std::vector<uint32_t> xpow(6144);
  const uint32_t g = crc_generator_mask(CrcKind::Crc24B);
  uint32_t r = 1;
  for (int j = 0; j < 6144; ++j) {
    xpow[j] = r;
    r <<= 1;
    if (r & (1u << 24)) r ^= (1u << 24) | g;
  }
  ok(cudaMemcpy(d.perm, perm.data(), perm.size() * 2, cudaMemcpyHostToDevice), "table upload");
  ok(cudaMemcpy(d.inv, inv.data(), inv.size() * 2, cudaMemcpyHostToDevice), "table upload");
  ok(cudaMemcpy(d.xpow, xpow.data(), xpow.size() * 4, cudaMemcpyHostToDevice), "table upload");
  d.ready = true;
  return d;
}

// Bump allocator over the static scratch array (256-byte aligned slices).
struct Carve {
  unsigned char* base;
  size_t used = 0;
  template <class T>
  T* take(size_t count) {
    used = (used + 255) & ~size_t{255};
    T* p = reinterpret_cast<T*>(base + used);
    used += count * sizeof(T);
    return p;
  }
};

}  // namespace

void decode_noalloc(const DecodeRequest& rq, size_t* bytes_needed) {
  int device = 0;
  ok(cudaGetDevice(&device), "cudaGetDevice");
  cudaStream_t st = static_cast<cudaStream_t>(rq.stream);
  // The block descriptors below are copied from host memory that lives only for this call, and
  // the first call's set-up copies synchronously; neither may be recorded into a graph.
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  ok(cudaStreamIsCapturing(st, &capture), "cudaStreamIsCapturing");
  if (capture != cudaStreamCaptureStatusNone)
    throw InvalidArgument("tc_decode_noalloc was called while its stream is being captured; its "
                          "descriptor copies read memory that lives only for the call");
  const DeviceState& ds = setup(device);
  const size_t n = rq.n_cb;
  if (reinterpret_cast<uintptr_t>(rq.llr) % 16 != 0)
    throw InvalidArgument("the LLR buffer must be 16-byte aligned");
  const int guard = rq.guard < 0 ? kDefaultGuard : rq.guard;
  if (guard % kGroup != 0) throw InvalidArgument("guard must be a multiple of 8");

  // ---- layout (as the decoder object's plain schedule) ----
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
    d.tab = ds.tab_offset[qi];
    d.window = rq.window > 0 ? std::min<int32_t>(rq.window, k) : std::min<int32_t>(kDefaultWindow, k);
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

  // ---- carve the scratch array; reject what does not fit ----
  Carve c{ds.scratch};
  DevCb* dcbs = c.take<DevCb>(n);
  int32_t* dwin = c.take<int32_t>(n_win);
  float* sysi = c.take<float>(work);
  float* e1i = c.take<float>(work);
  float* e2 = c.take<float>(work);
  float* seeds = c.take<float>(static_cast<size_t>(n_win) * 16 * 4);
  float4* ckpt = c.take<float4>(static_cast<size_t>(n_win) * 2 * max_ckpt);
  uint8_t* done = c.take<uint8_t>(n);
  uint32_t* iters = rq.iterations_used ? rq.iterations_used : c.take<uint32_t>(n);
  uint8_t* crc = rq.crc_ok ? rq.crc_ok : c.take<uint8_t>(n);
  if (bytes_needed) *bytes_needed = c.used;
  if (c.used > kNoAllocScratchBytes)
    throw CapacityExceeded("the code blocks need " + std::to_string(c.used) +
                           " bytes of scratch; tc_decode_noalloc has " +
                           std::to_string(kNoAllocScratchBytes));
  if (n == 0) return;

  // ---- same launch sequence as the plain schedule ----
  ok(cudaMemcpyAsync(dcbs, cbs.data(), n * sizeof(DevCb), cudaMemcpyHostToDevice, st), "copy cbs");
  ok(cudaMemcpyAsync(dwin, wincb.data(), n_win * sizeof(int32_t), cudaMemcpyHostToDevice, st),
     "copy windows");
  ok(cudaMemsetAsync(seeds, 0, static_cast<size_t>(n_win) * 16 * 4 * sizeof(float), st),
     "zero seeds");
  init_flags_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(
      static_cast<int>(n), done, iters, rq.max_iterations);
  launch_setup(dcbs, static_cast<int>(n), rq.llr, ds.perm, sysi, e2, st);
  ok(cudaGetLastError(), "set-up launch");
  const int blocks = (n_win + kThreads - 1) / kThreads;
  const size_t slab = static_cast<size_t>(n_win) * 16;
  float* seed_up[2] = {seeds, seeds + slab};
  float* seed_lo[2] = {seeds + 2 * slab, seeds + 3 * slab};
  for (uint32_t it = 0; it < rq.max_iterations; ++it) {
    const float s_up = rq.scales ? rq.scales[2 * it] : 1.0f;
    const float s_lo = rq.scales ? rq.scales[2 * it + 1] : 1.0f;
    const SisoIo up{rq.llr, sysi, e2, e1i, nullptr, ds.perm, ds.inv, seed_up[it & 1],
                    seed_up[(it + 1) & 1], s_up, guard};
    const SisoIo lo{rq.llr, sysi, e1i, e2, rq.posterior, ds.perm, ds.inv, seed_lo[it & 1],
                    seed_lo[(it + 1) & 1], s_lo, guard};
    const uint8_t* dn = rq.early_stop ? done : nullptr;
    const bool post_now = rq.early_stop || it + 1 == rq.max_iterations;
    siso_plain_kernel<kSub, 0, true><<<blocks, kThreads, 0, st>>>(dcbs, dwin, n_win, up, dn, ckpt,
                                                                  max_ckpt);
    if (post_now)
      siso_plain_kernel<kSub, 2, true><<<blocks, kThreads, 0, st>>>(dcbs, dwin, n_win, lo, dn, ckpt,
                                                                    max_ckpt);
    else
      siso_plain_kernel<kSub, 1, true><<<blocks, kThreads, 0, st>>>(dcbs, dwin, n_win, lo, dn, ckpt,
                                                                    max_ckpt);
    ok(cudaGetLastError(), "SISO launch");
    if (rq.early_stop) {
      crc_stop_kernel<<<static_cast<unsigned>((n * 32 + 255) / 256), 256, 0, st>>>(
          dcbs, static_cast<int>(n), rq.posterior, ds.xpow, done, iters, static_cast<int>(it));
      ok(cudaGetLastError(), "CRC launch");
    }
  }
  finish_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(static_cast<int>(n), done,
                                                                        crc, rq.early_stop ? 1 : 0);
  ok(cudaGetLastError(), "finish launch");
}

}  // namespace tcb
