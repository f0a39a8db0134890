// capi.cpp -- the extern "C" boundary (include/turbo_b200.h): status codes instead of
// exceptions, plain pointers instead of spans and vectors.
#include <cstring>
#include <exception>
#include <new>
#include <string>
#include <vector>

#include "../../include/turbo_b200.h"
#include "adjoint.hpp"
#include "decoder.hpp"
#include "lte_codec.hpp"

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* what) {
  g_last_error = what ? what : "";
  return code;
}

// Runs f() and maps the exception classes of the library to status codes.
template <class F>
int guarded(F&& f) {
  try {
    f();
    g_last_error.clear();
    return TC_OK;
  } catch (const tcb::OutOfRange& e) {
    return fail(TC_ERR_OUT_OF_RANGE, e.what());
  } catch (const tcb::InvalidArgument& e) {
    return fail(TC_ERR_INVALID_ARGUMENT, e.what());
  } catch (const tcb::NoDevice& e) {
    return fail(TC_ERR_NO_DEVICE, e.what());
  } catch (const tcb::CudaError& e) {
    return fail(TC_ERR_CUDA, e.what());
  } catch (const tcb::DeviceTimeout& e) {
    return fail(TC_ERR_TIMEOUT, e.what());
  } catch (const tcb::CapacityExceeded& e) {
    return fail(TC_ERR_CAPACITY, e.what());
  } catch (const std::bad_alloc&) {
    return fail(TC_ERR_RUNTIME, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(TC_ERR_RUNTIME, e.what());
  } catch (...) {
    return fail(TC_ERR_RUNTIME, "unknown error");
  }
}

void need(bool cond, const char* what) {
  if (!cond) throw tcb::InvalidArgument(what);
}

tcb::CrcKind crc_kind(int kind) {
  need(kind >= 0 && kind <= 3, "unknown CRC kind");
  return static_cast<tcb::CrcKind>(kind);
}

tcb::Convention convention_of(int c) {
  need(c == TC_CONVENTION_REFERENCE || c == TC_CONVENTION_3GPP, "unknown convention");
  return c == TC_CONVENTION_3GPP ? tcb::Convention::Std3gpp : tcb::Convention::Reference;
}

}  // namespace

struct tc_decoder {
  explicit tc_decoder(int device) : impl(device) {}
  tcb::Decoder impl;
};

struct tc_adjoint {
  explicit tc_adjoint(tcb::Decoder& d) : impl(d) {}
  tcb::Adjoint impl;
};

extern "C" {

const char* tc_status_name(int status) {
  switch (status) {
    case TC_OK: return "TC_OK";
    case TC_ERR_INVALID_ARGUMENT: return "TC_ERR_INVALID_ARGUMENT";
    case TC_ERR_OUT_OF_RANGE: return "TC_ERR_OUT_OF_RANGE";
    case TC_ERR_RUNTIME: return "TC_ERR_RUNTIME";
    case TC_ERR_CUDA: return "TC_ERR_CUDA";
    case TC_ERR_NO_DEVICE: return "TC_ERR_NO_DEVICE";
    case TC_ERR_TIMEOUT: return "TC_ERR_TIMEOUT";
    case TC_ERR_CAPACITY: return "TC_ERR_CAPACITY";
    default: return "TC_UNKNOWN_STATUS";
  }
}

const char* tc_last_error(void) { return g_last_error.c_str(); }

int tc_version(void) { return 100; }

int tc_qpp_table_size(void) { return tcb::kQppCount; }

int tc_qpp_entry(int index, int32_t* k, int32_t* f1, int32_t* f2) {
  return guarded([&] {
    need(k && f1 && f2, "null output pointer");
    const tcb::QppEntry e = tcb::qpp_entry(index);
    *k = e.k;
    *f1 = e.f1;
    *f2 = e.f2;
  });
}

int tc_qpp_index(int32_t k, int32_t* index) {
  return guarded([&] {
    need(index != nullptr, "null output pointer");
    const int i = tcb::qpp_index(k);
    if (i < 0) throw tcb::OutOfRange("unsupported QPP block size");
    *index = i;
  });
}

int tc_qpp_permutation(int32_t k, int32_t* perm) {
  return guarded([&] {
    need(perm != nullptr, "null output pointer");
    const auto p = tcb::qpp_permutation(k);
    std::memcpy(perm, p.data(), p.size() * sizeof(int32_t));
  });
}

int tc_qpp_inverse_permutation(int32_t k, int32_t* inv) {
  return guarded([&] {
    need(inv != nullptr, "null output pointer");
    const auto p = tcb::qpp_inverse_permutation(k);
    std::memcpy(inv, p.data(), p.size() * sizeof(int32_t));
  });
}

int tc_crc_append_conv(int convention, int kind, const uint8_t* bits, size_t n, uint8_t* out) {
  return guarded([&] {
    need(out != nullptr && (bits != nullptr || n == 0), "null pointer");
    tcb::crc_append(crc_kind(kind), bits, n, out, convention_of(convention));
  });
}

int tc_crc_append(int kind, const uint8_t* bits, size_t n, uint8_t* out) {
  return tc_crc_append_conv(TC_CONVENTION_REFERENCE, kind, bits, n, out);
}

int tc_crc_check_conv(int convention, int kind, const uint8_t* bits, size_t n, int* ok) {
  return guarded([&] {
    need(ok != nullptr && (bits != nullptr || n == 0), "null pointer");
    *ok = tcb::crc_check(crc_kind(kind), bits, n, convention_of(convention)) ? 1 : 0;
  });
}

int tc_crc_check(int kind, const uint8_t* bits, size_t n, int* ok) {
  return tc_crc_check_conv(TC_CONVENTION_REFERENCE, kind, bits, n, ok);
}

int tc_segment_transport_block_conv(int convention, const uint8_t* bits, size_t b,
                                    tc_segmentation* info, uint8_t* cb_bits, size_t cap) {
  return guarded([&] {
    need(info != nullptr, "null output pointer");
    need(bits != nullptr || b == 0, "null input");
    const tcb::Convention conv = convention_of(convention);
    const tcb::Segmentation s = tcb::segment_sizes(b);
    info->c = s.c;
    info->c_plus = s.c_plus;
    info->c_minus = s.c_minus;
    info->k_plus = s.k_plus;
    info->k_minus = s.k_minus;
    info->filler_bits = s.filler;
    info->l = s.l;
    if (cb_bits) {
      need(cap >= s.total_bits(), "code-block buffer too small");
      tcb::segment_bits(bits, b, s, cb_bits, conv);
    }
  });
}

int tc_segment_transport_block(const uint8_t* bits, size_t b, tc_segmentation* info,
                               uint8_t* cb_bits, size_t cap) {
  return tc_segment_transport_block_conv(TC_CONVENTION_REFERENCE, bits, b, info, cb_bits, cap);
}

int tc_turbo_encode_conv(int convention, int32_t k, int32_t filler, const uint8_t* cb_bits,
                         uint8_t* d012) {
  return guarded([&] {
    need(cb_bits && d012, "null pointer");
    const tcb::Convention conv = convention_of(convention);
    if (tcb::qpp_index(k) < 0) throw tcb::OutOfRange("unsupported QPP block size");
    need(filler >= 0 && filler < k, "invalid filler count");
    tcb::turbo_encode(k, filler, cb_bits, d012, conv);
  });
}

int tc_turbo_encode(int32_t k, int32_t filler, const uint8_t* cb_bits, uint8_t* d012) {
  return tc_turbo_encode_conv(TC_CONVENTION_REFERENCE, k, filler, cb_bits, d012);
}

int tc_compute_e(size_t r, size_t g_total, size_t c, uint32_t num_layers, uint32_t mod_order,
                 size_t* e) {
  return guarded([&] {
    need(e != nullptr, "null output pointer");
    *e = tcb::compute_e(r, g_total, c, num_layers, mod_order);
  });
}

int tc_rate_match(int32_t k, int32_t filler, const uint8_t* d012, size_t e, uint32_t rv,
                  uint8_t* out) {
  return guarded([&] {
    need(d012 && (out || e == 0), "null pointer");
    if (tcb::qpp_index(k) < 0) throw tcb::OutOfRange("unsupported QPP block size");
    need(filler >= 0 && filler < k && rv < 4, "invalid filler count or rv");
    tcb::rate_match(k, filler, d012, e, rv, out);
  });
}

int tc_derate_match_bits(int32_t k, int32_t filler, const uint8_t* e_bits, size_t e, uint32_t rv,
                         float* d012) {
  return guarded([&] {
    need(d012 && (e_bits || e == 0), "null pointer");
    if (tcb::qpp_index(k) < 0) throw tcb::OutOfRange("unsupported QPP block size");
    need(filler >= 0 && filler < k && rv < 4, "invalid filler count or rv");
    tcb::derate_match_bits(k, filler, e_bits, e, rv, d012);
  });
}

int tc_derate_match_llr(int32_t k, int32_t filler, const float* e_llr, size_t e, uint32_t rv,
                        float* d012) {
  return guarded([&] {
    need(d012 && (e_llr || e == 0), "null pointer");
    if (tcb::qpp_index(k) < 0) throw tcb::OutOfRange("unsupported QPP block size");
    need(filler >= 0 && filler < k && rv < 4, "invalid filler count or rv");
    tcb::derate_match_llr(k, filler, e_llr, e, rv, d012);
  });
}

int tc_random_bits(uint64_t seed, uint64_t first, size_t n, uint8_t* bits) {
  return guarded([&] {
    need(bits || n == 0, "null pointer");
    tcb::random_bits(seed, first, n, bits);
  });
}

int tc_awgn_llr(uint64_t seed, uint64_t first, const uint8_t* bits, size_t n, double sigma2,
                float* llr) {
  return guarded([&] {
    need((bits && llr) || n == 0, "null pointer");
    need(sigma2 > 0.0, "noise variance must be positive");
    tcb::awgn_llr(seed, first, bits, n, sigma2, llr);
  });
}

int tc_awgn_code_blocks(uint64_t seed, size_t n, const int32_t* k, const int32_t* filler,
                        const float* ebn0_db, int crc24b, uint8_t* bits, float* llr,
                        int threads) {
  return guarded([&] {
    need(n == 0 || (k && filler && ebn0_db && bits && llr), "null pointer");
    tcb::awgn_code_blocks(seed, n, k, filler, ebn0_db, crc24b != 0, bits, llr, threads);
  });
}

int tc_decoder_create(int device, tc_decoder** out) {
  return guarded([&] {
    need(out != nullptr, "null output pointer");
    *out = nullptr;
    *out = new tc_decoder(device);
  });
}

int tc_decoder_destroy(tc_decoder* dec) {
  return guarded([&] { delete dec; });
}

int tc_decode_options_init(tc_decode_options* o) {
  return guarded([&] {
    need(o != nullptr, "null options");
    std::memset(o, 0, sizeof *o);
    o->max_iterations = 8;
    o->window = 0;
    o->guard = -1;
    o->memory = TC_MEM_HOST;
    o->schedule = TC_SCHEDULE_PLAIN;
  });
}

int tc_decode(tc_decoder* dec, size_t n_cb, const tc_code_block* cbs, size_t llr_len,
              const float* llr, size_t post_len, float* posterior, uint8_t* crc_ok,
              uint32_t* iterations_used, const tc_decode_options* opts) {
  return guarded([&] {
    need(dec != nullptr, "null decoder");
    need(n_cb == 0 || (cbs && llr && posterior), "null pointer");
    tc_decode_options o;
    if (opts) o = *opts; else tc_decode_options_init(&o);
    need(o.memory == TC_MEM_HOST || o.memory == TC_MEM_DEVICE || o.memory == TC_MEM_HOST_ASYNC,
         "unknown memory kind");
    need(o.schedule == TC_SCHEDULE_PLAIN || o.schedule == TC_SCHEDULE_PERSISTENT ||
             o.schedule == TC_SCHEDULE_AUTO,
         "unknown schedule");
    need(o.max_iterations <= 64, "max_iterations above 64");
    static_assert(sizeof(tc_code_block) == sizeof(tcb::CodeBlockDesc), "descriptor layout");
    tcb::DecodeRequest rq;
    rq.n_cb = n_cb;
    rq.cbs = reinterpret_cast<const tcb::CodeBlockDesc*>(cbs);
    rq.llr_len = llr_len;
    rq.llr = llr;
    rq.post_len = post_len;
    rq.posterior = posterior;
    rq.crc_ok = crc_ok;
    rq.iterations_used = iterations_used;
    rq.max_iterations = o.max_iterations;
    rq.early_stop = o.early_stop != 0;
    rq.window = o.window;
    rq.guard = o.guard;
    rq.device_memory = o.memory == TC_MEM_DEVICE;
    rq.host_async = o.memory == TC_MEM_HOST_ASYNC;
    rq.persistent = o.schedule == TC_SCHEDULE_PERSISTENT;
    rq.auto_schedule = o.schedule == TC_SCHEDULE_AUTO;
    rq.graph = o.graph != 0;
    rq.scales = o.scales;
    rq.stream = o.stream;
    rq.std3gpp = convention_of(static_cast<int>(o.convention)) == tcb::Convention::Std3gpp;
    dec->impl.decode(rq);
  });
}

int tc_decode_noalloc(size_t n_cb, const tc_code_block* cbs, size_t llr_len, const float* llr,
                      size_t post_len, float* posterior, uint8_t* crc_ok,
                      uint32_t* iterations_used, const tc_decode_options* opts,
                      size_t* scratch_bytes) {
  return guarded([&] {
    need(n_cb == 0 || (cbs && llr && posterior), "null pointer");
    tc_decode_options o;
    if (opts) o = *opts; else tc_decode_options_init(&o);
    need(o.max_iterations <= 64, "max_iterations above 64");
    need(o.convention == TC_CONVENTION_REFERENCE,
         "tc_decode_noalloc decodes the reference convention only");
    tcb::DecodeRequest rq;
    rq.n_cb = n_cb;
    rq.cbs = reinterpret_cast<const tcb::CodeBlockDesc*>(cbs);
    rq.llr_len = llr_len;
    rq.llr = llr;
    rq.post_len = post_len;
    rq.posterior = posterior;
    rq.crc_ok = crc_ok;
    rq.iterations_used = iterations_used;
    rq.max_iterations = o.max_iterations;
    rq.early_stop = o.early_stop != 0;
    rq.window = o.window;
    rq.guard = o.guard;
    rq.device_memory = true;
    rq.scales = o.scales;
    rq.stream = o.stream;
    tcb::decode_noalloc(rq, scratch_bytes);
  });
}

int tc_autotune(tc_decoder* dec, size_t n_cb, const tc_code_block* cbs, size_t llr_len,
                const float* llr, size_t post_len, float* posterior,
                const tc_decode_options* opts, tc_tune_result* best) {
  return guarded([&] {
    need(dec != nullptr && cbs && llr && posterior, "null pointer");
    tc_decode_options o;
    if (opts) o = *opts; else tc_decode_options_init(&o);
    need(o.memory == TC_MEM_DEVICE, "autotuning needs TC_MEM_DEVICE buffers");
    tcb::DecodeRequest rq;
    rq.n_cb = n_cb;
    rq.cbs = reinterpret_cast<const tcb::CodeBlockDesc*>(cbs);
    rq.llr_len = llr_len;
    rq.llr = llr;
    rq.post_len = post_len;
    rq.posterior = posterior;
    rq.max_iterations = o.max_iterations;
    rq.early_stop = o.early_stop != 0;
    rq.guard = o.guard;
    rq.device_memory = true;
    rq.scales = o.scales;
    rq.stream = o.stream;
    rq.std3gpp = convention_of(static_cast<int>(o.convention)) == tcb::Convention::Std3gpp;
    const auto c = dec->impl.autotune(rq);
    if (best) {
      best->schedule = c.persistent ? TC_SCHEDULE_PERSISTENT : TC_SCHEDULE_PLAIN;
      best->window = c.window;
      best->ms = c.ms;
    }
  });
}

int tc_autotune_save(tc_decoder* dec, const char* path) {
  return guarded([&] {
    need(dec != nullptr && path != nullptr, "null pointer");
    dec->impl.save_tuning(path);
  });
}

int tc_autotune_load(tc_decoder* dec, const char* path) {
  return guarded([&] {
    need(dec != nullptr && path != nullptr, "null pointer");
    dec->impl.load_tuning(path);
  });
}

int tc_decoder_inject_stall(tc_decoder* dec, int task) {
  return guarded([&] {
    need(dec != nullptr, "null decoder");
    dec->impl.inject_stall(task);
  });
}

int tc_decoder_sync(tc_decoder* dec) {
  return guarded([&] {
    need(dec != nullptr, "null decoder");
    dec->impl.sync();
  });
}

int tc_derate_match_llr_device(tc_decoder* dec, size_t n_cb, const tc_rm_block* blocks,
                               size_t e_len, const float* e_llr, size_t llr_len, float* d012,
                               void* stream) {
  return guarded([&] {
    need(dec != nullptr && (n_cb == 0 || (blocks && e_llr && d012)), "null pointer");
    static_assert(sizeof(tc_rm_block) == sizeof(tcb::RmBlockDesc), "descriptor layout");
    dec->impl.derate_match_llr(n_cb, reinterpret_cast<const tcb::RmBlockDesc*>(blocks), e_llr,
                               e_len, d012, llr_len, stream);
  });
}

int tc_awgn_code_blocks_device(tc_decoder* dec, uint64_t seed, size_t n, const int32_t* k,
                               const int32_t* filler, const float* ebn0_db, int crc24b,
                               uint8_t* bits, float* llr, void* stream) {
  return guarded([&] {
    need(dec != nullptr && (n == 0 || (k && ebn0_db && bits && llr)), "null pointer");
    std::vector<int32_t> f(n, 0);
    if (filler) f.assign(filler, filler + n);
    dec->impl.awgn_code_blocks_device(seed, n, k, f.data(), ebn0_db, crc24b != 0, bits, llr,
                                      stream);
  });
}

int tc_turbo_encode_device(tc_decoder* dec, size_t n, const int32_t* k, const int32_t* filler,
                           const uint8_t* bits, uint8_t* d012, void* stream) {
  return guarded([&] {
    need(dec != nullptr && (n == 0 || (k && bits && d012)), "null pointer");
    std::vector<int32_t> f(n, 0);
    if (filler) f.assign(filler, filler + n);
    dec->impl.turbo_encode_device(n, k, f.data(), bits, d012, stream);
  });
}

int tc_rate_match_device(tc_decoder* dec, size_t n, const tc_rm_block* blocks, size_t d012_len,
                         const uint8_t* d012, size_t e_len, uint8_t* e_bits, void* stream) {
  return guarded([&] {
    need(dec != nullptr && (n == 0 || (blocks && d012 && e_bits)), "null pointer");
    dec->impl.rate_match_device(n, reinterpret_cast<const tcb::RmBlockDesc*>(blocks), d012,
                                d012_len, e_bits, e_len, stream);
  });
}

int tc_derate_combine_llr_device(tc_decoder* dec, size_t n_tx, const tc_rm_block* tx,
                                 size_t e_len, const float* e_llr, size_t llr_len, float* d012,
                                 void* stream) {
  return guarded([&] {
    need(dec != nullptr && (n_tx == 0 || (tx && e_llr && d012)), "null pointer");
    dec->impl.derate_combine_llr(n_tx, reinterpret_cast<const tcb::RmBlockDesc*>(tx), e_llr,
                                 e_len, d012, llr_len, stream);
  });
}

int tc_decode_transport_blocks(tc_decoder* dec, size_t n_tb, const tc_transport_block* tbs,
                               size_t n_cb, const tc_rm_block* cbs, size_t e_len,
                               const float* e_llr, size_t bits_len, uint8_t* tb_bits,
                               uint8_t* tb_crc_ok, uint8_t* cb_crc_ok, uint32_t* iterations_used,
                               float* posterior, const tc_decode_options* opts) {
  return guarded([&] {
    need(dec != nullptr, "null decoder");
    need(n_tb == 0 || (tbs && cbs && e_llr && tb_bits), "null pointer");
    static_assert(sizeof(tc_transport_block) == sizeof(tcb::TbDesc), "descriptor layout");
    tc_decode_options o;
    if (opts) o = *opts; else tc_decode_options_init(&o);
    need(o.max_iterations <= 64, "max_iterations above 64");
    need(o.schedule <= TC_SCHEDULE_AUTO, "unknown schedule");
    tcb::TbRequest q;
    q.n_tb = n_tb;
    q.tbs = reinterpret_cast<const tcb::TbDesc*>(tbs);
    q.n_cb = n_cb;
    q.cbs = reinterpret_cast<const tcb::RmBlockDesc*>(cbs);
    q.e_len = e_len;
    q.e_llr = e_llr;
    q.bits_len = bits_len;
    q.bits = tb_bits;
    q.tb_crc_ok = tb_crc_ok;
    q.cb_crc_ok = cb_crc_ok;
    q.iterations_used = iterations_used;
    q.posterior = posterior;
    need(o.memory == TC_MEM_HOST || o.memory == TC_MEM_DEVICE || o.memory == TC_MEM_HOST_ASYNC,
         "unknown memory kind");
    q.device_memory = o.memory == TC_MEM_DEVICE;
    q.host_async = o.memory == TC_MEM_HOST_ASYNC;
    q.stream = o.stream;
    q.decode.max_iterations = o.max_iterations;
    q.decode.early_stop = o.early_stop != 0;
    q.decode.window = o.window;
    q.decode.guard = o.guard;
    q.decode.persistent = o.schedule == TC_SCHEDULE_PERSISTENT;
    q.decode.auto_schedule = o.schedule == TC_SCHEDULE_AUTO;
    q.decode.graph = o.graph != 0;  // honoured with TC_MEM_DEVICE
    q.decode.scales = o.scales;
    q.decode.std3gpp = convention_of(static_cast<int>(o.convention)) == tcb::Convention::Std3gpp;
    dec->impl.decode_transport_blocks(q);
  });
}

int tc_decoder_set_timing(tc_decoder* dec, int enable) {
  return guarded([&] {
    need(dec != nullptr, "null decoder");
    dec->impl.set_timing(enable != 0);
  });
}

int tc_decoder_timing(tc_decoder* dec, tc_timing* out, int reset) {
  return guarded([&] {
    need(dec != nullptr && out != nullptr, "null pointer");
    const tcb::Timing t = dec->impl.timing(reset != 0);
    out->launches = t.launches;
    out->siso_launches = t.siso_launches;
    out->siso_ms = t.siso_ms;
    out->trellis_steps = t.trellis_steps;
  });
}

int tc_adjoint_create(tc_decoder* dec, tc_adjoint** out) {
  return guarded([&] {
    need(dec != nullptr && out != nullptr, "null pointer");
    *out = nullptr;
    *out = new tc_adjoint(dec->impl);
  });
}

int tc_adjoint_destroy(tc_adjoint* adj) {
  return guarded([&] { delete adj; });
}

int tc_adjoint_forward(tc_adjoint* adj, size_t n_cb, const tc_code_block* cbs, size_t llr_len,
                       const float* llr, size_t post_len, float* posterior, uint32_t iterations,
                       const float* scales, int32_t window, int32_t guard, void* stream,
                       uint64_t* tape) {
  return tc_adjoint_forward_conv(TC_CONVENTION_REFERENCE, adj, n_cb, cbs, llr_len, llr, post_len,
                                 posterior, iterations, scales, window, guard, stream, tape);
}

int tc_adjoint_forward_conv(int convention, tc_adjoint* adj, size_t n_cb,
                            const tc_code_block* cbs, size_t llr_len, const float* llr,
                            size_t post_len, float* posterior, uint32_t iterations,
                            const float* scales, int32_t window, int32_t guard, void* stream,
                            uint64_t* tape) {
  return guarded([&] {
    need(adj != nullptr && tape != nullptr, "null pointer");
    need(n_cb > 0 && cbs && llr && posterior, "null pointer or no code blocks");
    tcb::AdjointRequest rq;
    rq.n_cb = n_cb;
    rq.cbs = reinterpret_cast<const tcb::CodeBlockDesc*>(cbs);
    rq.llr_len = llr_len;
    rq.llr = llr;
    rq.post_len = post_len;
    rq.posterior = posterior;
    rq.iterations = iterations;
    rq.scales = scales;
    rq.window = window;
    rq.guard = guard;
    rq.stream = stream;
    rq.std3gpp = convention_of(convention) == tcb::Convention::Std3gpp;
    *tape = adj->impl.forward(rq);
  });
}

int tc_adjoint_backward(tc_adjoint* adj, uint64_t tape, const float* grad_posterior,
                        float* grad_llr, float* grad_scales, void* stream) {
  return guarded([&] {
    need(adj && grad_posterior && grad_llr && grad_scales, "null pointer");
    adj->impl.backward(tape, grad_posterior, grad_llr, grad_scales, stream);
  });
}

int tc_adjoint_launches(tc_adjoint* adj, uint64_t* launches) {
  return guarded([&] {
    need(adj && launches, "null pointer");
    *launches = adj->impl.launches();
  });
}

}  // extern "C"
