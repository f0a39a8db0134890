/*
 * turbo_b200.h -- C ABI of libturbo_b200.so, the B200 (sm_100a) LTE turbo decoder.
 *
 * Every function returns a tc_status (0 = TC_OK), never throws, and leaves a human-readable
 * detail of the last failure in tc_last_error() (per calling thread).  No CUDA or C++ types
 * appear here: device pointers, host pointers and streams are plain pointers.
 *
 * Each entry point names the Wiseung/Turbo_CPP interface it replaces
 * (include/turbo_cpp/lte_turbo.h and src/lte_turbo.cpp in that project).
 */
#ifndef TURBO_B200_H
#define TURBO_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define TC_API __attribute__((visibility("default")))
#else
#define TC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  TC_OK = 0,
  TC_ERR_INVALID_ARGUMENT = 1, /* reference: std::invalid_argument (sizes, descriptors)       */
  TC_ERR_OUT_OF_RANGE = 2,     /* reference: std::out_of_range (K not an LTE block size)     */
  TC_ERR_RUNTIME = 3,          /* reference: std::runtime_error (e.g. K+/K- selection)        */
  TC_ERR_CUDA = 4,             /* a CUDA runtime call failed                                  */
  TC_ERR_NO_DEVICE = 5,        /* no CUDA device visible                                      */
  TC_ERR_TIMEOUT = 6,          /* a bounded device-side wait gave up                          */
  TC_ERR_CAPACITY = 7          /* request exceeds a fixed capacity                            */
} tc_status;

TC_API const char* tc_status_name(int status);
TC_API const char* tc_last_error(void);
TC_API int tc_version(void); /* major*10000 + minor*100 + patch */

/* ---------------- QPP interleaver ----------------
 * replaces qpp_interleaver_table / qpp_entry_for_k / qpp_permutation /
 * qpp_inverse_permutation (lte_turbo.h:94-95, 108-109; lte_turbo.cpp:498-506, 606-622) */
TC_API int tc_qpp_table_size(void);
TC_API int tc_qpp_entry(int index, int32_t* k, int32_t* f1, int32_t* f2);
TC_API int tc_qpp_index(int32_t k, int32_t* index); /* TC_ERR_OUT_OF_RANGE for unsupported K */
TC_API int tc_qpp_permutation(int32_t k, int32_t* perm /* K */);
TC_API int tc_qpp_inverse_permutation(int32_t k, int32_t* inv /* K */);

/* ---------------- CRC ----------------
 * replaces append_crc24a/24b/16/8 and check_crc24a/24b/16/8 (lte_turbo.h:97-104) */
typedef enum { TC_CRC24A = 0, TC_CRC24B = 1, TC_CRC16 = 2, TC_CRC8 = 3 } tc_crc_kind;
TC_API int tc_crc_append(int kind, const uint8_t* bits, size_t n, uint8_t* out /* n + L */);
TC_API int tc_crc_check(int kind, const uint8_t* bits, size_t n, int* ok);

/* ---------------- code-block segmentation ----------------
 * replaces segment_transport_block (lte_turbo.h:83-92, 106; lte_turbo.cpp:540-604) */
typedef struct {
  size_t c, c_plus, c_minus, k_plus, k_minus, filler_bits, l;
} tc_segmentation;
/* cb_bits may be NULL (sizes only); otherwise it receives the C blocks back to back,
 * c_plus*k_plus + c_minus*k_minus bits, and cap is its capacity. */
TC_API int tc_segment_transport_block(const uint8_t* bits_with_crc, size_t b, tc_segmentation* info,
                               uint8_t* cb_bits, size_t cap);

/* ---------------- encoder and rate matching ----------------
 * replace turbo_encode_code_block (lte_turbo.h:111-112), the rate matching inside
 * encode_transport_block (lte_turbo.cpp:167-278, 690-720) and derate_match_code_block
 * (lte_turbo.h:116-118).  d012 = [d0 | d1 | d2], each K+4 entries. */
TC_API int tc_turbo_encode(int32_t k, int32_t filler, const uint8_t* cb_bits, uint8_t* d012);
TC_API int tc_compute_e(size_t r, size_t g_total, size_t c, uint32_t num_layers, uint32_t mod_order,
                 size_t* e);
TC_API int tc_rate_match(int32_t k, int32_t filler, const uint8_t* d012, size_t e, uint32_t rv,
                  uint8_t* out /* e bits */);
/* hard bits -> +-8.0 with repetition combining, exactly derate_match_code_block */
TC_API int tc_derate_match_bits(int32_t k, int32_t filler, const uint8_t* e_bits, size_t e, uint32_t rv,
                         float* d012_llr);
/* the same walk over soft channel LLRs (LLR-domain de-rate matching; new) */
TC_API int tc_derate_match_llr(int32_t k, int32_t filler, const float* e_llr, size_t e, uint32_t rv,
                        float* d012_llr);

/* ---------------- the TS 36.212 code (new; off by default) ----------------
 * Everything above follows the reference's code, which departs from TS 36.212 in its
 * constituent encoder (feedback g0 = 1+D+D^2 where 36.212 5.1.3.2.1 has 1+D^2+D^3;
 * lte_turbo.cpp:333-341), its CRC generators (the coefficient arrays of lte_turbo.cpp:104-116
 * instead of the 36.212 5.1.1 polynomials) and its trellis-termination multiplexing
 * (lte_turbo.cpp:664-677 instead of 36.212 5.1.3.2.2).  TC_CONVENTION_3GPP selects the 36.212
 * code in these functions and, through tc_decode_options.convention, in the decoders.  QPP
 * interleaving, segmentation sizes, filler handling, the circular buffer and rate matching are
 * common to both conventions (no limited-buffer rate matching in either).  The _conv functions
 * with TC_CONVENTION_REFERENCE are the functions above. */
enum { TC_CONVENTION_REFERENCE = 0, TC_CONVENTION_3GPP = 1 };
TC_API int tc_crc_append_conv(int convention, int kind, const uint8_t* bits, size_t n,
                              uint8_t* out /* n + L */);
TC_API int tc_crc_check_conv(int convention, int kind, const uint8_t* bits, size_t n, int* ok);
TC_API int tc_segment_transport_block_conv(int convention, const uint8_t* bits_with_crc, size_t b,
                                           tc_segmentation* info, uint8_t* cb_bits, size_t cap);
TC_API int tc_turbo_encode_conv(int convention, int32_t k, int32_t filler, const uint8_t* cb_bits,
                                uint8_t* d012);

/* ---------------- seeded test channel (new; used by tests and the benchmark) ---------------- */
TC_API int tc_random_bits(uint64_t seed, uint64_t first, size_t n, uint8_t* bits);
TC_API int tc_awgn_llr(uint64_t seed, uint64_t first, const uint8_t* bits, size_t n, double sigma2,
                float* llr);

/* n seeded code blocks: info bits (filler zeros first; last 24 bits CRC24B when crc24b), turbo
 * encoding, BPSK/AWGN at ebn0_db[i] (rate K/(3(K+4)), LLR = 2y/sigma^2), filler LLRs zeroed.
 * bits: sum K; llr: 3*sum(K+4), blocks back to back.  threads <= 0: all cores. */
TC_API int tc_awgn_code_blocks(uint64_t seed, size_t n, const int32_t* k, const int32_t* filler,
                               const float* ebn0_db, int crc24b, uint8_t* bits, float* llr,
                               int threads);

/* ---------------- GPU decoder ----------------
 * replaces turbo_decode_code_block_gpu_stage1 / _stage2 / _stage1_tile8_experimental
 * (lte_turbo.h:129-155) and their CUDA impls (lte_turbo_cuda.cu:1391-1899): any number of
 * code blocks of any LTE sizes per call, exact Log-MAP, posterior = Ls + e1 + e2 as
 * turbo_decode_code_block_cpu (lte_turbo.cpp:736-813). */
typedef struct tc_decoder tc_decoder;
TC_API int tc_decoder_create(int device, tc_decoder** out);
TC_API int tc_decoder_destroy(tc_decoder* dec);

typedef struct {
  int32_t k;          /* block size: one of the 188 LTE QPP sizes                       */
  int32_t filler;     /* filler bits at the block start (erasures; zeroed before CRC)   */
  int64_t llr_offset; /* float offset of [d0|d1|d2] (3*(K+4) floats); multiple of 4       */
  int64_t out_offset; /* float offset of the block's K posterior LLRs                     */
} tc_code_block;

/* HOST: synchronous, the call copies the LLRs in and the results out.  DEVICE: device pointers,
 * ordered on opts->stream, returns once enqueued (without a graph replay, the launch
 * descriptors' copy first waits for the work already on that stream, so back-to-back calls
 * return as each previous one finishes; a replayed graph never waits).  HOST_ASYNC (new): host
 * pointers; the call
 * enqueues copy-in, decode and copy-out on one of three internal device workspaces (used in
 * turn, each with its own stream) and returns, so that one call's copies run while earlier
 * calls decode; results are valid, and the input buffer may be reused, after tc_decoder_sync.
 * Pinned host memory is needed for the copies to overlap. */
enum { TC_MEM_HOST = 0, TC_MEM_DEVICE = 1, TC_MEM_HOST_ASYNC = 2 };
/* PLAIN: one launch per SISO half-iteration over all blocks (host-driven iteration loop).
 * PERSISTENT: one launch for all iterations, warps pull (task, half-iteration) items from a
 * device queue, blocks stop individually on CRC24B.  AUTO: the schedule and window that
 * tc_autotune found fastest for requests of the same signature (PLAIN, window 128 if none). */
enum { TC_SCHEDULE_PLAIN = 0, TC_SCHEDULE_PERSISTENT = 1, TC_SCHEDULE_AUTO = 2 };

typedef struct {
  uint32_t max_iterations; /* default 8                                                   */
  uint32_t early_stop;     /* stop a block once its hard decisions pass CRC24B            */
  int32_t window;          /* steps per window; 0 = default (128); >= K = full trellis    */
  int32_t guard;           /* warm-up steps on each side; < 0 = default (96); multiple of 8 */
  uint32_t memory;         /* TC_MEM_HOST, TC_MEM_DEVICE or TC_MEM_HOST_ASYNC              */
  uint32_t schedule;       /* TC_SCHEDULE_PLAIN, TC_SCHEDULE_PERSISTENT or TC_SCHEDULE_AUTO */
  const float* scales;     /* host array, 2 per iteration (upper, lower); NULL = 1.0     */
  uint32_t graph;          /* TC_MEM_DEVICE only (tc_decode, tc_decode_transport_blocks):
                              capture this request's launch sequence in a CUDA graph the first
                              time and replay it when the same shapes, buffers and options come
                              again (16 graphs kept per decoder);
                              needs a created stream (the legacy default stream cannot be
                              captured: TC_ERR_INVALID_ARGUMENT)                          */
  void* stream;            /* cudaStream_t; TC_MEM_DEVICE: used as given (NULL = the legacy
                              default stream); TC_MEM_HOST: NULL = the decoder's own stream */
  uint32_t convention;     /* TC_CONVENTION_REFERENCE (default) or TC_CONVENTION_3GPP: the code
                              the LLRs come from (trellis, tail multiplexing, CRC24B of the
                              early stop; CRC24A too in tc_decode_transport_blocks).  Honoured
                              by tc_decode (every schedule and memory kind), tc_autotune and
                              tc_decode_transport_blocks; tc_decode_noalloc refuses the 3GPP
                              code (TC_ERR_INVALID_ARGUMENT); the differentiable decoder takes
                              it through tc_adjoint_forward_conv */
} tc_decode_options;

TC_API int tc_decode_options_init(tc_decode_options* opts);

/* Autotuning (new): decodes the given TC_MEM_DEVICE request with each candidate schedule and
 * window length (plain 128..256, persistent 192..320; a few decodes each), keeps the fastest for
 * requests of the same signature (early stop, iterations, block count and mean K, rounded) and
 * reports it.  tc_autotune_save/load write and read the table as text. */
typedef struct {
  int32_t schedule; /* TC_SCHEDULE_PLAIN or TC_SCHEDULE_PERSISTENT */
  int32_t window;
  double ms;        /* time of one decode with that choice */
} tc_tune_result;
TC_API int tc_autotune(tc_decoder* dec, size_t n_cb, const tc_code_block* cbs, size_t llr_len,
                       const float* llr, size_t post_len, float* posterior,
                       const tc_decode_options* opts, tc_tune_result* best);
TC_API int tc_autotune_save(tc_decoder* dec, const char* path);
TC_API int tc_autotune_load(tc_decoder* dec, const char* path);

/* Waits until the work this decoder has enqueued is done.  Returns TC_ERR_TIMEOUT (once) when a
 * persistent-schedule wait on the device gave up since the last check; host-memory calls report
 * that themselves, device-memory callers learn it here. */
TC_API int tc_decoder_sync(tc_decoder* dec);

/* Testing hook for the failure path (new): while set, persistent decodes on this decoder make
 * the warps working on task `task` (the task queue's order: largest blocks first) wait for a
 * progress count that is never reached.  The device-side wait limit (one second) runs out, the
 * kernel still finishes, and the call reports TC_ERR_TIMEOUT (host memory) or tc_decoder_sync
 * does (device memory); the results of that call are not valid.  -1 turns it off. */
TC_API int tc_decoder_inject_stall(tc_decoder* dec, int task);

/* Decodes n_cb code blocks.  llr has llr_len floats, posterior post_len floats; crc_ok
 * (n_cb bytes) and iterations_used (n_cb words) may be NULL.  With TC_MEM_HOST the call is
 * synchronous; with TC_MEM_DEVICE it is ordered on opts->stream and returns once enqueued
 * (see the memory kinds above for when that waits). */
TC_API int tc_decode(tc_decoder* dec, size_t n_cb, const tc_code_block* cbs, size_t llr_len,
              const float* llr, size_t post_len, float* posterior, uint8_t* crc_ok,
              uint32_t* iterations_used, const tc_decode_options* opts);

/* ---------------- transport-block chain on the device (new) ----------------
 * LLR-domain de-rate matching of many code blocks on the GPU: bit-identical to
 * tc_derate_match_llr (the reference's walk of lte_turbo.cpp:280-325 with soft values).  e_llr
 * and d012 are device pointers; ordered on `stream` (NULL = legacy default stream). */
typedef struct {
  int32_t k;          /* block size                                                  */
  int32_t filler;     /* filler bits (first code block of a transport block)         */
  int32_t e;          /* rate-matched LLRs of the block                               */
  uint32_t rv;        /* redundancy version 0..3                                      */
  int64_t e_offset;   /* float offset of its E rate-matched LLRs                     */
  int64_t llr_offset; /* float offset of its [d0|d1|d2] output (multiple of 4)       */
} tc_rm_block;
TC_API int tc_derate_match_llr_device(tc_decoder* dec, size_t n_cb, const tc_rm_block* blocks,
                                      size_t e_len, const float* e_llr, size_t llr_len,
                                      float* d012, void* stream);

/* ---------------- test-vector generation on the device (new) ----------------
 * tc_awgn_code_blocks_device: the device version of tc_awgn_code_blocks (same seed, same
 * layout: K information bits per block back to back in `bits`, [d0|d1|d2] LLRs per block back
 * to back in `llr`, both device memory; k, filler (may be NULL: none) and ebn0_db are host
 * arrays of n).  Bits (and their CRC24B) and encoded streams are bit-identical to the host
 * generator; the LLRs are equal up to the last bit of double log/cos on the device against the
 * host C library.  tc_turbo_encode_device: turbo_encode_code_block (lte_turbo.cpp:624-688) of
 * many blocks (bits in, 3(K+4) encoded bits per block out, back to back, device memory).
 * tc_rate_match_device: rate matching (lte_turbo.cpp:250-278) of many blocks: tc_rm_block
 * gives K, filler, E, rv, the output offset (e_offset) and the offset of the block's encoded
 * [d0|d1|d2] bits in d012 (llr_offset).  All ordered on `stream`. */
TC_API int tc_awgn_code_blocks_device(tc_decoder* dec, uint64_t seed, size_t n, const int32_t* k,
                                      const int32_t* filler, const float* ebn0_db, int crc24b,
                                      uint8_t* bits, float* llr, void* stream);
TC_API int tc_turbo_encode_device(tc_decoder* dec, size_t n, const int32_t* k,
                                  const int32_t* filler, const uint8_t* bits, uint8_t* d012,
                                  void* stream);
TC_API int tc_rate_match_device(tc_decoder* dec, size_t n, const tc_rm_block* blocks,
                                size_t d012_len, const uint8_t* d012, size_t e_len,
                                uint8_t* e_bits, void* stream);

/* HARQ soft combining (new; the reference de-rate matches a single transmission,
 * lte_turbo.cpp:280-325): the n_tx entries of tx are transmissions; those of one code block are
 * consecutive and share llr_offset, K and filler (at most 8 per code block), each with its own
 * rv, E and e_offset.  Each code block's [d0|d1|d2] becomes the sum, in the given order, of its
 * transmissions' de-rate-matched LLRs -- bit-identical to tc_derate_match_llr per transmission
 * followed by elementwise addition in that order.  Device pointers, ordered on `stream`. */
TC_API int tc_derate_combine_llr_device(tc_decoder* dec, size_t n_tx, const tc_rm_block* tx,
                                        size_t e_len, const float* e_llr, size_t llr_len,
                                        float* d012, void* stream);

/* Decodes many transport blocks at once (replaces decode_transport_block, lte_turbo.h:157-159,
 * lte_turbo.cpp:891-980, for any number of transport blocks per call): device de-rate matching,
 * batched turbo decoding with opts (schedule, early stop on CRC24B, iterations, ...), then per
 * transport block hard decisions, filler strip, CRC24B check and strip (C > 1), concatenation
 * and CRC24A.  The code blocks of transport block t are cbs[first_cb .. first_cb + n_cb); their
 * llr_offset is ignored.  tb_bits receives one byte (0/1) per decoded bit at bits_offset;
 * tb_crc_ok (n_tb), cb_crc_ok, iterations_used (n_cb) and posterior (sum K, may be NULL) follow
 * opts->memory like the rate-matched LLRs.  TC_MEM_HOST_ASYNC (new): host pointers; the call
 * is enqueued on one of the decoder's three worker workspaces and returns, so that one call's
 * copies overlap earlier calls' decoding; results are valid, and the inputs may be reused,
 * after tc_decoder_sync (pinned buffers for the overlap).  TC_SCHEDULE_AUTO takes the schedule
 * and window that tc_autotune found for the code blocks' decode request (same signature); with
 * TC_MEM_DEVICE and opts->graph the whole chain -- de-rate matching, decoding, finish -- is
 * captured in one CUDA graph per request key (descriptors, buffers, options) and replayed. */
typedef struct {
  int64_t tbs;         /* transport block size, without CRC24A */
  int32_t first_cb;
  int32_t n_cb;
  int64_t bits_offset; /* first output bit of the block */
} tc_transport_block;
TC_API int tc_decode_transport_blocks(tc_decoder* dec, size_t n_tb, const tc_transport_block* tbs,
                                      size_t n_cb, const tc_rm_block* cbs, size_t e_len,
                                      const float* e_llr, size_t bits_len, uint8_t* tb_bits,
                                      uint8_t* tb_crc_ok, uint8_t* cb_crc_ok,
                                      uint32_t* iterations_used, float* posterior,
                                      const tc_decode_options* opts);

/* ---------------- decoding without device allocation ----------------
 * No counterpart in the reference.  The same plain-schedule decode as tc_decode with
 * TC_MEM_DEVICE, for callers that must not allocate device memory: a real-time receiver thread
 * that cannot absorb the synchronisation and latency of cudaMalloc/cudaFree, a program whose
 * device memory belongs to another allocator, a plug-in handed only its input and output
 * buffers.  No decoder object is needed; it runs on the current device, ordered on
 * opts->stream (NULL = the legacy default stream), and returns once enqueued (after the work
 * already on that stream: its descriptor copy waits for it).  llr, posterior,
 * crc_ok and iterations_used are device pointers (the last two may be NULL).
 *
 * Every other device buffer comes from a fixed 32 MiB array compiled into the library (held on
 * each GPU that loads it until the library is unloaded); a request that needs more is refused
 * with TC_ERR_CAPACITY before any work is enqueued (*scratch_bytes, when given, receives the
 * bytes the request needs; about 135 KB per K=6144 code block, i.e. ~240 such blocks).  The
 * first call on a device copies constant tables synchronously: make it before any stream
 * capture begins.  Every call copies its block descriptors from memory that lives only for the
 * call, so a call made while its stream is capturing is refused (TC_ERR_INVALID_ARGUMENT).
 * Those tables are uploaded once per device and process: after cudaDeviceReset the entry point
 * must not be used again in that process (a module reloaded at another address is detected and
 * set up again; one reloaded at the same address is not).  All calls on a device share the
 * array; calls that overlap on the GPU race. */
TC_API int tc_decode_noalloc(size_t n_cb, const tc_code_block* cbs, size_t llr_len,
                             const float* llr, size_t post_len, float* posterior,
                             uint8_t* crc_ok, uint32_t* iterations_used,
                             const tc_decode_options* opts, size_t* scratch_bytes);

/* ---------------- kernel accounting (new) ----------------
 * Every kernel launch is counted.  With timing on, each SISO half-iteration launch is
 * bracketed by CUDA events on its launching stream; tc_decoder_timing waits for those events
 * and returns the sums (optionally resetting them). */
typedef struct {
  uint64_t launches;      /* kernels launched by this decoder                  */
  uint64_t siso_launches; /* SISO launches timed                               */
  double siso_ms;         /* summed device time of the timed SISO launches     */
  uint64_t trellis_steps; /* output trellis steps (sum of K) of those launches */
} tc_timing;
TC_API int tc_decoder_set_timing(tc_decoder* dec, int enable);
TC_API int tc_decoder_timing(tc_decoder* dec, tc_timing* out, int reset);

/* ---------------- differentiable decoder and its adjoint (new) ----------------
 * No counterpart in the reference, which has no gradient code; the forward function is the
 * reference decoder (turbo_decode_code_block_cpu, lte_turbo.cpp:736-813) unrolled for
 * `iterations` iterations without early stop, with the extrinsic of SISO j (j = 2*it upper,
 * 2*it+1 lower) multiplied by scales[j] before it becomes the other SISO's a-priori and before
 * it enters the posterior Ls + e1 + e2, run on the windowed schedule (window, guard;
 * 0 / -1 = 64 / 32; window >= K is the full trellis) whose next-iteration seeds are constants
 * of the function.  The adjoint is hand-written: alpha checkpoints every 4 steps kept by the
 * forward pass, beta checkpointed on the backward pass, both recomputed between checkpoints,
 * the transposed softmax weights of every max*.
 * All buffers are device memory ordered on `stream` (NULL = the legacy default stream);
 * `scales` is host memory (2*iterations floats, NULL = all 1).  The LLR buffer must stay
 * unchanged between a forward pass and its backward pass.  A forward pass returns a tape id;
 * the backward pass of an older tape (replaced by a later forward pass on the same handle)
 * fails with TC_ERR_INVALID_ARGUMENT. */
typedef struct tc_adjoint tc_adjoint;
TC_API int tc_adjoint_create(tc_decoder* dec, tc_adjoint** out);
TC_API int tc_adjoint_destroy(tc_adjoint* adj);
TC_API int tc_adjoint_forward(tc_adjoint* adj, size_t n_cb, const tc_code_block* cbs,
                              size_t llr_len, const float* llr, size_t post_len, float* posterior,
                              uint32_t iterations, const float* scales, int32_t window,
                              int32_t guard, void* stream, uint64_t* tape);
/* The same on the code `convention` selects (TC_CONVENTION_REFERENCE or TC_CONVENTION_3GPP);
 * the backward pass differentiates the code of its tape. */
TC_API int tc_adjoint_forward_conv(int convention, tc_adjoint* adj, size_t n_cb,
                                   const tc_code_block* cbs, size_t llr_len, const float* llr,
                                   size_t post_len, float* posterior, uint32_t iterations,
                                   const float* scales, int32_t window, int32_t guard,
                                   void* stream, uint64_t* tape);
/* grad_posterior: post_len floats (posterior layout); grad_llr: llr_len floats (LLR layout,
 * 0 outside every block; 16-byte aligned, as the LLR buffer); grad_scales: 2*iterations
 * floats. */
TC_API int tc_adjoint_backward(tc_adjoint* adj, uint64_t tape, const float* grad_posterior,
                               float* grad_llr, float* grad_scales, void* stream);
TC_API int tc_adjoint_launches(tc_adjoint* adj, uint64_t* launches);

#ifdef __cplusplus
}
#endif
#endif
