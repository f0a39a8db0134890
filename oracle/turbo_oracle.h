/*
 * turbo_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the Wiseung/Turbo_CPP CPU codec chain (src/lte_turbo.cpp), used as
 * the correctness oracle for the turbo_cpp_b200 CUDA decoder.  Only tests/, the smoke() check
 * in __graft_entry__.py and the cpu_baseline leg of bench.py may load it; the product library
 * never links or calls it.
 *
 * Parity status: pinned.  tests/test_oracle.py checks every function here against golden
 * fixtures produced by the reference itself (oracle/_ref, built from the reference sources by
 * oracle/Makefile) and, when oracle/_ref is present, against the live reference bit for bit.
 *
 * Conventions reproduced exactly (the reference deviates from TS 36.212 in these places):
 *   - RSC feedback u^s1^s2, parity fb^s0^s2, state (s2 s1 s0)       lte_turbo.cpp:333-341
 *   - CRC generators as the reference's bit arrays                   lte_turbo.cpp:104-155
 *   - tail multiplexing of d0/d1/d2                                  lte_turbo.cpp:664-677
 *   - decoder tail-LLR mapping (lower mapping does not mirror the mux) lte_turbo.cpp:758-773
 *   - filler bits are erasures; bit -> +-8.0 de-rate matching         lte_turbo.cpp:201,301
 *   - k0 = R*(2*ceil(Ncb/(8R))*rv + 2), Ncb = 3*K_pi (no LBRM)        lte_turbo.cpp:243,263
 */
#ifndef TURBO_ORACLE_H
#define TURBO_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- QPP interleaver (lte_turbo.cpp:54-102, 606-622) ---- */
int or_qpp_count(void);
void or_qpp_entry(int index, int32_t* k, int32_t* f1, int32_t* f2);
int or_qpp_index(int32_t k); /* -1 when K is not an LTE turbo block size */
void or_qpp_perm(int32_t k, int32_t* perm);

/* ---- CRC (lte_turbo.cpp:104-155, 508-538); kind: 0=24A 1=24B 2=16 3=8 ---- */
int or_crc_len(int kind);
void or_crc_append(int kind, const uint8_t* bits, size_t n, uint8_t* out /* n + len */);
int or_crc_check(int kind, const uint8_t* bits, size_t n);

/* ---- segmentation (lte_turbo.cpp:540-604) ---- */
typedef struct {
  size_t c, c_plus, c_minus, k_plus, k_minus, filler, l;
} or_seg_info;
/* cb_out receives the C code blocks back to back (sum of their K); may be NULL. */
int or_segment(const uint8_t* bits_with_crc, size_t b, or_seg_info* info, uint8_t* cb_out);

/* ---- encoder (lte_turbo.cpp:333-353, 624-688); d0/d1/d2 each K+4 ---- */
void or_turbo_encode(int32_t k, int32_t filler, const uint8_t* cb, uint8_t* d0, uint8_t* d1,
                     uint8_t* d2);

/* ---- rate matching / de-rate matching (lte_turbo.cpp:167-325, 690-734) ---- */
int64_t or_compute_e(size_t r, size_t g_total, size_t c, size_t num_layers, size_t mod_order);
void or_rate_match(int32_t d, int32_t filler, const uint8_t* d0, const uint8_t* d1,
                   const uint8_t* d2, size_t e, int32_t rv, uint8_t* out);
/* bits -> +-8.0 with repetition combining; out = [d0|d1|d2], 3*d floats */
void or_derate_bits(int32_t d, int32_t filler, const uint8_t* e_bits, size_t e, int32_t rv,
                    float* out);
/* the same walk over soft channel LLRs instead of hard bits */
void or_derate_llr(int32_t d, int32_t filler, const float* e_llr, size_t e, int32_t rv,
                   float* out);

/* ---- exact Log-MAP turbo decoder (lte_turbo.cpp:357-486, 736-813) ----
 * llr = [d0|d1|d2], each K+4.  Matches turbo_decode_code_block_cpu bit for bit. */
void or_decode_cb(int32_t k, int32_t filler, const float* llr, int32_t max_iterations,
                  int32_t early_stop, float* posterior, int32_t* crc_ok,
                  int32_t* iterations_used);

/* Many code blocks on `threads` POSIX threads (0 = all cores).  llr_off/out_off in floats. */
void or_decode_batch(int32_t n, const int32_t* k, const int32_t* filler, const int64_t* llr_off,
                     const float* llr, const int64_t* out_off, float* posterior,
                     int32_t max_iterations, int32_t early_stop, int32_t* crc_ok,
                     int32_t* iterations_used, int32_t threads);

/* ---- window-parallel schedule (restates the GPU fast mode's arithmetic order) ----
 * The block is cut into windows of `window` steps.  Each window's forward recursion starts
 * `guard` steps before the window and its backward recursion `guard` steps after it (warm-up).
 * A start at the block edge uses the true edge metric (state 0 / tail metrics); every other
 * start is seeded with the metric the neighbouring window computed at that position in the
 * previous iteration (next-iteration initialisation, NII); first-iteration seeds are all
 * zero (uniform).  This is the schedule the CUDA kernels run; tests compare the GPU against it
 * with a 1e-3 tolerance.  A window >= K reproduces the full trellis exactly. */
void or_decode_cb_windowed(int32_t k, int32_t filler, const float* llr, int32_t max_iterations,
                           int32_t early_stop, int32_t window, int32_t guard, float* posterior,
                           int32_t* crc_ok, int32_t* iterations_used);
void or_decode_batch_windowed(int32_t n, const int32_t* k, const int32_t* filler,
                              const int64_t* llr_off, const float* llr, const int64_t* out_off,
                              float* posterior, int32_t max_iterations, int32_t early_stop,
                              int32_t window, int32_t guard, int32_t* crc_ok,
                              int32_t* iterations_used, int32_t threads);

/* ---- FP64 differentiable decoder and its adjoint (checker of the GPU adjoint) ----
 * The windowed schedule of or_decode_cb_windowed (window, guard, next-iteration seeds) in
 * natural-log FP64, `iters` iterations, no early stop, the extrinsic of SISO j (j = 2*it upper,
 * 2*it+1 lower) multiplied by scales[j] before it is the other SISO's a-priori and before it
 * enters the posterior Ls + e1 + e2.  The seeds are constants of the function; window <= 0 or
 * >= K is the full trellis (no seeds).  Seeds are [2*iters][windows][16] (alpha 0..7, beta
 * 8..15, the values SISO j used in window w).  frozen_seeds (may be NULL) replaces the
 * schedule's own seeds; seeds_out (may be NULL) receives the seeds used.  grad_post (may be
 * NULL: forward only) is d loss / d posterior; then grad_llr (3(K+4)) and grad_scales
 * (2*iters) receive the vector-Jacobian product. */
int64_t or_adj_seed_count(int32_t k, int32_t iters, int32_t window);
void or_adj_vjp(int32_t k, const double* llr, int32_t iters, const double* scales,
                int32_t window, int32_t guard, const double* frozen_seeds,
                const double* grad_post, double* posterior, double* grad_llr,
                double* grad_scales, double* seeds_out);

/* ---- the TS 36.212 code (no reference counterpart; restated from 36.212 5.1.1 and
 * 5.1.3.2): CRC generator polynomials, constituent encoder g0 = 1+D^2+D^3 / g1 = 1+D+D^3, trellis
 * termination and tail multiplexing, and the windowed decoder above on that code.  Pinned by
 * the published CRC check values and by encode/decode round trips, not by the reference. ---- */
void or_std_crc_append(int kind, const uint8_t* bits, size_t n, uint8_t* out /* n + len */);
int or_std_crc_check(int kind, const uint8_t* bits, size_t n);
void or_std_turbo_encode(int32_t k, int32_t filler, const uint8_t* cb, uint8_t* d0, uint8_t* d1,
                         uint8_t* d2);
void or_std_decode_cb_windowed(int32_t k, int32_t filler, const float* llr,
                               int32_t max_iterations, int32_t early_stop, int32_t window,
                               int32_t guard, float* posterior, int32_t* crc_ok,
                               int32_t* iterations_used);

/* The FP64 differentiable decoder and its adjoint (or_adj_vjp) on the TS 36.212 code. */
void or_std_adj_vjp(int32_t k, const double* llr, int32_t iters, const double* scales,
                    int32_t window, int32_t guard, const double* frozen_seeds,
                    const double* grad_post, double* posterior, double* grad_llr,
                    double* grad_scales, double* seeds_out);

#ifdef __cplusplus
}
#endif
#endif
