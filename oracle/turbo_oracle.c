/*
 * turbo_oracle.c -- TEST INFRASTRUCTURE ONLY (see turbo_oracle.h).
 *
 * Plain-C restatement of the Wiseung/Turbo_CPP CPU codec chain.  Every function cites the
 * reference lines (src/lte_turbo.cpp) whose behaviour it follows.  The floating-point
 * operations are written in the reference's order and compiled with -ffp-contract=off so that
 * or_decode_cb is bitwise identical to turbo_decode_code_block_cpu.
 */
#include "turbo_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* ------------------------------------------------------------------------------------------ */
/* QPP table: TS 36.212 Table 5.1.3-3 as carried by lte_turbo.cpp:54-102.  The block sizes    */
/* follow the standard's four step regions, so only (f1, f2) are listed.                      */
/* ------------------------------------------------------------------------------------------ */
static const int16_t kF1F2[188][2] = {
    {3, 10},    {7, 12},    {19, 42},   {7, 16},    {7, 18},    {11, 20},   {5, 22},
    {11, 24},   {7, 26},    {41, 84},   {103, 90},  {15, 32},   {9, 34},    {17, 108},
    {9, 38},    {21, 120},  {101, 84},  {21, 44},   {57, 46},   {23, 48},   {13, 50},
    {27, 52},   {11, 36},   {27, 56},   {85, 58},   {29, 60},   {33, 62},   {15, 32},
    {17, 198},  {33, 68},   {103, 210}, {19, 36},   {19, 74},   {37, 76},   {19, 78},
    {21, 120},  {21, 82},   {115, 84},  {193, 86},  {21, 44},   {133, 90},  {81, 46},
    {45, 94},   {23, 48},   {243, 98},  {151, 40},  {155, 102}, {25, 52},   {51, 106},
    {47, 72},   {91, 110},  {29, 168},  {29, 114},  {247, 58},  {29, 118},  {89, 180},
    {91, 122},  {157, 62},  {55, 84},   {31, 64},   {17, 66},   {35, 68},   {227, 420},
    {65, 96},   {19, 74},   {37, 76},   {41, 234},  {39, 80},   {185, 82},  {43, 252},
    {21, 86},   {155, 44},  {79, 120},  {139, 92},  {23, 94},   {217, 48},  {25, 98},
    {17, 80},   {127, 102}, {25, 52},   {239, 106}, {17, 48},   {137, 110}, {215, 112},
    {29, 114},  {15, 58},   {147, 118}, {29, 60},   {59, 122},  {65, 124},  {55, 84},
    {31, 64},   {17, 66},   {171, 204}, {67, 140},  {35, 72},   {19, 74},   {39, 76},
    {19, 78},   {199, 240}, {21, 82},   {211, 252}, {21, 86},   {43, 88},   {149, 60},
    {45, 92},   {49, 846},  {71, 48},   {13, 28},   {17, 80},   {25, 102},  {183, 104},
    {55, 954},  {127, 96},  {27, 110},  {29, 112},  {29, 114},  {57, 116},  {45, 354},
    {31, 120},  {59, 610},  {185, 124}, {113, 420}, {31, 64},   {17, 66},   {171, 136},
    {209, 420}, {253, 216}, {367, 444}, {265, 456}, {181, 468}, {39, 80},   {27, 164},
    {127, 504}, {143, 172}, {43, 88},   {29, 300},  {45, 92},   {157, 188}, {47, 96},
    {13, 28},   {111, 240}, {443, 204}, {51, 104},  {51, 212},  {451, 192}, {257, 220},
    {57, 336},  {313, 228}, {271, 232}, {179, 236}, {331, 120}, {363, 244}, {375, 248},
    {127, 168}, {31, 64},   {33, 130},  {43, 264},  {33, 134},  {477, 408}, {35, 138},
    {233, 280}, {357, 142}, {337, 480}, {37, 146},  {71, 444},  {71, 120},  {37, 152},
    {39, 462},  {127, 234}, {39, 158},  {39, 80},   {31, 96},   {113, 902}, {41, 166},
    {251, 336}, {43, 170},  {21, 86},   {43, 174},  {45, 176},  {45, 178},  {161, 120},
    {89, 182},  {323, 184}, {47, 186},  {23, 94},   {47, 190},  {263, 480},
};

static int32_t qpp_k_of_index(int i) {
  if (i < 60) return 40 + 8 * i;             /* 40..512 step 8 */
  if (i < 92) return 528 + 16 * (i - 60);    /* 528..1024 step 16 */
  if (i < 124) return 1056 + 32 * (i - 92);  /* 1056..2048 step 32 */
  return 2112 + 64 * (i - 124);              /* 2112..6144 step 64 */
}

int or_qpp_count(void) { return 188; }

void or_qpp_entry(int index, int32_t* k, int32_t* f1, int32_t* f2) {
  *k = qpp_k_of_index(index);
  *f1 = kF1F2[index][0];
  *f2 = kF1F2[index][1];
}

int or_qpp_index(int32_t k) {
  for (int i = 0; i < 188; ++i)
    if (qpp_k_of_index(i) == k) return i;
  return -1;
}

/* lte_turbo.cpp:606-613: perm[i] = (f1*i + f2*i*i) mod K, evaluated in 64 bits. */
void or_qpp_perm(int32_t k, int32_t* perm) {
  const int idx = or_qpp_index(k);
  const uint64_t f1 = (uint64_t)kF1F2[idx][0], f2 = (uint64_t)kF1F2[idx][1];
  for (int32_t i = 0; i < k; ++i) {
    const uint64_t ii = (uint64_t)i;
    perm[i] = (int32_t)((f1 * ii + f2 * ii * ii) % (uint64_t)k);
  }
}

/* ------------------------------------------------------------------------------------------ */
/* CRC: bit-serial long division by the reference's generator arrays (lte_turbo.cpp:104-155). */
/* g[j] is the coefficient of D^(L-1-j); the leading D^L term is implicit.                     */
/* ------------------------------------------------------------------------------------------ */
static const uint8_t kG24A[24] = {1, 1, 0, 0, 0, 0, 0, 1, 1, 0, 0, 1,
                                  1, 0, 0, 1, 1, 0, 1, 1, 1, 1, 1, 1};
static const uint8_t kG24B[24] = {1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                                  0, 0, 0, 0, 0, 1, 1, 0, 0, 0, 1, 1};
static const uint8_t kG16[16] = {1, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 1};
static const uint8_t kG8[8] = {1, 1, 0, 1, 1, 0, 0, 1};

static const uint8_t* crc_poly(int kind, int* len) {
  switch (kind) {
    case 0: *len = 24; return kG24A;
    case 1: *len = 24; return kG24B;
    case 2: *len = 16; return kG16;
    default: *len = 8; return kG8;
  }
}

int or_crc_len(int kind) {
  int len;
  crc_poly(kind, &len);
  return len;
}

/* TS 36.212 5.1.1 generator polynomials, written the same way (no reference counterpart):
 * gCRC24A = D^24+D^23+D^18+D^17+D^14+D^11+D^10+D^7+D^6+D^5+D^4+D^3+D+1,
 * gCRC24B = D^24+D^23+D^6+D^5+D+1, gCRC16 = D^16+D^12+D^5+1, gCRC8 = D^8+D^7+D^4+D^3+D+1 */
static const uint8_t kS24A[24] = {1, 0, 0, 0, 0, 1, 1, 0, 0, 1, 0, 0,
                                  1, 1, 0, 0, 1, 1, 1, 1, 1, 0, 1, 1};
static const uint8_t kS24B[24] = {1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                                  0, 0, 0, 0, 0, 1, 1, 0, 0, 0, 1, 1};
static const uint8_t kS16[16] = {0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
static const uint8_t kS8[8] = {1, 0, 0, 1, 1, 0, 1, 1};

static const uint8_t* crc_poly_conv(int conv, int kind, int* len) {
  if (!conv) return crc_poly(kind, len);
  switch (kind) {
    case 0: *len = 24; return kS24A;
    case 1: *len = 24; return kS24B;
    case 2: *len = 16; return kS16;
    default: *len = 8; return kS8;
  }
}

static void crc_append_g(const uint8_t* g, int len, const uint8_t* bits, size_t n, uint8_t* out);
static int crc_check_g(const uint8_t* g, int len, const uint8_t* bits, size_t n);

void or_crc_append(int kind, const uint8_t* bits, size_t n, uint8_t* out) {
  int len;
  const uint8_t* g = crc_poly(kind, &len);
  crc_append_g(g, len, bits, n, out);
}

int or_crc_check(int kind, const uint8_t* bits, size_t n) {
  int len;
  const uint8_t* g = crc_poly(kind, &len);
  return crc_check_g(g, len, bits, n);
}

void or_std_crc_append(int kind, const uint8_t* bits, size_t n, uint8_t* out) {
  int len;
  const uint8_t* g = crc_poly_conv(1, kind, &len);
  crc_append_g(g, len, bits, n, out);
}

int or_std_crc_check(int kind, const uint8_t* bits, size_t n) {
  int len;
  const uint8_t* g = crc_poly_conv(1, kind, &len);
  return crc_check_g(g, len, bits, n);
}

/* lte_turbo.cpp:118-135 */
static void crc_append_g(const uint8_t* g, int len, const uint8_t* bits, size_t n, uint8_t* out) {
  uint8_t* work = (uint8_t*)calloc(n + (size_t)len, 1);
  memcpy(work, bits, n);
  for (size_t i = 0; i < n; ++i) {
    if (!(work[i] & 1u)) continue;
    work[i] = 0;
    for (int j = 0; j < len; ++j) work[i + 1 + (size_t)j] ^= g[j];
  }
  memmove(out, bits, n);
  memcpy(out + n, work + n, (size_t)len);
  free(work);
}

/* lte_turbo.cpp:137-155: divide all but the last L bits; remainder must be zero. */
static int crc_check_g(const uint8_t* g, int len, const uint8_t* bits, size_t n) {
  if (n < (size_t)len) return 0;
  uint8_t* work = (uint8_t*)malloc(n ? n : 1);
  memcpy(work, bits, n);
  for (size_t i = 0; i + (size_t)len < n; ++i) {
    if (!(work[i] & 1u)) continue;
    work[i] = 0;
    for (int j = 0; j < len; ++j) work[i + 1 + (size_t)j] ^= g[j];
  }
  int ok = 1;
  for (size_t i = n - (size_t)len; i < n; ++i) ok &= (work[i] == 0);
  free(work);
  return ok;
}

/* ------------------------------------------------------------------------------------------ */
/* Segmentation (lte_turbo.cpp:540-604)                                                       */
/* ------------------------------------------------------------------------------------------ */
static size_t ceil_div(size_t a, size_t b) { return (a + b - 1u) / b; }

int or_segment(const uint8_t* bits, size_t b, or_seg_info* info, uint8_t* cb_out) {
  if (b == 0) return -1;
  or_seg_info s;
  memset(&s, 0, sizeof s);
  size_t b_prime = b;
  if (b <= 6144) {
    s.l = 0;
    s.c = 1;
  } else {
    s.l = 24;
    s.c = ceil_div(b, 6144 - s.l);
    b_prime = b + s.c * s.l;
  }
  int up = -1;
  for (int i = 0; i < 188; ++i)
    if (s.c * (size_t)qpp_k_of_index(i) >= b_prime) {
      up = i;
      break;
    }
  if (up < 0) return -2;
  s.k_plus = (size_t)qpp_k_of_index(up);
  if (s.c == 1) {
    s.c_plus = 1;
  } else {
    if (up == 0) return -3;
    s.k_minus = (size_t)qpp_k_of_index(up - 1); /* largest table K below K+ */
    s.c_minus = (s.c * s.k_plus - b_prime) / (s.k_plus - s.k_minus);
    s.c_plus = s.c - s.c_minus;
  }
  s.filler = s.c_plus * s.k_plus + s.c_minus * s.k_minus - b_prime;
  if (cb_out) {
    size_t cursor = 0, out_pos = 0;
    for (size_t r = 0; r < s.c; ++r) {
      const size_t kr = (r < s.c_minus) ? s.k_minus : s.k_plus;
      uint8_t* blk = cb_out + out_pos;
      memset(blk, 0, kr);
      const size_t off = (r == 0) ? s.filler : 0;
      const size_t payload = kr - off - s.l;
      memcpy(blk + off, bits + cursor, payload);
      cursor += payload;
      if (s.l == 24) {
        uint8_t* tmp = (uint8_t*)malloc(payload + 24);
        or_crc_append(1, blk + off, payload, tmp);
        memcpy(blk + off + payload, tmp + payload, 24);
        free(tmp);
      }
      out_pos += kr;
    }
  }
  *info = s;
  return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* RSC constituent code (lte_turbo.cpp:333-353).  state = (s2 s1 s0).                          */
/* ------------------------------------------------------------------------------------------ */
static void rsc_step(uint8_t state, uint8_t u, uint8_t* parity, uint8_t* next) {
  const uint8_t s0 = state & 1u, s1 = (state >> 1) & 1u, s2 = (state >> 2) & 1u;
  const uint8_t fb = u ^ s1 ^ s2;
  *parity = fb ^ s0 ^ s2;
  *next = (uint8_t)((fb << 2) | (s2 << 1) | s1);
}

static void termination(uint8_t state, uint8_t in[3]) {
  for (int i = 0; i < 3; ++i) {
    const uint8_t u = ((state >> 1) & 1u) ^ ((state >> 2) & 1u);
    uint8_t p;
    in[i] = u;
    rsc_step(state, u, &p, &state);
  }
}

/* TS 36.212 5.1.3.2.1 (no reference counterpart): transfer function [1, g1(D)/g0(D)],
 * g0 = 1 + D^2 + D^3, g1 = 1 + D + D^3.  The register holds r1 (delay D), r2 (D^2), r3 (D^3);
 * state = r1 | r2 << 1 | r3 << 2, a labelling of this file's own. */
static void rsc_step_std(uint8_t state, uint8_t u, uint8_t* parity, uint8_t* next) {
  const uint8_t r1 = state & 1u, r2 = (state >> 1) & 1u, r3 = (state >> 2) & 1u;
  const uint8_t a = u ^ r2 ^ r3; /* register input: g0 taps D^2, D^3 fed back */
  *parity = a ^ r1 ^ r3;         /* g1 taps 1, D, D^3 */
  *next = (uint8_t)(a | (r1 << 1) | (r2 << 2));
}

/* 5.1.3.2.2: with the switch in the lower position the input is the feedback r2^r3, so the
 * register input is 0; the systematic tail bit is that input. */
static uint8_t term_input_std(uint8_t state) { return ((state >> 1) & 1u) ^ ((state >> 2) & 1u); }

void or_std_turbo_encode(int32_t k, int32_t filler, const uint8_t* cb, uint8_t* d0, uint8_t* d1,
                         uint8_t* d2) {
  int32_t* perm = (int32_t*)malloc(sizeof(int32_t) * (size_t)k);
  or_qpp_perm(k, perm);
  uint8_t su = 0, sl = 0, p, n;
  for (int32_t i = 0; i < k; ++i) { /* 5.1.3.2.1, filler bits as <NULL> in d0 and d1 */
    rsc_step_std(su, cb[i], &p, &n);
    su = n;
    d0[i] = (i < filler) ? 0 : cb[i];
    d1[i] = (i < filler) ? 0 : p;
    rsc_step_std(sl, cb[perm[i]], &p, &n);
    sl = n;
    d2[i] = p;
  }
  uint8_t x[3], z[3], xp[3], zp[3]; /* x_K+i, z_K+i, x'_K+i, z'_K+i */
  for (int i = 0; i < 3; ++i) {
    x[i] = term_input_std(su);
    rsc_step_std(su, x[i], &z[i], &su);
    xp[i] = term_input_std(sl);
    rsc_step_std(sl, xp[i], &zp[i], &sl);
  }
  /* 5.1.3.2.2: d0 = x_K z_K+1 x'_K z'_K+1, d1 = z_K x_K+2 z'_K x'_K+2,
   * d2 = x_K+1 z_K+2 x'_K+1 z'_K+2 */
  d0[k + 0] = x[0]; d0[k + 1] = z[1]; d0[k + 2] = xp[0]; d0[k + 3] = zp[1];
  d1[k + 0] = z[0]; d1[k + 1] = x[2]; d1[k + 2] = zp[0]; d1[k + 3] = xp[2];
  d2[k + 0] = x[1]; d2[k + 1] = z[2]; d2[k + 2] = xp[1]; d2[k + 3] = zp[2];
  free(perm);
}

/* lte_turbo.cpp:624-688 */
void or_turbo_encode(int32_t k, int32_t filler, const uint8_t* cb, uint8_t* d0, uint8_t* d1,
                     uint8_t* d2) {
  int32_t* perm = (int32_t*)malloc(sizeof(int32_t) * (size_t)k);
  or_qpp_perm(k, perm);
  uint8_t su = 0, sl = 0, p, n;
  for (int32_t i = 0; i < k; ++i) {
    rsc_step(su, cb[i], &p, &n);
    su = n;
    d0[i] = (i < filler) ? 0 : cb[i];
    d1[i] = (i < filler) ? 0 : p;
    rsc_step(sl, cb[perm[i]], &p, &n);
    sl = n;
    d2[i] = p;
  }
  uint8_t ui[3], li[3], us[3], up[3], ls[3], lp[3];
  termination(su, ui);
  termination(sl, li);
  for (int i = 0; i < 3; ++i) {
    us[i] = ui[i];
    rsc_step(su, ui[i], &up[i], &su);
    ls[i] = li[i];
    rsc_step(sl, li[i], &lp[i], &sl);
  }
  /* tail multiplexing exactly as lte_turbo.cpp:664-677 */
  d0[k + 0] = us[0]; d0[k + 1] = up[1]; d0[k + 2] = us[1]; d0[k + 3] = up[2];
  d1[k + 0] = up[0]; d1[k + 1] = us[1]; d1[k + 2] = up[2]; d1[k + 3] = ls[0];
  d2[k + 0] = lp[0]; d2[k + 1] = ls[1]; d2[k + 2] = lp[1]; d2[k + 3] = ls[2];
  free(perm);
}

/* ------------------------------------------------------------------------------------------ */
/* Rate matching (lte_turbo.cpp:167-325)                                                      */
/* ------------------------------------------------------------------------------------------ */
static const uint8_t kColPerm[32] = {0, 16, 8, 24, 4, 20, 12, 28, 2, 18, 10, 26, 6, 22, 14, 30,
                                     1, 17, 9, 25, 5, 21, 13, 29, 3, 19, 11, 27, 7, 23, 15, 31};

/* lte_turbo.cpp:167-185 */
int64_t or_compute_e(size_t r, size_t g_total, size_t c, size_t num_layers, size_t mod_order) {
  if (c == 0 || num_layers == 0 || mod_order == 0) return -1;
  const size_t nlqm = num_layers * mod_order;
  if (g_total % nlqm) return -1;
  const size_t gp = g_total / nlqm;
  const size_t gamma = gp % c;
  return (int64_t)((r + gamma + 1 <= c) ? nlqm * (gp / c) : nlqm * ceil_div(gp, c));
}

typedef struct {
  int32_t d, rows, kpi, ncb;
  int32_t* map[3]; /* source index into the stream, -1 for <NULL> */
} layout_t;

/* lte_turbo.cpp:195-248 */
static void layout_build(layout_t* L, int32_t d, int32_t filler) {
  L->d = d;
  L->rows = (int32_t)ceil_div((size_t)d, 32);
  L->kpi = L->rows * 32;
  L->ncb = 3 * L->kpi;
  const int32_t dummy = L->kpi - d;
  int32_t* y = (int32_t*)malloc(sizeof(int32_t) * (size_t)L->kpi);
  for (int s = 0; s < 3; ++s) L->map[s] = (int32_t*)malloc(sizeof(int32_t) * (size_t)L->kpi);
  /* d0/d1: rows of 32, columns permuted, read column by column; filler -> NULL */
  for (int32_t i = 0; i < L->kpi; ++i) y[i] = -1;
  for (int32_t i = 0; i < d; ++i) y[dummy + i] = (i < filler) ? -1 : i;
  int32_t pos = 0;
  for (int c = 0; c < 32; ++c)
    for (int32_t r = 0; r < L->rows; ++r) {
      const int32_t v = y[r * 32 + kColPerm[c]];
      L->map[0][pos] = v;
      L->map[1][pos] = v;
      ++pos;
    }
  /* d2: pi(k) = (P[k/R] + 32*(k%R) + 1) mod K_pi, no filler nulling */
  for (int32_t i = 0; i < L->kpi; ++i) y[i] = -1;
  for (int32_t i = 0; i < d; ++i) y[dummy + i] = i;
  for (int32_t k = 0; k < L->kpi; ++k) {
    const int32_t idx = kColPerm[k / L->rows] + 32 * (k % L->rows) + 1;
    L->map[2][k] = y[idx % L->kpi];
  }
  free(y);
}

static void layout_free(layout_t* L) {
  for (int s = 0; s < 3; ++s) free(L->map[s]);
}

/* circular-buffer position -> (stream, source index); -1 when <NULL> (lte_turbo.cpp:255-262) */
static int32_t circ_src(const layout_t* L, int32_t idx, int* stream) {
  if (idx < L->kpi) {
    *stream = 0;
    return L->map[0][idx];
  }
  const int32_t local = idx - L->kpi;
  *stream = (local & 1) ? 2 : 1;
  return L->map[*stream][local >> 1];
}

static int32_t k0_of(const layout_t* L, int32_t rv) {
  return L->rows * (2 * (int32_t)ceil_div((size_t)L->ncb, 8 * (size_t)L->rows) * rv + 2);
}

/* lte_turbo.cpp:250-278 */
void or_rate_match(int32_t d, int32_t filler, const uint8_t* d0, const uint8_t* d1,
                   const uint8_t* d2, size_t e, int32_t rv, uint8_t* out) {
  layout_t L;
  layout_build(&L, d, filler);
  const uint8_t* st[3] = {d0, d1, d2};
  const int32_t k0 = k0_of(&L, rv);
  size_t k = 0;
  int64_t j = 0;
  while (k < e) {
    int s;
    const int32_t src = circ_src(&L, (int32_t)((k0 + j) % L.ncb), &s);
    if (src >= 0) out[k++] = st[s][src];
    ++j;
  }
  layout_free(&L);
}

/* lte_turbo.cpp:280-325 (values: +-8 per bit) generalised over a value array */
static void derate_core(int32_t d, int32_t filler, const uint8_t* bits, const float* llr,
                        size_t e, int32_t rv, float* out) {
  layout_t L;
  layout_build(&L, d, filler);
  float* circ = (float*)calloc((size_t)L.ncb, sizeof(float));
  uint8_t* valid = (uint8_t*)calloc((size_t)L.ncb, 1);
  const int32_t k0 = k0_of(&L, rv);
  size_t k = 0;
  int64_t j = 0;
  while (k < e) {
    const int32_t idx = (int32_t)((k0 + j) % L.ncb);
    int s;
    if (circ_src(&L, idx, &s) >= 0) {
      circ[idx] += bits ? (bits[k] ? 8.0f : -8.0f) : llr[k];
      valid[idx] = 1;
      ++k;
    }
    ++j;
  }
  memset(out, 0, sizeof(float) * 3u * (size_t)d);
  for (int32_t i = 0; i < L.kpi; ++i) {
    if (L.map[0][i] >= 0 && valid[i]) out[L.map[0][i]] += circ[i];
    if (L.map[1][i] >= 0 && valid[L.kpi + 2 * i]) out[d + L.map[1][i]] += circ[L.kpi + 2 * i];
    if (L.map[2][i] >= 0 && valid[L.kpi + 2 * i + 1])
      out[2 * d + L.map[2][i]] += circ[L.kpi + 2 * i + 1];
  }
  free(circ);
  free(valid);
  layout_free(&L);
}

void or_derate_bits(int32_t d, int32_t filler, const uint8_t* e_bits, size_t e, int32_t rv,
                    float* out) {
  derate_core(d, filler, e_bits, NULL, e, rv, out);
}

void or_derate_llr(int32_t d, int32_t filler, const float* e_llr, size_t e, int32_t rv,
                   float* out) {
  derate_core(d, filler, NULL, e_llr, e, rv, out);
}

/* ------------------------------------------------------------------------------------------ */
/* Exact Log-MAP (lte_turbo.cpp:357-486)                                                       */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
  uint8_t parity[8][2], next[8][2];
  uint8_t term[8]; /* the input that zeroes the register input (trellis termination) */
  int std;         /* 1: the TS 36.212 code (tail mapping and CRC too) */
} trellis_t;

static trellis_t make_trellis_conv(int std) {
  trellis_t t;
  t.std = std;
  for (int s = 0; s < 8; ++s) {
    for (int u = 0; u < 2; ++u) {
      if (std) rsc_step_std((uint8_t)s, (uint8_t)u, &t.parity[s][u], &t.next[s][u]);
      else rsc_step((uint8_t)s, (uint8_t)u, &t.parity[s][u], &t.next[s][u]);
    }
    uint8_t in[3];
    termination((uint8_t)s, in);
    t.term[s] = std ? term_input_std((uint8_t)s) : in[0];
  }
  return t;
}

static trellis_t make_trellis(void) { return make_trellis_conv(0); }

/* lte_turbo.cpp:380-390 */
static float max_star(float x, float y) {
  if (!isfinite(x)) return y;
  if (!isfinite(y)) return x;
  const float hi = x > y ? x : y;
  const float lo = x > y ? y : x;
  return hi + log1pf(expf(lo - hi));
}

/* lte_turbo.cpp:392-402 */
static void normalize8(float* m) {
  float mx = m[0];
  for (int s = 1; s < 8; ++s)
    if (m[s] > mx) mx = m[s];
  if (!isfinite(mx)) return;
  for (int s = 0; s < 8; ++s)
    if (isfinite(m[s])) m[s] -= mx;
}

/* lte_turbo.cpp:357-378 */
static void tail_beta(const trellis_t* T, const float ts[4], const float tp[4], float beta[8]) {
  for (int s = 0; s < 8; ++s) {
    uint8_t cur = (uint8_t)s;
    float metric = 0.0f;
    for (int i = 0; i < 3; ++i) {
      const uint8_t in = T->term[cur], p = T->parity[cur][in];
      cur = T->next[cur][in];
      const float sys_term = 0.5f * ((in ? 1.0f : -1.0f) * ts[i]);
      const float par_term = 0.5f * ((p ? 1.0f : -1.0f) * tp[i]);
      metric += sys_term + par_term;
    }
    beta[s] = (cur == 0) ? metric : -INFINITY;
  }
  normalize8(beta);
}

static inline float branch(const trellis_t* T, int s, int u, float sa, float par) {
  /* lte_turbo.cpp:437-438: 0.5 * (+-(sys+apr) +- parity) */
  return 0.5f * ((u ? 1.0f : -1.0f) * sa + (T->parity[s][u] ? 1.0f : -1.0f) * par);
}

/*
 * One SISO over the output segment [lo, hi) of the trellis.  The forward recursion starts at
 * a_lo <= lo from the metric a_in and the backward recursion at b_hi >= hi from b_in (the
 * steps outside [lo, hi) are warm-up steps).  alpha/beta scratch hold (b_hi-a_lo+1)*8 floats.
 * Writes the extrinsic for lo..hi-1; returns the alpha at position a_rec and the beta at
 * position b_rec (the metrics the neighbouring windows take as next-iteration seeds).
 * With a_lo=lo=0, hi=b_hi=K, a_in = state 0 and b_in = tail metrics this is
 * decode_siso_log_map (lte_turbo.cpp:410-486) step for step.
 */
static void siso_segment(const trellis_t* T, const float* sys, const float* par, const float* apr,
                         int32_t a_lo, int32_t lo, int32_t hi, int32_t b_hi, const float a_in[8],
                         const float b_in[8], float* alpha, float* beta, float* ext,
                         int32_t a_rec, float a_out[8], int32_t b_rec, float b_out[8]) {
  const int32_t n = b_hi - a_lo; /* scratch rows are positions a_lo..b_hi */
  for (int32_t i = 0; i <= n; ++i)
    for (int s = 0; s < 8; ++s) {
      alpha[8 * i + s] = -INFINITY;
      beta[8 * i + s] = -INFINITY;
    }
  memcpy(alpha, a_in, 8 * sizeof(float));
  memcpy(beta + 8 * n, b_in, 8 * sizeof(float));

  for (int32_t p = a_lo; p < hi; ++p) { /* lte_turbo.cpp:430-446 */
    const int32_t i = p - a_lo;
    const float sa = sys[p] + apr[p];
    const float* a = alpha + 8 * i;
    float* an = alpha + 8 * (i + 1);
    for (int s = 0; s < 8; ++s) {
      if (!isfinite(a[s])) continue;
      for (int u = 0; u < 2; ++u) {
        const int nx = T->next[s][u];
        const float v = a[s] + branch(T, s, u, sa, par[p]);
        an[nx] = isfinite(an[nx]) ? max_star(an[nx], v) : v;
      }
    }
    normalize8(an);
  }
  for (int32_t p = b_hi; p-- > lo;) { /* lte_turbo.cpp:448-464 */
    const int32_t i = p - a_lo;
    const float sa = sys[p] + apr[p];
    const float* bn = beta + 8 * (i + 1);
    float* b = beta + 8 * i;
    for (int s = 0; s < 8; ++s)
      for (int u = 0; u < 2; ++u) {
        const int nx = T->next[s][u];
        if (!isfinite(bn[nx])) continue;
        const float v = bn[nx] + branch(T, s, u, sa, par[p]);
        b[s] = isfinite(b[s]) ? max_star(b[s], v) : v;
      }
    normalize8(b);
  }
  for (int32_t p = lo; p < hi; ++p) { /* lte_turbo.cpp:466-485 */
    const int32_t i = p - a_lo;
    const float sa = sys[p] + apr[p];
    float l0 = -INFINITY, l1 = -INFINITY;
    for (int s = 0; s < 8; ++s)
      for (int u = 0; u < 2; ++u) {
        const float m = alpha[8 * i + s] + branch(T, s, u, sa, par[p]) +
                        beta[8 * (i + 1) + T->next[s][u]];
        if (u == 0)
          l0 = isfinite(l0) ? max_star(l0, m) : m;
        else
          l1 = isfinite(l1) ? max_star(l1, m) : m;
      }
    ext[p] = (l1 - l0) - sys[p] - apr[p];
  }
  if (a_out) memcpy(a_out, alpha + 8 * (a_rec - a_lo), 8 * sizeof(float));
  if (b_out) memcpy(b_out, beta + 8 * (b_rec - a_lo), 8 * sizeof(float));
}

/* Tail LLRs as gathered by lte_turbo.cpp:758-773 (the lower mapping is the reference's own). */
static void gather_tails(int32_t k, const float* d0, const float* d1, const float* d2,
                         float uts[4], float utp[4], float lts[4], float ltp[4]) {
  uts[0] = d0[k + 0]; uts[1] = d0[k + 2]; uts[2] = 0.0f; uts[3] = 0.0f;
  utp[0] = d1[k + 0]; utp[1] = d0[k + 1]; utp[2] = d1[k + 2]; utp[3] = 0.0f;
  lts[0] = d1[k + 3]; lts[1] = d2[k + 0]; lts[2] = d2[k + 2]; lts[3] = 0.0f;
  ltp[0] = d2[k + 1]; ltp[1] = d0[k + 3]; ltp[2] = d2[k + 3]; ltp[3] = 0.0f;
}

/* The tail LLRs of the TS 36.212 multiplexing (5.1.3.2.2; no reference counterpart):
 * upper systematic x_K..x_K+2 = d0[K], d2[K], d1[K+1], parity z_K..z_K+2 = d1[K], d0[K+1],
 * d2[K+1]; lower x'_K.. = d0[K+2], d2[K+2], d1[K+3], z'_K.. = d1[K+2], d0[K+3], d2[K+3]. */
static void gather_tails_std(int32_t k, const float* d0, const float* d1, const float* d2,
                             float uts[4], float utp[4], float lts[4], float ltp[4]) {
  uts[0] = d0[k + 0]; uts[1] = d2[k + 0]; uts[2] = d1[k + 1]; uts[3] = 0.0f;
  utp[0] = d1[k + 0]; utp[1] = d0[k + 1]; utp[2] = d2[k + 1]; utp[3] = 0.0f;
  lts[0] = d0[k + 2]; lts[1] = d2[k + 2]; lts[2] = d1[k + 3]; lts[3] = 0.0f;
  ltp[0] = d1[k + 2]; ltp[1] = d0[k + 3]; ltp[2] = d2[k + 3]; ltp[3] = 0.0f;
}

/* hard decision >= 0 -> 1, zero the filler, CRC24B over the rest (lte_turbo.cpp:488-494,
 * 792-797) */
static int early_stop_crc(const float* post, int32_t k, int32_t filler, uint8_t* hard, int std) {
  for (int32_t i = 0; i < k; ++i) hard[i] = post[i] >= 0.0f ? 1u : 0u;
  for (int32_t i = 0; i < filler; ++i) hard[i] = 0;
  return std ? or_std_crc_check(1, hard + filler, (size_t)(k - filler))
             : or_crc_check(1, hard + filler, (size_t)(k - filler));
}

/*
 * Shared driver for the full-trellis and the windowed schedules (lte_turbo.cpp:736-813).
 * window <= 0 or >= K: one segment, i.e. the reference decoder exactly.
 * Otherwise window w covers [w*W, min((w+1)*W, K)).  Its forward recursion starts `guard`
 * steps early, at lo-guard, and its backward recursion `guard` steps late, at hi+guard; a
 * start that reaches the block edge uses the true edge metric (state 0 / tail), any other
 * start uses the metric the neighbouring window produced at that position in the previous
 * iteration (all zero in the first iteration).
 */
static void decode_common(int32_t k, int32_t filler, const float* llr, int32_t max_iterations,
                          int32_t early_stop, int32_t window, int32_t guard, float* posterior,
                          int32_t* crc_ok, int32_t* iterations_used, int std) {
  const trellis_t T = make_trellis_conv(std);
  const float* d0 = llr;
  const float* d1 = llr + (k + 4);
  const float* d2 = llr + 2 * (k + 4);
  if (window <= 0 || window > k) window = k;
  if (guard < 0) guard = 0;
  if (guard > window) guard = window;
  const int32_t nw = (k + window - 1) / window;

  int32_t* perm = (int32_t*)malloc(sizeof(int32_t) * (size_t)k);
  or_qpp_perm(k, perm);
  float* apr = (float*)calloc((size_t)k, sizeof(float));
  float* e1 = (float*)calloc((size_t)k, sizeof(float));
  float* e2 = (float*)calloc((size_t)k, sizeof(float));
  float* sys_i = (float*)malloc(sizeof(float) * (size_t)k);
  float* apr_i = (float*)malloc(sizeof(float) * (size_t)k);
  float* e2_i = (float*)malloc(sizeof(float) * (size_t)k);
  const size_t rows = (size_t)(window + 2 * guard + 1);
  float* alpha = (float*)malloc(sizeof(float) * 8u * rows);
  float* beta = (float*)malloc(sizeof(float) * 8u * rows);
  uint8_t* hard = (uint8_t*)malloc((size_t)k);
  /* seeds: [siso][window][8]; alpha seed of window w, beta seed of window w */
  float* aseed = (float*)calloc(2u * (size_t)nw * 8u, sizeof(float));
  float* bseed = (float*)calloc(2u * (size_t)nw * 8u, sizeof(float));
  float* arec = (float*)malloc(sizeof(float) * 8u * (size_t)nw);
  float* brec = (float*)malloc(sizeof(float) * 8u * (size_t)nw);
  for (int32_t i = 0; i < k; ++i) sys_i[i] = d0[perm[i]];

  float tails[4][4];
  if (std) gather_tails_std(k, d0, d1, d2, tails[0], tails[1], tails[2], tails[3]);
  else gather_tails(k, d0, d1, d2, tails[0], tails[1], tails[2], tails[3]);
  float tb[2][8];
  tail_beta(&T, tails[0], tails[1], tb[0]);
  tail_beta(&T, tails[2], tails[3], tb[1]);
  float a_start[8];
  for (int s = 0; s < 8; ++s) a_start[s] = s == 0 ? 0.0f : -INFINITY;

  int ok = 0;
  memset(posterior, 0, sizeof(float) * (size_t)k);
  for (int32_t it = 0; it < max_iterations; ++it) {
    for (int pass = 0; pass < 2; ++pass) {
      const float* sys = pass ? sys_i : d0;
      const float* par = pass ? d2 : d1;
      const float* ap = pass ? apr_i : apr;
      float* ex = pass ? e2_i : e1;
      if (pass == 1)
        for (int32_t i = 0; i < k; ++i) apr_i[i] = e1[perm[i]]; /* lte_turbo.cpp:780-783 */
      float* as = aseed + (size_t)pass * nw * 8;
      float* bs = bseed + (size_t)pass * nw * 8;
      for (int32_t w = 0; w < nw; ++w) {
        const int32_t lo = w * window, hi = (lo + window < k) ? lo + window : k;
        int32_t a_lo = lo - guard, b_hi = hi + guard;
        const float* ain = as + 8 * w;
        const float* bin = bs + 8 * w;
        if (a_lo <= 0) { a_lo = 0; ain = a_start; }
        if (b_hi >= k) { b_hi = k; bin = tb[pass]; }
        const int32_t a_rec = hi - guard;                       /* seed of window w+1 */
        const int32_t b_rec = (lo + guard < b_hi) ? lo + guard : b_hi; /* seed of w-1 */
        siso_segment(&T, sys, par, ap, a_lo, lo, hi, b_hi, ain, bin, alpha, beta, ex, a_rec,
                     arec + 8 * w, b_rec, brec + 8 * w);
      }
      /* next-iteration initialisation: seeds for the following iteration */
      for (int32_t w = 0; w + 1 < nw; ++w) {
        memcpy(as + 8 * (w + 1), arec + 8 * w, 8 * sizeof(float));
        memcpy(bs + 8 * w, brec + 8 * (w + 1), 8 * sizeof(float));
      }
    }
    for (int32_t i = 0; i < k; ++i) e2[perm[i]] = e2_i[i]; /* = e2_i[inv_perm[j]] */
    for (int32_t i = 0; i < k; ++i) {
      apr[i] = e2[i];
      posterior[i] = d0[i] + e1[i] + e2[i];
    }
    if (iterations_used) *iterations_used = it + 1;
    if (early_stop) {
      ok = early_stop_crc(posterior, k, filler, hard, std);
      if (ok) break;
    }
  }
  if (crc_ok) *crc_ok = ok;
  free(perm); free(apr); free(e1); free(e2); free(sys_i); free(apr_i); free(e2_i);
  free(alpha); free(beta); free(hard); free(aseed); free(bseed); free(arec); free(brec);
}

void or_decode_cb(int32_t k, int32_t filler, const float* llr, int32_t max_iterations,
                  int32_t early_stop, float* posterior, int32_t* crc_ok,
                  int32_t* iterations_used) {
  if (iterations_used) *iterations_used = 0;
  decode_common(k, filler, llr, max_iterations, early_stop, 0, 0, posterior, crc_ok,
                iterations_used, 0);
}

void or_decode_cb_windowed(int32_t k, int32_t filler, const float* llr, int32_t max_iterations,
                           int32_t early_stop, int32_t window, int32_t guard, float* posterior,
                           int32_t* crc_ok, int32_t* iterations_used) {
  if (iterations_used) *iterations_used = 0;
  decode_common(k, filler, llr, max_iterations, early_stop, window, guard, posterior, crc_ok,
                iterations_used, 0);
}

/* The same schedule on the TS 36.212 code (trellis, tail mapping, CRC24B of the early stop). */
void or_std_decode_cb_windowed(int32_t k, int32_t filler, const float* llr,
                               int32_t max_iterations, int32_t early_stop, int32_t window,
                               int32_t guard, float* posterior, int32_t* crc_ok,
                               int32_t* iterations_used) {
  if (iterations_used) *iterations_used = 0;
  decode_common(k, filler, llr, max_iterations, early_stop, window, guard, posterior, crc_ok,
                iterations_used, 1);
}

/* ------------------------------------------------------------------------------------------ */
/* Thread pool over code blocks                                                                */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
  int32_t n;
  const int32_t *k, *filler;
  const int64_t *llr_off, *out_off;
  const float* llr;
  float* post;
  int32_t iters, early, window, guard;
  int32_t *crc, *used;
  int32_t next; /* shared work index */
  pthread_mutex_t mu;
} batch_t;

static void* batch_worker(void* p) {
  batch_t* b = (batch_t*)p;
  for (;;) {
    pthread_mutex_lock(&b->mu);
    const int32_t i = b->next++;
    pthread_mutex_unlock(&b->mu);
    if (i >= b->n) break;
    int32_t c = 0, u = 0;
    decode_common(b->k[i], b->filler[i], b->llr + b->llr_off[i], b->iters, b->early, b->window,
                  b->guard, b->post + b->out_off[i], &c, &u, 0);
    if (b->crc) b->crc[i] = c;
    if (b->used) b->used[i] = u;
  }
  return NULL;
}

static void run_batch(batch_t* b, int32_t threads) {
  if (threads <= 0) threads = (int32_t)sysconf(_SC_NPROCESSORS_ONLN);
  if (threads < 1) threads = 1;
  if (threads > b->n) threads = b->n > 0 ? b->n : 1;
  pthread_mutex_init(&b->mu, NULL);
  b->next = 0;
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)threads);
  for (int32_t t = 0; t < threads; ++t) pthread_create(&th[t], NULL, batch_worker, b);
  for (int32_t t = 0; t < threads; ++t) pthread_join(th[t], NULL);
  free(th);
  pthread_mutex_destroy(&b->mu);
}

void or_decode_batch(int32_t n, const int32_t* k, const int32_t* filler, const int64_t* llr_off,
                     const float* llr, const int64_t* out_off, float* posterior,
                     int32_t max_iterations, int32_t early_stop, int32_t* crc_ok,
                     int32_t* iterations_used, int32_t threads) {
  batch_t b = {n, k, filler, llr_off, out_off, llr, posterior, max_iterations, early_stop, 0,
               0, crc_ok, iterations_used, 0};
  run_batch(&b, threads);
}

void or_decode_batch_windowed(int32_t n, const int32_t* k, const int32_t* filler,
                              const int64_t* llr_off, const float* llr, const int64_t* out_off,
                              float* posterior, int32_t max_iterations, int32_t early_stop,
                              int32_t window, int32_t guard, int32_t* crc_ok,
                              int32_t* iterations_used, int32_t threads) {
  batch_t b = {n, k, filler, llr_off, out_off, llr, posterior, max_iterations, early_stop,
               window, guard, crc_ok, iterations_used, 0};
  run_batch(&b, threads);
}

/* ------------------------------------------------------------------------------------------ */
/* FP64 differentiable decoder and its hand-written adjoint                                    */
/* ------------------------------------------------------------------------------------------ */
/*
 * The differentiated function: the windowed schedule of decode_common (window W, guard G,
 * next-iteration-initialisation seeds) in natural-log FP64, no early stop, the extrinsic of SISO
 * j (j = 2*it upper, 2*it+1 lower) multiplied by scales[j] before it becomes the other SISO's
 * a-priori and enters the posterior Ls + e1 + e2.  The seeds are constants of the function (the
 * gradient stops at them); with W >= K there are none and this is the reference's full-trellis
 * decoder (turbo_decode_code_block_cpu, lte_turbo.cpp:736-813) with the scales inserted.
 * Per-step normalisations subtract a common value from all 8 metrics; every extrinsic is a
 * difference of two log-sums over the same metrics, so they are constants of the function too.
 */
static double lse2(double x, double y) {
  if (x == -INFINITY) return y;
  if (y == -INFINITY) return x;
  const double m = x > y ? x : y;
  return m + log1p(exp(-fabs(x - y)));
}

/* branch metric (u ? a : -a) + (p ? b : -b), a = (Ls+La)/2, b = Lp/2 (lte_turbo.cpp:437-438) */
static inline double gam(const trellis_t* T, int s, int u, double a, double b) {
  return (u ? a : -a) + (T->parity[s][u] ? b : -b);
}

/* beta at the block end from the three termination steps (lte_turbo.cpp:357-378), and its
 * derivatives w.r.t. the tail systematic (ts) and parity (tp) LLRs */
static void tail_beta64(const trellis_t* T, const double ts[3], const double tp[3], double beta[8],
                        double dts[8][3], double dtp[8][3]) {
  for (int s = 0; s < 8; ++s) {
    uint8_t cur = (uint8_t)s;
    double m = 0.0;
    for (int i = 0; i < 3; ++i) {
      const uint8_t in = T->term[cur], p = T->parity[cur][in];
      cur = T->next[cur][in];
      dts[s][i] = in ? 0.5 : -0.5;
      dtp[s][i] = p ? 0.5 : -0.5;
      m += dts[s][i] * ts[i] + dtp[s][i] * tp[i];
    }
    beta[s] = m;
  }
}

/* one window: alpha over positions [a_lo, hi] from a_in (NULL: the start state), beta over
 * [lo, b_hi] from b_in (NULL: the tail metric), extrinsic over [lo, hi) */
typedef struct {
  int32_t a_lo, lo, hi, b_hi;
  int start, tail; /* edge metric used instead of a seed */
} seg64_t;

static seg64_t seg64(int32_t k, int32_t W, int32_t G, int32_t w) {
  seg64_t g;
  g.lo = w * W;
  g.hi = g.lo + W < k ? g.lo + W : k;
  g.a_lo = g.lo - G;
  g.b_hi = g.hi + G;
  g.start = g.a_lo <= 0;
  g.tail = g.b_hi >= k;
  if (g.start) g.a_lo = 0;
  if (g.tail) g.b_hi = k;
  return g;
}

static void seg64_forward(const trellis_t* T, const double* sys, const double* par,
                          const double* apr, seg64_t g, const double* a_in, const double* b_in,
                          const double ts[3], const double tp[3], double* alpha, double* beta,
                          double* ext) {
  for (int s = 0; s < 8; ++s) alpha[s] = a_in ? a_in[s] : (s == 0 ? 0.0 : -INFINITY);
  for (int32_t p = g.a_lo; p < g.hi; ++p) {
    const double a = 0.5 * (sys[p] + apr[p]), b = 0.5 * par[p];
    const double* at = alpha + 8 * (p - g.a_lo);
    double* an = alpha + 8 * (p + 1 - g.a_lo);
    for (int s = 0; s < 8; ++s) an[s] = -INFINITY;
    for (int s = 0; s < 8; ++s)
      for (int u = 0; u < 2; ++u) {
        const int n = T->next[s][u];
        an[n] = lse2(an[n], at[s] + gam(T, s, u, a, b));
      }
    const double c = an[0];
    for (int s = 0; s < 8; ++s) an[s] -= c;
  }
  double* bk = beta + 8 * (g.b_hi - g.lo);
  if (b_in) {
    for (int s = 0; s < 8; ++s) bk[s] = b_in[s];
  } else {
    double dts[8][3], dtp[8][3];
    tail_beta64(T, ts, tp, bk, dts, dtp);
  }
  for (int32_t p = g.b_hi; p-- > g.lo;) {
    const double a = 0.5 * (sys[p] + apr[p]), b = 0.5 * par[p];
    const double* bn = beta + 8 * (p + 1 - g.lo);
    double* bt = beta + 8 * (p - g.lo);
    for (int s = 0; s < 8; ++s) {
      bt[s] = -INFINITY;
      for (int u = 0; u < 2; ++u) bt[s] = lse2(bt[s], bn[T->next[s][u]] + gam(T, s, u, a, b));
    }
    const double c = bt[0];
    for (int s = 0; s < 8; ++s) bt[s] -= c;
  }
  for (int32_t p = g.lo; p < g.hi; ++p) {
    const double b = 0.5 * par[p];
    const double* at = alpha + 8 * (p - g.a_lo);
    const double* bn = beta + 8 * (p + 1 - g.lo);
    double l[2] = {-INFINITY, -INFINITY};
    for (int s = 0; s < 8; ++s)
      for (int u = 0; u < 2; ++u)
        l[u] = lse2(l[u], at[s] + bn[T->next[s][u]] + (T->parity[s][u] ? b : -b));
    ext[p] = l[1] - l[0];
  }
}

/* Adjoint of seg64_forward: g_ext over [lo, hi) in, accumulates d/d(Ls+La) and d/d(Lp) over
 * [a_lo, b_hi) and, when the tail metric was used, d/d ts and d/d tp.  Reverse mode through
 * the softmax weights of every log-sum; alpha/beta as seg64_forward left them. */
static void seg64_adjoint(const trellis_t* T, const double* sys, const double* par,
                          const double* apr, seg64_t g, const double ts[3], const double tp[3],
                          const double* alpha, const double* beta, const double* g_ext,
                          double* g_sa, double* g_par, double g_ts[3], double g_tp[3]) {
  const int32_t na = g.hi - g.a_lo + 1, nb = g.b_hi - g.lo + 1;
  double* ab = (double*)calloc(8u * (size_t)na, sizeof(double));
  double* bb = (double*)calloc(8u * (size_t)nb, sizeof(double));
  for (int32_t p = g.lo; p < g.hi; ++p) { /* extrinsic = LSE1 - LSE0 */
    const double b = 0.5 * par[p];
    const double* at = alpha + 8 * (p - g.a_lo);
    const double* bn = beta + 8 * (p + 1 - g.lo);
    double m[8][2], l[2] = {-INFINITY, -INFINITY};
    for (int s = 0; s < 8; ++s)
      for (int u = 0; u < 2; ++u) {
        m[s][u] = at[s] + bn[T->next[s][u]] + (T->parity[s][u] ? b : -b);
        l[u] = lse2(l[u], m[s][u]);
      }
    for (int s = 0; s < 8; ++s)
      for (int u = 0; u < 2; ++u) {
        if (m[s][u] == -INFINITY) continue;
        const double v = exp(m[s][u] - l[u]) * (u ? 1.0 : -1.0) * g_ext[p];
        ab[8 * (p - g.a_lo) + s] += v;
        bb[8 * (p + 1 - g.lo) + T->next[s][u]] += v;
        g_par[p] += 0.5 * v * (T->parity[s][u] ? 1.0 : -1.0);
      }
  }
  for (int32_t p = g.lo; p < g.b_hi; ++p) { /* beta_p = LSE_u(beta_{p+1}[n] + gamma), forward */
    const double a = 0.5 * (sys[p] + apr[p]), b = 0.5 * par[p];
    const double* bn = beta + 8 * (p + 1 - g.lo);
    for (int s = 0; s < 8; ++s) {
      const double gs = bb[8 * (p - g.lo) + s];
      if (gs == 0.0) continue;
      double v[2], l = -INFINITY;
      for (int u = 0; u < 2; ++u) {
        v[u] = bn[T->next[s][u]] + gam(T, s, u, a, b);
        l = lse2(l, v[u]);
      }
      for (int u = 0; u < 2; ++u) {
        const double q = exp(v[u] - l) * gs;
        bb[8 * (p + 1 - g.lo) + T->next[s][u]] += q;
        g_sa[p] += 0.5 * q * (u ? 1.0 : -1.0);
        g_par[p] += 0.5 * q * (T->parity[s][u] ? 1.0 : -1.0);
      }
    }
  }
  for (int32_t p = g.hi; p-- > g.a_lo;) { /* alpha_{p+1}[n] = LSE over (s,u)->n, backward */
    const double a = 0.5 * (sys[p] + apr[p]), b = 0.5 * par[p];
    const double* at = alpha + 8 * (p - g.a_lo);
    double l[8];
    for (int n = 0; n < 8; ++n) l[n] = -INFINITY;
    for (int s = 0; s < 8; ++s)
      for (int u = 0; u < 2; ++u)
        l[T->next[s][u]] = lse2(l[T->next[s][u]], at[s] + gam(T, s, u, a, b));
    for (int s = 0; s < 8; ++s)
      for (int u = 0; u < 2; ++u) {
        const int n = T->next[s][u];
        const double gn = ab[8 * (p + 1 - g.a_lo) + n];
        if (gn == 0.0 || at[s] == -INFINITY) continue;
        const double v = exp(at[s] + gam(T, s, u, a, b) - l[n]) * gn;
        ab[8 * (p - g.a_lo) + s] += v;
        g_sa[p] += 0.5 * v * (u ? 1.0 : -1.0);
        g_par[p] += 0.5 * v * (T->parity[s][u] ? 1.0 : -1.0);
      }
  }
  if (g.tail) {
    double bk[8], dts[8][3], dtp[8][3];
    tail_beta64(T, ts, tp, bk, dts, dtp);
    for (int s = 0; s < 8; ++s)
      for (int i = 0; i < 3; ++i) {
        g_ts[i] += bb[8 * (nb - 1) + s] * dts[s][i];
        g_tp[i] += bb[8 * (nb - 1) + s] * dtp[s][i];
      }
  }
  free(ab);
  free(bb);
}

static int32_t adj_window(int32_t k, int32_t window) {
  return (window <= 0 || window > k) ? k : window;
}

int64_t or_adj_seed_count(int32_t k, int32_t iters, int32_t window) {
  const int32_t W = adj_window(k, window);
  return (int64_t)2 * iters * ((k + W - 1) / W) * 16;
}

/* tail LLRs of both SISOs (gather_tails, lte_turbo.cpp:758-773) and where they come from in
 * [d0|d1|d2] (offsets into the 3(K+4) LLRs) */
static void tails64(int32_t k, const double* llr, double ts[2][3], double tp[2][3],
                    int32_t its[2][3], int32_t itp[2][3], int std) {
  const int32_t o0 = 0, o1 = k + 4, o2 = 2 * (k + 4);
  const int32_t r_s[2][3] = {{o0 + k, o0 + k + 2, -1}, {o1 + k + 3, o2 + k, o2 + k + 2}};
  const int32_t r_p[2][3] = {{o1 + k, o0 + k + 1, o1 + k + 2}, {o2 + k + 1, o0 + k + 3, o2 + k + 3}};
  /* TS 36.212 5.1.3.2.2 (gather_tails_std) */
  const int32_t t_s[2][3] = {{o0 + k, o2 + k, o1 + k + 1}, {o0 + k + 2, o2 + k + 2, o1 + k + 3}};
  const int32_t t_p[2][3] = {{o1 + k, o0 + k + 1, o2 + k + 1}, {o1 + k + 2, o0 + k + 3, o2 + k + 3}};
  const int32_t(*s_idx)[3] = std ? t_s : r_s;
  const int32_t(*p_idx)[3] = std ? t_p : r_p;
  for (int h = 0; h < 2; ++h)
    for (int i = 0; i < 3; ++i) {
      its[h][i] = s_idx[h][i];
      itp[h][i] = p_idx[h][i];
      ts[h][i] = s_idx[h][i] >= 0 ? llr[s_idx[h][i]] : 0.0;
      tp[h][i] = llr[p_idx[h][i]];
    }
}

static void adj_vjp(int32_t k, const double* llr, int32_t iters, const double* scales,
                    int32_t window, int32_t guard, const double* frozen_seeds,
                    const double* grad_post, double* posterior, double* grad_llr,
                    double* grad_scales, double* seeds_out, int std) {
  const trellis_t T = make_trellis_conv(std);
  const int32_t W = adj_window(k, window);
  const int32_t G = guard < 0 ? 0 : (guard > W ? W : guard);
  const int32_t nw = (k + W - 1) / W, nj = 2 * iters;
  const double* d0 = llr;
  const double* d1 = llr + (k + 4);
  const double* d2 = llr + 2 * (k + 4);
  double ts[2][3], tp[2][3];
  int32_t its[2][3], itp[2][3];
  tails64(k, llr, ts, tp, its, itp, std);
  int32_t* perm = (int32_t*)malloc(sizeof(int32_t) * (size_t)k);
  or_qpp_perm(k, perm);
  const size_t rows = (size_t)(W + 2 * G + 1);
  double* alpha = (double*)malloc(sizeof(double) * 8u * rows);
  double* beta = (double*)malloc(sizeof(double) * 8u * rows);
  double* sys_i = (double*)malloc(sizeof(double) * (size_t)k);
  double* e1 = (double*)calloc((size_t)k, sizeof(double));
  double* e2 = (double*)calloc((size_t)k, sizeof(double));
  double* x = (double*)malloc(sizeof(double) * (size_t)k);
  /* tape: a-priori and extrinsic (unscaled) per SISO, seeds per SISO and window */
  double* tape_apr = (double*)malloc(sizeof(double) * (size_t)k * (size_t)nj);
  double* tape_x = (double*)malloc(sizeof(double) * (size_t)k * (size_t)nj);
  double* seeds = (double*)calloc((size_t)(nj + 2) * (size_t)nw * 16u, sizeof(double));
  for (int32_t i = 0; i < k; ++i) sys_i[i] = d0[perm[i]];
  for (int32_t it = 0; it < iters; ++it)
    for (int h = 0; h < 2; ++h) {
      const int j = 2 * it + h;
      const double* sys = h ? sys_i : d0;
      const double* par = h ? d2 : d1;
      double* apr = tape_apr + (size_t)j * k;
      if (h)
        for (int32_t i = 0; i < k; ++i) apr[i] = e1[perm[i]];
      else
        memcpy(apr, e2, sizeof(double) * (size_t)k);
      double* sj = frozen_seeds ? (double*)frozen_seeds + (size_t)j * nw * 16
                                : seeds + (size_t)j * nw * 16;
      double* snext = seeds + (size_t)(j + 2) * nw * 16;
      for (int32_t w = 0; w < nw; ++w) {
        const seg64_t g = seg64(k, W, G, w);
        seg64_forward(&T, sys, par, apr, g, g.start ? NULL : sj + 16 * w,
                      g.tail ? NULL : sj + 16 * w + 8, ts[h], tp[h], alpha, beta, x);
        /* next-iteration seeds: alpha at hi-G for window w+1, beta at lo+G for window w-1 */
        if (w + 1 < nw && g.hi - G > 0)
          memcpy(snext + 16 * (w + 1), alpha + 8 * (g.hi - G - g.a_lo), 8 * sizeof(double));
        if (w > 0 && g.lo + G < k)
          memcpy(snext + 16 * (w - 1) + 8, beta + 8 * (g.lo + G - g.lo), 8 * sizeof(double));
      }
      memcpy(tape_x + (size_t)j * k, x, sizeof(double) * (size_t)k);
      if (h)
        for (int32_t i = 0; i < k; ++i) e2[perm[i]] = scales[j] * x[i];
      else
        for (int32_t i = 0; i < k; ++i) e1[i] = scales[j] * x[i];
    }
  if (seeds_out) {
    if (frozen_seeds)
      memcpy(seeds_out, frozen_seeds, sizeof(double) * (size_t)nj * nw * 16);
    else
      memcpy(seeds_out, seeds, sizeof(double) * (size_t)nj * nw * 16);
  }
  if (posterior)
    for (int32_t i = 0; i < k; ++i) posterior[i] = d0[i] + e1[i] + e2[i];

  if (grad_post) {
    const double* sd = frozen_seeds ? frozen_seeds : seeds;
    memset(grad_llr, 0, sizeof(double) * 3u * (size_t)(k + 4));
    memset(grad_scales, 0, sizeof(double) * (size_t)nj);
    double* g0 = grad_llr;
    double* g1 = grad_llr + (k + 4);
    double* g2 = grad_llr + 2 * (k + 4);
    double* ge1 = (double*)calloc((size_t)k, sizeof(double)); /* d/d e1, natural order */
    double* ge2 = (double*)calloc((size_t)k, sizeof(double)); /* d/d e2, natural order */
    double* gx = (double*)malloc(sizeof(double) * (size_t)k);
    double* gsa = (double*)malloc(sizeof(double) * (size_t)k);
    double* gpar = (double*)malloc(sizeof(double) * (size_t)k);
    for (int32_t i = 0; i < k; ++i) { /* posterior = Ls + e1 + e2 */
      g0[i] += grad_post[i];
      ge1[i] = grad_post[i];
      ge2[i] = grad_post[i];
    }
    for (int32_t it = iters; it-- > 0;)
      for (int h = 1; h >= 0; --h) {
        const int j = 2 * it + h;
        const double* X = tape_x + (size_t)j * k;
        const double* sys = h ? sys_i : d0;
        const double* par = h ? d2 : d1;
        const double* apr = tape_apr + (size_t)j * k;
        for (int32_t i = 0; i < k; ++i) { /* e = scale * x, lower in interleaved order */
          const double ge = h ? ge2[perm[i]] : ge1[i];
          grad_scales[j] += ge * X[i];
          gx[i] = ge * scales[j];
        }
        memset(gsa, 0, sizeof(double) * (size_t)k);
        memset(gpar, 0, sizeof(double) * (size_t)k);
        double gts[3] = {0, 0, 0}, gtp[3] = {0, 0, 0};
        const double* sj = sd + (size_t)j * nw * 16;
        for (int32_t w = 0; w < nw; ++w) {
          const seg64_t g = seg64(k, W, G, w);
          seg64_forward(&T, sys, par, apr, g, g.start ? NULL : sj + 16 * w,
                        g.tail ? NULL : sj + 16 * w + 8, ts[h], tp[h], alpha, beta, x);
          seg64_adjoint(&T, sys, par, apr, g, ts[h], tp[h], alpha, beta, gx, gsa, gpar, gts,
                        gtp);
        }
        for (int i = 0; i < 3; ++i) {
          if (its[h][i] >= 0) grad_llr[its[h][i]] += gts[i];
          grad_llr[itp[h][i]] += gtp[i];
        }
        if (h) { /* sys_i[i] = d0[perm[i]], a-priori[i] = e1[perm[i]] */
          for (int32_t i = 0; i < k; ++i) {
            g0[perm[i]] += gsa[i];
            g2[i] += gpar[i];
          }
          memset(ge1, 0, sizeof(double) * (size_t)k); /* e1 of iteration it: only via this SISO */
          if (it + 1 == iters)
            for (int32_t i = 0; i < k; ++i) ge1[i] = grad_post[i];
          for (int32_t i = 0; i < k; ++i) ge1[perm[i]] += gsa[i];
        } else { /* a-priori = e2 of iteration it-1 (zero for it = 0) */
          for (int32_t i = 0; i < k; ++i) {
            g0[i] += gsa[i];
            g1[i] += gpar[i];
            ge2[i] = gsa[i];
          }
        }
      }
    free(ge1); free(ge2); free(gx); free(gsa); free(gpar);
  }
  free(perm); free(alpha); free(beta); free(sys_i); free(e1); free(e2); free(x);
  free(tape_apr); free(tape_x); free(seeds);
}

void or_adj_vjp(int32_t k, const double* llr, int32_t iters, const double* scales,
                int32_t window, int32_t guard, const double* frozen_seeds,
                const double* grad_post, double* posterior, double* grad_llr,
                double* grad_scales, double* seeds_out) {
  adj_vjp(k, llr, iters, scales, window, guard, frozen_seeds, grad_post, posterior, grad_llr,
          grad_scales, seeds_out, 0);
}

/* The same on the TS 36.212 code (trellis, termination, tail mapping). */
void or_std_adj_vjp(int32_t k, const double* llr, int32_t iters, const double* scales,
                    int32_t window, int32_t guard, const double* frozen_seeds,
                    const double* grad_post, double* posterior, double* grad_llr,
                    double* grad_scales, double* seeds_out) {
  adj_vjp(k, llr, iters, scales, window, guard, frozen_seeds, grad_post, posterior, grad_llr,
          grad_scales, seeds_out, 1);
}
