// circular_buffer.cuh -- the LTE rate-matching circular buffer on the device, shared by the
// de-rate matchers (chain.cu) and the rate matcher (generate.cu).
//
// The buffer of a code block interlaces the sub-block-interleaved systematic stream with the two
// interleaved parity streams (lte_turbo.cpp:195-262); some of its Ncb positions are <NULL>
// (dummy padding, and the filler bits of d0 and d1).  Rate matching walks it from k0 and takes
// the non-<NULL> positions in order, wrapping around: the E values of a block land, in order,
// on the valid positions of rank (rank(k0) + kk) mod Nv.  One CTA per block finds every valid
// position's rank with a block-wide scan over contiguous chunks of positions.
#pragma once
#include <cstdint>

namespace tcb {
namespace {

// The inter-column permutation of the sub-block interleaver (TS 36.212 Table 5.1.4-1,
// lte_turbo.cpp:195-236) is the 5-bit reversal of the column index, its own inverse: one
// instruction, where a table in constant memory would serialise a warp whose lanes read
// different columns.
__device__ __forceinline__ int col_perm(int c) { return static_cast<int>(__brev(static_cast<unsigned>(c)) >> 27); }

constexpr int kCircThreads = 512;  // threads per CTA of the kernels that use CircularScan

// Circular-buffer position -> index into [d0|d1|d2], -1 for <NULL> (sub-block interleavers of
// lte_turbo.cpp:195-236 in closed form; interlacing lte_turbo.cpp:256-262).
__device__ __forceinline__ int rm_source(int pos, int d, int rows, int kpi, int filler) {
  const int dummy = kpi - d;
  if (pos < kpi) {  // systematic, read column by column
    const int y = (pos % rows) * 32 + col_perm(pos / rows) - dummy;
    return (y < 0 || y < filler) ? -1 : y;
  }
  const int local = pos - kpi, lane = local >> 1;
  if ((local & 1) == 0) {  // parity 1: same permutation as the systematic stream
    const int y = (lane % rows) * 32 + col_perm(lane / rows) - dummy;
    return (y < 0 || y < filler) ? -1 : d + y;
  }
  const int y = (col_perm(lane / rows) + 32 * (lane % rows) + 1) % kpi - dummy;
  return y < 0 ? -1 : 2 * d + y;  // parity 2: no filler nulling
}

// Sources of consecutive circular-buffer positions from p on, with the divisions by `rows` of
// rm_source done once: the position's (or, in the parity part, its interlaced lane's) quotient
// and remainder by `rows` are advanced incrementally.  next() returns the source of the current
// position (as rm_source) and moves to the following one.
struct CircularWalk {
  int d, rows, kpi, dummy, filler;
  int pos, q, r;  // systematic part: pos = q*rows + r; parity part: lane = q*rows + r

  __device__ __forceinline__ CircularWalk(int p, int d_, int rows_, int kpi_, int filler_)
      : d(d_), rows(rows_), kpi(kpi_), dummy(kpi_ - d_), filler(filler_), pos(p) {
    const int idx = p < kpi ? p : (p - kpi) >> 1;
    q = idx / rows;
    r = idx - q * rows;
  }

  __device__ __forceinline__ int next() {
    int src;
    if (pos < kpi) {  // systematic, read column by column
      const int y = r * 32 + col_perm(q) - dummy;
      src = (y < 0 || y < filler) ? -1 : y;
      if (++r == rows) {
        r = 0;
        ++q;
      }
      if (++pos == kpi) q = r = 0;  // the parity part starts at lane 0
      return src;
    }
    if (((pos - kpi) & 1) == 0) {  // parity 1: same permutation as the systematic stream
      const int y = r * 32 + col_perm(q) - dummy;
      src = (y < 0 || y < filler) ? -1 : d + y;
    } else {  // parity 2: no filler nulling; the lane advances after its second stream
      int y = col_perm(q) + 32 * r + 1;
      if (y >= kpi) y -= kpi;
      y -= dummy;
      src = y < 0 ? -1 : 2 * d + y;
      if (++r == rows) {
        r = 0;
        ++q;
      }
    }
    ++pos;
    return src;
  }
};

// The circular buffer of one code block as one CTA of kCircThreads threads sees it: each thread
// owns the positions [p0, p1); `before` is the number of valid positions before p0.
struct CircularScan {
  int d, rows, kpi, ncb, filler;
  int p0, p1, before;
  int total;  // valid positions (Nv), after scan()

  __device__ __forceinline__ CircularScan(int k, int filler_bits) {
    d = k + 4;
    rows = (d + 31) / 32;
    kpi = rows * 32;
    ncb = 3 * kpi;
    filler = filler_bits;
    const int chunk = (ncb + static_cast<int>(blockDim.x) - 1) / static_cast<int>(blockDim.x);
    p0 = min(ncb, static_cast<int>(threadIdx.x) * chunk);
    p1 = min(ncb, p0 + chunk);
    before = total = 0;
  }

  __device__ __forceinline__ int source(int pos) const { return rm_source(pos, d, rows, kpi, filler); }

  // k0 of redundancy version rv (lte_turbo.cpp:294-295), reduced modulo Ncb
  __device__ __forceinline__ int k0(int rv) const {
    return rows * (2 * ((ncb + 8 * rows - 1) / (8 * rows)) * rv + 2) % ncb;
  }

  // the sources of positions p, p+1, ... in order
  __device__ __forceinline__ CircularWalk walk(int p) const {
    return CircularWalk(p, d, rows, kpi, filler);
  }

  // Block-wide exclusive scan of the valid-position counts; every thread must call it.
  // warp_sum: kCircThreads / 32 ints of shared memory; s_total: one shared int.
  __device__ __forceinline__ void scan(int* warp_sum, int* s_total) {
    int cnt = 0;
    CircularWalk wk = walk(p0);
    for (int p = p0; p < p1; ++p) cnt += wk.next() >= 0;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) warp_sum[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      int v = lane < kCircThreads / 32 ? warp_sum[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
      }
      if (lane < kCircThreads / 32) warp_sum[lane] = v;  // inclusive per warp
    }
    __syncthreads();
    before = (wid ? warp_sum[wid - 1] : 0) + incl - cnt;
    if (threadIdx.x == blockDim.x - 1) *s_total = before + cnt;
  }

  // The thread whose chunk holds position `pos` writes its rank to *out (no barrier here).
  __device__ __forceinline__ void rank_of(int pos, int* out) const {
    if (pos >= p0 && pos < p1) {
      int r = before;
      CircularWalk wk = walk(p0);
      for (int p = p0; p < pos; ++p) r += wk.next() >= 0;
      *out = r;
    }
  }
};

// The ranks of circular-buffer positions in closed form, and each [d0|d1|d2] element's
// position.  The column permutation of the sub-block interleaver is a 5-bit reversal, its own
// inverse.  In a column q (32 columns of `rows` rows, read top to bottom) the <NULL> entries of
// the systematic stream and of parity 1 are the top rows r with r*32 + perm[q] < dummy + filler
// (cnt1[q] of them); parity 2 is <NULL> in row 0 when perm[q] + 1 < dummy and in the last row of
// the column with perm[q] = 31 when dummy > 0 (its index wraps to 0).  The <NULL> entries before
// a position are therefore a prefix over whole columns plus a count inside its column, and
// rank(p) = p - that number.  setup() is run by the first warp of the CTA (tables in shared
// memory: kRankTableInts ints), followed by a barrier.
constexpr int kRankTableInts = 32 + 2 * 33;
struct CircularRank {
  int d, rows, kpi, ncb, filler, dummy;
  int* cnt1;   // [32]: <NULL> rows at the top of column q (systematic, parity 1)
  int* pre1;   // [33]: prefix of cnt1 over the columns
  int* pre12;  // [33]: prefix of cnt1 + the parity-2 <NULL>s over the columns

  __device__ __forceinline__ CircularRank(int k, int filler_bits, int* smem)
      : d(k + 4), rows((k + 4 + 31) / 32), filler(filler_bits), cnt1(smem), pre1(smem + 32),
        pre12(smem + 65) {
    kpi = rows * 32;
    ncb = 3 * kpi;
    dummy = kpi - d;
  }

  __device__ __forceinline__ bool p2_row0_null(int q) const { return col_perm(q) + 1 < dummy; }

  // first warp: the per-column tables
  __device__ __forceinline__ void setup() {
    if (threadIdx.x >= 32) return;
    const int q = threadIdx.x, pq = col_perm(q);
    const int t = dummy + filler - pq;
    const int c1 = t <= 0 ? 0 : min(rows, (t + 31) >> 5);
    const int c2 = (pq + 1 < dummy ? 1 : 0) + (pq == 31 && dummy > 0 ? 1 : 0);
    cnt1[q] = c1;
    int a = c1, b = c1 + c2;  // inclusive prefixes over columns 0..q
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int ua = __shfl_up_sync(0xffffffffu, a, o), ub = __shfl_up_sync(0xffffffffu, b, o);
      if (q >= o) {
        a += ua;
        b += ub;
      }
    }
    pre1[q + 1] = a;
    pre12[q + 1] = b;
    if (q == 0) pre1[0] = pre12[0] = 0;
  }

  __device__ __forceinline__ int valid() const { return ncb - pre1[32] - pre12[32]; }  // Nv
  // rank of the systematic position of column q, row r
  __device__ __forceinline__ int rank_sys(int q, int r) const {
    return q * rows + r - (pre1[q] + min(r, cnt1[q]));
  }
  // rank of the parity-1 (odd = 0) or parity-2 (odd = 1) position of lane (q, r)
  __device__ __forceinline__ int rank_par(int q, int r, int odd) const {
    const int nulls = pre1[32] + pre12[q] + min(r, cnt1[q]) + (r > 0 && p2_row0_null(q) ? 1 : 0) +
                      (odd && r < cnt1[q] ? 1 : 0);
    return kpi + 2 * (q * rows + r) + odd - nulls;
  }
  // rank of any position p in [0, Ncb) (valid positions before it)
  __device__ __forceinline__ int rank(int p) const {
    if (p < kpi) return rank_sys(p / rows, p % rows);
    const int lane = (p - kpi) >> 1;
    return rank_par(lane / rows, lane % rows, (p - kpi) & 1);
  }
  // the rank of [d0|d1|d2] element i (stream i / d), or -1 for the filler elements of d0 and d1
  // (<NULL> in the buffer)
  __device__ __forceinline__ int rank_of_element(int i) const {
    const int s = i >= d ? (i >= 2 * d ? 2 : 1) : 0;
    const int y = i - s * d;
    if (s < 2) {
      if (y < filler) return -1;
      const int yy = y + dummy;
      const int q = col_perm(yy & 31), r = yy >> 5;
      return s == 0 ? rank_sys(q, r) : rank_par(q, r, 0);
    }
    const int y2 = y + dummy;
    const int v = y2 > 0 ? y2 - 1 : kpi - 1;
    return rank_par(col_perm(v & 31), v >> 5, 1);
  }
  // k0 of redundancy version rv (lte_turbo.cpp:294-295), reduced modulo Ncb
  __device__ __forceinline__ int k0(int rv) const {
    return rows * (2 * ((ncb + 8 * rows - 1) / (8 * rows)) * rv + 2) % ncb;
  }
};

}  // namespace
}  // namespace tcb
