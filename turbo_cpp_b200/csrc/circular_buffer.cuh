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

__constant__ uint8_t c_col_perm[32] = {0, 16, 8, 24, 4, 20, 12, 28, 2, 18, 10, 26, 6, 22, 14, 30,
                                       1, 17, 9, 25, 5, 21, 13, 29, 3, 19, 11, 27, 7, 23, 15, 31};

constexpr int kCircThreads = 512;  // threads per CTA of the kernels that use CircularScan

// Circular-buffer position -> index into [d0|d1|d2], -1 for <NULL> (sub-block interleavers of
// lte_turbo.cpp:195-236 in closed form; interlacing lte_turbo.cpp:256-262).
__device__ __forceinline__ int rm_source(int pos, int d, int rows, int kpi, int filler) {
  const int dummy = kpi - d;
  if (pos < kpi) {  // systematic, read column by column
    const int y = (pos % rows) * 32 + c_col_perm[pos / rows] - dummy;
    return (y < 0 || y < filler) ? -1 : y;
  }
  const int local = pos - kpi, lane = local >> 1;
  if ((local & 1) == 0) {  // parity 1: same permutation as the systematic stream
    const int y = (lane % rows) * 32 + c_col_perm[lane / rows] - dummy;
    return (y < 0 || y < filler) ? -1 : d + y;
  }
  const int y = (c_col_perm[lane / rows] + 32 * (lane % rows) + 1) % kpi - dummy;
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
      const int y = r * 32 + c_col_perm[q] - dummy;
      src = (y < 0 || y < filler) ? -1 : y;
      if (++r == rows) {
        r = 0;
        ++q;
      }
      if (++pos == kpi) q = r = 0;  // the parity part starts at lane 0
      return src;
    }
    if (((pos - kpi) & 1) == 0) {  // parity 1: same permutation as the systematic stream
      const int y = r * 32 + c_col_perm[q] - dummy;
      src = (y < 0 || y < filler) ? -1 : d + y;
    } else {  // parity 2: no filler nulling; the lane advances after its second stream
      int y = c_col_perm[q] + 32 * r + 1;
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

}  // namespace
}  // namespace tcb
