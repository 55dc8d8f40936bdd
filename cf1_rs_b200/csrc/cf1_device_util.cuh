// Device-side building blocks shared by several kernels.
#pragma once
#include "cf1_common.cuh"

namespace cf1 {

constexpr unsigned FULL = 0xFFFFFFFFu;

CF1_D unsigned lane_id() { return threadIdx.x & 31; }
CF1_D unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <class T>
CF1_D T warp_inclusive_scan(T x) {
  unsigned lane = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(FULL, x, o);
    if (lane >= (unsigned)o) x += y;
  }
  return x;
}

template <class T>
CF1_D T warp_sum(T x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(FULL, x, o);
  return x;
}

// Block-wide exclusive scan of one value per thread.  `sm` holds BLOCK/32
// entries.  Ends with a barrier, so `sm` may be reused right after.
template <int BLOCK, class T>
CF1_D T block_exclusive_scan(T v, T *sm, T &total) {
  constexpr int NW = BLOCK / 32;
  unsigned lane = lane_id(), warp = threadIdx.x >> 5;
  T x = warp_inclusive_scan(v);
  if (lane == 31) sm[warp] = x;
  __syncthreads();
  if (warp == 0) {
    T w = lane < (unsigned)NW ? sm[lane] : T(0);
    w = warp_inclusive_scan(w);
    if (lane < (unsigned)NW) sm[lane] = w;
  }
  __syncthreads();
  T pre = warp ? sm[warp - 1] : T(0);
  total = sm[NW - 1];
  __syncthreads();
  return pre + x - v;
}

template <int BLOCK, class T>
CF1_D T block_sum(T v, T *sm) {
  T tot;
  block_exclusive_scan<BLOCK>(v, sm, tot);
  return tot;
}

// Order-preserving selection over [0, len) by a whole block: pred(i) picks
// indices, emit(i, rank) receives each picked index with its rank among the
// picked ones.  Each warp owns one contiguous slice and walks it 32
// consecutive indices at a time, so consecutive lanes touch consecutive
// elements (no shared-memory bank conflicts).  Returns the count; ends with
// a barrier.  `sm` holds BLOCK/32 entries.
template <int BLOCK, class Pred, class Emit>
CF1_D uint32_t block_select(uint32_t len, Pred pred, Emit emit, uint32_t *sm) {
  constexpr int NW = BLOCK / 32;
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
  const uint32_t per = ((len + NW - 1) / NW + 31) & ~31u;
  const uint32_t lo = warp * per, hi = lo + per < len ? lo + per : len;
  uint32_t c = 0;
  for (uint32_t base = lo; base < hi; base += 32) {
    uint32_t i = base + lane;
    c += __popc(__ballot_sync(FULL, i < hi && pred(i)));
  }
  if (lane == 0) sm[warp] = c;
  __syncthreads();
  uint32_t pre = 0, tot = 0;
  for (int w = 0; w < NW; w++) {
    uint32_t v = sm[w];
    pre += (unsigned)w < warp ? v : 0;
    tot += v;
  }
  const unsigned lt = lanemask_lt();
  for (uint32_t base = lo; base < hi; base += 32) {
    uint32_t i = base + lane;
    bool f = i < hi && pred(i);
    unsigned b = __ballot_sync(FULL, f);
    if (f) emit(i, pre + __popc(b & lt));
    pre += __popc(b);
  }
  __syncthreads();
  return tot;
}

// Largest b in [0, nseg) with off[b] <= t, for nondecreasing off[0..nseg].
template <class T>
CF1_D uint32_t upper_segment(const T *off, uint32_t nseg, T t) {
  uint32_t lo = 0, hi = nseg;  // invariant: off[lo] <= t < off[hi] (off[nseg] > t)
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (off[mid] <= t) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Segment of tile t over segments seg_off[0..nseg] cut into tiles of `tile`
// elements (tiles never cross a segment edge; tile_off from segment_tiles).
struct TileSpan {
  uint32_t seg;
  uint64_t start, end;
  uint32_t first_tile, ntiles;
};
CF1_D TileSpan tile_span(const uint64_t *seg_off, const uint32_t *tile_off, uint32_t nseg, uint32_t t, uint32_t tile) {
  TileSpan s;
  s.seg = upper_segment(tile_off, nseg, t);
  s.first_tile = tile_off[s.seg];
  s.ntiles = tile_off[s.seg + 1] - s.first_tile;
  s.start = seg_off[s.seg] + (uint64_t)(t - s.first_tile) * tile;
  uint64_t e = s.start + tile;
  s.end = e < seg_off[s.seg + 1] ? e : seg_off[s.seg + 1];
  return s;
}
// Tile t over gapped segments: segment b holds cnt[b] items from start[b].
CF1_D TileSpan tile_span_gapped(const uint64_t *start, const uint64_t *cnt, const uint32_t *tile_off, uint32_t nseg,
                                uint32_t t, uint32_t tile) {
  TileSpan s;
  s.seg = upper_segment(tile_off, nseg, t);
  s.first_tile = tile_off[s.seg];
  s.ntiles = tile_off[s.seg + 1] - s.first_tile;
  s.start = start[s.seg] + (uint64_t)(t - s.first_tile) * tile;
  uint64_t e = s.start + tile, stop = start[s.seg] + cnt[s.seg];
  s.end = e < stop ? e : stop;
  return s;
}

}  // namespace cf1
