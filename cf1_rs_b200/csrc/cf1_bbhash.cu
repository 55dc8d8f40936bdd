// Per-bin GPU BBHash construction (the "plain" MPHF of this library).
//
// The reference builds one ph::fmph::Function over all distinct keys
// (src/mphf.rs:144-190; BBHash-style levels with relative_level_size 200).
// Here every bin gets its own levels so that phase 4, which walks the bins in
// order, touches one bin's bit arrays at a time.  Per level, over the keys not
// yet placed:
//   mark   : set the key's bit with atomicOr; a key that finds its bit set
//            marks the collision array instead;
//   clean  : bits that collided are cleared; a popcount prefix gives ranks;
//   filter : keys whose bit survived are placed, the rest go to the next level.
// A bin's local slot of a key placed at level l is the number of keys of the
// bin placed at earlier levels plus the key's rank inside its level block.
// All levels live in one array of {bit word, level rank} entries, addressed
// through the per-(level, bin) BBMeta table.
#include <algorithm>
#include <cstring>

#include "../../include/cf1gpu.h"
#include "cf1_bbhash.cuh"
#include "cf1_device_util.cuh"
#include "cf1_mphf.cuh"

namespace cf1 {

namespace {

constexpr int BB_BLOCK = 256;
constexpr uint32_t BB_TILE = 4096;

__global__ void bb_sel_counts_kernel(const uint64_t *seg_off, const uint32_t *sel, uint32_t nbins, uint64_t *cnt) {
  uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nbins) cnt[b] = (sel == nullptr || sel[b]) ? seg_off[b + 1] - seg_off[b] : 0;
}

template <class KeyT>
__global__ void __launch_bounds__(BB_BLOCK) bb_copy_sel_kernel(const KeyT *keys, const uint64_t *seg_off,
                                                               const uint32_t *tile_off, uint32_t nbins,
                                                               const uint32_t *sel, const uint64_t *new_off,
                                                               KeyT *out) {
  const uint32_t t = blockIdx.x;
  if (t >= tile_off[nbins]) return;
  TileSpan sp = tile_span(seg_off, tile_off, nbins, t, BB_TILE);
  if (sel && !sel[sp.seg]) return;
  uint64_t delta = new_off[sp.seg] - seg_off[sp.seg];
  for (uint64_t i = sp.start + threadIdx.x; i < sp.end; i += BB_BLOCK) out[i + delta] = keys[i];
}

__global__ void bb_sizes_kernel(const uint64_t *rem_off, uint32_t nbins, uint64_t *wcnt) {
  uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nbins) {
    uint64_t n = rem_off[b + 1] - rem_off[b];
    uint64_t words = (2 * n + 63) / 64;
    wcnt[b] = n ? (words ? words : 1) : 0;
  }
}

// AR points at this level's first entry; woff are the level-relative block
// offsets of the bins.
template <class KeyT>
__global__ void __launch_bounds__(BB_BLOCK) bb_mark_kernel(const KeyT *rem, const uint64_t *rem_off,
                                                           const uint32_t *tile_off, uint32_t nbins,
                                                           const uint64_t *woff, uint32_t level, ulonglong2 *AR,
                                                           uint64_t *C) {
  const uint32_t t = blockIdx.x;
  if (t >= tile_off[nbins]) return;
  TileSpan sp = tile_span(rem_off, tile_off, nbins, t, BB_TILE);
  const uint64_t w0 = woff[sp.seg];
  const uint32_t nw = (uint32_t)(woff[sp.seg + 1] - w0);
  for (uint64_t i = sp.start + threadIdx.x; i < sp.end; i += BB_BLOCK) {
    uint64_t pos = bb_pos(bb_key_hash(rem[i]), level, nw);
    uint64_t wi = w0 + (pos >> 6);
    uint64_t bit = 1ull << (pos & 63);
    unsigned long long old = atomicOr(&AR[wi].x, (unsigned long long)bit);
    if (old & bit) atomicOr(reinterpret_cast<unsigned long long *>(C + wi), (unsigned long long)bit);
  }
}

__global__ void bb_clean_kernel(ulonglong2 *AR, const uint64_t *C, uint32_t *pc, uint64_t nw) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nw) {
    uint64_t a = AR[i].x & ~C[i];
    AR[i].x = a;
    pc[i] = (uint32_t)__popcll(a);
  }
}

__global__ void bb_rank_kernel(ulonglong2 *AR, const uint64_t *R, uint64_t nw) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nw) AR[i].y = R[i];
}

__global__ void bb_meta_kernel(const uint64_t *woff, const uint64_t *R, uint64_t level_base, uint64_t *base,
                               BBMeta *meta, uint32_t nbins) {
  uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbins) return;
  uint64_t w0 = woff[b], w1 = woff[b + 1];
  BBMeta m;
  m.word_off = level_base + w0;
  m.nwords = (uint32_t)(w1 - w0);
  m.rank_adj = (uint32_t)(base[b] - R[w0]);
  meta[b] = m;
  base[b] += R[w1] - R[w0];
}

template <class KeyT>
CF1_D bool bb_placed(const KeyT &key, uint32_t level, uint64_t w0, uint32_t nw, const ulonglong2 *AR) {
  uint64_t pos = bb_pos(bb_key_hash(key), level, nw);
  return (AR[w0 + (pos >> 6)].x >> (pos & 63)) & 1;
}

template <class KeyT>
__global__ void __launch_bounds__(BB_BLOCK) bb_filter_count_kernel(const KeyT *rem, const uint64_t *rem_off,
                                                                   const uint32_t *tile_off, uint32_t nbins,
                                                                   const uint64_t *woff, uint32_t level,
                                                                   const ulonglong2 *A, uint32_t *tile_cnt) {
  __shared__ uint32_t sm[BB_BLOCK / 32];
  const uint32_t t = blockIdx.x;
  if (t >= tile_off[nbins]) {
    if (threadIdx.x == 0) tile_cnt[t] = 0;
    return;
  }
  TileSpan sp = tile_span(rem_off, tile_off, nbins, t, BB_TILE);
  const uint64_t w0 = woff[sp.seg];
  const uint32_t nw = (uint32_t)(woff[sp.seg + 1] - w0);
  uint32_t c = 0;
  for (uint64_t i = sp.start + threadIdx.x; i < sp.end; i += BB_BLOCK) c += bb_placed(rem[i], level, w0, nw, A) ? 0 : 1;
  uint32_t tot = block_sum<BB_BLOCK>(c, sm);
  if (threadIdx.x == 0) tile_cnt[t] = tot;
}

template <class KeyT>
__global__ void __launch_bounds__(BB_BLOCK) bb_filter_write_kernel(const KeyT *rem, const uint64_t *rem_off,
                                                                   const uint32_t *tile_off, uint32_t nbins,
                                                                   const uint64_t *woff, uint32_t level,
                                                                   const ulonglong2 *A, const uint64_t *tile_out,
                                                                   KeyT *out) {
  constexpr int ITEMS = BB_TILE / BB_BLOCK;
  __shared__ uint32_t sm[BB_BLOCK / 32];
  const uint32_t t = blockIdx.x;
  if (t >= tile_off[nbins]) return;
  TileSpan sp = tile_span(rem_off, tile_off, nbins, t, BB_TILE);
  const uint64_t w0 = woff[sp.seg];
  const uint32_t nw = (uint32_t)(woff[sp.seg + 1] - w0);
  uint64_t i0 = sp.start + (uint64_t)threadIdx.x * ITEMS;
  uint32_t flags = 0, c = 0;
#pragma unroll
  for (int j = 0; j < ITEMS; j++) {
    uint64_t i = i0 + j;
    bool keep = i < sp.end && !bb_placed(rem[i], level, w0, nw, A);
    flags |= (uint32_t)keep << j;
    c += keep;
  }
  uint32_t tot;
  uint32_t pre = block_exclusive_scan<BB_BLOCK>(c, sm, tot);
  uint64_t o = tile_out[t] + pre;
#pragma unroll
  for (int j = 0; j < ITEMS; j++)
    if ((flags >> j) & 1) out[o++] = rem[i0 + j];
}

__global__ void offsets_from_tiles_kernel(const uint32_t *tile_off, uint32_t nseg, const uint64_t *tile_out,
                                          uint64_t *out_off) {
  uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b <= nseg) out_off[b] = tile_out[tile_off[b]];
}

uint64_t d2h_u64(const uint64_t *p, cudaStream_t s) {
  uint64_t v = 0;
  CF1_CUDA(cudaMemcpyAsync(&v, p, sizeof(v), cudaMemcpyDeviceToHost, s));
  CF1_CUDA(cudaStreamSynchronize(s));
  return v;
}

}  // namespace

template <class KeyT>
void BBHashBuild<KeyT>::clear() {
  nwords.clear();
  level_off.clear();
  total_words = 0;
  levels = 0;
  bytes = 0;
}

template <class KeyT>
void BBHashBuild<KeyT>::reserve_entries(uint64_t words, uint64_t keep, cudaStream_t s) {
  const size_t need = words * sizeof(ulonglong2);
  if (ar_.p && need <= ar_.cap) return;
  size_t cap = std::max<size_t>(need + need / 4, 4096);
  void *np = nullptr;
  CF1_CUDA(cudaMalloc(&np, cap));
  if (keep && ar_.p) {
    CF1_CUDA(cudaMemcpyAsync(np, ar_.p, keep * sizeof(ulonglong2), cudaMemcpyDeviceToDevice, s));
    CF1_CUDA(cudaStreamSynchronize(s));
  }
  ar_.release();
  ar_.p = np;
  ar_.cap = cap;
}

template <class KeyT>
void BBHashBuild<KeyT>::build(const KeyT *keys, const uint64_t *seg_off, uint32_t nb, const uint32_t *sel,
                              cudaStream_t s, KeyT *ws0, KeyT *ws1, uint64_t ws_cap) {
  clear();
  nbins = nb;
  {  // local slots are 32-bit: every bin must hold fewer than 2^32 keys
    std::vector<uint64_t> h(nbins + 1);
    CF1_CUDA(cudaMemcpyAsync(h.data(), seg_off, (nbins + 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    CF1_CUDA(cudaStreamSynchronize(s));
    for (uint32_t b = 0; b < nbins; b++)
      if (h[b + 1] - h[b] >= (1ull << 32))
        throw Error(CF1GPU_ERR_INVALID_ARG, "BBHash: a bin holds 2^32 or more distinct keys; use more bins");
  }
  uint64_t *base = base_.get<uint64_t>(nbins);
  CF1_CUDA(cudaMemsetAsync(base, 0, nbins * sizeof(uint64_t), s));
  BBMeta *meta = meta_.get<BBMeta>((size_t)BB_MAX_LEVELS * nbins);
  CF1_CUDA(cudaMemsetAsync(meta, 0, (size_t)BB_MAX_LEVELS * nbins * sizeof(BBMeta), s));

  uint64_t *cnt = wcnt_.get<uint64_t>(nbins + 1);
  uint64_t *off0 = rem_off_[0].get<uint64_t>(nbins + 1);
  uint64_t *off1 = rem_off_[1].get<uint64_t>(nbins + 1);
  uint32_t *tile_off = tile_off_.get<uint32_t>(nbins + 1);
  uint64_t n_all = d2h_u64(seg_off + nbins, s);
  uint64_t n = n_all;
  // level workspace: two key arrays of n keys (the caller's, when big enough)
  KeyT *r[2];
  r[0] = (ws0 && ws_cap >= n + 1) ? ws0 : rem_[0].get<KeyT>(n + 1);
  r[1] = (ws1 && ws_cap >= n + 1) ? ws1 : rem_[1].get<KeyT>(n + 1);
  uint64_t *roffs[2] = {off0, off1};
  const KeyT *rem = keys;
  const uint64_t *roff = seg_off;
  if (sel) {  // keys of the selected bins -> r[0]
    bb_sel_counts_kernel<<<(unsigned)ceil_div(nbins, 256), 256, 0, s>>>(seg_off, sel, nbins, cnt);
    CF1_LAUNCH_CHECK();
    exclusive_scan_u64(cnt, off0, nbins, scan_tmp_, s);
    n = d2h_u64(off0 + nbins, s);
    if (n) {
      uint32_t ub = (uint32_t)(ceil_div(n_all, BB_TILE) + nbins);
      segment_tiles(seg_off, nbins, BB_TILE, tile_off, s);
      bb_copy_sel_kernel<KeyT><<<ub, BB_BLOCK, 0, s>>>(keys, seg_off, tile_off, nbins, sel, off0, r[0]);
      CF1_LAUNCH_CHECK();
    }
    rem = r[0];
    roff = off0;
  }
  // room for the usual level sizes (2 bits per key, then ~40% fewer keys per
  // level) so that the entry array rarely grows in mid-build
  reserve_entries((2 * n / 64 + nbins) * 2 + 64, 0, s);
  int cur = 1;  // level l reads rem (keys, then r[cur^1]) and writes r[cur]
  uint64_t remaining = n;
  uint32_t l = 0;
  while (remaining > 0) {
    if (l >= BB_MAX_LEVELS) throw Error(CF1GPU_ERR_BIJECTION, "BBHash: keys left after the last level");
    KeyT *nxt = r[cur];
    uint64_t *noff = roffs[cur];
    uint64_t *woff = woff_.get<uint64_t>(nbins + 1);
    bb_sizes_kernel<<<(unsigned)ceil_div(nbins, 256), 256, 0, s>>>(roff, nbins, cnt);
    CF1_LAUNCH_CHECK();
    exclusive_scan_u64(cnt, woff, nbins, scan_tmp_, s);
    uint64_t nw = d2h_u64(woff + nbins, s);
    reserve_entries(total_words + nw, total_words, s);
    nwords.push_back(nw);
    level_off.push_back(total_words);
    ulonglong2 *Al = ar_.as<ulonglong2>() + total_words;
    uint64_t *Rl = rtmp_.get<uint64_t>(nw + 1);
    uint64_t *C = C_.get<uint64_t>(nw);
    uint32_t *pc = pc_.get<uint32_t>(nw);
    CF1_CUDA(cudaMemsetAsync(Al, 0, nw * sizeof(ulonglong2), s));
    CF1_CUDA(cudaMemsetAsync(C, 0, nw * 8, s));
    uint32_t ub = (uint32_t)(ceil_div(remaining, BB_TILE) + nbins);
    segment_tiles(roff, nbins, BB_TILE, tile_off, s);
    bb_mark_kernel<KeyT><<<ub, BB_BLOCK, 0, s>>>(rem, roff, tile_off, nbins, woff, l, Al, C);
    CF1_LAUNCH_CHECK();
    bb_clean_kernel<<<(unsigned)ceil_div(nw, 256), 256, 0, s>>>(Al, C, pc, nw);
    CF1_LAUNCH_CHECK();
    exclusive_scan_u32(pc, Rl, nw, scan_tmp_, s);
    bb_rank_kernel<<<(unsigned)ceil_div(nw, 256), 256, 0, s>>>(Al, Rl, nw);
    CF1_LAUNCH_CHECK();
    bb_meta_kernel<<<(unsigned)ceil_div(nbins, 256), 256, 0, s>>>(woff, Rl, total_words, base, meta + (size_t)l * nbins,
                                                                  nbins);
    CF1_LAUNCH_CHECK();
    uint32_t *tc = tile_cnt_.get<uint32_t>(ub + 1);
    uint64_t *to = tile_out_.get<uint64_t>(ub + 2);
    bb_filter_count_kernel<KeyT><<<ub, BB_BLOCK, 0, s>>>(rem, roff, tile_off, nbins, woff, l, Al, tc);
    CF1_LAUNCH_CHECK();
    exclusive_scan_u32(tc, to, ub, scan_tmp_, s);
    bb_filter_write_kernel<KeyT><<<ub, BB_BLOCK, 0, s>>>(rem, roff, tile_off, nbins, woff, l, Al, to, nxt);
    CF1_LAUNCH_CHECK();
    offsets_from_tiles_kernel<<<(unsigned)ceil_div(nbins + 1, 256), 256, 0, s>>>(tile_off, nbins, to, noff);
    CF1_LAUNCH_CHECK();
    total_words += nw;
    remaining = d2h_u64(noff + nbins, s);
    rem = nxt;
    roff = noff;
    cur ^= 1;
    l++;
  }
  levels = l;
  bytes = total_words * sizeof(ulonglong2) + (size_t)levels * nbins * sizeof(BBMeta);
  CF1_CUDA(cudaStreamSynchronize(s));
}

template <class KeyT>
BBView BBHashBuild<KeyT>::view() const {
  BBView v;
  v.AR = ar_.as<const ulonglong2>();
  v.meta = meta_.as<const BBMeta>();
  v.levels = levels;
  v.nbins = nbins;
  return v;
}

template <class KeyT>
uint64_t BBHashBuild<KeyT>::level_words(uint32_t l) const {
  return l < nwords.size() ? nwords[l] : 0;
}

template struct BBHashBuild<uint64_t>;
template struct BBHashBuild<Key2>;

}  // namespace cf1
