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

// Keys of bin b at level 0: all its distinct keys when selected.
__global__ void bb_init_counts_kernel(const uint64_t *seg_off, const uint32_t *sel, uint32_t nbins, uint64_t *cnt) {
  uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nbins) cnt[b] = (sel == nullptr || sel[b]) ? seg_off[b + 1] - seg_off[b] : 0;
}

// Bits per key of a level: 8 at every level (ph::fmph uses gamma 2,
// src/mphf.rs:155-160).  A wide level places ~88% of its keys instead of
// ~61%, so a query -- and a warp of queries, which waits for its deepest
// lane -- walks fewer levels, and the build runs fewer.  At 2.7e9 keys the
// first level costs ~6.1 GB of HBM and the rest ~0.8 GB.  Measured at 3.1
// Gbp: 4 bits at level 0 ran phases 1-4 3% slower, 16 bits 1% slower (its
// first level's passes outweigh the shorter probes); 8 bits after level 0
// instead of 2 took the classification kernel from 50.9 to 46.3 ms and the
// build from 21.8 to 18.1 ms (16 levels down to 10).
constexpr uint32_t BB_GAMMA0 = 8, BB_GAMMA = 8;

// Words of each bin's block at this level (gamma bits per key, at least one
// word for a non-empty bin) and the level's totals {keys, words}.
__global__ void bb_sizes_kernel(const uint64_t *cnt, uint32_t nbins, uint32_t gamma, uint64_t *wcnt,
                                unsigned long long *tot) {
  uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  uint64_t n = 0, words = 0;
  if (b < nbins) {
    n = cnt[b];
    words = n ? (gamma * n + 63) / 64 : 0;
    wcnt[b] = words;
  }
  n = warp_sum(n);
  words = warp_sum(words);
  if (lane_id() == 0 && (n | words)) {
    atomicAdd(&tot[0], (unsigned long long)n);
    atomicAdd(&tot[1], (unsigned long long)words);
  }
}

// Marks every key's bit in this level's block of its bin.  The entry's rank
// half (y) collects the bits that more than one key set; AR points at this
// level's first entry and woff are the level-relative block offsets.  Keys
// of bin b are rem[start[b], start[b] + cnt[b]).
//
// When a tile's keys fall in a narrow stretch of the block -- at level 0 the
// unsorted phase-3 output is ordered by the same hash's top bits -- the tile
// marks a shared-memory copy of that stretch and merges it with one atomicOr
// per word (and one more per word with a collision) instead of one per key.
constexpr uint32_t BB_WIN = 2048;  // words of the shared-memory stretch
template <class KeyT>
__global__ void __launch_bounds__(BB_BLOCK) bb_mark_kernel(const KeyT *rem, const uint64_t *start, const uint64_t *cnt,
                                                           const uint32_t *tile_off, uint32_t nbins,
                                                           const uint64_t *woff, uint32_t level, ulonglong2 *AR) {
  __shared__ unsigned long long s_set[BB_WIN], s_col[BB_WIN];
  __shared__ unsigned long long s_lo, s_hi;
  const uint32_t t = blockIdx.x;
  if (t >= tile_off[nbins]) return;
  TileSpan sp = tile_span_gapped(start, cnt, tile_off, nbins, t, BB_TILE);
  const uint64_t w0 = woff[sp.seg];
  const uint32_t nw = (uint32_t)(woff[sp.seg + 1] - w0);
  if (threadIdx.x == 0) {
    s_lo = ~0ull;
    s_hi = 0;
  }
  __syncthreads();
  unsigned long long lo = ~0ull, hi = 0;
  for (uint64_t i = sp.start + threadIdx.x; i < sp.end; i += BB_BLOCK) {
    const unsigned long long wi = bb_pos(bb_key_hash(rem[i]), level, nw) >> 6;
    lo = wi < lo ? wi : lo;
    hi = wi > hi ? wi : hi;
  }
  atomicMin(&s_lo, lo);
  atomicMax(&s_hi, hi);
  __syncthreads();
  const uint64_t wlo = s_lo, span = s_hi >= s_lo ? s_hi - s_lo + 1 : 0;
  if (span > 0 && span <= BB_WIN) {
    for (uint32_t j = threadIdx.x; j < span; j += BB_BLOCK) s_set[j] = s_col[j] = 0;
    __syncthreads();
    for (uint64_t i = sp.start + threadIdx.x; i < sp.end; i += BB_BLOCK) {
      const uint64_t pos = bb_pos(bb_key_hash(rem[i]), level, nw);
      const uint32_t j = (uint32_t)((pos >> 6) - wlo);
      const unsigned long long bit = 1ull << (pos & 63);
      if (atomicOr(&s_set[j], bit) & bit) atomicOr(&s_col[j], bit);
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < span; j += BB_BLOCK) {
      const unsigned long long set = s_set[j];
      if (!set) continue;
      ulonglong2 *e = AR + w0 + wlo + j;
      const unsigned long long col = s_col[j] | (atomicOr(&e->x, set) & set);
      if (col) atomicOr(&e->y, col);
    }
    return;
  }
  for (uint64_t i = sp.start + threadIdx.x; i < sp.end; i += BB_BLOCK) {
    uint64_t pos = bb_pos(bb_key_hash(rem[i]), level, nw);
    ulonglong2 *e = AR + w0 + (pos >> 6);
    unsigned long long bit = 1ull << (pos & 63);
    unsigned long long old = atomicOr(&e->x, bit);
    if (old & bit) atomicOr(&e->y, bit);
  }
}

// Clears the bits set by more than one key; popcount per word for the ranks.
__global__ void bb_clean_kernel(ulonglong2 *AR, uint32_t *pc, uint64_t nw) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nw) {
    ulonglong2 e = AR[i];
    uint64_t a = e.x & ~e.y;
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

// A sliced level (levels 0 and 1 of the phase-3 dedup): each entry holds
// {placed bits, placed bits of its slice before it}; R = the exclusive scan
// of the slices' placed counts over the whole level (slices of bin b are
// [b << P, (b + 1) << P)).  srank[j] = the placed keys of slice j's bin
// before slice j; the bin's metadata takes the keys earlier levels placed as
// its rank adjustment.
__global__ void bb_srank_kernel(const uint64_t *R, int P, uint64_t nsub, uint32_t *srank) {
  const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j < nsub) srank[j] = (uint32_t)(R[j] - R[(j >> P) << P]);
}

__global__ void bb_meta_sliced_kernel(const uint64_t *woff, const uint64_t *R, int P, uint64_t level_base,
                                      uint64_t *base, BBMeta *meta, uint32_t nbins) {
  uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbins) return;
  const uint64_t r0 = R[(uint64_t)b << P], r1 = R[(uint64_t)(b + 1) << P];
  BBMeta m;
  m.word_off = level_base + woff[b];
  m.nwords = (uint32_t)(woff[b + 1] - woff[b]);
  m.rank_adj = (uint32_t)base[b];
  meta[b] = m;
  base[b] += r1 - r0;
}

// Keys whose bit did not survive go to the next level: each tile appends its
// survivors to out[start[b] + ...] behind one atomic on the bin's next count
// (the order of the keys inside a bin does not matter to BBHash).
template <class KeyT>
__global__ void __launch_bounds__(BB_BLOCK) bb_filter_kernel(const KeyT *rem, const uint64_t *start, const uint64_t *cnt,
                                                             const uint32_t *tile_off, uint32_t nbins,
                                                             const uint64_t *woff, uint32_t level, const ulonglong2 *AR,
                                                             unsigned long long *cnt_next, KeyT *out) {
  constexpr int ITEMS = BB_TILE / BB_BLOCK;
  __shared__ uint32_t sm[BB_BLOCK / 32];
  __shared__ unsigned long long s_base;
  const uint32_t t = blockIdx.x;
  if (t >= tile_off[nbins]) return;
  TileSpan sp = tile_span_gapped(start, cnt, tile_off, nbins, t, BB_TILE);
  const uint64_t w0 = woff[sp.seg];
  const uint32_t nw = (uint32_t)(woff[sp.seg + 1] - w0);
  uint64_t i0 = sp.start + (uint64_t)threadIdx.x * ITEMS;
  uint32_t flags = 0, c = 0;
#pragma unroll
  for (int j = 0; j < ITEMS; j++) {
    uint64_t i = i0 + j;
    bool keep = false;
    if (i < sp.end) {
      uint64_t pos = bb_pos(bb_key_hash(rem[i]), level, nw);
      keep = ((AR[w0 + (pos >> 6)].x >> (pos & 63)) & 1) == 0;
    }
    flags |= (uint32_t)keep << j;
    c += keep;
  }
  uint32_t tot;
  uint32_t pre = block_exclusive_scan<BB_BLOCK>(c, sm, tot);
  if (threadIdx.x == 0) s_base = tot ? atomicAdd(&cnt_next[sp.seg], (unsigned long long)tot) : 0;
  __syncthreads();
  uint64_t o = start[sp.seg] + s_base + pre;
#pragma unroll
  for (int j = 0; j < ITEMS; j++)
    if ((flags >> j) & 1) out[o++] = rem[i0 + j];
}

}  // namespace

template <class KeyT>
void BBHashBuild<KeyT>::clear() {
  nwords.clear();
  level_off.clear();
  total_words = 0;
  levels = 0;
  bytes = 0;
  l1_slice_bits = -1;
  srank_words = 0;
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
void BBHashBuild<KeyT>::begin(uint32_t nb, cudaStream_t s) {
  clear();
  nbins = nb;
  uint64_t *base = base_.get<uint64_t>(nbins);
  CF1_CUDA(cudaMemsetAsync(base, 0, nbins * sizeof(uint64_t), s));
  BBMeta *meta = meta_.get<BBMeta>((size_t)BB_MAX_LEVELS * nbins);
  CF1_CUDA(cudaMemsetAsync(meta, 0, (size_t)BB_MAX_LEVELS * nbins * sizeof(BBMeta), s));
  cnt_[0].get<uint64_t>(nbins);
  cnt_[1].get<uint64_t>(nbins);
  wcnt_.get<uint64_t>(nbins + 1);
  woff_.get<uint64_t>(nbins + 1);
  tile_off_.get<uint32_t>(nbins + 1);
  tot_.get<uint64_t>(2);
}

// Ranks and metadata of a level whose cleaned bits are in place: AR =
// entries [total_words, total_words + nw), woff = the bins' level-relative
// block offsets.
template <class KeyT>
void BBHashBuild<KeyT>::finish_level(uint32_t l, const uint64_t *woff, uint64_t nw, cudaStream_t s) {
  ulonglong2 *Al = ar_.as<ulonglong2>() + total_words;
  uint64_t *Rl = rtmp_.get<uint64_t>(nw + 1);
  uint32_t *pc = pc_.get<uint32_t>(nw);
  bb_clean_kernel<<<(unsigned)ceil_div(nw, 256), 256, 0, s>>>(Al, pc, nw);
  CF1_LAUNCH_CHECK();
  exclusive_scan_u32(pc, Rl, nw, scan_tmp_, s);
  bb_rank_kernel<<<(unsigned)ceil_div(nw, 256), 256, 0, s>>>(Al, Rl, nw);
  CF1_LAUNCH_CHECK();
  bb_meta_kernel<<<(unsigned)ceil_div(nbins, 256), 256, 0, s>>>(woff, Rl, total_words, base_.as<uint64_t>(),
                                                                meta_.as<BBMeta>() + (size_t)l * nbins, nbins);
  CF1_LAUNCH_CHECK();
}

// Levels l, l+1, ... until no key is left.  Level l's keys: bin b's are
// rem[start[b], start[b] + cnt_[l & 1][b]); each level writes the keys it
// does not place to r0 / r1 in turn at the same offsets.
template <class KeyT>
void BBHashBuild<KeyT>::run_levels(uint32_t l, const KeyT *rem, const uint64_t *start, KeyT *r0, KeyT *r1,
                                   cudaStream_t s) {
  KeyT *r[2] = {r0, r1};
  uint64_t *wcnt = wcnt_.as<uint64_t>(), *woff = woff_.as<uint64_t>();
  uint32_t *tile_off = tile_off_.as<uint32_t>();
  unsigned long long *tot = reinterpret_cast<unsigned long long *>(tot_.as<uint64_t>());
  for (;; l++) {
    uint64_t *cur = cnt_[l & 1].as<uint64_t>(), *nxt_cnt = cnt_[(l + 1) & 1].as<uint64_t>();
    CF1_CUDA(cudaMemsetAsync(tot, 0, 2 * sizeof(unsigned long long), s));
    bb_sizes_kernel<<<(unsigned)ceil_div(nbins, 256), 256, 0, s>>>(cur, nbins, l ? BB_GAMMA : BB_GAMMA0, wcnt, tot);
    CF1_LAUNCH_CHECK();
    uint64_t ht[2] = {0, 0};
    CF1_CUDA(cudaMemcpyAsync(ht, tot, sizeof(ht), cudaMemcpyDeviceToHost, s));
    CF1_CUDA(cudaStreamSynchronize(s));
    const uint64_t remaining = ht[0], nw = ht[1];
    if (remaining == 0) break;
    if (l >= BB_MAX_LEVELS) throw Error(CF1GPU_ERR_BIJECTION, "BBHash: keys left after the last level");
    exclusive_scan_u64(wcnt, woff, nbins, scan_tmp_, s);
    reserve_entries(total_words + nw, total_words, s);
    nwords.push_back(nw);
    level_off.push_back(total_words);
    ulonglong2 *Al = ar_.as<ulonglong2>() + total_words;
    CF1_CUDA(cudaMemsetAsync(Al, 0, nw * sizeof(ulonglong2), s));
    uint32_t ub = (uint32_t)(ceil_div(remaining, BB_TILE) + nbins);
    segment_tiles_counts(cur, nbins, BB_TILE, tile_off, s);
    bb_mark_kernel<KeyT><<<ub, BB_BLOCK, 0, s>>>(rem, start, cur, tile_off, nbins, woff, l, Al);
    CF1_LAUNCH_CHECK();
    finish_level(l, woff, nw, s);
    KeyT *out = r[l & 1];
    CF1_CUDA(cudaMemsetAsync(nxt_cnt, 0, nbins * sizeof(uint64_t), s));
    bb_filter_kernel<KeyT><<<ub, BB_BLOCK, 0, s>>>(rem, start, cur, tile_off, nbins, woff, l, Al,
                                                   reinterpret_cast<unsigned long long *>(nxt_cnt), out);
    CF1_LAUNCH_CHECK();
    total_words += nw;
    rem = out;
  }
  levels = l;
  bytes = total_words * sizeof(ulonglong2) + (size_t)levels * nbins * sizeof(BBMeta);
  CF1_CUDA(cudaStreamSynchronize(s));
}

template <class KeyT>
void BBHashBuild<KeyT>::build(const KeyT *keys, const uint64_t *seg_off, uint32_t nb, const uint32_t *sel,
                              cudaStream_t s, KeyT *ws0, KeyT *ws1, uint64_t ws_cap) {
  begin(nb, s);
  std::vector<uint64_t> hoff(nbins + 1);
  CF1_CUDA(cudaMemcpyAsync(hoff.data(), seg_off, (nbins + 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  CF1_CUDA(cudaStreamSynchronize(s));
  for (uint32_t b = 0; b < nbins; b++)  // local slots are 32-bit
    if (hoff[b + 1] - hoff[b] >= (1ull << 32))
      throw Error(CF1GPU_ERR_INVALID_ARG, "BBHash: a bin holds 2^32 or more distinct keys; use more bins");
  const uint64_t n_all = hoff[nbins];
  // Keys of bin b at every level sit at [seg_off[b], seg_off[b] + cnt[b]) of
  // the level's key array: the distinct keys at level 0, then the two
  // workspaces in turn (the caller's, when big enough).
  KeyT *r0 = (ws0 && ws_cap >= n_all + 1) ? ws0 : rem_[0].get<KeyT>(n_all + 1);
  KeyT *r1 = (ws1 && ws_cap >= n_all + 1) ? ws1 : rem_[1].get<KeyT>(n_all + 1);
  bb_init_counts_kernel<<<(unsigned)ceil_div(nbins, 256), 256, 0, s>>>(seg_off, sel, nbins, cnt_[0].as<uint64_t>());
  CF1_LAUNCH_CHECK();
  // room for the usual level sizes (gamma0 bits per key, then ~12% and
  // fewer keys per level) so that the entry array rarely grows in mid-build
  reserve_entries((BB_GAMMA0 * n_all / 64 + nbins) * 3 / 2 + 64 * nbins + 64, 0, s);
  run_levels(0, keys, seg_off, r0, r1, s);
}

template <class KeyT>
ulonglong2 *BBHashBuild<KeyT>::prepare_levels01(uint64_t words0, uint64_t words1, cudaStream_t s) {
  const uint64_t words = words0 + words1;
  reserve_entries(words + words / 4 + 64 * 1024, 0, s);
  return ar_.as<ulonglong2>();
}

template <class KeyT>
void BBHashBuild<KeyT>::finish_sliced(uint32_t l, const uint64_t *woff, const uint32_t *placed, int P,
                                      cudaStream_t s) {
  const uint64_t nsub = (uint64_t)nbins << P;
  uint64_t *R = rtmp_.get<uint64_t>(nsub + 1);
  exclusive_scan_u32(placed, R, nsub, scan_tmp_, s);
  bb_srank_kernel<<<(unsigned)ceil_div(nsub, 256), 256, 0, s>>>(R, P, nsub, srank_[l].get<uint32_t>(nsub + 1));
  CF1_LAUNCH_CHECK();
  bb_meta_sliced_kernel<<<(unsigned)ceil_div(nbins, 256), 256, 0, s>>>(
      woff, R, P, total_words, base_.as<uint64_t>(), meta_.as<BBMeta>() + (size_t)l * nbins, nbins);
  CF1_LAUNCH_CHECK();
}

template <class KeyT>
void BBHashBuild<KeyT>::build_from_levels01(uint32_t nb, int P, const uint64_t *woff0, uint64_t words0,
                                            const uint32_t *placed0, const uint64_t *woff1, uint64_t words1,
                                            const uint32_t *placed1, const KeyT *surv, const uint64_t *surv_off,
                                            const uint64_t *surv_cnt, uint64_t surv_total, cudaStream_t s, KeyT *ws0,
                                            KeyT *ws1, uint64_t ws_cap) {
  begin(nb, s);
  nwords.push_back(words0);
  level_off.push_back(0);
  finish_sliced(0, woff0, placed0, P, s);
  total_words = words0;
  nwords.push_back(words1);
  level_off.push_back(words0);
  finish_sliced(1, woff1, placed1, P, s);
  total_words += words1;
  l1_slice_bits = P;
  srank_words = (uint64_t)nbins << P;
  CF1_CUDA(cudaMemcpyAsync(cnt_[0].as<uint64_t>(), surv_cnt, nbins * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
  KeyT *r0 = (ws0 && ws_cap >= surv_total + 1) ? ws0 : rem_[0].get<KeyT>(surv_total + 1);
  KeyT *r1 = (ws1 && ws_cap >= surv_total + 1) ? ws1 : rem_[1].get<KeyT>(surv_total + 1);
  run_levels(2, surv, surv_off, r0, r1, s);  // level l reads cnt_[l & 1] and writes r[l & 1]
  levels = std::max<uint32_t>(levels, 2);
  bytes = total_words * sizeof(ulonglong2) + (size_t)levels * nbins * sizeof(BBMeta) + 2 * srank_words * sizeof(uint32_t);
}

template <class KeyT>
BBView BBHashBuild<KeyT>::view() const {
  BBView v;
  v.AR = ar_.as<const ulonglong2>();
  v.meta = meta_.as<const BBMeta>();
  v.levels = levels;
  v.nbins = nbins;
  v.l1_slice_bits = l1_slice_bits;
  v.pad = 0;
  v.srank[0] = l1_slice_bits >= 0 ? srank_[0].as<const uint32_t>() : nullptr;
  v.srank[1] = l1_slice_bits >= 0 ? srank_[1].as<const uint32_t>() : nullptr;
  return v;
}

template <class KeyT>
uint64_t BBHashBuild<KeyT>::level_words(uint32_t l) const {
  return l < nwords.size() ? nwords[l] : 0;
}

template struct BBHashBuild<uint64_t>;
template struct BBHashBuild<Key2>;

}  // namespace cf1
