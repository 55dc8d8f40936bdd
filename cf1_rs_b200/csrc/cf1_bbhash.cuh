// Host-side owner of a per-bin BBHash (built by cf1_bbhash.cu).
#pragma once
#include "cf1_internal.cuh"

namespace cf1 {

template <class KeyT>
struct BBHashBuild {
  std::vector<uint64_t> nwords;    // words of each level in use
  std::vector<uint64_t> level_off; // first entry of each level in the entry array
  uint64_t total_words = 0;        // entries of all levels
  uint32_t levels = 0, nbins = 0;
  uint64_t bytes = 0;
  int l1_slice_bits = -1;          // see BBView
  uint64_t srank_words = 0;        // entries of each sliced level's srank table

  BBHashBuild() = default;
  BBHashBuild(const BBHashBuild &) = delete;
  BBHashBuild &operator=(const BBHashBuild &) = delete;

  // Builds over the bins with sel[b] != 0 (sel == nullptr: every bin); the
  // other bins get no levels.  Synchronises the stream between levels.
  // ws0/ws1 (optional, ws_cap keys each, not aliasing keys) hold the keys
  // still unplaced between levels; without them the builder allocates.
  void build(const KeyT *keys, const uint64_t *seg_off, uint32_t nbins, const uint32_t *sel, cudaStream_t s,
             KeyT *ws0 = nullptr, KeyT *ws1 = nullptr, uint64_t ws_cap = 0);
  // Levels 0 and 1 built elsewhere (the unsorted phase-3 dedup, one
  // exclusive slice of each per sub-bucket; level 1 sliced, see BBView):
  // prepare_levels01 gives the entry array to fill with level 0's cleaned
  // bit words at [0, words0) and level 1's at [words0, words0 + words1), as
  // {bits, placed bits of the slice before the word}; build_from_levels01
  // ranks both from the slices' placed counts (placed0 / placed1, one per
  // sub-bucket) and builds the later levels over the keys level 1 left (bin
  // b's at surv[surv_off[b] + [0, surv_cnt[b])]).  woff0 / woff1: the bins'
  // block offsets [nbins + 1] of levels 0 and 1; P: the slice bits.
  ulonglong2 *prepare_levels01(uint64_t words0, uint64_t words1, cudaStream_t s);
  void build_from_levels01(uint32_t nbins, int P, const uint64_t *woff0, uint64_t words0, const uint32_t *placed0,
                           const uint64_t *woff1, uint64_t words1, const uint32_t *placed1, const KeyT *surv,
                           const uint64_t *surv_off, const uint64_t *surv_cnt, uint64_t surv_total, cudaStream_t s,
                           KeyT *ws0 = nullptr, KeyT *ws1 = nullptr, uint64_t ws_cap = 0);
  BBView view() const;
  void clear();
  uint64_t level_words(uint32_t l) const;
  const BBMeta *meta_device() const { return meta_.as<const BBMeta>(); }
  // {bit word, level rank} entries of all levels (total_words of them)
  const ulonglong2 *entries_device() const { return ar_.as<const ulonglong2>(); }
  // per-slice start ranks of sliced level l (srank_words of them)
  const uint32_t *srank_device(int l) const { return srank_[l].as<const uint32_t>(); }

 private:
  // Grows the entry array to hold `words` entries, keeping the first `keep`.
  void reserve_entries(uint64_t words, uint64_t keep, cudaStream_t s);
  void begin(uint32_t nbins, cudaStream_t s);
  void finish_level(uint32_t l, const uint64_t *woff, uint64_t nw, cudaStream_t s);
  void finish_sliced(uint32_t l, const uint64_t *woff, const uint32_t *placed, int P, cudaStream_t s);
  void run_levels(uint32_t l, const KeyT *rem, const uint64_t *start, KeyT *r0, KeyT *r1, cudaStream_t s);

  // The entry array and the level buffers are kept across builds and grown on
  // demand, so a rebuild allocates nothing once sizes settle.
  DevBuf ar_, meta_, base_, rem_[2], cnt_[2], tot_, tile_off_, wcnt_, woff_, pc_, rtmp_, scan_tmp_, srank_[2];
};

}  // namespace cf1
