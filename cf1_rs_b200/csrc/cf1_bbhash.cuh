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

  BBHashBuild() = default;
  BBHashBuild(const BBHashBuild &) = delete;
  BBHashBuild &operator=(const BBHashBuild &) = delete;

  // Builds over the bins with sel[b] != 0 (sel == nullptr: every bin); the
  // other bins get no levels.  Synchronises the stream between levels.
  // ws0/ws1 (optional, ws_cap keys each, not aliasing keys) hold the keys
  // still unplaced between levels; without them the builder allocates.
  void build(const KeyT *keys, const uint64_t *seg_off, uint32_t nbins, const uint32_t *sel, cudaStream_t s,
             KeyT *ws0 = nullptr, KeyT *ws1 = nullptr, uint64_t ws_cap = 0);
  BBView view() const;
  void clear();
  uint64_t level_words(uint32_t l) const;
  const BBMeta *meta_device() const { return meta_.as<const BBMeta>(); }
  // {bit word, level rank} entries of all levels (total_words of them)
  const ulonglong2 *entries_device() const { return ar_.as<const ulonglong2>(); }

 private:
  // Grows the entry array to hold `words` entries, keeping the first `keep`.
  void reserve_entries(uint64_t words, uint64_t keep, cudaStream_t s);

  // The entry array and the level buffers are kept across builds and grown on
  // demand, so a rebuild allocates nothing once sizes settle.
  DevBuf ar_, meta_, base_, rem_[2], cnt_[2], tot_, tile_off_, wcnt_, woff_, pc_, rtmp_, scan_tmp_;
};

}  // namespace cf1
