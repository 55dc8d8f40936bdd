// Phase 3a in MSD form (cf1_msdsort.cu): per-bin multisplit on the top bits,
// shared-memory sort + unique of each sub-bucket.
#pragma once
#include "cf1_internal.cuh"

namespace cf1 {

struct MsdScratch {
  DevBuf tile_off, hist, hscan, scan_tmp, sb_off, sb_off1, cnt, out_off, flag, clist, ccount, coff, ov, ovc;
  uint32_t last_overflow = 0;  // sub-buckets the last unsorted run left to the block kernel
  cudaEvent_t ev[2] = {nullptr, nullptr};  // around the last dedup kernel launch
  float ms_dedup = 0;                      // its device time
  ~MsdScratch() {
    for (auto e : ev)
      if (e) cudaEventDestroy(e);
  }
};

// Top bits to split on so that the largest bin's sub-buckets hold about a
// third of the shared-memory capacity.
template <class KeyT>
int msd_prefix_bits(uint64_t max_bin_keys, bool sorted);

// keys: n keys segmented by bin (seg_off[0..nbins]); alt: n scratch keys.
// Writes the distinct keys of every bin to dist and their offsets to
// dist_off[0..nbins]: sorted within each bin, or (sorted = false) in
// sub-bucket order with any order inside a sub-bucket.  Returns false
// (nothing written) when a sub-bucket is larger than the shared-memory
// capacity; keys are then clobbered and the caller re-expands and takes the
// LSD path.
// Level 0 of the BBHash form, built by the unsorted (64-bit) dedup: with the
// sub-buckets split on the top P bits of key * KEY_SPREAD_MUL -- level 0's own
// hash -- and every bin's level-0 block a multiple of 2^P words, sub-bucket
// j of bin b owns words [j, j + 1) * (block / 2^P) of it alone, so its CTA
// marks, clears and writes them with no atomics in global memory and lists
// the keys it does not place.
// BBHash levels 0 and 1 built by the unsorted dedup: each sub-bucket j (bin
// b, slice sub) marks its keys in its slice of level 0 (sw0 words), and the
// keys level 0 leaves in its slice of level 1 (sw1 words; level 1 is sliced,
// see BBView); the keys level 1 leaves are listed for level 2.
struct Level0Out {
  ulonglong2 *AR = nullptr;                // level-0 entries (each slice writes all of its); nullptr: off
  const uint64_t *woff = nullptr;          // [nbins + 1] level-0 block offsets (sw0 << P words per bin)
  ulonglong2 *AR1 = nullptr;               // level-1 entries (each slice writes all of its)
  const uint64_t *woff1 = nullptr;         // [nbins + 1] level-1 block offsets (sw1 << P words per bin)
  uint64_t *surv = nullptr;                // keys level 1 leaves: bin b's from surv_off[b]
  const uint64_t *surv_off = nullptr;      // [nbins + 1]; bin b's room is surv_off[b+1] - surv_off[b]
  unsigned long long *surv_cnt = nullptr;  // [nbins], zeroed
  uint32_t *err = nullptr;                 // set when a slice or a bin's room is too small
  // Each slice's entries are written as {placed bits, placed bits of the
  // slice before the word}; placed[j] / placed1[j] = the keys level 0 / 1
  // places in sub-bucket j, from which the build turns the entries' ranks
  // into level-wide ones.
  uint32_t *placed = nullptr;   // [nsub]
  uint32_t *placed1 = nullptr;  // [nsub]
  // Joined side sets (payload bytes beside the keys): a key level 0 places
  // gets local rank r inside its slice (the set bits before its bit), and
  // its byte goes to l0pay[sub-bucket start + r]; a key level 1 places, rank
  // r1 in its level-1 slice, to l0pay[sub-bucket start + placed[j] + r1]; a
  // key level 1 leaves takes its byte along to surv_pay.
  bool with_pay = false;
  uint8_t *l0pay = nullptr;    // filled by msd_sort_unique: the payload buffer the kept bytes are not in
  uint8_t *surv_pay = nullptr; // beside surv
};

// With dist = nullptr the distinct keys stay where the dedup left them, at
// the start of each sub-bucket's range of *kept (keys or alt), and
// msd_compact writes dist later; dist_off is written either way.
// With pkeys/palt (one payload byte per key, beside keys and alt), each
// distinct key leaves with the OR of its copies' payloads at the same place
// of *kept_pay (pkeys or palt, beside *kept).
template <class KeyT>
bool msd_sort_unique(KeyT *keys, KeyT *alt, uint64_t n, const uint64_t *seg_off, uint32_t nbins, int key_bits, int P,
                     KeyT *dist, uint64_t *dist_off, MsdScratch &sc, cudaStream_t s, bool sorted = true,
                     const Level0Out *l0 = nullptr, KeyT **kept = nullptr, uint8_t *pkeys = nullptr,
                     uint8_t *palt = nullptr, uint8_t **kept_pay = nullptr, uint8_t **l0pay_buf = nullptr);

// The deferred copy: distinct keys of the last msd_sort_unique (nsub
// sub-buckets, left in `kept`) to dist, bins in order.
template <class KeyT>
void msd_compact(const KeyT *kept, uint64_t nsub, KeyT *dist, MsdScratch &sc, cudaStream_t s);

}  // namespace cf1
