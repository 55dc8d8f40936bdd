// Phase 3a in MSD form (cf1_msdsort.cu): per-bin multisplit on the top bits,
// shared-memory sort + unique of each sub-bucket.
#pragma once
#include "cf1_internal.cuh"

namespace cf1 {

struct MsdScratch {
  DevBuf tile_off, hist, hscan, scan_tmp, sb_off, sb_off1, cnt, out_off, flag;
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
template <class KeyT>
bool msd_sort_unique(KeyT *keys, KeyT *alt, uint64_t n, const uint64_t *seg_off, uint32_t nbins, int key_bits, int P,
                     KeyT *dist, uint64_t *dist_off, MsdScratch &sc, cudaStream_t s, bool sorted = true);

}  // namespace cf1
