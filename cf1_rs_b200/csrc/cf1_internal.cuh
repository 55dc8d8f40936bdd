// Host-side plumbing shared by the kernels' launchers and the pipeline.
#pragma once
#include <atomic>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "cf1_common.cuh"

namespace cf1 {

// A failed CUDA call or a broken invariant inside the library; the C ABI turns
// it into a status code and a message.
struct Error : std::runtime_error {
  int status;
  Error(int st, const std::string &m) : std::runtime_error(m), status(st) {}
};

#define CF1_CUDA(call)                                                                 \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      throw ::cf1::Error(e_ == cudaErrorMemoryAllocation ? -2 : -3,                    \
                         std::string(#call) + ": " + cudaGetErrorString(e_));          \
  } while (0)

// Kernels launched by this library (every launch is followed by
// CF1_LAUNCH_CHECK, which counts it).
extern std::atomic<uint64_t> g_launches;
#define CF1_LAUNCH_CHECK()                                        \
  do {                                                            \
    ::cf1::g_launches.fetch_add(1, std::memory_order_relaxed);    \
    CF1_CUDA(cudaGetLastError());                                 \
  } while (0)

// Device allocation that grows on demand and keeps its capacity.
struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
  void *reserve(size_t bytes) {
    if (bytes <= cap && p) return p;
    release();
    size_t b = bytes ? bytes : 16;
    CF1_CUDA(cudaMalloc(&p, b));
    cap = b;
    return p;
  }
  template <class T>
  T *as() const { return static_cast<T *>(p); }
  template <class T>
  T *get(size_t n) { return static_cast<T *>(reserve(n * sizeof(T))); }
  // Grows to at least `bytes` (by a quarter more), keeping the first `keep`
  // bytes; synchronises the stream when it moves them.
  void *reserve_keep(size_t bytes, size_t keep, cudaStream_t s) {
    if (bytes <= cap && p) return p;
    size_t b = bytes + bytes / 4 + 16;
    void *np = nullptr;
    CF1_CUDA(cudaMalloc(&np, b));
    if (keep && p) {
      CF1_CUDA(cudaMemcpyAsync(np, p, keep, cudaMemcpyDeviceToDevice, s));
      CF1_CUDA(cudaStreamSynchronize(s));
    }
    release();
    p = np;
    cap = b;
    return p;
  }
};

inline uint64_t ceil_div(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

// CTAs of a persistent (work-queue) launch: `requested` when positive, else
// one full wave -- the CTAs of `kernel` resident per SM times the SMs; never
// more than `items` work items.
template <class Kernel>
unsigned persistent_grid(Kernel kernel, int block, size_t smem, int requested, uint64_t items) {
  uint64_t g;
  if (requested > 0) {
    g = (uint64_t)requested;
  } else {
    int dev = 0, sms = 0, per_sm = 0;
    CF1_CUDA(cudaGetDevice(&dev));
    CF1_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CF1_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem));
    g = (uint64_t)(per_sm > 0 ? per_sm : 1) * (uint64_t)sms;
  }
  if (g > items) g = items;
  return (unsigned)(g ? g : 1);
}

// ------------------------------------------------------------ util kernels ----
// Exclusive prefix sum of n values into out[0..n] (out[n] = total).
// `scratch` grows as needed.
void exclusive_scan_u32(const uint32_t *in, uint64_t *out, uint64_t n, DevBuf &scratch, cudaStream_t s);
void exclusive_scan_u64(const uint64_t *in, uint64_t *out, uint64_t n, DevBuf &scratch, cudaStream_t s);

// Tiles of TILE elements over segments given by seg_off[0..nseg]; a tile never
// crosses a segment edge.  tile_off[0..nseg] (u32) gets the first tile of each
// segment; tile_off[nseg] is the tile count.
void segment_tiles(const uint64_t *seg_off, uint32_t nseg, uint32_t tile, uint32_t *tile_off, cudaStream_t s);
// The same over gapped segments given by item counts cnt[0..nseg).
void segment_tiles_counts(const uint64_t *cnt, uint32_t nseg, uint32_t tile, uint32_t *tile_off, cudaStream_t s);

// ------------------------------------------------------------ phase kernels ----
void launch_pack(const uint8_t *ascii, uint64_t L, uint64_t *W, uint64_t *NM, cudaStream_t s);
// The same for the W/NM words [w0, w1) only (64 bases per word of NM).
void launch_pack_words(const uint8_t *ascii, uint64_t L, uint64_t *W, uint64_t *NM, uint64_t w0, uint64_t w1,
                       cudaStream_t s);

struct SuperkmerArgs {
  const uint64_t *W;
  const uint64_t *NM;
  uint64_t L;
  int k, m, w;
  uint32_t tile;          // k-mer positions per tile
  uint64_t n_tiles;       // tiles [tile_begin, n_tiles) of this launch
  uint64_t tile_begin;    // first tile (one CTA per tile from here; 0 in persistent mode)
  uint32_t *tile_counter; // persistent mode: atomic work queue (zeroed); nullptr = one CTA per tile
  uint32_t *hist;         // [65536] super k-mers per bucket (zeroed)
  unsigned long long *n_kmers;    // valid k-mer windows (zeroed)
  uint64_t *rec_tmp;      // unordered super k-mers (rec_pack with bin 0) ...
  uint16_t *rec_bucket;   // ... and their histogram buckets
  unsigned long long *rec_count;  // records produced (zeroed); only the first rec_cap are stored
  uint64_t rec_cap;
  uint32_t *err;
};
// The default k (31, with m = 15 and w = 17 by src/params.rs:221-228) gets a
// minimizer scan with k, m and w as compile-time constants (phase 1 27.3 ->
// 24.4 ms at 3.1 Gbp); other k run the same code with them read at run
// time.  (The same for the classification and expansion kernels measured
// slower or no faster: their register allocation changed.)
constexpr int K_FIXED = 31, M_FIXED = 15, W_FIXED = 17;
// Phase 1: minimizer histogram + unordered super k-mer list.
void launch_superkmer_scan(const SuperkmerArgs &a, int persistent_ctas, cudaStream_t s);
// Phase 2: route the list into per-bin ranges rec_off[0..num_bins] of records
// (rec_bucket nullptr: the records already carry their bin).
void launch_bin_scatter(const uint64_t *rec_tmp, const uint16_t *rec_bucket, uint64_t n, const uint16_t *lut,
                        uint32_t num_bins, const uint64_t *rec_off, uint32_t *cursor, uint64_t *records, uint32_t *err,
                        cudaStream_t s);
// Greedy partition of the histogram (src/minimizer.rs:116-172) into the
// bucket->bin table, plus per-bin record offsets rec_off[0..num_bins].
void launch_partition(const uint32_t *hist, uint32_t num_bins, uint16_t *lut, uint64_t *rec_off, uint32_t *n_bins_eff,
                      cudaStream_t s);

// ------------------------------------------------------------ phase 3 ----
template <class KeyT>
struct SortScratch {
  DevBuf alt, hist, hscan, tile_off, tile_cnt, tile_out, scan_tmp;
};

// Per record k-mer offsets: kpre[i] = sum of n over records < i (kpre[n_rec] = total).
void record_kmer_prefix(const uint64_t *records, uint64_t n_rec, uint64_t *kpre, DevBuf &lens, DevBuf &scratch,
                        cudaStream_t s);

// Writes each k-mer's canonical form; keys[kpre[i] + j] is k-mer j of record
// i.  Writes past n_keys or reads past base L are skipped and flagged in err.
template <class KeyT>
void launch_expand(const uint64_t *records, uint64_t n_rec, const uint64_t *kpre, const uint64_t *W, int k, KeyT *keys,
                   uint64_t n_keys, uint64_t L, uint32_t *queue, uint32_t *err, int persistent_ctas, cudaStream_t s,
                   const uint64_t *NM = nullptr, uint8_t *sides = nullptr);

// Sorts each segment [seg_off[b], seg_off[b+1]) of keys ascending (LSD radix,
// segmented).  The result is in `keys` on return.
template <class KeyT>
void segmented_sort(KeyT *keys, uint64_t n, const uint64_t *seg_off, uint32_t nseg, int key_bits, SortScratch<KeyT> &sc,
                    cudaStream_t s);

// Adjacent-unique per segment: writes distinct keys to `out` and their segment
// offsets to out_off[0..nseg].
template <class KeyT>
void segmented_unique(const KeyT *keys, uint64_t n, const uint64_t *seg_off, uint32_t nseg, KeyT *out, uint64_t *out_off,
                      SortScratch<KeyT> &sc, cudaStream_t s);

// ------------------------------------------------------------ MPHF ----
// One (level, bin) block of a per-bin BBHash; 16 bytes, one load per probe.
struct __align__(16) BBMeta {
  uint64_t word_off;  // first entry of the block in the entry array (all levels)
  uint32_t nwords;    // block size in 64-bit words (0: bin has no keys at this level)
  uint32_t rank_adj;  // bin-local slot base minus the level rank at word_off (mod 2^32; bins hold < 2^32 keys)
};

// Device view of a per-bin BBHash (read by query kernels).  All levels share
// one array of {bit word, exclusive popcount of the level before it}
// entries: one 16-byte load gives a probe both the bit and the rank.
struct BBView {
  const ulonglong2 *AR;  // {cleaned bit word, level rank}, levels back to back
  const BBMeta *meta;    // [levels * nbins]
  uint32_t levels, nbins;
  // >= 0: levels 0 and 1 were built by the phase-3 dedup, one slice per
  // sub-bucket: a bin's block of either level is 2^l1_slice_bits slices of
  // equal size, and a key's bit lies in the slice its level-0 hash's top
  // l1_slice_bits bits name (level 0's bit is its hash scaled to the block,
  // level 1's its own hash scaled to the slice).  Their entries' rank halves
  // count the placed bits of the slice before the word, srank[l][slice] the
  // placed bits of the bin's slices before it, and a bin's rank_adj is the
  // keys its earlier levels placed.  -1: every level hashes over its bin's
  // whole block and the entries hold level-wide ranks.
  int32_t l1_slice_bits;
  uint32_t pad;
  const uint32_t *srank[2];  // [nbins << l1_slice_bits] each, when sliced
};

constexpr int LI_HIDDEN = 16;
// The trained root, stored as the piecewise-linear function it computes: the
// hidden ramps tile [0, 1] (ramp j over [knot[j], knot[j+1])), so on piece j
// every earlier ramp is saturated and every later one is 0, and
// root(x) = base[j] + slope[j] * (x - knot[j]).
struct LIRoot {
  float knot[LI_HIDDEN], base[LI_HIDDEN], slope[LI_HIDDEN];
  uint64_t hmin;     // high64 of the bin's smallest key
  float inv_range;   // 1 / (high64(max) - high64(min))
  uint32_t n_leaves; // leaves of this bin
  uint64_t leaf_off; // first leaf of this bin in the leaf table
  uint32_t use_learned;  // 0: bin served by BBHash
  uint32_t max_err;
};
struct LILeaf {
  uint64_t hfirst;   // high64 of the leaf's first key
  uint32_t first_rank;
  uint32_t err;      // max |prediction - rank| over the leaf's keys
  float slope;       // ranks per unit of high64
  uint32_t n;        // keys routed to the leaf (0: empty)
};
struct LIView {
  const LIRoot *roots;  // [nbins]
  const LILeaf *leaves;
  int k;
};

// Everything a slot query needs: bin -> local slot, then + dist_off[bin].
template <class KeyT>
struct MphfView {
  const KeyT *keys;        // distinct keys, bins in order, each bin sorted
  const uint64_t *dist_off;  // [nbins+1]
  BBView bb;
  LIView li;
  int learned;             // 0: BBHash for every bin
};

}  // namespace cf1
