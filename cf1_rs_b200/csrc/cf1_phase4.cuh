// Launchers of the phase-4 and MPHF-query kernels (cf1_phase4.cu).
#pragma once
#include "cf1_internal.cuh"

namespace cf1 {

template <class KeyT>
struct ClassifyArgs {
  const uint64_t *records;
  uint64_t n_rec;
  const uint64_t *W;
  const uint64_t *NM;
  uint64_t L;
  int k;
  MphfView<KeyT> mphf;
  unsigned long long *states;   // CAS mode: ceil(n_distinct/12) words, zeroed
  uint32_t *sides;              // side-set mode: 12 * ceil(n_distinct/12) bytes, zeroed; nullptr = CAS mode
  uint32_t *queue;              // persistent mode work counter (zeroed), else nullptr
  uint32_t *err;
  unsigned long long *cas_retries;
};

template <class KeyT>
void launch_classify(const ClassifyArgs<KeyT> &a, int persistent_ctas, cudaStream_t s);

// Phase 4 when phase 3 has joined the occurrences: the side-set byte left
// beside each distinct key (kept[sb_off[j] + i], i < cnt[j], for the
// sub-buckets j in [j0, j1) of 2^P per bin) goes to its vertex's slot --
// the key's rank (out_off[j] + i) in a bin the learned index serves, its
// BBHash slot in any other bin.  A slot outside the bin flags DEV_MPHF_MISS.
// The keys are read from the dense array (dense[out_off[j] + i]) when it is
// given, else from beside the bytes (kept[sb_off[j] + i]).
template <class KeyT>
void launch_place_sides(const MphfView<KeyT> &m, const KeyT *kept, const KeyT *dense, const uint8_t *kept_pay,
                        const uint64_t *sb_off, const uint32_t *cnt, const uint64_t *out_off, uint64_t j0, uint64_t j1,
                        int P, uint8_t *sides, uint32_t *err, cudaStream_t s);

// The same for the BBHash form whose levels 0 and 1 the dedup built
// (Level0Out with payloads): the keys level 0 places in sub-bucket j have
// the consecutive slots from its level-0 slice's first rank on, those level
// 1 places the ones from its level-1 slice's first rank on, and their bytes
// wait in rank order at l0pay[sb_off[j] ...] (level 0's placed[j], then
// level 1's placed1[j]) -- two contiguous copies each; the keys
// level 1 left (bin b's at surv[surv_off[b] ...], surv_cnt[b] of them, bytes
// beside them) walk the levels from 2.  Sub-buckets [j0, j1), bins [b0, b1).
void launch_place_l0(const BBView &bb, const uint64_t *dist_off, const uint64_t *sb_off, const uint32_t *placed,
                     const uint32_t *placed1, const uint8_t *l0pay, uint64_t j0, uint64_t j1, int P, uint8_t *sides,
                     uint32_t *err, cudaStream_t s);
void launch_place_surv(const BBView &bb, const uint64_t *dist_off, const uint64_t *surv, const uint8_t *surv_pay,
                       const uint64_t *surv_off, const unsigned long long *surv_cnt, uint32_t b0, uint32_t b1,
                       uint8_t *sides, uint32_t *err, cudaStream_t s);

// Packs side-set bytes (3 u32 per state word) into state words [w0, w1).
void launch_sideset_pack(const uint32_t *sides, uint64_t w0, uint64_t w1, unsigned long long *states,
                         cudaStream_t s);

template <class KeyT>
void launch_dump(const MphfView<KeyT> &m, uint32_t nbins, uint64_t n, const unsigned long long *states, uint64_t *keys_out,
                 uint8_t *states_out, cudaStream_t s);

template <class KeyT>
void launch_verify(const MphfView<KeyT> &m, uint32_t nbins, uint64_t n, uint32_t *seen, uint32_t *err, cudaStream_t s);

template <class KeyT>
void launch_query(const MphfView<KeyT> &m, const uint16_t *lut, int k, int mlen, const uint64_t *in, uint64_t n,
                  uint64_t *out, cudaStream_t s);

}  // namespace cf1
