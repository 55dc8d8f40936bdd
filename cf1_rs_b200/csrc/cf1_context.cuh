// The library context behind the C ABI (cf1gpu_ctx).
#pragma once
#include <string>
#include <utility>
#include <vector>

#include "../../include/cf1gpu.h"
#include "cf1_bbhash.cuh"
#include "cf1_internal.cuh"
#include "cf1_learned.cuh"
#include "cf1_msdsort.cuh"
#include "cf1_tuner.cuh"

namespace cf1 {

// Pinned host staging for the concatenated input.
struct PinnedBuf {
  uint8_t *p = nullptr;
  size_t cap = 0;
  PinnedBuf() = default;
  PinnedBuf(const PinnedBuf &) = delete;
  PinnedBuf &operator=(const PinnedBuf &) = delete;
  ~PinnedBuf() {
    if (p) cudaFreeHost(p);
  }
  // Grows to at least `bytes`, keeping the first `keep` bytes.
  void reserve(size_t bytes, size_t keep);
};

template <class KeyT>
struct Backend {
  SortScratch<KeyT> sort;
  MsdScratch msd;
  BBHashBuild<KeyT> bb;
  LearnedBuild<KeyT> li;
};

struct Tuning {
  uint32_t sk_tile = 2048;      // k-mer positions per minimizer tile (1024/2048/4096)
  int persistent_ctas = 0;      // 0: derived from the SM count in batched mode
  uint32_t leaf_size = 32;      // learned index keys per leaf
  int msd_delta = 0;            // added to the phase-3 MSD split width
};

}  // namespace cf1

struct cf1gpu_ctx {
  cf1gpu_opts opts;
  int k = 31, m = 15, w = 17;
  bool wide = false;  // k > 32: 128-bit keys
  std::string last_error;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;  // streamed runs: host<->device copies beside the kernels
  cudaEvent_t ev[12] = {};
  cudaEvent_t stage_ev[8] = {};        // streamed runs: a phase-4 stage's words are packed
  int num_sms = 148;
  cf1::Tuning tune;
  cf1::LearnedOpts learned;

  // host input: records concatenated, one placeholder after each
  cf1::PinnedBuf host;
  uint64_t L = 0;
  uint64_t n_records = 0;
  uint64_t n_bases = 0;
  std::vector<std::pair<std::string, uint64_t>> short_seqs;
  bool uploaded = false;
  // Leading bytes of the concatenation already on the device: records given
  // in page-locked host memory are copied there directly (no staging), the
  // rest wait in `host` for cf1gpu_upload.
  uint64_t dev_valid = 0;
  double ms_intake = 0;  // device time of those direct copies since the last upload
  bool ran = false;

  // device buffers
  cf1::DevBuf d_l0, d_l0surv, d_binfile, d_binimg, d_raw, d_intake, d_shard, d_ascii, d_W, d_NM, d_hist, d_lut, d_rec_off, d_small, d_cursor, d_records, d_kpre, d_lens, d_seg,
      d_keys, d_dist, d_dist_off, d_states, d_scan, d_seen, d_qin, d_qout, d_queue;
  // state_update 0: one side-set byte per key beside the sort's two key buffers
  cf1::DevBuf d_pay, d_pay_alt;
  // ... and, with BBHash level 0 built by the dedup, the bytes of the keys it
  // leaves and the placed count of every slice
  cf1::DevBuf d_l0survpay, d_l0placed;
  uint64_t rec_cap_hint = 0;  // phase-1 record list size of the last run
  // exchange-based sharding: the scanned slice's records wait in d_keys for
  // routing; d_xsend holds them grouped by owner shard, d_xcnt the counts
  cf1::DevBuf d_xsend, d_xcnt;
  int x_step = 0;              // 0 nothing pending, 1 slice scanned, 2 slice routed
  uint64_t x_local = 0;        // records of the scanned slice
  uint64_t x_rec_cap = 0;      // capacity of their list in d_keys
  double x_ms_scan = 0;        // device time of the slice's scan and routing
  uint64_t x_launches0 = 0;    // kernel launch count when the scan began
  // autotuner: cache file ("" = off), the key the current tuning is for
  std::string tuner_path;
  cf1::TuneKey tuned_key;
  bool tune_valid = false;
  int tuner_state = 0;  // last run: 0 off, 1 from the cache, 2 measured
  cf1::Backend<uint64_t> b64;
  cf1::Backend<cf1::Key2> b128;

  // results of the last run
  uint64_t n_super = 0, n_occ = 0, n_distinct = 0, n_bins_eff = 0, cas_retries = 0;
  // BBHash form: the distinct keys wait in their sub-buckets (dist_kept, one
  // of the sort buffers) until d_dist is asked for
  bool dist_pending = false;
  void *dist_kept = nullptr;
  uint64_t dist_nsub = 0;
  int msd_bits = 0;        // top bits split on by the MSD sort (-1: LSD path ran)
  bool force_lsd = false;  // opts.sort_mode == 1
  uint32_t nbins = 0;
  cf1gpu_stats stats{};
};

namespace cf1 {
template <class KeyT>
inline Backend<KeyT> &ctx_backend(cf1gpu_ctx *c);
template <>
inline Backend<uint64_t> &ctx_backend<uint64_t>(cf1gpu_ctx *c) { return c->b64; }
template <>
inline Backend<Key2> &ctx_backend<Key2>(cf1gpu_ctx *c) { return c->b128; }
}  // namespace cf1
