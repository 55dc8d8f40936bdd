// Orchestration of phases 1-4 (src/pipeline.rs:66-105) and the C ABI.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <thread>

#include "cf1_context.cuh"
#include "cf1_device_util.cuh"
#include "cf1_mphf.cuh"
#include "cf1_phase4.cuh"
#include "cf1_pipeline.cuh"

using cf1::DevBuf;
using cf1::Error;
using cf1::Key2;

namespace cf1 {

void PinnedBuf::reserve(size_t bytes, size_t keep) {
  if (bytes <= cap) return;
  size_t ncap = std::max(bytes, cap + cap / 2);
  uint8_t *np = nullptr;
  CF1_CUDA(cudaHostAlloc((void **)&np, ncap, cudaHostAllocDefault));
  if (p) {
    if (keep) std::memcpy(np, p, keep);
    cudaFreeHost(p);
  }
  p = np;
  cap = ncap;
}

namespace {

// Small device counters of one run.
struct Small {
  unsigned long long n_kmers;
  unsigned long long cas_retries;
  unsigned long long rec_count;
  uint32_t err;
  uint32_t n_bins_eff;
  uint32_t l0_err;  // the phase-3 dedup could not build BBHash level 0
  uint32_t queues[8];
};

__global__ void seg_gather_kernel(const uint64_t *kpre, const uint64_t *rec_off, uint32_t nbins, uint64_t *seg) {
  uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b <= nbins) seg[b] = kpre[rec_off[b]];
}

// Bin sharding: records of the bins this shard keeps (b % shards == idx).
__global__ void shard_counts_kernel(const uint64_t *rec_off, uint32_t nbins, uint32_t idx, uint32_t shards,
                                    uint64_t *cnt) {
  uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nbins) cnt[b] = b % shards == idx ? rec_off[b + 1] - rec_off[b] : 0;
}

constexpr uint32_t SH_TILE = 4096;
__global__ void shard_copy_kernel(const uint64_t *in, const uint64_t *rec_off, const uint32_t *tile_off, uint32_t nbins,
                                  uint32_t idx, uint32_t shards, const uint64_t *new_off, uint64_t *out) {
  const uint32_t t = blockIdx.x;
  if (t >= tile_off[nbins]) return;
  TileSpan sp = tile_span(rec_off, tile_off, nbins, t, SH_TILE);
  if (sp.seg % shards != idx) return;
  const uint64_t delta = new_off[sp.seg] - rec_off[sp.seg];
  for (uint64_t i = sp.start + threadIdx.x; i < sp.end; i += blockDim.x) out[i + delta] = in[i];
}

// Exchange-based sharding.  Route: the scanned slice's records, tagged with
// their bins, grouped by owner shard (bin % shards); a CTA counts its records
// per owner in shared memory and reserves each owner's places with one atomic.
constexpr int XR_BLOCK = 256, XR_ITEMS = 8;
__global__ void __launch_bounds__(XR_BLOCK) xroute_count_kernel(const uint16_t *bucket, uint64_t n, const uint16_t *lut,
                                                                uint32_t shards, unsigned long long *cnt) {
  extern __shared__ uint32_t xr_cnt[];  // [shards]
  for (uint32_t i = threadIdx.x; i < shards; i += XR_BLOCK) xr_cnt[i] = 0;
  __syncthreads();
  for (uint64_t r = (uint64_t)blockIdx.x * XR_BLOCK + threadIdx.x; r < n; r += (uint64_t)gridDim.x * XR_BLOCK)
    atomicAdd(&xr_cnt[lut[bucket[r]] % shards], 1u);
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < shards; i += XR_BLOCK)
    if (xr_cnt[i]) atomicAdd(&cnt[i], (unsigned long long)xr_cnt[i]);
}

__global__ void __launch_bounds__(XR_BLOCK) xroute_scatter_kernel(const uint64_t *rec, const uint16_t *bucket, uint64_t n,
                                                                  const uint16_t *lut, uint32_t shards,
                                                                  const uint64_t *off, unsigned long long *cursor,
                                                                  uint64_t *out, uint32_t *err) {
  extern __shared__ uint64_t xr_base[];  // [shards], then the counts
  uint32_t *s_cnt = reinterpret_cast<uint32_t *>(xr_base + shards);
  for (uint32_t i = threadIdx.x; i < shards; i += XR_BLOCK) s_cnt[i] = 0;
  __syncthreads();
  const uint64_t r0 = (uint64_t)blockIdx.x * XR_BLOCK * XR_ITEMS;
  uint32_t bin[XR_ITEMS], li[XR_ITEMS];
#pragma unroll
  for (int i = 0; i < XR_ITEMS; i++) {
    const uint64_t r = r0 + (uint64_t)i * XR_BLOCK + threadIdx.x;
    bin[i] = 0xFFFFFFFFu;
    if (r < n) {
      bin[i] = lut[bucket[r]];
      li[i] = atomicAdd(&s_cnt[bin[i] % shards], 1u);
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < XR_ITEMS; i++) {
    if (bin[i] == 0xFFFFFFFFu || li[i]) continue;
    const uint32_t d = bin[i] % shards;
    xr_base[d] = off[d] + atomicAdd(&cursor[d], (unsigned long long)s_cnt[d]);
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < XR_ITEMS; i++) {
    if (bin[i] == 0xFFFFFFFFu) continue;
    const uint32_t d = bin[i] % shards;
    const uint64_t r = r0 + (uint64_t)i * XR_BLOCK + threadIdx.x, t = rec[r], idx = xr_base[d] + li[i];
    if (idx < off[d + 1]) out[idx] = rec_pack(rec_pos(t), rec_n(t), bin[i]);
    else atomicOr(err, (uint32_t)DEV_OVERFLOW);
  }
}

// Finish: records per bin of the records this shard received; a record of
// another shard's bin, or one reaching past the input, is refused.
__global__ void __launch_bounds__(XR_BLOCK) xrecv_count_kernel(const uint64_t *rec, uint64_t n, uint32_t nbins,
                                                               uint32_t idx, uint32_t shards, uint64_t L, int k,
                                                               unsigned long long *cnt, uint32_t *err) {
  extern __shared__ uint32_t xr_cnt[];  // [nbins]
  for (uint32_t b = threadIdx.x; b < nbins; b += XR_BLOCK) xr_cnt[b] = 0;
  __syncthreads();
  for (uint64_t r = (uint64_t)blockIdx.x * XR_BLOCK + threadIdx.x; r < n; r += (uint64_t)gridDim.x * XR_BLOCK) {
    const uint64_t x = rec[r];
    const uint32_t b = rec_bin(x);
    if (b >= nbins || b % shards != idx || rec_pos(x) + rec_n(x) + (uint64_t)k - 1 > L) atomicOr(err, (uint32_t)DEV_FOREIGN);
    else atomicAdd(&xr_cnt[b], 1u);
  }
  __syncthreads();
  for (uint32_t b = threadIdx.x; b < nbins; b += XR_BLOCK)
    if (xr_cnt[b]) atomicAdd(&cnt[b], (unsigned long long)xr_cnt[b]);
}

unsigned stride_grid(uint64_t n, int num_sms) {
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(ceil_div(n, XR_BLOCK), (uint64_t)num_sms * 8));
}

template <class KeyT>
Backend<KeyT> &backend(cf1gpu_ctx *c) {
  return ctx_backend<KeyT>(c);
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0;
  CF1_CUDA(cudaEventElapsedTime(&ms, a, b));
  return ms;
}

void check_device_errors(uint32_t err) {
  if (err & DEV_CAS_LIMIT) throw Error(CF1GPU_ERR_DEVICE_TIMEOUT, "phase 4: a state CAS loop passed its bound");
  if (err & DEV_WAIT_LIMIT) throw Error(CF1GPU_ERR_DEVICE_TIMEOUT, "a bounded device wait gave up");
  if (err & DEV_OVERFLOW) throw Error(CF1GPU_ERR_QUEUE_OVERRUN, "a device buffer bound was hit");
  if (err & DEV_MPHF_MISS) throw Error(CF1GPU_ERR_BIJECTION, "phase 4: a k-mer was not found by the MPHF");
  if (err & DEV_BIJECTION) throw Error(CF1GPU_ERR_BIJECTION, "MPHF is not a bijection onto [0, n)");
  if (err & DEV_FOREIGN)
    throw Error(CF1GPU_ERR_INVALID_ARG, "a received record is not this shard's (bin, position or length out of range)");
}

template <class KeyT>
MphfView<KeyT> make_view(cf1gpu_ctx *c) {
  Backend<KeyT> &be = backend<KeyT>(c);
  MphfView<KeyT> v;
  v.keys = c->d_dist.as<const KeyT>();
  v.dist_off = c->d_dist_off.as<const uint64_t>();
  v.bb = be.bb.view();
  v.learned = c->opts.mphf_mode == CF1GPU_MPHF_LEARNED;
  v.li = be.li.view(c->k);
  return v;
}

// Direct intake of records given in page-locked host memory: one DMA of the
// caller's bytes into a device buffer, then tiles of it are moved to their
// places in the concatenation, a placeholder after each record.
struct IntakeTile {
  uint64_t src, dst;
  uint32_t len, last;  // last: the tile ends its record
};
constexpr uint32_t INTAKE_TILE = 1u << 16;

__global__ void intake_kernel(const uint8_t *raw, const IntakeTile *tiles, uint8_t *out) {
  const IntakeTile t = tiles[blockIdx.x];
  for (uint32_t i = threadIdx.x; i < t.len; i += blockDim.x) out[t.dst + i] = raw[t.src + i];
  if (t.last && threadIdx.x == 0) out[t.dst + t.len] = 'N';
}

// The host ends of a streamed run (cf1gpu_run_streamed).  In: the caller's
// record bytes arrive in d_raw chunk by chunk on the copy stream; phase 1
// places, packs and scans each stretch as soon as its chunk is in.  Out:
// phase 4 runs in stages of whole bins, and the state words every stage
// completes go back to the caller on the copy stream while the next stage
// classifies.
struct StreamIO {
  const uint8_t *raw = nullptr;            // device copy of the record bytes
  const IntakeTile *tiles = nullptr;       // device intake tiles, in source order
  std::vector<IntakeTile> htiles;          // the same on the host
  std::vector<uint64_t> chunk_end;         // raw bytes in place after chunk c
  std::vector<cudaEvent_t> chunk_ev;       // recorded on the copy stream after chunk c
  uint64_t *host_words = nullptr;          // caller's state-word buffer
  uint64_t host_cap = 0;                   // its size in words
  bool words_done = false;                 // the run copied all words back
};
constexpr int STREAM_STAGES = 8;

// One run of phases 1-4 (FULL), or one of the two device steps of an
// exchange-sharded run: XSCAN is phase 1 over this shard's slice of the
// minimizer tiles (the histogram goes to the caller, the records wait for
// routing); XFINISH runs phases 2-4 on the records the shards routed here.
enum class Step { FULL, XSCAN, XFINISH };
struct XShard {
  uint32_t *hist_out = nullptr;    // XSCAN: the slice's histogram (host or device memory)
  const uint64_t *recv = nullptr;  // XFINISH: received records (host or device memory)
  uint64_t n_recv = 0;
};

template <class KeyT>
void run_impl(cf1gpu_ctx *c, StreamIO *io = nullptr, Step step = Step::FULL, const XShard *xs = nullptr) {
  cudaStream_t s = c->stream;
  Backend<KeyT> &be = backend<KeyT>(c);
  const uint64_t L = c->L;
  const int k = c->k;
  const uint32_t B = c->opts.num_bins;
  const bool batched = c->opts.batched != 0;
  const uint32_t shards = c->opts.shard_count > 1 ? c->opts.shard_count : 1;
  c->nbins = B;
  c->dist_pending = false;  // the sort buffers are about to be reused
  const uint64_t launches0 = step == Step::XFINISH ? c->x_launches0 : g_launches.load();
  // The learned index needs each bin's keys sorted; BBHash needs them
  // distinct (128-bit keys always take the sorted path).
  const bool sorted = c->opts.mphf_mode == CF1GPU_MPHF_LEARNED || c->opts.sort_mode == 1 || KOps<KeyT>::WORDS == 2;
  // autotuner: parameters of this input class from the cache, or measured
  // in this run and stored
  bool tune_now = false;  // (streamed runs do not measure: their phase 1 waits on the input)
  TuneValue tuned;
  tuned.sk_tile = c->tune.sk_tile;
  c->tuner_state = 0;
  if (!c->tuner_path.empty()) {
    TuneKey key;
    key.wide = c->wide;
    key.sorted = sorted;
    key.batched = batched;
    for (uint64_t x = L; x > 1; x >>= 1) key.size_class++;
    TuneValue v;
    if (c->tune_valid && c->tuned_key == key) {
      c->tuner_state = 1;
    } else if (tuner_lookup(c->tuner_path, key, v)) {
      if (c->opts.sk_tile == 0) c->tune.sk_tile = v.sk_tile;
      c->tune.msd_delta = v.msd_delta;
      c->tuned_key = key;
      c->tune_valid = true;
      c->tuner_state = 1;
    } else if (!io && step == Step::FULL) {
      c->tuned_key = key;
      c->tune_valid = false;
      tune_now = true;
    }
  }
  Small *sm = c->d_small.get<Small>(1);
  CF1_CUDA(cudaMemsetAsync(sm, 0, sizeof(Small), s));
  CF1_CUDA(cudaEventRecord(c->ev[0], s));

  // ---- phase 1: pack, minimizer histogram, partition
  uint64_t n_nm = ceil_div(L, 64);
  uint64_t *W = c->d_W.get<uint64_t>(2 * n_nm + 4);
  uint64_t *NM = c->d_NM.get<uint64_t>(n_nm + 2);
  CF1_CUDA(cudaMemsetAsync(W + 2 * n_nm, 0, 4 * sizeof(uint64_t), s));
  CF1_CUDA(cudaMemsetAsync(NM + n_nm, 0xFF, 2 * sizeof(uint64_t), s));
  if (!io && step != Step::XFINISH) launch_pack(c->d_ascii.as<uint8_t>(), L, W, NM, s);
  uint32_t *hist = c->d_hist.get<uint32_t>(NUM_BUCKETS);
  SuperkmerArgs a{};
  a.W = W;
  a.NM = NM;
  a.L = L;
  a.k = k;
  a.m = c->m;
  a.w = c->w;
  a.hist = hist;
  a.n_kmers = &sm->n_kmers;
  a.rec_count = &sm->rec_count;
  a.err = &sm->err;
  // persistent launches: the tuned CTA count, else one full wave (-1)
  int pctas = batched ? (c->tune.persistent_ctas > 0 ? c->tune.persistent_ctas : -1) : 0;
  a.tile_counter = batched ? &sm->queues[0] : nullptr;
  uint16_t *lut = c->d_lut.get<uint16_t>(NUM_BUCKETS);
  uint64_t *rec_off = c->d_rec_off.get<uint64_t>(B + 1);
  // The record list is sized from the last run (or a quarter of the input,
  // ~2x the density of random sequence); if it overflows, the scan reruns
  // with the exact count.
  // The list lives in the key buffer, which phase 3 only fills after phase 2
  // has routed the list.
  Small hs;
  const bool xscan = step == Step::XSCAN;
  auto phase1 = [&](uint32_t tile) {
    a.tile = tile;
    a.n_tiles = L >= (uint64_t)k ? ceil_div(L - k + 1, a.tile) : 0;
    if (xscan) {  // this shard's slice of the tiles, in plain launches
      const uint64_t nt = a.n_tiles;
      a.tile_begin = nt * c->opts.shard_index / shards;
      a.n_tiles = nt * (c->opts.shard_index + 1) / shards;
      a.tile_counter = nullptr;
    }
    for (int attempt = 0;; attempt++) {
      a.rec_cap = std::max<uint64_t>(c->rec_cap_hint, L / 4 + 1024);
      uint8_t *rbuf = static_cast<uint8_t *>(c->d_keys.reserve(a.rec_cap * (sizeof(uint64_t) + sizeof(uint16_t))));
      a.rec_tmp = reinterpret_cast<uint64_t *>(rbuf);
      a.rec_bucket = reinterpret_cast<uint16_t *>(rbuf + a.rec_cap * sizeof(uint64_t));
      CF1_CUDA(cudaMemsetAsync(hist, 0, NUM_BUCKETS * sizeof(uint32_t), s));
      CF1_CUDA(cudaMemsetAsync(sm, 0, sizeof(Small), s));
      launch_superkmer_scan(a, xscan ? 0 : pctas, s);
      if (!xscan) launch_partition(hist, B, lut, rec_off, &sm->n_bins_eff, s);
      CF1_CUDA(cudaMemcpyAsync(&hs, sm, sizeof(Small), cudaMemcpyDeviceToHost, s));
      if (!xscan) CF1_CUDA(cudaMemcpyAsync(&c->n_super, rec_off + B, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
      CF1_CUDA(cudaStreamSynchronize(s));
      if (!xscan && hs.rec_count != c->n_super)
        throw Error(CF1GPU_ERR_QUEUE_OVERRUN, "phase 1: record count != histogram total");
      if (hs.rec_count <= a.rec_cap) break;
      if (attempt) throw Error(CF1GPU_ERR_QUEUE_OVERRUN, "phase 1: record list overflowed twice");
      c->rec_cap_hint = hs.rec_count;
    }
  };
  if (step == Step::XFINISH) {
    // phase 1 ran in the scan step; the records arrive below
  } else if (io) {
    // Streamed intake: as chunk c of the record bytes lands, place the intake
    // tiles it completes, pack the W/NM words wholly inside the placed
    // prefix, and scan the minimizer tiles whose bases are all packed.  The
    // scan is the usual one, launched over tile ranges (no persistent queue).
    uint8_t *ascii = c->d_ascii.as<uint8_t>();
    a.tile = c->tune.sk_tile;
    a.n_tiles = L >= (uint64_t)k ? ceil_div(L - k + 1, a.tile) : 0;
    a.tile_counter = nullptr;
    a.rec_cap = std::max<uint64_t>(c->rec_cap_hint, L / 4 + 1024);
    uint8_t *rbuf = static_cast<uint8_t *>(c->d_keys.reserve(a.rec_cap * (sizeof(uint64_t) + sizeof(uint16_t))));
    a.rec_tmp = reinterpret_cast<uint64_t *>(rbuf);
    a.rec_bucket = reinterpret_cast<uint16_t *>(rbuf + a.rec_cap * sizeof(uint64_t));
    CF1_CUDA(cudaMemsetAsync(hist, 0, NUM_BUCKETS * sizeof(uint32_t), s));
    CF1_CUDA(cudaMemsetAsync(sm, 0, sizeof(Small), s));
    const uint64_t ntiles_in = io->htiles.size(), T = a.tile;
    uint64_t placed = 0, packed = 0, scanned = 0;
    for (size_t ch = 0; ch < io->chunk_ev.size(); ch++) {
      const bool last = ch + 1 == io->chunk_ev.size();
      CF1_CUDA(cudaStreamWaitEvent(s, io->chunk_ev[ch], 0));
      uint64_t t_end = placed;
      while (t_end < ntiles_in && io->htiles[t_end].src + io->htiles[t_end].len <= io->chunk_end[ch]) t_end++;
      if (t_end > placed) {
        intake_kernel<<<(unsigned)(t_end - placed), 256, 0, s>>>(io->raw, io->tiles + placed, ascii);
        CF1_LAUNCH_CHECK();
        placed = t_end;
      }
      const uint64_t prefix = (last || placed == ntiles_in) ? L : io->htiles[placed].dst;
      const uint64_t pw = last ? n_nm : prefix / 64;
      launch_pack_words(ascii, L, W, NM, packed, pw, s);
      packed = std::max(packed, pw);
      // a tile reads bases up to (t+1) T + k - 1, W and NM one word beyond
      uint64_t ready = a.n_tiles;
      if (!last) {
        const uint64_t bases = packed * 64;
        ready = bases > (uint64_t)k + 128 + T ? (bases - k - 128) / T : 0;
        if (ready > a.n_tiles) ready = a.n_tiles;
      }
      if (ready > scanned) {
        a.tile_begin = scanned;
        const uint64_t nt = a.n_tiles;
        a.n_tiles = ready;
        launch_superkmer_scan(a, 0, s);
        a.n_tiles = nt;
        scanned = ready;
      }
    }
    a.tile_begin = 0;
    launch_partition(hist, B, lut, rec_off, &sm->n_bins_eff, s);
    CF1_CUDA(cudaMemcpyAsync(&hs, sm, sizeof(Small), cudaMemcpyDeviceToHost, s));
    CF1_CUDA(cudaMemcpyAsync(&c->n_super, rec_off + B, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    CF1_CUDA(cudaStreamSynchronize(s));
    if (hs.rec_count != c->n_super) throw Error(CF1GPU_ERR_QUEUE_OVERRUN, "phase 1: record count != histogram total");
    if (hs.rec_count > a.rec_cap) {  // the list overflowed: all bases are in place now, scan again
      c->rec_cap_hint = hs.rec_count;
      a.tile_counter = batched ? &sm->queues[0] : nullptr;
      phase1(c->tune.sk_tile);
    }
  } else if (tune_now && c->opts.sk_tile == 0) {  // autotuner: time each tile, keep the fastest
    double best = 1e30;
    for (uint32_t t : TUNE_TILES) {
      CF1_CUDA(cudaEventRecord(c->ev[10], s));
      phase1(t);
      CF1_CUDA(cudaEventRecord(c->ev[11], s));
      CF1_CUDA(cudaEventSynchronize(c->ev[11]));
      const double ms = elapsed(c->ev[10], c->ev[11]);
      if (ms < best) {
        best = ms;
        tuned.sk_tile = t;
        tuned.p1_ms = ms;
      }
    }
    c->tune.sk_tile = tuned.sk_tile;
    phase1(c->tune.sk_tile);
  } else {
    phase1(c->tune.sk_tile);
  }
  CF1_CUDA(cudaEventRecord(c->ev[1], s));
  if (xscan) {  // the slice's histogram to the caller; its records wait for routing
    check_device_errors(hs.err);
    CF1_CUDA(cudaMemcpyAsync(xs->hist_out, hist, NUM_BUCKETS * sizeof(uint32_t), cudaMemcpyDefault, s));
    CF1_CUDA(cudaStreamSynchronize(s));
    c->x_local = hs.rec_count;
    c->x_rec_cap = a.rec_cap;
    c->x_ms_scan = elapsed(c->ev[0], c->ev[1]);
    return;
  }
  if (step != Step::XFINISH) {
    c->n_occ = hs.n_kmers;
    c->n_bins_eff = hs.n_bins_eff;
  }

  // ---- phase 2: route super k-mers into bins
  if (step == Step::XFINISH) {
    // The received records carry their bins: count them per bin for the
    // ranges, after checking that every one is this shard's.
    const uint64_t n = xs->n_recv;
    uint64_t *rin = static_cast<uint64_t *>(c->d_keys.reserve((n + 1) * sizeof(uint64_t)));
    if (n) CF1_CUDA(cudaMemcpyAsync(rin, xs->recv, n * sizeof(uint64_t), cudaMemcpyDefault, s));
    uint64_t *cnt = c->d_xcnt.get<uint64_t>(B + 1);
    CF1_CUDA(cudaMemsetAsync(cnt, 0, B * sizeof(uint64_t), s));
    if (n) {
      xrecv_count_kernel<<<stride_grid(n, c->num_sms), XR_BLOCK, B * sizeof(uint32_t), s>>>(
          rin, n, B, c->opts.shard_index, shards, L, k, reinterpret_cast<unsigned long long *>(cnt), &sm->err);
      CF1_LAUNCH_CHECK();
    }
    exclusive_scan_u64(cnt, rec_off, B, c->d_scan, s);
    CF1_CUDA(cudaMemcpyAsync(&hs.err, &sm->err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    CF1_CUDA(cudaStreamSynchronize(s));
    check_device_errors(hs.err);
    a.rec_tmp = rin;
    a.rec_bucket = nullptr;
    c->n_super = n;
  }
  uint64_t NS = c->n_super;
  uint64_t *records = c->d_records.get<uint64_t>(NS + 1);
  CF1_CUDA(cudaMemsetAsync(records, 0, (NS + 1) * sizeof(uint64_t), s));
  uint32_t *cursor = c->d_cursor.get<uint32_t>(B);
  CF1_CUDA(cudaMemsetAsync(cursor, 0, B * sizeof(uint32_t), s));
  launch_bin_scatter(a.rec_tmp, a.rec_bucket, NS, lut, B, rec_off, cursor, records, &sm->err, s);
  if (shards > 1 && step == Step::FULL) {
    // Keep this shard's bins: their records, moved to the front through the
    // free key buffer (the phase-1 list in it has been routed); the other
    // bins keep empty ranges, so they get no keys, slots or states.
    uint64_t *cnt = c->d_shard.get<uint64_t>(3 * (size_t)(B + 1));
    uint64_t *new_off = cnt + (B + 1);
    uint32_t *tile_off = reinterpret_cast<uint32_t *>(new_off + (B + 1));
    shard_counts_kernel<<<(unsigned)ceil_div(B, 256), 256, 0, s>>>(rec_off, B, c->opts.shard_index, shards, cnt);
    CF1_LAUNCH_CHECK();
    exclusive_scan_u64(cnt, new_off, B, c->d_scan, s);
    segment_tiles(rec_off, B, SH_TILE, tile_off, s);
    uint64_t *tmp = static_cast<uint64_t *>(c->d_keys.reserve((NS + 1) * sizeof(uint64_t)));
    shard_copy_kernel<<<(unsigned)(ceil_div(NS, SH_TILE) + B), 256, 0, s>>>(records, rec_off, tile_off, B,
                                                                            c->opts.shard_index, shards, new_off, tmp);
    CF1_LAUNCH_CHECK();
    CF1_CUDA(cudaMemcpyAsync(&NS, new_off + B, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    CF1_CUDA(cudaStreamSynchronize(s));
    if (NS) CF1_CUDA(cudaMemcpyAsync(records, tmp, NS * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    CF1_CUDA(cudaMemcpyAsync(rec_off, new_off, (B + 1) * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
  }
  uint64_t *kpre = c->d_kpre.get<uint64_t>(NS + 1);
  record_kmer_prefix(records, NS, kpre, c->d_lens, c->d_scan, s);
  if (shards > 1 || step == Step::XFINISH) {  // the k-mer windows of this shard's records
    CF1_CUDA(cudaMemcpyAsync(&c->n_occ, kpre + NS, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    CF1_CUDA(cudaStreamSynchronize(s));
  }
  CF1_CUDA(cudaEventRecord(c->ev[2], s));

  // ---- phase 3a: expand, sort per bin, unique
  const uint64_t NO = c->n_occ;
  KeyT *keys = c->d_keys.get<KeyT>(NO + 1);
  // state_update 0: every occurrence's side-set byte travels with its key
  // through the MSD sort, whose dedup joins a vertex's occurrences, so phase
  // 4 only places each distinct key's byte in its slot (the LSD fallback has
  // no payloads: phase 4 then classifies the occurrences as before)
  const bool join3 = c->opts.state_update == 0 && !c->force_lsd;
  uint8_t *pay = join3 ? c->d_pay.get<uint8_t>(NO + 16) : nullptr;
  uint8_t *pay_alt = join3 ? c->d_pay_alt.get<uint8_t>(NO + 16) : nullptr;
  launch_expand<KeyT>(records, NS, kpre, W, k, keys, NO, L, batched ? &sm->queues[2] : nullptr, &sm->err, pctas, s, NM,
                      pay);
  uint64_t *seg = c->d_seg.get<uint64_t>(B + 1);
  seg_gather_kernel<<<(unsigned)ceil_div(B + 1, 256), 256, 0, s>>>(kpre, rec_off, B, seg);
  CF1_LAUNCH_CHECK();
  // the dense distinct-key array, allocated when a step writes it
  auto dist_buf = [&]() { return c->d_dist.get<KeyT>(NO + 1); };
  uint64_t *dist_off = c->d_dist_off.get<uint64_t>(B + 1);
  std::vector<uint64_t> hseg(B + 1);
  CF1_CUDA(cudaMemcpyAsync(hseg.data(), seg, (B + 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  CF1_CUDA(cudaStreamSynchronize(s));
  uint64_t max_bin = 0;
  for (uint32_t b = 0; b < B; b++) max_bin = std::max(max_bin, hseg[b + 1] - hseg[b]);
  KeyT *alt = be.sort.alt.template get<KeyT>(NO + 1);
  const int P0 = c->force_lsd ? -1 : msd_prefix_bits<KeyT>(max_bin, sorted);
  auto msd_width = [&](int delta) { return P0 < 0 ? -1 : std::min(16, std::max(0, P0 + delta)); };
  auto expand_again = [&]() {
    launch_expand<KeyT>(records, NS, kpre, W, k, keys, NO, L, batched ? &sm->queues[4] : nullptr, &sm->err, pctas, s,
                        NM, pay);
  };
  if (tune_now && P0 >= 0) {  // autotuner: time each MSD width, keep the fastest
    double best = 1e30;
    int tried = -2;
    for (int d : TUNE_MSD_DELTAS) {
      const int P = msd_width(d);
      if (P == tried) continue;
      if (tried != -2) expand_again();  // the previous try consumed the keys
      if (batched) CF1_CUDA(cudaMemsetAsync(&sm->queues[4], 0, sizeof(uint32_t), s));
      CF1_CUDA(cudaEventRecord(c->ev[10], s));
      const bool ok = msd_sort_unique<KeyT>(keys, alt, NO, seg, B, 2 * k, P, dist_buf(), dist_off, be.msd, s, sorted,
                                            nullptr, nullptr, pay, pay_alt);
      CF1_CUDA(cudaEventRecord(c->ev[11], s));
      CF1_CUDA(cudaEventSynchronize(c->ev[11]));
      const double ms = elapsed(c->ev[10], c->ev[11]);
      if (ok && ms < best) {
        best = ms;
        tuned.msd_delta = d;
        tuned.p3_ms = ms;
      }
      tried = P;
    }
    c->tune.msd_delta = tuned.msd_delta;
    expand_again();
    if (batched) CF1_CUDA(cudaMemsetAsync(&sm->queues[4], 0, sizeof(uint32_t), s));
  }
  int P = msd_width(c->tune.msd_delta);
  // BBHash form, 64-bit keys: the dedup builds BBHash levels 0 and 1 on the
  // way (Level0Out): level 0 with 8 bits per k-mer occurrence of the bin
  // rounded up to a multiple of the bin's 2^P slices, level 1 with an eighth
  // of level 0's words per slice (the keys level 0 leaves are ~10% of its
  // distinct keys, so ~10 bits each); the keys level 1 leaves go to a list
  // with room for a quarter of the bin's occurrences.
  const bool l0_fuse = !sorted && !c->wide && c->opts.mphf_mode == CF1GPU_MPHF_BBHASH && P >= 0;
  Level0Out l0;
  uint64_t l0_words = 0, l1_words = 0, l0_room = 0;
  if (l0_fuse) {
    std::vector<uint64_t> hw(B + 1, 0), hw1(B + 1, 0), hr(B + 1, 0);
    const uint64_t slices = 1ull << P;
    for (uint32_t b = 0; b < B; b++) {
      const uint64_t occ = hseg[b + 1] - hseg[b];
      const uint64_t sw0 = occ ? ceil_div(ceil_div(8 * occ, 64), slices) : 0;
      hw[b + 1] = hw[b] + sw0 * slices;
      hw1[b + 1] = hw1[b] + ceil_div(sw0, 8) * slices;
      hr[b + 1] = hr[b] + (occ ? occ / 4 + 64 : 0);
    }
    l0_words = hw[B];
    l1_words = hw1[B];
    l0_room = hr[B];
    uint64_t *woff0 = c->d_l0.get<uint64_t>(4 * (size_t)(B + 1));
    uint64_t *room_off = woff0 + (B + 1);
    unsigned long long *scnt = reinterpret_cast<unsigned long long *>(room_off + (B + 1));
    uint64_t *woff1 = room_off + 2 * (size_t)(B + 1);
    CF1_CUDA(cudaMemcpyAsync(woff0, hw.data(), (B + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
    CF1_CUDA(cudaMemcpyAsync(woff1, hw1.data(), (B + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
    CF1_CUDA(cudaMemcpyAsync(room_off, hr.data(), (B + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
    CF1_CUDA(cudaMemsetAsync(scnt, 0, B * sizeof(uint64_t), s));
    l0.AR = be.bb.prepare_levels01(l0_words, l1_words, s);  // every slice writes all of its entries
    l0.woff = woff0;
    l0.AR1 = l0.AR + l0_words;
    l0.woff1 = woff1;
    l0.surv = c->d_l0surv.get<uint64_t>(l0_room + 1);
    l0.surv_off = room_off;
    l0.surv_cnt = scnt;
    l0.err = &sm->l0_err;
    uint32_t *placed = c->d_l0placed.get<uint32_t>(2 * (((uint64_t)B << P) + 1));
    l0.placed = placed;
    l0.placed1 = placed + ((uint64_t)B << P) + 1;
    if (join3) {  // joined side sets: levels 0 and 1 place their keys' bytes by rank (see Level0Out)
      l0.with_pay = true;
      l0.surv_pay = c->d_l0survpay.get<uint8_t>(l0_room + 1);
    }
  }
  // The BBHash form leaves the distinct keys in their sub-buckets (kept):
  // nothing on the path reads them, so the dense copy waits until a
  // verification or dump asks for it.
  KeyT *kept = nullptr;
  uint8_t *kept_pay = nullptr, *l0pay = nullptr;
  bool done = P >= 0 && msd_sort_unique<KeyT>(keys, alt, NO, seg, B, 2 * k, P, l0_fuse ? nullptr : dist_buf(), dist_off,
                                              be.msd, s, sorted, l0_fuse ? &l0 : nullptr, &kept, pay, pay_alt,
                                              &kept_pay, &l0pay);
  c->msd_bits = done ? P : -1;
  if (tune_now) {
    tuned.sk_tile = c->tune.sk_tile;
    tuned.msd_delta = c->tune.msd_delta;
    tuner_store(c->tuner_path, c->tuned_key, tuned);
    c->tune_valid = true;
    c->tuner_state = 2;
  }
  if (!done) {  // a sub-bucket overflowed shared memory: expand again, LSD path
    if (P >= 0) {
      if (batched) CF1_CUDA(cudaMemsetAsync(&sm->queues[5], 0, sizeof(uint32_t), s));
      launch_expand<KeyT>(records, NS, kpre, W, k, keys, NO, L, batched ? &sm->queues[5] : nullptr, &sm->err, pctas, s);
    }
    segmented_sort<KeyT>(keys, NO, seg, B, 2 * k, be.sort, s);
    segmented_unique<KeyT>(keys, NO, seg, B, dist_buf(), dist_off, be.sort, s);
  }
  KeyT *dist = c->d_dist.as<KeyT>();
  CF1_CUDA(cudaMemcpyAsync(&c->n_distinct, dist_off + B, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  uint32_t l0_err = 1;
  if (l0_fuse) CF1_CUDA(cudaMemcpyAsync(&l0_err, &sm->l0_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  CF1_CUDA(cudaStreamSynchronize(s));
  const bool l0_ready = l0_fuse && done && l0_err == 0;
  const uint64_t nsub = done && P >= 0 ? (uint64_t)B << P : 0;
  const bool joined = join3 && done && kept_pay != nullptr;  // phase 3 joined the occurrences' side sets
  if (l0_fuse && done && !l0_ready) {  // level 0 did not fit: the plain build reads the dense keys
    dist = dist_buf();
    msd_compact<KeyT>(kept, nsub, dist, be.msd, s);
  }
  c->dist_pending = l0_ready;
  c->dist_kept = kept;
  c->dist_nsub = nsub;
  CF1_CUDA(cudaEventRecord(c->ev[3], s));

  // ---- phase 3b: MPHF
  // the sort's buffers (NO keys each) are free now: BBHash levels use them,
  // except the one holding the kept keys, whose twin they share
  KeyT *ws1 = be.sort.alt.template as<KeyT>();
  KeyT *twin = kept == keys ? ws1 : keys;
  const uint64_t half = (NO + 1) / 2;
  if (c->opts.mphf_mode == CF1GPU_MPHF_LEARNED) {
    be.li.build(dist, dist_off, B, k, c->learned, s);
    be.bb.build(dist, dist_off, B, be.li.fallback_sel(), s, keys, ws1, NO + 1);
  } else if (l0_ready) {
    be.bb.build_from_levels01(B, P, l0.woff, l0_words, l0.placed, l0.woff1, l1_words, l0.placed1,
                              reinterpret_cast<const KeyT *>(l0.surv), l0.surv_off,
                              reinterpret_cast<const uint64_t *>(l0.surv_cnt), l0_room, s, twin, twin + half, half);
  } else {
    be.bb.build(dist, dist_off, B, nullptr, s, keys, ws1, NO + 1);
  }
  CF1_CUDA(cudaEventRecord(c->ev[4], s));

  // ---- phase 4: classification
  // Side-set mode keeps one byte per vertex in a sort buffer, which is free
  // once the MPHF is built (12 * nwords <= n_distinct + 11 <= 8 * (NO + 1)):
  // the key buffer, or the twin of the kept keys.
  const uint64_t nwords = ceil_div(c->n_distinct, 12);
  const bool sideset = c->opts.state_update != 1;
  unsigned long long *states = c->d_states.get<unsigned long long>(nwords + 1);
  // joined: phase 3 left each distinct key's side-set byte beside it, and
  // the other payload buffer takes the bytes in slot order
  // (with level 0 placed by rank, the other payload buffer holds the level-0
  // bytes in rank order, so the free sort buffer takes the slots)
  const bool joined_l0 = joined && l0_ready;
  uint32_t *sides = !sideset ? nullptr
                    : (joined && !joined_l0) ? reinterpret_cast<uint32_t *>(kept_pay == pay ? pay_alt : pay)
                                             : reinterpret_cast<uint32_t *>(c->dist_pending ? twin : keys);
  // the phase-4 work of a stage of bins [b0, b1)
  auto place = [&](uint32_t b0, uint32_t b1) {
    uint8_t *sb = reinterpret_cast<uint8_t *>(sides);
    const uint64_t *sbo = be.msd.sb_off.template as<const uint64_t>();
    if (joined_l0) {
      launch_place_l0(be.bb.view(), dist_off, sbo, l0.placed, l0.placed1, l0pay, (uint64_t)b0 << P,
                      (uint64_t)b1 << P, P, sb, &sm->err, s);
      launch_place_surv(be.bb.view(), dist_off, reinterpret_cast<const uint64_t *>(l0.surv), l0.surv_pay, l0.surv_off,
                        l0.surv_cnt, b0, b1, sb, &sm->err, s);
    } else {
      launch_place_sides<KeyT>(make_view<KeyT>(c), kept, c->dist_pending ? nullptr : c->d_dist.as<const KeyT>(),
                               kept_pay, sbo, be.msd.cnt.template as<const uint32_t>(),
                               be.msd.out_off.template as<const uint64_t>(), (uint64_t)b0 << P, (uint64_t)b1 << P, P, sb,
                               &sm->err, s);
    }
  };
  if (sideset) {
    if (joined) {  // every slot gets its byte; only the last word's unused tail is cleared
      if (nwords * 12 > c->n_distinct)
        CF1_CUDA(cudaMemsetAsync(reinterpret_cast<uint8_t *>(sides) + c->n_distinct, 0, nwords * 12 - c->n_distinct, s));
    } else {
      CF1_CUDA(cudaMemsetAsync(sides, 0, nwords * 12, s));
    }
    CF1_CUDA(cudaMemsetAsync(states + nwords, 0, sizeof(unsigned long long), s));
  } else {
    CF1_CUDA(cudaMemsetAsync(states, 0, (nwords + 1) * sizeof(unsigned long long), s));
  }
  ClassifyArgs<KeyT> ca;
  ca.records = records;
  ca.n_rec = NS;
  ca.W = W;
  ca.NM = NM;
  ca.L = L;
  ca.k = k;
  ca.mphf = make_view<KeyT>(c);
  ca.states = states;
  ca.sides = sides;
  ca.queue = batched ? &sm->queues[3] : nullptr;
  ca.err = &sm->err;
  ca.cas_retries = &sm->cas_retries;
  CF1_CUDA(cudaEventRecord(c->ev[5], s));
  if (io && io->host_cap >= nwords && nwords) {
    // Staged: bins in STREAM_STAGES groups of about equal record counts; the
    // words whose slots all belong to finished bins go back while the next
    // group classifies.
    std::vector<uint64_t> hro(B + 1), hdo(B + 1);
    CF1_CUDA(cudaMemcpyAsync(hro.data(), rec_off, (B + 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    CF1_CUDA(cudaMemcpyAsync(hdo.data(), dist_off, (B + 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    CF1_CUDA(cudaStreamSynchronize(s));
    uint32_t b0 = 0;
    uint64_t w_done = 0;
    for (int st = 0; st < STREAM_STAGES && b0 < B; st++) {
      uint32_t b1 = B;
      if (st + 1 < STREAM_STAGES) {
        const uint64_t target = hro[B] * (uint64_t)(st + 1) / STREAM_STAGES;
        b1 = b0 + 1;
        while (b1 < B && hro[b1] < target) b1++;
      }
      if (joined) {
        place(b0, b1);
      } else {
        ClassifyArgs<KeyT> cs = ca;
        cs.records = records + hro[b0];
        cs.n_rec = hro[b1] - hro[b0];
        if (batched) CF1_CUDA(cudaMemsetAsync(ca.queue, 0, sizeof(uint32_t), s));
        launch_classify<KeyT>(cs, pctas, s);
      }
      const uint64_t w_fin = b1 == B ? nwords : hdo[b1] / 12;
      if (w_fin > w_done) {
        if (sideset) launch_sideset_pack(sides, w_done, w_fin, states, s);
        CF1_CUDA(cudaEventRecord(c->stage_ev[st], s));
        CF1_CUDA(cudaStreamWaitEvent(c->copy_stream, c->stage_ev[st], 0));
        CF1_CUDA(cudaMemcpyAsync(io->host_words + w_done, states + w_done, (w_fin - w_done) * sizeof(uint64_t),
                                 cudaMemcpyDeviceToHost, c->copy_stream));
        w_done = w_fin;
      }
      b0 = b1;
    }
    CF1_CUDA(cudaEventRecord(c->ev[6], s));
    CF1_CUDA(cudaStreamSynchronize(c->copy_stream));
    io->words_done = true;
  } else {
    if (joined)
      place(0, B);
    else
      launch_classify<KeyT>(ca, pctas, s);
    CF1_CUDA(cudaEventRecord(c->ev[6], s));
    if (sideset) launch_sideset_pack(sides, 0, nwords, states, s);
  }
  CF1_CUDA(cudaEventRecord(c->ev[7], s));
  CF1_CUDA(cudaMemcpyAsync(&hs, sm, sizeof(Small), cudaMemcpyDeviceToHost, s));
  CF1_CUDA(cudaStreamSynchronize(s));
  check_device_errors(hs.err);
  c->cas_retries = hs.cas_retries;

  cf1gpu_stats &st = c->stats;
  double h2d = st.ms_h2d;
  std::memset(&st, 0, sizeof(st));
  st.ms_h2d = h2d;
  st.n_bases = c->n_bases;
  st.n_records = c->n_records;
  st.n_short = c->short_seqs.size();
  st.n_superkmers = NS;
  st.n_kmer_occurrences = NO;
  st.n_distinct = c->n_distinct;
  st.n_bins = c->n_bins_eff;
  st.n_state_words = nwords;
  st.bbhash_levels = be.bb.levels;
  st.mphf_bytes = be.bb.bytes + (c->opts.mphf_mode == CF1GPU_MPHF_LEARNED ? be.li.stats.bytes : 0);
  st.learned_bins = c->opts.mphf_mode == CF1GPU_MPHF_LEARNED ? be.li.stats.learned_bins : 0;
  st.fallback_bins = c->opts.mphf_mode == CF1GPU_MPHF_LEARNED ? be.li.stats.fallback_bins : 0;
  st.learned_max_err = c->opts.mphf_mode == CF1GPU_MPHF_LEARNED ? be.li.stats.max_err : 0;
  st.classify_cas_retries = c->cas_retries;
  st.n_kernel_launches = g_launches.load() - launches0;
  st.sort_msd_bits = c->msd_bits >= 0 ? (uint64_t)c->msd_bits : ~0ull;
  st.tuner_state = (uint64_t)c->tuner_state;
  st.sk_tile = c->tune.sk_tile;
  // an exchange-sharded run's phase 1 is the slice's scan and routing
  const double p1_before = step == Step::XFINISH ? c->x_ms_scan : 0.0;
  st.ms_phase1 = elapsed(c->ev[0], c->ev[1]) + p1_before;
  st.ms_phase2 = elapsed(c->ev[1], c->ev[2]);
  st.ms_phase3_sort = elapsed(c->ev[2], c->ev[3]);
  st.ms_phase3_mphf = elapsed(c->ev[3], c->ev[4]);
  st.ms_phase4 = elapsed(c->ev[4], c->ev[7]);
  st.ms_classify_kernel = elapsed(c->ev[5], c->ev[6]);
  st.ms_dedup_kernel = done ? be.msd.ms_dedup : 0.0;
  st.dedup_overflow = done && !sorted ? be.msd.last_overflow : 0;
  st.state_path = joined ? 0 : (c->opts.state_update == 1 ? 1 : 2);
  st.ms_total = elapsed(c->ev[0], c->ev[7]) + p1_before;
}

// The dense distinct-key array of a run that left it for later.
template <class KeyT>
void ensure_dist(cf1gpu_ctx *c) {
  if (!c->dist_pending) return;
  msd_compact<KeyT>(static_cast<const KeyT *>(c->dist_kept), c->dist_nsub, c->d_dist.get<KeyT>(c->n_distinct + 1),
                    backend<KeyT>(c).msd, c->stream);
  c->dist_pending = false;
}

template <class KeyT>
void dump_impl(cf1gpu_ctx *c, uint64_t *keys, uint8_t *states) {
  ensure_dist<KeyT>(c);
  cudaStream_t s = c->stream;
  uint64_t n = c->n_distinct;
  uint64_t *dk = c->d_qout.get<uint64_t>(n * cf1::KOps<KeyT>::WORDS + 1);
  uint8_t *ds = c->d_qin.get<uint8_t>(n + 1);
  launch_dump<KeyT>(make_view<KeyT>(c), c->nbins, n, c->d_states.as<const unsigned long long>(), dk, ds, s);
  CF1_CUDA(cudaMemcpyAsync(keys, dk, n * cf1::KOps<KeyT>::WORDS * 8, cudaMemcpyDeviceToHost, s));
  CF1_CUDA(cudaMemcpyAsync(states, ds, n, cudaMemcpyDeviceToHost, s));
  CF1_CUDA(cudaStreamSynchronize(s));
}

template <class KeyT>
void verify_impl(cf1gpu_ctx *c) {
  ensure_dist<KeyT>(c);
  cudaStream_t s = c->stream;
  uint64_t n = c->n_distinct;
  Small *sm = c->d_small.get<Small>(1);
  CF1_CUDA(cudaMemsetAsync(&sm->err, 0, sizeof(uint32_t), s));
  uint32_t *seen = c->d_seen.get<uint32_t>(n + 1);
  launch_verify<KeyT>(make_view<KeyT>(c), c->nbins, n, seen, &sm->err, s);
  uint32_t err = 0;
  CF1_CUDA(cudaMemcpyAsync(&err, &sm->err, 4, cudaMemcpyDeviceToHost, s));
  CF1_CUDA(cudaStreamSynchronize(s));
  if (err) throw Error(CF1GPU_ERR_BIJECTION, "MPHF is not a bijection onto [0, total_kmers)");
}

template <class KeyT>
void query_impl(cf1gpu_ctx *c, const uint64_t *keys, size_t n, uint64_t *slots) {
  cudaStream_t s = c->stream;
  constexpr int KW = cf1::KOps<KeyT>::WORDS;
  uint64_t *din = c->d_qin.get<uint64_t>(n * KW + 1);
  uint64_t *dout = c->d_qout.get<uint64_t>(n + 1);
  CF1_CUDA(cudaMemcpyAsync(din, keys, n * KW * 8, cudaMemcpyHostToDevice, s));
  launch_query<KeyT>(make_view<KeyT>(c), c->d_lut.as<const uint16_t>(), c->k, c->m, din, n, dout, s);
  CF1_CUDA(cudaMemcpyAsync(slots, dout, n * 8, cudaMemcpyDeviceToHost, s));
  CF1_CUDA(cudaStreamSynchronize(s));
}

bool page_locked(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    (void)cudaGetLastError();  // not a pointer CUDA knows: pageable
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// dst[i]: the record's place in the concatenation (~0 for records below k
// bases); end: the concatenation's length after the records.
void intake_direct(cf1gpu_ctx *c, const uint8_t *seqs, const uint64_t *off, size_t n, const std::vector<uint64_t> &dst,
                   uint64_t end) {
  cudaStream_t s = c->stream;
  const uint64_t first = off[0], raw = off[n] - first;
  c->d_ascii.reserve_keep(end + 16, c->dev_valid, s);
  std::vector<IntakeTile> tiles;
  for (size_t i = 0; i < n; i++) {
    if (dst[i] == ~0ull) continue;
    const uint64_t len = off[i + 1] - off[i];
    for (uint64_t t = 0; t < len; t += INTAKE_TILE) {
      const uint64_t m = std::min<uint64_t>(INTAKE_TILE, len - t);
      tiles.push_back(IntakeTile{off[i] - first + t, dst[i] + t, (uint32_t)m, t + m == len ? 1u : 0u});
    }
  }
  if (!tiles.empty()) {
    uint8_t *r = c->d_raw.get<uint8_t>(raw + 1);
    IntakeTile *dt = c->d_intake.get<IntakeTile>(tiles.size());
    CF1_CUDA(cudaEventRecord(c->ev[10], s));
    CF1_CUDA(cudaMemcpyAsync(r, seqs + first, raw, cudaMemcpyHostToDevice, s));
    CF1_CUDA(cudaEventRecord(c->ev[11], s));
    CF1_CUDA(cudaMemcpyAsync(dt, tiles.data(), tiles.size() * sizeof(IntakeTile), cudaMemcpyHostToDevice, s));
    intake_kernel<<<(unsigned)tiles.size(), 256, 0, s>>>(r, dt, c->d_ascii.as<uint8_t>());
    CF1_LAUNCH_CHECK();
    CF1_CUDA(cudaStreamSynchronize(s));  // the caller may free its buffer on return
    c->ms_intake += elapsed(c->ev[10], c->ev[11]);
  }
  c->L = c->dev_valid = end;
}

void append_record(cf1gpu_ctx *c, const uint8_t *seq, size_t len) {
  c->host.reserve(c->L + len + 1, c->L);
  if (len) std::memcpy(c->host.p + c->L, seq, len);
  c->host.p[c->L + len] = 'N';
  c->L += len + 1;
}

std::string first_token(const char *name, size_t n) {
  size_t i = 0;
  while (i < n && (name[i] == ' ' || name[i] == '\t' || name[i] == '\n' || name[i] == '\r')) i++;
  size_t j = i;
  while (j < n && !(name[j] == ' ' || name[j] == '\t' || name[j] == '\n' || name[j] == '\r')) j++;
  return std::string(name + i, j - i);
}

}  // namespace

// ---- entry points used by the C ABI (and by the C++ host mirror) ----
void run_resident(cf1gpu_ctx *c) {
  if (!c->uploaded) throw Error(CF1GPU_ERR_STATE, "no input on the device: call cf1gpu_upload first");
  c->x_step = 0;
  if (c->wide) run_impl<Key2>(c);
  else run_impl<uint64_t>(c);
  c->ran = true;
}

size_t run_streamed(cf1gpu_ctx *c, const uint8_t *seqs, const uint64_t *off, size_t n, uint64_t *words, size_t cap) {
  // the input of cf1gpu_reset_input + cf1gpu_add_records, without staging
  c->L = 0;
  c->dev_valid = 0;
  c->ms_intake = 0;
  c->n_records = 0;
  c->n_bases = 0;
  c->short_seqs.clear();
  c->uploaded = false;
  c->ran = false;
  c->x_step = 0;
  std::vector<uint64_t> dst(n + 1);
  uint64_t pos = 0;
  for (size_t i = 0; i < n; i++) {
    const uint64_t len = off[i + 1] - off[i];
    dst[i] = pos;
    c->n_records++;
    c->n_bases += len;
    if (len < (uint64_t)c->k) {
      if (c->opts.track_short_seqs) c->short_seqs.emplace_back(std::string(), len);
      dst[i] = ~0ull;
      continue;
    }
    pos += len + 1;
  }
  cudaStream_t s = c->stream, cs = c->copy_stream;
  StreamIO io;
  const uint64_t first = n ? off[0] : 0, raw = n ? off[n] - first : 0;
  for (size_t i = 0; i < n; i++) {
    if (dst[i] == ~0ull) continue;
    const uint64_t len = off[i + 1] - off[i];
    for (uint64_t t = 0; t < len; t += INTAKE_TILE) {
      const uint64_t m = std::min<uint64_t>(INTAKE_TILE, len - t);
      io.htiles.push_back(IntakeTile{off[i] - first + t, dst[i] + t, (uint32_t)m, t + m == len ? 1u : 0u});
    }
  }
  c->d_ascii.reserve_keep(pos + 16, 0, s);
  uint8_t *r = c->d_raw.get<uint8_t>(raw + 1);
  IntakeTile *dt = c->d_intake.get<IntakeTile>(io.htiles.size() + 1);
  if (!io.htiles.empty())
    CF1_CUDA(cudaMemcpyAsync(dt, io.htiles.data(), io.htiles.size() * sizeof(IntakeTile), cudaMemcpyHostToDevice, s));
  CF1_CUDA(cudaStreamSynchronize(s));  // buffers in place before the copy stream writes them
  io.raw = r;
  io.tiles = dt;
  io.host_words = words;
  io.host_cap = cap;
  // the record bytes in about 16 chunks (1 MB to 256 MB each) on the copy stream
  const uint64_t CHUNK = std::max<uint64_t>(1ull << 20, std::min<uint64_t>(256ull << 20, ceil_div(raw, 16)));
  const size_t nch = raw ? (size_t)ceil_div(raw, CHUNK) : 1;
  io.chunk_ev.resize(nch);
  io.chunk_end.resize(nch);
  for (auto &e : io.chunk_ev) CF1_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  struct EvGuard {
    std::vector<cudaEvent_t> &v;
    ~EvGuard() {
      for (auto e : v) cudaEventDestroy(e);
    }
  } guard_ev{io.chunk_ev};
  CF1_CUDA(cudaEventRecord(c->ev[8], cs));
  for (size_t ch = 0; ch < nch; ch++) {
    const uint64_t b = ch * CHUNK, e = std::min(raw, b + CHUNK);
    if (e > b) CF1_CUDA(cudaMemcpyAsync(r + b, seqs + first + b, e - b, cudaMemcpyHostToDevice, cs));
    CF1_CUDA(cudaEventRecord(io.chunk_ev[ch], cs));
    io.chunk_end[ch] = e;
  }
  CF1_CUDA(cudaEventRecord(c->ev[9], cs));
  c->L = pos;
  c->dev_valid = pos;
  c->uploaded = true;
  if (c->wide) run_impl<Key2>(c, &io);
  else run_impl<uint64_t>(c, &io);
  c->ran = true;
  c->stats.ms_h2d = elapsed(c->ev[8], c->ev[9]);
  const uint64_t nw = ceil_div(c->n_distinct, 12);
  if (!io.words_done && nw) {  // staged copy-back skipped (no buffer or too small)
    if (cap < nw) throw Error(CF1GPU_ERR_INVALID_ARG, "state word buffer too small: need " + std::to_string(nw));
    CF1_CUDA(cudaMemcpyAsync(words, c->d_states.p, nw * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    CF1_CUDA(cudaStreamSynchronize(s));
  }
  return nw;
}

void xshard_scan(cf1gpu_ctx *c, uint32_t *hist, uint64_t *n_local) {
  upload(c);
  c->ran = false;
  c->x_step = 0;
  c->x_launches0 = g_launches.load();
  XShard xs;
  xs.hist_out = hist;
  if (c->wide) run_impl<Key2>(c, nullptr, Step::XSCAN, &xs);
  else run_impl<uint64_t>(c, nullptr, Step::XSCAN, &xs);
  c->x_step = 1;
  *n_local = c->x_local;
}

void xshard_route(cf1gpu_ctx *c, const uint32_t *hist_in, uint64_t *send, size_t cap, uint64_t *counts) {
  if (c->x_step != 1) throw Error(CF1GPU_ERR_STATE, "no scanned slice to route: call cf1gpu_xshard_scan first");
  const uint64_t n = c->x_local;
  if (cap < n) throw Error(CF1GPU_ERR_INVALID_ARG, "record buffer too small: need " + std::to_string(n));
  cudaStream_t s = c->stream;
  const uint32_t B = c->opts.num_bins;
  const uint32_t N = c->opts.shard_count > 1 ? c->opts.shard_count : 1;
  CF1_CUDA(cudaEventRecord(c->ev[10], s));
  // the partition of the summed histogram: the same on every shard
  uint32_t *hist = c->d_hist.get<uint32_t>(NUM_BUCKETS);
  CF1_CUDA(cudaMemcpyAsync(hist, hist_in, NUM_BUCKETS * sizeof(uint32_t), cudaMemcpyDefault, s));
  uint16_t *lut = c->d_lut.get<uint16_t>(NUM_BUCKETS);
  uint64_t *rec_off = c->d_rec_off.get<uint64_t>(B + 1);
  Small *sm = c->d_small.get<Small>(1);
  CF1_CUDA(cudaMemsetAsync(sm, 0, sizeof(Small), s));
  launch_partition(hist, B, lut, rec_off, &sm->n_bins_eff, s);
  // the slice's records, grouped by owner shard
  const uint8_t *rbuf = c->d_keys.as<const uint8_t>();
  const uint64_t *rec = reinterpret_cast<const uint64_t *>(rbuf);
  const uint16_t *bucket = reinterpret_cast<const uint16_t *>(rbuf + c->x_rec_cap * sizeof(uint64_t));
  uint64_t *cnt = c->d_xcnt.get<uint64_t>(3 * (size_t)(N + 1));
  uint64_t *off = cnt + (N + 1), *cur = off + (N + 1);
  CF1_CUDA(cudaMemsetAsync(cnt, 0, 3 * (size_t)(N + 1) * sizeof(uint64_t), s));
  uint64_t *out = c->d_xsend.get<uint64_t>(n + 1);
  if (n) {
    xroute_count_kernel<<<stride_grid(n, c->num_sms), XR_BLOCK, N * sizeof(uint32_t), s>>>(
        bucket, n, lut, N, reinterpret_cast<unsigned long long *>(cnt));
    CF1_LAUNCH_CHECK();
  }
  exclusive_scan_u64(cnt, off, N, c->d_scan, s);
  if (n) {
    xroute_scatter_kernel<<<(unsigned)ceil_div(n, (uint64_t)XR_BLOCK * XR_ITEMS), XR_BLOCK,
                            N * (sizeof(uint64_t) + sizeof(uint32_t)), s>>>(
        rec, bucket, n, lut, N, off, reinterpret_cast<unsigned long long *>(cur), out, &sm->err);
    CF1_LAUNCH_CHECK();
    CF1_CUDA(cudaMemcpyAsync(send, out, n * sizeof(uint64_t), cudaMemcpyDefault, s));
  }
  CF1_CUDA(cudaMemcpyAsync(counts, cnt, N * sizeof(uint64_t), cudaMemcpyDefault, s));
  CF1_CUDA(cudaEventRecord(c->ev[11], s));
  Small hs;
  CF1_CUDA(cudaMemcpyAsync(&hs, sm, sizeof(Small), cudaMemcpyDeviceToHost, s));
  CF1_CUDA(cudaStreamSynchronize(s));
  check_device_errors(hs.err);
  c->n_bins_eff = hs.n_bins_eff;
  c->x_ms_scan += elapsed(c->ev[10], c->ev[11]);
  c->x_step = 2;
}

void xshard_finish(cf1gpu_ctx *c, const uint64_t *recv, size_t n) {
  if (c->x_step != 2) throw Error(CF1GPU_ERR_STATE, "the slice is not routed: call cf1gpu_xshard_route first");
  XShard xs;
  xs.recv = recv;
  xs.n_recv = n;
  c->x_step = 0;
  if (c->wide) run_impl<Key2>(c, nullptr, Step::XFINISH, &xs);
  else run_impl<uint64_t>(c, nullptr, Step::XFINISH, &xs);
  c->ran = true;
}

void upload(cf1gpu_ctx *c) {
  cudaStream_t s = c->stream;
  uint8_t *d = static_cast<uint8_t *>(c->d_ascii.reserve_keep(c->L + 16, c->dev_valid, s));
  CF1_CUDA(cudaEventRecord(c->ev[8], s));
  if (c->L > c->dev_valid)
    CF1_CUDA(cudaMemcpyAsync(d + c->dev_valid, c->host.p + c->dev_valid, c->L - c->dev_valid, cudaMemcpyHostToDevice, s));
  CF1_CUDA(cudaEventRecord(c->ev[9], s));
  CF1_CUDA(cudaEventSynchronize(c->ev[9]));
  float ms = 0;
  CF1_CUDA(cudaEventElapsedTime(&ms, c->ev[8], c->ev[9]));
  c->stats.ms_h2d = ms + c->ms_intake;
  c->ms_intake = 0;
  c->dev_valid = c->L;
  c->uploaded = true;
}

void add_record(cf1gpu_ctx *c, const char *name, size_t name_len, const uint8_t *seq, size_t len) {
  c->n_records++;
  c->n_bases += len;
  c->uploaded = false;
  if (len < (size_t)c->k) {  // src/classify.rs:550-561
    if (c->opts.track_short_seqs) c->short_seqs.emplace_back(name ? first_token(name, name_len) : std::string(), len);
    return;
  }
  append_record(c, seq, len);
}

void add_records(cf1gpu_ctx *c, const uint8_t *seqs, const uint64_t *off, size_t n) {
  // Records of k bases or more are copied into the pinned buffer by several
  // threads (or, when the caller's buffer is page-locked, DMA'd to the
  // device); shorter ones only update the short-sequence list.
  std::vector<uint64_t> dst(n + 1);
  uint64_t pos = c->L;
  for (size_t i = 0; i < n; i++) {
    uint64_t len = off[i + 1] - off[i];
    dst[i] = pos;
    c->n_records++;
    c->n_bases += len;
    if (len < (uint64_t)c->k) {
      if (c->opts.track_short_seqs) c->short_seqs.emplace_back(std::string(), len);
      dst[i] = ~0ull;
      continue;
    }
    pos += len + 1;
  }
  // page-locked records go straight to the device while nothing is staged
  if (n && c->dev_valid == c->L && page_locked(seqs + off[0])) {
    intake_direct(c, seqs, off, n, dst, pos);
    c->uploaded = false;
    return;
  }
  c->host.reserve(pos + 1, c->L);
  uint8_t *h = c->host.p;
  uint64_t total = pos - c->L;
  unsigned nt = total > (64ull << 20) ? std::max(1u, std::min(16u, std::thread::hardware_concurrency())) : 1;
  auto work = [&](unsigned t) {
    // record i goes to thread t when its destination start falls in t's share
    uint64_t lo = c->L + total * t / nt, hi = c->L + total * (t + 1) / nt;
    for (size_t i = 0; i < n; i++) {
      if (dst[i] == ~0ull) continue;
      uint64_t len = off[i + 1] - off[i];
      uint64_t a = std::max(dst[i], lo), b = std::min(dst[i] + len + 1, hi);
      if (a >= b) continue;
      uint64_t e = std::min(b, dst[i] + len);
      if (a < e) std::memcpy(h + a, seqs + off[i] + (a - dst[i]), e - a);
      if (b == dst[i] + len + 1) h[dst[i] + len] = 'N';
    }
  };
  if (nt == 1) work(0);
  else {
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; t++) th.emplace_back(work, t);
    for (auto &x : th) x.join();
  }
  c->L = pos;
  c->uploaded = false;
}

void dump_states(cf1gpu_ctx *c, uint64_t *keys, uint8_t *states) {
  if (c->wide) dump_impl<Key2>(c, keys, states);
  else dump_impl<uint64_t>(c, keys, states);
}

void verify_bijection(cf1gpu_ctx *c) {
  if (c->wide) verify_impl<Key2>(c);
  else verify_impl<uint64_t>(c);
}

void query(cf1gpu_ctx *c, const uint64_t *keys, size_t n, uint64_t *slots) {
  if (c->wide) query_impl<Key2>(c, keys, n, slots);
  else query_impl<uint64_t>(c, keys, n, slots);
}

void learned_summary(const cf1gpu_ctx *c, double out5[5]) {
  const LearnedStats &ls = c->wide ? c->b128.li.stats : c->b64.li.stats;
  out5[0] = ls.mean_err;
  out5[1] = ls.mean_window;
  out5[2] = ls.train_loss;
  out5[3] = (double)ls.max_err_all;
  out5[4] = (double)ls.verify_miss_bins;
}

}  // namespace cf1
