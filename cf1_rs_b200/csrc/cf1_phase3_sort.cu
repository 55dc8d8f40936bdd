// Phase 3a on the device: expand every routed super k-mer into canonical
// k-mers, sort each bin, keep one copy of each key (src/mphf.rs:284-363:
// decode, canonicalise, radix sort, dedup per bin).
#include "cf1_device_util.cuh"
#include "cf1_internal.cuh"

namespace cf1 {

namespace {

constexpr int RS_BLOCK = 256;
constexpr int RS_ITEMS = 16;
constexpr uint32_t RS_TILE = RS_BLOCK * RS_ITEMS;  // 4096 keys
constexpr int RS_BITS = 8;
constexpr uint32_t RS_DIGITS = 1u << RS_BITS;
constexpr int RS_NW = RS_BLOCK / 32;

CF1_D uint64_t ceil_div_dev(uint64_t n) { return (n + 31) / 32; }

__global__ void record_len_kernel(const uint64_t *records, uint64_t n, uint32_t *len) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) len[i] = rec_n(records[i]);
}

// Warp-cooperative expansion: a warp takes 32 records, and its lanes walk the
// records' k-mers in one flattened index space, so output stores are
// contiguous whatever the record lengths.  With `sides` (and NM), each
// occurrence also writes its side-set byte: the (front, back) contribution
// its true neighbours in the sequence give the vertex (src/classify.rs:
// 65-518 as the per-side join), so phase 3 can join a vertex's occurrences
// while it removes their duplicate keys.
template <class KeyT>
__global__ void __launch_bounds__(256) expand_kernel(const uint64_t *records, uint64_t n_rec, const uint64_t *kpre,
                                                     const uint64_t *W, int k, KeyT *keys, uint64_t n_keys,
                                                     uint64_t L, uint32_t *queue, uint32_t *err, const uint64_t *NM,
                                                     uint8_t *sides) {
  const unsigned lane = lane_id();
  const uint64_t n_chunks = ceil_div_dev(n_rec);
  uint64_t chunk = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  for (;;) {
    if (queue) {
      uint32_t c = 0;
      if (lane == 0) c = atomicAdd(queue, 1u);
      chunk = __shfl_sync(FULL, c, 0);
    }
    if (chunk >= n_chunks) break;
    uint64_t r = chunk * 32 + lane;
    bool valid = r < n_rec;
    uint64_t rec = valid ? records[r] : 0;
    uint32_t n = valid ? rec_n(rec) : 0;
    uint64_t pos = rec_pos(rec);
    uint64_t off = valid ? kpre[r] : 0;
    // whether the record's first k-mer has a base before it and its last one
    // a base after it (inside a super k-mer the windows before and after are
    // valid, so only these two can lack a neighbour): read once per record,
    // not in the k-mer loop
    uint32_t ends = 0;
    if (sides && valid) {
      const uint64_t q = pos + n - 1;  // the last k-mer
      ends = (uint32_t)(pos > 0 && !is_n(NM, pos - 1)) | ((uint32_t)(q + k < L && !is_n(NM, q + k)) << 1);
    }
    uint32_t incl = warp_inclusive_scan(n);
    uint32_t total = __shfl_sync(FULL, incl, 31);
    uint32_t excl = incl - n;
    for (uint32_t base = 0; base < total; base += 32) {
      uint32_t j = base + lane;
      int lo = 0;
#pragma unroll
      for (int step = 16; step >= 1; step >>= 1) {
        uint32_t v = __shfl_sync(FULL, incl, lo + step - 1);
        if (v <= j) lo += step;
      }
      uint64_t opos = __shfl_sync(FULL, pos, lo);
      uint32_t oex = __shfl_sync(FULL, excl, lo);
      uint64_t ooff = __shfl_sync(FULL, off, lo);
      const uint32_t onrec = __shfl_sync(FULL, n, lo), oends = __shfl_sync(FULL, ends, lo);
      if (j < total) {
        uint32_t t = j - oex;
        if (ooff + t < n_keys && opos + t + k <= L) {
          const uint64_t p = opos + t;
          if (sides) {
            // the neighbours come from the words the k-mer is read from
            const bool hp = t > 0 || (oends & 1u);
            const bool hn = t + 1 < onrec || (oends & 2u);
            uint32_t pb, nb;
            KeyT fw = KOps<KeyT>::extract_nb(W, p, k, hp, pb, nb);
            KeyT rc = KOps<KeyT>::rc(fw, k);
            keys[ooff + t] = kmin(fw, rc);
            sides[ooff + t] = (uint8_t)contribution_sideset(fw, rc, hp, pb, hn, hn ? nb : 0u, k);
          } else {
            KeyT fw = KOps<KeyT>::extract(W, p, k);
            KeyT rc = KOps<KeyT>::rc(fw, k);
            keys[ooff + t] = kmin(fw, rc);
          }
        } else {
          atomicOr(err, (uint32_t)DEV_OVERFLOW);
        }
      }
    }
    if (!queue) break;
  }
}

// Rolling expansion (64-bit keys, k <= 31, with side-set bytes).  A warp
// takes 32 records, whose keys are consecutive in the output; each round,
// every lane takes a run of `er` consecutive occurrences of the warp's
// flattened index space (er <= XR_E, the same for all lanes, so the lanes
// stay balanced whatever the record lengths).  A lane extracts its run's
// first k-mer from the packed words once, then rolls forward and backward
// forms one base at a time (src/kmer.rs:240-262) from a 32-base look-ahead
// word; when its run crosses into the next record it takes that record's
// first k-mer, look-ahead and preceding base, prepared once per record by
// the record's own lane, through shuffles.  The rolled k-mer is also the
// "next k-mer" the side-set byte needs for its self-loop test.  Keys and
// bytes are staged per warp in shared memory and written out contiguously.
constexpr int XR_E = 16;                       // most occurrences a lane takes per round
constexpr int XR_WARPS = 8;
constexpr uint32_t XR_SPAN = 32 * XR_E;        // occurrences a warp takes per round at most
constexpr uint32_t XR_PAD = XR_SPAN + XR_SPAN / 16;
constexpr uint32_t XR_BPAD = XR_SPAN + XR_SPAN / 4;
// Staging slots of key i and byte i: a pad word per 16 keys and four pad
// bytes per 16 bytes, so that the lanes' runs (stride er) fall on different
// shared-memory banks.
CF1_D uint32_t xr_slot(uint32_t i) { return i + (i >> 4); }
CF1_D uint32_t xr_bslot(uint32_t i) { return i + ((i >> 4) << 2); }

// The k-mer starting at base p (k <= 31), the 32 bases after it (p + k ...,
// most significant first) and, with want_prev, the base before it.  Reads
// words p/32 .. p/32 + 2, which the packed sequence's padding covers for any
// p < L.
CF1_D void xr_window(const uint64_t *W, uint64_t p, int k, bool want_prev, uint64_t &fw, uint64_t &ahead,
                     uint32_t &prev) {
  const uint64_t i = p >> 5;
  const int s = (int)(p & 31) * 2;
  const uint64_t w0 = W[i], w1 = W[i + 1], w2 = W[i + 2];
  const uint64_t t0 = s ? ((w0 << s) | (w1 >> (64 - s))) : w0;  // bases p .. p + 31
  const uint64_t t1 = s ? ((w1 << s) | (w2 >> (64 - s))) : w1;  // bases p + 32 .. p + 63
  fw = t0 >> (64 - 2 * k);
  ahead = (t0 << (2 * k)) | (t1 >> (64 - 2 * k));
  prev = want_prev ? (s ? (uint32_t)(w0 >> (64 - s)) & 3 : (uint32_t)W[i - 1] & 3) : 0u;
}

__global__ void __launch_bounds__(XR_WARPS * 32) expand_roll_kernel(const uint64_t *records, uint64_t n_rec,
                                                                    const uint64_t *kpre, const uint64_t *W, int k,
                                                                    uint64_t *keys, uint64_t n_keys, uint64_t L,
                                                                    uint32_t *queue, uint32_t *err,
                                                                    const uint64_t *NM, uint8_t *sides) {
  __shared__ uint64_t skey[XR_WARPS][XR_PAD];
  __shared__ uint8_t sside[XR_WARPS][XR_BPAD];
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
  uint64_t *sk = skey[warp];
  uint8_t *ss = sside[warp];
  const uint64_t n_chunks = ceil_div_dev(n_rec);
  const uint64_t kmask = KOps<uint64_t>::mask(k);
  const int top = 2 * k - 2;
  uint64_t chunk = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  for (;;) {
    if (queue) {
      uint32_t c = 0;
      if (lane == 0) c = atomicAdd(queue, 1u);
      chunk = __shfl_sync(FULL, c, 0);
    }
    if (chunk >= n_chunks) break;
    const uint64_t r = chunk * 32 + lane;
    const bool valid = r < n_rec;
    const uint64_t rec = valid ? records[r] : 0;
    const uint32_t n = valid ? rec_n(rec) : 0;
    const uint64_t pos = rec_pos(rec);
    const uint64_t out0 = kpre[chunk * 32];  // the chunk's records are consecutive in the key array
    // a record whose windows leave the input is flagged and its bases are
    // never read (its keys' slots get zeros)
    const bool inb = valid && pos + n - 1 + k <= L;
    if (valid && !inb) atomicOr(err, (uint32_t)DEV_OVERFLOW);
    uint32_t ends = 0, pb0 = 0;
    uint64_t fw0 = 0, rc0 = 0, ah0 = 0;
    if (inb) {
      const uint64_t q = pos + n - 1;  // the last k-mer
      ends = (uint32_t)(pos > 0 && !is_n(NM, pos - 1)) | ((uint32_t)(q + k < L && !is_n(NM, q + k)) << 1);
      xr_window(W, pos, k, ends & 1u, fw0, ah0, pb0);
      rc0 = KOps<uint64_t>::rc(fw0, k);
    }
    // n (13 bits), whether the record has a base before / after (2), the
    // base before it (2), whether its bases may be read (1)
    const uint32_t info0 = n | (ends << 16) | (pb0 << 18) | ((uint32_t)inb << 20);
    const uint32_t incl = warp_inclusive_scan(n);
    const uint32_t total = __shfl_sync(FULL, incl, 31);
    for (uint32_t base = 0; base < total;) {
      const uint32_t rem = total - base;
      const uint32_t er = rem >= XR_SPAN ? (uint32_t)XR_E : (rem + 31) / 32;
      const uint32_t j0 = base + lane * er;
      // the record holding j0: the number of records ending at or before it
      int cur = 0;
#pragma unroll
      for (int step = 16; step >= 1; step >>= 1) {
        const uint32_t v = __shfl_sync(FULL, incl, cur + step - 1);
        if (v <= j0) cur += step;
      }
      uint32_t info = __shfl_sync(FULL, info0, cur);
      uint32_t rec_end = __shfl_sync(FULL, incl, cur);
      const uint64_t cpos = __shfl_sync(FULL, pos, cur);
      uint32_t t = j0 - (rec_end - (info & 0x1FFFu));
      uint64_t fw = 0, rc = 0, ah = 0;
      uint32_t prevb = 0;
      if (j0 < total && (info >> 20 & 1u)) {
        xr_window(W, cpos + t, k, t > 0 || (info >> 16 & 1u), fw, ah, prevb);
        rc = KOps<uint64_t>::rc(fw, k);
      }
      for (uint32_t e = 0; e < er; e++) {
        const uint32_t j = j0 + e;
        // the next record's first k-mer, taken when the run crosses into it
        const int nx = cur < 31 ? cur + 1 : 31;
        const uint64_t fwN = __shfl_sync(FULL, fw0, nx), rcN = __shfl_sync(FULL, rc0, nx),
                       ahN = __shfl_sync(FULL, ah0, nx);
        const uint32_t infoN = __shfl_sync(FULL, info0, nx), endN = __shfl_sync(FULL, incl, nx);
        if (j == rec_end && j < total) {
          cur = nx;
          fw = fwN;
          rc = rcN;
          ah = ahN;
          info = infoN;
          rec_end = endN;
          t = 0;
          prevb = (infoN >> 18) & 3u;
        }
        const bool hp = t > 0 || (info >> 16 & 1u);
        const bool hn = t + 1 < (info & 0x1FFFu) || (info >> 17 & 1u);
        const uint32_t nb = (uint32_t)(ah >> 62);
        const uint64_t nf = ((fw << 2) | nb) & kmask;
        const uint64_t nr = (rc >> 2) | ((uint64_t)(3 - nb) << top);
        if (j < total) {
          const uint32_t i = lane * er + e;
          sk[xr_slot(i)] = kmin(fw, rc);
          ss[xr_bslot(i)] = (uint8_t)contribution_sideset_rolled(fw, rc, nf, nr, hp, prevb, hn, nb);
        }
        prevb = (uint32_t)(fw >> top);  // this k-mer's first base precedes the next one
        fw = nf;
        rc = nr;
        ah <<= 2;
        t++;
      }
      __syncwarp();
      const uint32_t span = 32 * er;
      for (uint32_t i = lane; i < span; i += 32) {
        const uint64_t o = out0 + base + i;
        if (base + i < total) {
          if (o < n_keys) {
            keys[o] = sk[xr_slot(i)];
            sides[o] = ss[xr_bslot(i)];
          } else {
            atomicOr(err, (uint32_t)DEV_OVERFLOW);
          }
        }
      }
      __syncwarp();
      base += span;
    }
    if (!queue) break;
  }
}

// Per tile digit counts, stored segment-major then digit-major so that one
// exclusive scan over the array yields every (segment, digit, tile) output
// position: previous segments' sizes + smaller digits of this segment +
// earlier tiles of this digit.
template <class KeyT>
__global__ void __launch_bounds__(RS_BLOCK) rs_hist_kernel(const KeyT *keys, const uint64_t *seg_off,
                                                           const uint32_t *tile_off, uint32_t nseg, int shift,
                                                           uint32_t *H) {
  __shared__ uint32_t h[RS_DIGITS];
  const uint32_t t = blockIdx.x;
  const uint32_t total = tile_off[nseg];
  if (t >= total) {
    for (uint32_t d = threadIdx.x; d < RS_DIGITS; d += RS_BLOCK) H[(uint64_t)t * RS_DIGITS + d] = 0;
    return;
  }
  for (uint32_t d = threadIdx.x; d < RS_DIGITS; d += RS_BLOCK) h[d] = 0;
  __syncthreads();
  TileSpan sp = tile_span(seg_off, tile_off, nseg, t, RS_TILE);
  for (uint64_t i = sp.start + threadIdx.x; i < sp.end; i += RS_BLOCK)
    atomicAdd(&h[KOps<KeyT>::digit(keys[i], shift, RS_DIGITS - 1)], 1u);
  __syncthreads();
  for (uint32_t d = threadIdx.x; d < RS_DIGITS; d += RS_BLOCK)
    H[(uint64_t)sp.first_tile * RS_DIGITS + (uint64_t)d * sp.ntiles + (t - sp.first_tile)] = h[d];
}

// Stable scatter of one tile: keys are taken in rounds of RS_BLOCK (round r,
// thread i holds tile element r*RS_BLOCK + i), ranked inside each warp with
// match_any, and the per (round, warp, digit) counts are turned into
// per-digit offsets by one pass per digit over the shared table.
template <class KeyT>
__global__ void __launch_bounds__(RS_BLOCK) rs_scatter_kernel(const KeyT *in, KeyT *out, const uint64_t *seg_off,
                                                              const uint32_t *tile_off, uint32_t nseg, int shift,
                                                              const uint64_t *Hs) {
  extern __shared__ uint16_t cnt[];  // [RS_ITEMS][RS_NW][RS_DIGITS]
  __shared__ uint64_t s_base[RS_DIGITS];
  const uint32_t t = blockIdx.x;
  if (t >= tile_off[nseg]) return;
  TileSpan sp = tile_span(seg_off, tile_off, nseg, t, RS_TILE);
  const unsigned tid = threadIdx.x, warp = tid >> 5;
  {
    uint32_t *c32 = reinterpret_cast<uint32_t *>(cnt);
    for (uint32_t i = tid; i < RS_ITEMS * RS_NW * RS_DIGITS / 2; i += RS_BLOCK) c32[i] = 0;
  }
  for (uint32_t d = tid; d < RS_DIGITS; d += RS_BLOCK)
    s_base[d] = Hs[(uint64_t)sp.first_tile * RS_DIGITS + (uint64_t)d * sp.ntiles + (t - sp.first_tile)];
  __syncthreads();
  KeyT key[RS_ITEMS];
  uint32_t dg[RS_ITEMS];
  uint32_t wr[RS_ITEMS];
  const unsigned lt = lanemask_lt();
#pragma unroll
  for (int r = 0; r < RS_ITEMS; r++) {
    uint64_t i = sp.start + (uint64_t)r * RS_BLOCK + tid;
    bool act = i < sp.end;
    key[r] = act ? in[i] : KeyT();
    dg[r] = act ? KOps<KeyT>::digit(key[r], shift, RS_DIGITS - 1) : 0xFFFFFFFFu;
    unsigned peers = __match_any_sync(FULL, dg[r]);
    wr[r] = __popc(peers & lt);
    if (act && wr[r] == 0) cnt[(r * RS_NW + warp) * RS_DIGITS + dg[r]] = (uint16_t)__popc(peers);
  }
  __syncthreads();
  for (uint32_t d = tid; d < RS_DIGITS; d += RS_BLOCK) {
    uint32_t run = 0;
    for (int r = 0; r < RS_ITEMS; r++)
      for (int w = 0; w < RS_NW; w++) {
        uint16_t &c = cnt[(r * RS_NW + w) * RS_DIGITS + d];
        uint32_t v = c;
        c = (uint16_t)run;
        run += v;
      }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < RS_ITEMS; r++) {
    if (dg[r] != 0xFFFFFFFFu) {
      uint64_t pos = s_base[dg[r]] + cnt[(r * RS_NW + warp) * RS_DIGITS + dg[r]] + wr[r];
      out[pos] = key[r];
    }
  }
}

// ---- segmented unique ----
template <class KeyT>
__global__ void __launch_bounds__(RS_BLOCK) uq_count_kernel(const KeyT *keys, const uint64_t *seg_off,
                                                            const uint32_t *tile_off, uint32_t nseg,
                                                            uint32_t *tile_cnt) {
  __shared__ uint32_t sm[RS_NW];
  const uint32_t t = blockIdx.x;
  if (t >= tile_off[nseg]) {
    if (threadIdx.x == 0) tile_cnt[t] = 0;
    return;
  }
  TileSpan sp = tile_span(seg_off, tile_off, nseg, t, RS_TILE);
  const uint64_t seg_start = seg_off[sp.seg];
  uint32_t c = 0;
  for (uint64_t i = sp.start + threadIdx.x; i < sp.end; i += RS_BLOCK)
    c += (i == seg_start || keys[i] != keys[i - 1]) ? 1u : 0u;
  uint32_t tot = block_sum<RS_BLOCK>(c, sm);
  if (threadIdx.x == 0) tile_cnt[t] = tot;
}

template <class KeyT>
__global__ void __launch_bounds__(RS_BLOCK) uq_write_kernel(const KeyT *keys, const uint64_t *seg_off,
                                                            const uint32_t *tile_off, uint32_t nseg,
                                                            const uint64_t *tile_out, KeyT *out) {
  __shared__ uint32_t sm[RS_NW];
  const uint32_t t = blockIdx.x;
  if (t >= tile_off[nseg]) return;
  TileSpan sp = tile_span(seg_off, tile_off, nseg, t, RS_TILE);
  const uint64_t seg_start = seg_off[sp.seg];
  uint64_t i0 = sp.start + (uint64_t)threadIdx.x * RS_ITEMS;
  uint32_t flags = 0, c = 0;
#pragma unroll
  for (int j = 0; j < RS_ITEMS; j++) {
    uint64_t i = i0 + j;
    bool f = i < sp.end && (i == seg_start || keys[i] != keys[i - 1]);
    flags |= (uint32_t)f << j;
    c += f;
  }
  uint32_t tot;
  uint32_t pre = block_exclusive_scan<RS_BLOCK>(c, sm, tot);
  uint64_t o = tile_out[t] + pre;
#pragma unroll
  for (int j = 0; j < RS_ITEMS; j++)
    if ((flags >> j) & 1) out[o++] = keys[i0 + j];
}

__global__ void seg_out_off_kernel(const uint32_t *tile_off, uint32_t nseg, const uint64_t *tile_out, uint64_t *out_off) {
  uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b <= nseg) out_off[b] = tile_out[tile_off[b]];
}

}  // namespace

void record_kmer_prefix(const uint64_t *records, uint64_t n_rec, uint64_t *kpre, DevBuf &lens, DevBuf &scratch,
                        cudaStream_t s) {
  uint32_t *len = lens.get<uint32_t>(n_rec + 1);
  if (n_rec) {
    record_len_kernel<<<(unsigned)ceil_div(n_rec, 256), 256, 0, s>>>(records, n_rec, len);
    CF1_LAUNCH_CHECK();
  }
  exclusive_scan_u32(len, kpre, n_rec, scratch, s);
}

template <class KeyT>
void launch_expand(const uint64_t *records, uint64_t n_rec, const uint64_t *kpre, const uint64_t *W, int k, KeyT *keys,
                   uint64_t n_keys, uint64_t L, uint32_t *queue, uint32_t *err, int persistent_ctas, cudaStream_t s,
                   const uint64_t *NM, uint8_t *sides) {
  if (n_rec == 0) return;
  uint64_t warps = ceil_div(n_rec, 32);
  if constexpr (KOps<KeyT>::WORDS == 1) {
    if (sides && k <= 31) {
      unsigned grid = persistent_ctas ? persistent_grid(expand_roll_kernel, XR_WARPS * 32, 0, persistent_ctas,
                                                        ceil_div(warps, XR_WARPS))
                                      : (unsigned)ceil_div(warps, XR_WARPS);
      expand_roll_kernel<<<grid, XR_WARPS * 32, 0, s>>>(records, n_rec, kpre, W, k, keys, n_keys, L,
                                                        persistent_ctas ? queue : nullptr, err, NM, sides);
      CF1_LAUNCH_CHECK();
      return;
    }
  }
  unsigned grid = persistent_ctas ? persistent_grid(expand_kernel<KeyT>, 256, 0, persistent_ctas, ceil_div(warps, 8))
                                  : (unsigned)ceil_div(warps, 8);
  expand_kernel<KeyT><<<grid, 256, 0, s>>>(records, n_rec, kpre, W, k, keys, n_keys, L,
                                           persistent_ctas ? queue : nullptr, err, NM, sides);
  CF1_LAUNCH_CHECK();
}

template <class KeyT>
void segmented_sort(KeyT *keys, uint64_t n, const uint64_t *seg_off, uint32_t nseg, int key_bits, SortScratch<KeyT> &sc,
                    cudaStream_t s) {
  if (n == 0) return;
  uint32_t ub_tiles = (uint32_t)(ceil_div(n, RS_TILE) + nseg);
  uint32_t *tile_off = sc.tile_off.template get<uint32_t>(nseg + 1);
  segment_tiles(seg_off, nseg, RS_TILE, tile_off, s);
  KeyT *alt = sc.alt.template get<KeyT>(n + 1);
  uint32_t *H = sc.hist.template get<uint32_t>((uint64_t)ub_tiles * RS_DIGITS);
  uint64_t *Hs = sc.hscan.template get<uint64_t>((uint64_t)ub_tiles * RS_DIGITS + 1);
  size_t smem = (size_t)RS_ITEMS * RS_NW * RS_DIGITS * sizeof(uint16_t);
  CF1_CUDA(cudaFuncSetAttribute(rs_scatter_kernel<KeyT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  KeyT *src = keys, *dst = alt;
  int passes = (key_bits + RS_BITS - 1) / RS_BITS;
  for (int p = 0; p < passes; p++) {
    int shift = p * RS_BITS;
    rs_hist_kernel<KeyT><<<ub_tiles, RS_BLOCK, 0, s>>>(src, seg_off, tile_off, nseg, shift, H);
    CF1_LAUNCH_CHECK();
    exclusive_scan_u32(H, Hs, (uint64_t)ub_tiles * RS_DIGITS, sc.scan_tmp, s);
    rs_scatter_kernel<KeyT><<<ub_tiles, RS_BLOCK, smem, s>>>(src, dst, seg_off, tile_off, nseg, shift, Hs);
    CF1_LAUNCH_CHECK();
    KeyT *t = src; src = dst; dst = t;
  }
  if (src != keys) CF1_CUDA(cudaMemcpyAsync(keys, src, n * sizeof(KeyT), cudaMemcpyDeviceToDevice, s));
}

template <class KeyT>
void segmented_unique(const KeyT *keys, uint64_t n, const uint64_t *seg_off, uint32_t nseg, KeyT *out, uint64_t *out_off,
                      SortScratch<KeyT> &sc, cudaStream_t s) {
  uint32_t ub_tiles = (uint32_t)(ceil_div(n, RS_TILE) + nseg);
  uint32_t *tile_off = sc.tile_off.template get<uint32_t>(nseg + 1);
  segment_tiles(seg_off, nseg, RS_TILE, tile_off, s);
  uint32_t *tc = sc.tile_cnt.template get<uint32_t>(ub_tiles + 1);
  uint64_t *to = sc.tile_out.template get<uint64_t>(ub_tiles + 2);
  if (ub_tiles) {
    uq_count_kernel<KeyT><<<ub_tiles, RS_BLOCK, 0, s>>>(keys, seg_off, tile_off, nseg, tc);
    CF1_LAUNCH_CHECK();
  }
  exclusive_scan_u32(tc, to, ub_tiles, sc.scan_tmp, s);
  if (ub_tiles) {
    uq_write_kernel<KeyT><<<ub_tiles, RS_BLOCK, 0, s>>>(keys, seg_off, tile_off, nseg, to, out);
    CF1_LAUNCH_CHECK();
  }
  seg_out_off_kernel<<<(unsigned)ceil_div(nseg + 1, 256), 256, 0, s>>>(tile_off, nseg, to, out_off);
  CF1_LAUNCH_CHECK();
}

#define CF1_INST(KT)                                                                                                 \
  template void launch_expand<KT>(const uint64_t *, uint64_t, const uint64_t *, const uint64_t *, int, KT *,        \
                                  uint64_t, uint64_t, uint32_t *, uint32_t *, int, cudaStream_t, const uint64_t *,  \
                                  uint8_t *);                                                                       \
  template void segmented_sort<KT>(KT *, uint64_t, const uint64_t *, uint32_t, int, SortScratch<KT> &, cudaStream_t); \
  template void segmented_unique<KT>(const KT *, uint64_t, const uint64_t *, uint32_t, KT *, uint64_t *,            \
                                     SortScratch<KT> &, cudaStream_t);
CF1_INST(uint64_t)
CF1_INST(Key2)
#undef CF1_INST

}  // namespace cf1
