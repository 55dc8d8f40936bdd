// Phase 3a, MSD form: distinct canonical k-mers per bin, sorted or not.
//
//   1. one or two multisplit passes on the top P bits of the keys (sorted) or
//      of key * KEY_SPREAD_MUL (distinct only), segmented by bin (P chosen so
//      a sub-bucket fits shared memory);
//   2. one CTA per sub-bucket: a shared-memory hash set keeps one copy of
//      each key; the sorted form then counting-sorts on the next 10 bits,
//      insertion-sorts the small buckets (bitonic sort of the whole
//      sub-bucket if any bucket is large); distinct keys are written back at
//      the sub-bucket's start;
//   3. a scan of the per-sub-bucket counts and a copy into the dense distinct
//      array; a bin's first sub-bucket gives its slot offset.
// A sub-bucket above CAP keys (long homopolymers, huge tandem arrays) makes
// the caller fall back to the LSD path (cf1_phase3_sort.cu) for the run.
#include "cf1_device_util.cuh"
#include "cf1_internal.cuh"
#include "cf1_mphf.cuh"
#include "cf1_msdsort.cuh"

namespace cf1 {

namespace {

constexpr int MS_BLOCK = 256;
constexpr int MS_ITEMS = 16;
constexpr uint32_t MS_TILE = MS_BLOCK * MS_ITEMS;  // 4096 keys per pass tile
constexpr int MS_NW = MS_BLOCK / 32;
constexpr int CS_BLOCK = 512;  // 16 warps: shared memory allows 2 CTAs per SM
constexpr int CS_BITS = 10;
constexpr uint32_t CS_BUCKETS = 1u << CS_BITS;
// Insertion sort up to this many keys per bucket.  Repeats put hundreds of
// copies of one k-mer in a bucket; insertion sort passes over equal keys at
// once, so large buckets of few distinct values stay cheap.
constexpr uint32_t CS_SMALL = 512;
constexpr uint32_t CS_DEDUP_MIN = 64;  // 64-bit sub-buckets above this size are deduplicated first

// Keys a sub-bucket's shared-memory sort holds.  The unsorted (deduplicate
// only) path keeps 64-bit sub-buckets at half that size, so its shared memory
// fits four CTAs per SM instead of two.
constexpr uint32_t cs_cap_for(bool wide, bool sorted) { return wide ? 4096u : (sorted ? 8192u : 4096u); }
template <class KeyT, bool SORTED = true>
constexpr uint32_t cs_cap() { return cs_cap_for(KOps<KeyT>::WORDS == 2, SORTED); }

// Digit of a key in a multisplit pass: bits [shift, shift + width) of the key
// or, when only the distinct keys and not their order are needed (hashed),
// of key * MS_HASH_MUL.  The product's top bits spread any key set evenly,
// where the key's own top bits -- the first bases of a canonical k-mer --
// are skewed several-fold.  (64-bit keys; wider keys always sort.)
constexpr uint64_t MS_HASH_MUL = KEY_SPREAD_MUL;
template <class KeyT>
CF1_D uint32_t ms_digit(const KeyT &k, int shift, uint32_t mask, bool hashed);
template <>
CF1_D uint32_t ms_digit<uint64_t>(const uint64_t &k, int shift, uint32_t mask, bool hashed) {
  return (uint32_t)((hashed ? k * MS_HASH_MUL : k) >> shift) & mask;
}
template <>
CF1_D uint32_t ms_digit<Key2>(const Key2 &k, int shift, uint32_t mask, bool) {
  return KOps<Key2>::digit(k, shift, mask);
}


// ---------------------------------------------------------------- multisplit pass
template <class KeyT, int BITS>
__global__ void __launch_bounds__(MS_BLOCK) ms_hist_kernel(const KeyT *keys, const uint64_t *seg_off,
                                                           const uint32_t *tile_off, uint32_t nseg, int shift,
                                                           bool hashed, uint32_t *H) {
  constexpr uint32_t DIG = 1u << BITS;
  __shared__ uint32_t h[DIG];
  const uint32_t t = blockIdx.x;
  if (t >= tile_off[nseg]) {
    for (uint32_t d = threadIdx.x; d < DIG; d += MS_BLOCK) H[(uint64_t)t * DIG + d] = 0;
    return;
  }
  for (uint32_t d = threadIdx.x; d < DIG; d += MS_BLOCK) h[d] = 0;
  __syncthreads();
  TileSpan sp = tile_span(seg_off, tile_off, nseg, t, MS_TILE);
  for (uint64_t i = sp.start + threadIdx.x; i < sp.end; i += MS_BLOCK)
    atomicAdd(&h[ms_digit(keys[i], shift, DIG - 1, hashed)], 1u);
  __syncthreads();
  for (uint32_t d = threadIdx.x; d < DIG; d += MS_BLOCK)
    H[(uint64_t)sp.first_tile * DIG + (uint64_t)d * sp.ntiles + (t - sp.first_tile)] = h[d];
}

// Multisplit of one tile: warp w ranks the keys of the w-th 512-key slice of
// the tile by a shared-memory atomic add on its per-warp digit count (the
// order inside a digit does not matter: every sub-bucket is sorted or
// deduplicated whole afterwards), a per-digit prefix over warps gives
// tile-local positions, the tile is staged in shared memory in digit order,
// and each digit's run is written out with consecutive threads on
// consecutive addresses.  Four CTAs per SM (64 registers): at 3.1 Gbp the
// two 64-bit passes took 3.3 ms less than with three CTAs and 80 registers.
// With pin/pout, each key's payload byte (its side-set byte) moves with it;
// with PACK (pin, no pout; hashed 64-bit keys, pack = the pass's bits) the
// byte goes into the key's packed output word (see pay_code).
template <class KeyT, int BITS, bool PACK>
__global__ void __launch_bounds__(MS_BLOCK, 4) ms_scatter_kernel(const KeyT *in, KeyT *out, const uint64_t *seg_off,
                                                                 const uint32_t *tile_off, uint32_t nseg, int shift,
                                                                 bool hashed, const uint64_t *Hs, const uint8_t *pin,
                                                                 uint8_t *pout, int pack) {
  constexpr uint32_t DIG = 1u << BITS;
  extern __shared__ __align__(16) unsigned char ms_smem[];
  KeyT *stage = reinterpret_cast<KeyT *>(ms_smem);                            // [MS_TILE]
  uint32_t *whist = reinterpret_cast<uint32_t *>(stage + MS_TILE);           // [MS_NW][DIG]
  uint32_t *lstart = whist + MS_NW * DIG;                                     // [DIG]
  uint64_t *base = reinterpret_cast<uint64_t *>(lstart + DIG);                // [DIG]
  uint8_t *pstage = reinterpret_cast<uint8_t *>(base + DIG);                  // [MS_TILE] when pin
  __shared__ uint32_t sm[MS_BLOCK / 32];
  const uint32_t t = blockIdx.x;
  if (t >= tile_off[nseg]) return;
  TileSpan sp = tile_span(seg_off, tile_off, nseg, t, MS_TILE);
  const unsigned tid = threadIdx.x, lane = lane_id(), warp = tid >> 5;
  for (uint32_t i = tid; i < MS_NW * DIG; i += MS_BLOCK) whist[i] = 0;
  for (uint32_t d = tid; d < DIG; d += MS_BLOCK)
    base[d] = Hs[(uint64_t)sp.first_tile * DIG + (uint64_t)d * sp.ntiles + (t - sp.first_tile)];
  __syncthreads();
  const uint32_t n = (uint32_t)(sp.end - sp.start);
  // per key: (rank in the warp's slice for its digit) << 8 | digit, or ~0
  // for lanes past the tile (128-bit keys are read again when staged, which
  // keeps their register count down)
  uint32_t pk[MS_ITEMS];
  uint32_t *wh = whist + warp * DIG;
  // 64-bit keys: all of the thread's loads are issued before the first is
  // used, and the keys stay in registers for the staging step
  constexpr bool HOLD = KOps<KeyT>::WORDS == 1;
  KeyT kk[HOLD ? MS_ITEMS : 1];
  // the payload bytes are loaded with the keys, four to a register, so their
  // latency is not paid again when the tile is staged
  uint32_t pb[MS_ITEMS / 4];
#pragma unroll
  for (int q = 0; q < MS_ITEMS / 4; q++) pb[q] = 0;
  if constexpr (HOLD) {
#pragma unroll
    for (int r = 0; r < MS_ITEMS; r++) {
      uint32_t li = warp * (MS_ITEMS * 32) + r * 32 + lane;
      kk[r] = li < n ? in[sp.start + li] : KeyT{};
      if (pin && li < n) pb[r >> 2] |= (uint32_t)pin[sp.start + li] << (8 * (r & 3));
    }
  }
#pragma unroll
  for (int r = 0; r < MS_ITEMS; r++) {
    uint32_t li = warp * (MS_ITEMS * 32) + r * 32 + lane;
    pk[r] = 0xFFFFFFFFu;
    if (li < n) {
      uint32_t d = ms_digit(HOLD ? kk[HOLD ? r : 0] : in[sp.start + li], shift, DIG - 1, hashed);
      pk[r] = (atomicAdd(&wh[d], 1u) << 8) | d;
    }
  }
  __syncthreads();
  // per digit: exclusive prefix over warps; tile total per digit
  uint32_t tot_d = 0;
  for (uint32_t d = tid; d < DIG; d += MS_BLOCK) {
    uint32_t run = 0;
    for (int w = 0; w < MS_NW; w++) {
      uint32_t v = whist[w * DIG + d];
      whist[w * DIG + d] = run;
      run += v;
    }
    if (DIG <= MS_BLOCK) tot_d = run;
    else lstart[d] = run;
  }
  __syncthreads();
  // tile-local start of each digit: exclusive scan over digits (one digit a
  // thread; the threads past the digits add nothing)
  if (DIG <= MS_BLOCK) {
    uint32_t tot;
    uint32_t pre = block_exclusive_scan<MS_BLOCK>(tot_d, sm, tot);
    if (tid < DIG) lstart[tid] = pre;
  } else if (tid == 0) {
    uint32_t run = 0;
    for (uint32_t d = 0; d < DIG; d++) {
      uint32_t v = lstart[d];
      lstart[d] = run;
      run += v;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < MS_ITEMS; r++) {
    if (pk[r] != 0xFFFFFFFFu) {
      uint32_t d = pk[r] & 0xFF, li = warp * (MS_ITEMS * 32) + r * 32 + lane;
      const uint32_t at = lstart[d] + wh[d] + (pk[r] >> 8);
      stage[at] = HOLD ? kk[HOLD ? r : 0] : in[sp.start + li];
      if (pin) pstage[at] = HOLD ? (uint8_t)(pb[r >> 2] >> (8 * (r & 3))) : pin[sp.start + li];
    }
  }
  __syncthreads();
  for (uint32_t i = tid; i < n; i += MS_BLOCK) {
    KeyT kk = stage[i];
    uint32_t d = ms_digit(kk, shift, DIG - 1, hashed);
    const uint64_t o = base[d] + (i - lstart[d]);
    if constexpr (PACK) {  // hashed 64-bit keys with payloads: the packed word (see pay_code)
      out[o] = ((kk * MS_HASH_MUL) << pack) | pay_code(pstage[i]);
    } else {
      out[o] = kk;
      if (pout) pout[o] = pstage[i];
    }
  }
}

// Sub-bucket starts after the last pass: sub-bucket (segment s, digit d)
// begins at the scanned histogram entry of its first tile.
template <int BITS>
__global__ void ms_subbucket_kernel(const uint64_t *seg_off, const uint32_t *tile_off, uint32_t nseg,
                                    const uint64_t *Hs, uint64_t *sb_off) {
  constexpr uint32_t DIG = 1u << BITS;
  uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint64_t nsub = (uint64_t)nseg * DIG;
  if (j > nsub) return;
  if (j == nsub) {
    sb_off[j] = seg_off[nseg];
    return;
  }
  uint32_t s = (uint32_t)(j / DIG), d = (uint32_t)(j % DIG);
  uint32_t ft = tile_off[s], nt = tile_off[s + 1] - ft;
  sb_off[j] = nt ? Hs[(uint64_t)ft * DIG + (uint64_t)d * nt] : seg_off[s];
}

// ---------------------------------------------------------------- chunk sort
template <class KeyT>
CF1_D void cs_swap_if(KeyT &a, KeyT &b, bool up) {
  if ((b < a) == up) {
    KeyT t = a;
    a = b;
    b = t;
  }
}

// Replaces T[a, a+n) by its distinct keys (any order) through an
// open-addressing set in shared memory; returns their count, or ~0u when
// they do not fit in three quarters of the set.  Every probe sequence is
// bounded by the set size.  Warps step through the keys together, so the
// insert count and the give-up test are per warp; the set is emptied into T
// a warp-sized group of slots at a time.  With TP (payload bytes parallel to
// T), the payloads of a key's copies are ORed into its slot's byte of SPw
// (cap bytes of shared memory) and written beside the key: the per-side join
// of the vertex's occurrences.  A pass that gives up leaves T and TP as they
// were.
CF1_D uint32_t cs_hash_dedup(uint64_t *T, uint64_t a, uint64_t n, uint64_t *S, uint32_t cap, uint32_t *s_cnt,
                             uint32_t *sm, uint8_t *TP = nullptr, uint32_t *SPw = nullptr) {
  (void)sm;
  const unsigned tid = threadIdx.x, lane = lane_id();
  const uint64_t EMPTY = ~0ull;  // above every key (keys use at most 62 bits)
  uint32_t tsize = 64, tbits = 6;  // a power of two >= 1.5 n, at most cap
  while (tsize < cap && (uint64_t)tsize < n + n / 2) {
    tsize <<= 1;
    tbits++;
  }
  for (uint32_t i = tid; i < tsize; i += CS_BLOCK) S[i] = EMPTY;
  if (TP)
    for (uint32_t i = tid; i < tsize / 4; i += CS_BLOCK) SPw[i] = 0;
  if (tid == 0) *s_cnt = 0;
  __syncthreads();
  const uint32_t limit = tsize / 4 * 3;
  for (uint64_t base = tid - lane; base < n; base += CS_BLOCK) {
    uint32_t seen = 0;
    if (lane == 0) seen = *reinterpret_cast<volatile uint32_t *>(s_cnt);
    if (__shfl_sync(FULL, seen, 0) > limit) break;
    const uint64_t i = base + lane;
    bool added = false;
    if (i < n) {
      const uint64_t key = T[a + i];
      const uint32_t pay = TP ? TP[a + i] : 0u;  // loaded beside the key, not after the probe
      uint32_t h = (uint32_t)((key * 0x9E3779B97F4A7C15ull) >> (64 - tbits));  // multiplicative hashing
      for (uint32_t probe = 0; probe < tsize; probe++) {
        unsigned long long old = atomicCAS(reinterpret_cast<unsigned long long *>(S + h), EMPTY, key);
        if (old == EMPTY || old == key) {
          added = old == EMPTY;
          if (TP) atomicOr(&SPw[h >> 2], pay << (8 * (h & 3)));
          break;
        }
        h = (h + 1) & (tsize - 1);
      }
    }
    const unsigned b = __ballot_sync(FULL, added);
    if (lane == 0 && b) atomicAdd(s_cnt, (uint32_t)__popc(b));
  }
  __syncthreads();
  const uint32_t d = *s_cnt;
  __syncthreads();
  if (d > limit) return ~0u;
  if (tid == 0) *s_cnt = 0;
  __syncthreads();
  for (uint32_t base = tid - lane; base < tsize; base += CS_BLOCK) {
    const uint64_t v = S[base + lane];
    const bool f = v != EMPTY;
    const unsigned b = __ballot_sync(FULL, f);
    uint32_t o = 0;
    if (lane == 0 && b) o = atomicAdd(s_cnt, (uint32_t)__popc(b));
    o = __shfl_sync(FULL, o, 0);
    if (f) {
      const uint64_t at = a + o + __popc(b & lanemask_lt());
      T[at] = v;
      if (TP) TP[at] = (uint8_t)(SPw[(base + lane) >> 2] >> (8 * ((base + lane) & 3)));
    }
  }
  __syncthreads();
  return d;
}

// Bucket of a key for the shared-memory counting sort: the bits
// [s1, s1+b1) minus off1, followed by the bits [s2, s2+b2).  A plain
// sub-bucket uses the next bits below its prefix (b2 = 0); a chunk of pieces
// of a split sub-bucket uses the piece index relative to the chunk's first
// piece, then further bits.
struct CsDigit {
  int s1, b1, s2, b2;
  uint32_t off1;
  template <class KeyT>
  CF1_D uint32_t operator()(const KeyT &k) const {
    uint32_t d1 = b1 ? KOps<KeyT>::digit(k, s1, (1u << b1) - 1) - off1 : 0u;
    uint32_t d2 = b2 ? KOps<KeyT>::digit(k, s2, (1u << b2) - 1) : 0u;
    return (d1 << b2) | d2;
  }
};

struct CsShared {
  uint32_t *hist, *cur, *sm;
  int *big;
  uint8_t *SP = nullptr;  // payload bytes beside S (CAP), when the keys carry payloads
};

template <class KeyT>
CF1_D void cs_swap_if(KeyT &a, KeyT &b, uint8_t *pa, uint8_t *pb, bool up) {
  if ((b < a) == up) {
    KeyT t = a;
    a = b;
    b = t;
    if (pa) {
      uint8_t u = *pa;
      *pa = *pb;
      *pb = u;
    }
  }
}

// Sorted distinct keys of src[0, m) (m <= CAP, keys all in [0, 1024) buckets
// of dig) into out[0, tot); returns tot.  src is fully read into shared
// memory before out is written, so they may overlap.  With srcP/outP (and
// sh.SP), each key's payload byte moves with it and the payloads of a key's
// copies are ORed.  All threads call it.
template <class KeyT>
CF1_D uint32_t cs_sort_unique_range(const KeyT *src, uint32_t m, const CsDigit &dig, KeyT *S, const CsShared &sh,
                                    KeyT *out, bool distinct, const uint8_t *srcP = nullptr,
                                    uint8_t *outP = nullptr) {
  uint8_t *SP = srcP ? sh.SP : nullptr;
  constexpr uint32_t CAP = cs_cap<KeyT>();
  const unsigned tid = threadIdx.x;
  for (uint32_t i = tid; i < CS_BUCKETS; i += CS_BLOCK) sh.hist[i] = 0;
  if (tid == 0) *sh.big = 0;
  __syncthreads();
  for (uint32_t i = tid; i < m; i += CS_BLOCK) atomicAdd(&sh.hist[dig(src[i])], 1u);
  __syncthreads();
  {
    constexpr int PER = CS_BUCKETS / CS_BLOCK;
    uint32_t v[PER], s = 0;
#pragma unroll
    for (int q = 0; q < PER; q++) {
      v[q] = sh.hist[tid * PER + q];
      s += v[q];
    }
    uint32_t tot;
    uint32_t pre = block_exclusive_scan<CS_BLOCK>(s, sh.sm, tot);
#pragma unroll
    for (int q = 0; q < PER; q++) {
      sh.hist[tid * PER + q] = pre;
      sh.cur[tid * PER + q] = pre;
      pre += v[q];
    }
  }
  __syncthreads();
  for (uint32_t i = tid; i < m; i += CS_BLOCK) {
    KeyT key = src[i];
    const uint32_t at = atomicAdd(&sh.cur[dig(key)], 1u);
    S[at] = key;
    if (SP) SP[at] = srcP[i];
  }
  __syncthreads();
  // insertion sort per bucket (bucket b spans [hist[b], cur[b]))
  for (uint32_t b = tid; b < CS_BUCKETS; b += CS_BLOCK) {
    uint32_t lo = sh.hist[b], hi = sh.cur[b];
    if (hi - lo > CS_SMALL) {
      *sh.big = 1;
      continue;
    }
    for (uint32_t i = lo + 1; i < hi; i++) {
      KeyT x = S[i];
      const uint8_t xp = SP ? SP[i] : 0;
      uint32_t q = i;
      while (q > lo && x < S[q - 1]) {
        S[q] = S[q - 1];
        if (SP) SP[q] = SP[q - 1];
        q--;
      }
      S[q] = x;
      if (SP) SP[q] = xp;
    }
  }
  __syncthreads();
  if (*sh.big) {  // bitonic sort of the whole range, padded to a power of two
    uint32_t P2 = 1;
    while (P2 < m) P2 <<= 1;
    for (uint32_t i = m + tid; i < P2; i += CS_BLOCK) {
      S[i] = KOps<KeyT>::max_key();
      if (SP) SP[i] = 0;
    }
    __syncthreads();
    for (uint32_t size = 2; size <= P2; size <<= 1) {
      for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
        for (uint32_t i = tid; i < P2 / 2; i += CS_BLOCK) {
          uint32_t lo = 2 * i - (i & (stride - 1));
          cs_swap_if(S[lo], S[lo + stride], SP ? SP + lo : nullptr, SP ? SP + lo + stride : nullptr,
                     (lo & size) == 0);
        }
        __syncthreads();
      }
    }
  }
  (void)CAP;
  if (distinct) {  // already one copy per key: plain copy out
    for (uint32_t i = tid; i < m; i += CS_BLOCK) {
      out[i] = S[i];
      if (SP) outP[i] = SP[i];
    }
    __syncthreads();
    return m;
  }
  // adjacent-unique; a run's first key takes the OR of the run's payloads
  return block_select<CS_BLOCK>(
      m, [&](uint32_t i) { return i == 0 || S[i] != S[i - 1]; },
      [&](uint32_t i, uint32_t r) {
        out[r] = S[i];
        if (SP) {
          uint32_t p = SP[i];
          for (uint32_t j = i + 1; j < m && S[j] == S[i]; j++) p |= SP[j];
          outP[r] = (uint8_t)p;
        }
      },
      sh.sm);
}

// Level-0 and level-1 slices of sub-bucket j (bin j >> P, slice j mod 2^P)
// over its n distinct keys (see Level0Out); set/col: L0_SW_MAX words of
// shared memory each (level 0's sw words, then level 1's sw1); lb: lb_cap
// u16 of shared memory for the keys' bits in the slices (a slice has at most
// L0_SW_MAX * 64 < 2^16 - 2 bits).  All threads call it.
constexpr uint32_t L0_SW_MAX = 768;
// With kpay (the keys' joined payload bytes) and o.with_pay, the payloads go
// out as Level0Out describes; pw: L0_SW_MAX u32 of shared memory.
CF1_D void l0_slice(const uint64_t *keys, uint32_t n, uint64_t j, int P, const Level0Out &o,
                    unsigned long long *set, unsigned long long *col, uint16_t *lb, uint32_t lb_cap, uint32_t *sm,
                    unsigned long long *s_base, const uint8_t *kpay, uint64_t a, uint32_t *pw) {
  constexpr uint16_t BAD = 0xFFFF, AT0 = 0xFFFE;  // lb[i]: no bit / placed at level 0 / else its level-1 bit
  const bool pay = o.with_pay && kpay;
  const unsigned tid = threadIdx.x;
  const uint32_t bin = (uint32_t)(j >> P), sub = (uint32_t)(j & ((1ull << P) - 1));
  const uint64_t W = o.woff[bin + 1] - o.woff[bin];
  const uint32_t sw = (uint32_t)(W >> P);
  const uint32_t sw1 = (uint32_t)((o.woff1[bin + 1] - o.woff1[bin]) >> P);
  const uint64_t first1 = o.woff1[bin] + (uint64_t)sub * sw1;
  if (n == 0) {  // every slice writes all its entries (the array is not cleared first)
    for (uint32_t w = tid; w < sw; w += CS_BLOCK)
      o.AR[o.woff[bin] + (uint64_t)sub * sw + w] = make_ulonglong2(0ull, 0ull);
    for (uint32_t w = tid; w < sw1; w += CS_BLOCK) o.AR1[first1 + w] = make_ulonglong2(0ull, 0ull);
    if (tid == 0) o.placed[j] = o.placed1[j] = 0;
    return;
  }
  // level 1 uses the words of set, col and pw after level 0's
  if (sw > L0_SW_MAX || sw + sw1 > L0_SW_MAX || sw1 > CS_BLOCK || sw == 0 || n > lb_cap) {
    if (tid == 0) {
      atomicOr(o.err, 1u);
      o.placed[j] = o.placed1[j] = 0;
    }
    return;
  }
  const uint64_t first = o.woff[bin] + (uint64_t)sub * sw;  // the slice's first entry
  const uint64_t lo_bit = (uint64_t)sub * sw * 64;
  for (uint32_t w = tid; w < sw; w += CS_BLOCK) set[w] = col[w] = 0;
  __syncthreads();
  for (uint32_t i = tid; i < n; i += CS_BLOCK) {
    const uint64_t b = bb_pos(keys[i], 0, (uint32_t)W) - lo_bit;
    if (b >= (uint64_t)sw * 64) {  // not this slice's key: cannot happen with the shared hash
      atomicOr(o.err, 1u);
      lb[i] = BAD;
      continue;
    }
    lb[i] = (uint16_t)b;
    const unsigned long long bit = 1ull << (b & 63);
    if (atomicOr(&set[b >> 6], bit) & bit) atomicOr(&col[b >> 6], bit);
  }
  __syncthreads();
  // the placed bits of the slice before each word (words 2t and 2t+1 per
  // thread: sw <= L0_SW_MAX <= 2 CS_BLOCK), written beside the word
  uint32_t placed0 = 0;
  {
    const uint32_t w0 = 2 * tid, w1 = w0 + 1;
    const uint32_t c0 = w0 < sw ? (uint32_t)popc64(set[w0] & ~col[w0]) : 0u;
    const uint32_t c1 = w1 < sw ? (uint32_t)popc64(set[w1] & ~col[w1]) : 0u;
    const uint32_t pre_w = block_exclusive_scan<CS_BLOCK>(c0 + c1, sm, placed0);
    if (w0 < sw) {
      pw[w0] = pre_w;
      o.AR[first + w0] = make_ulonglong2(set[w0] & ~col[w0], (unsigned long long)pre_w);
    }
    if (w1 < sw) {
      pw[w1] = pre_w + c0;
      o.AR[first + w1] = make_ulonglong2(set[w1] & ~col[w1], (unsigned long long)(pre_w + c0));
    }
  }
  if (pay) {
    // a placed key's rank in the slice: the placed bits before its bit
    __syncthreads();
    for (uint32_t i = tid; i < n; i += CS_BLOCK) {
      const uint32_t b = lb[i];
      if (b == BAD) continue;
      const uint64_t fin = set[b >> 6] & ~col[b >> 6];
      const uint64_t bit = 1ull << (b & 63);
      if (fin & bit) o.l0pay[a + pw[b >> 6] + (uint32_t)popc64(fin & (bit - 1))] = kpay[i];
    }
  }
  // level 1 (sliced, sw1 words): the keys whose level-0 bit collided
  unsigned long long *set1 = set + sw, *col1 = col + sw;
  uint32_t *pw1 = pw + sw;
  for (uint32_t w = tid; w < sw1; w += CS_BLOCK) set1[w] = col1[w] = 0;
  __syncthreads();
  for (uint32_t i = tid; i < n; i += CS_BLOCK) {
    const uint32_t b = lb[i];
    if (b == BAD) continue;
    if (!((col[b >> 6] >> (b & 63)) & 1)) {
      lb[i] = AT0;
      continue;
    }
    const uint32_t p1 = bb_slice_pos(keys[i], 1, sw1);
    const unsigned long long bit = 1ull << (p1 & 63);
    if (atomicOr(&set1[p1 >> 6], bit) & bit) atomicOr(&col1[p1 >> 6], bit);
    lb[i] = (uint16_t)p1;
  }
  __syncthreads();
  const unsigned long long g1 = tid < sw1 ? set1[tid] & ~col1[tid] : 0ull;  // sw1 <= CS_BLOCK
  uint32_t placed1;
  const uint32_t pre1 = block_exclusive_scan<CS_BLOCK>((uint32_t)popc64(g1), sm, placed1);
  if (tid < sw1) {
    pw1[tid] = pre1;
    o.AR1[first1 + tid] = make_ulonglong2(g1, (unsigned long long)pre1);
  }
  if (tid == 0) {
    o.placed[j] = placed0;
    o.placed1[j] = placed1;
  }
  __syncthreads();
  // level-1 ranks, and the keys level 1 leaves go on to level 2
  uint32_t c = 0;
  for (uint32_t i = tid; i < n; i += CS_BLOCK) {
    const uint32_t p1 = lb[i];
    if (p1 == BAD || p1 == AT0) continue;
    const uint64_t fin = set1[p1 >> 6] & ~col1[p1 >> 6], bit = 1ull << (p1 & 63);
    if (!(fin & bit)) c++;
    else if (pay) o.l0pay[a + placed0 + pw1[p1 >> 6] + (uint32_t)popc64(fin & (bit - 1))] = kpay[i];
  }
  uint32_t tot;
  uint32_t pre = block_exclusive_scan<CS_BLOCK>(c, sm, tot);
  if (tid == 0) {
    unsigned long long base = ~0ull;
    if (tot) {
      base = atomicAdd(&o.surv_cnt[bin], (unsigned long long)tot);
      if (base + tot > o.surv_off[bin + 1] - o.surv_off[bin]) {
        atomicOr(o.err, 1u);
        base = ~0ull;
      }
    }
    *s_base = base;
  }
  __syncthreads();
  if (*s_base != ~0ull) {
    uint64_t out = o.surv_off[bin] + *s_base + pre;
    for (uint32_t i = tid; i < n; i += CS_BLOCK) {
      const uint32_t p1 = lb[i];
      if (p1 == BAD || p1 == AT0) continue;
      if (!(((set1[p1 >> 6] & ~col1[p1 >> 6]) >> (p1 & 63)) & 1)) {
        if (pay) o.surv_pay[out] = kpay[i];
        o.surv[out++] = keys[i];
      }
    }
  }
  __syncthreads();
}

// Sorted distinct keys of one sub-bucket T[a, a+n), written back at a
// (SORTED = false: distinct keys in any order -- 64-bit keys then skip the
// sort whenever the shared-memory set holds the sub-bucket).
// Sub-buckets above CAP keys: 64-bit keys are first reduced to one copy each
// through a shared-memory set; if still above CAP, the sub-bucket is split on
// its next `bits` bits into U[a, a+n) (the free ping-pong buffer), runs of
// consecutive pieces up to CAP keys are sorted one after another, and their
// distinct keys are appended at T[a].  Only a single piece above CAP keys
// makes the kernel report the sub-bucket as oversized.
// With TP/UP (payload bytes parallel to T and U), every distinct key leaves
// with the OR of its copies' payloads beside it in TP.
// Chunks (sorted form): with clist, CTA c takes the run of consecutive
// sub-buckets [j0, j1) of one bin that the plan packed together (coff: the
// plan's chunks per bin, scanned), sorts the run as one range -- its bucket is
// the sub-bucket's place in the run, then the next key bits -- and credits
// all its distinct keys to sub-bucket j0.
template <class KeyT, bool SORTED>
__global__ void __launch_bounds__(CS_BLOCK, SORTED ? 2 : 4) cs_sort_unique_kernel(KeyT *T, KeyT *U, const uint64_t *sb_off,
                                                                  uint64_t nsub, int shift, int bits, uint32_t *cnt,
                                                                  uint32_t *oversize, int P, Level0Out l0,
                                                                  uint8_t *TP, uint8_t *UP, const uint2 *clist,
                                                                  const uint64_t *coff, uint32_t nbins,
                                                                  const uint32_t *jlist) {
  constexpr uint32_t CAP = cs_cap<KeyT, SORTED>();
  constexpr bool L0 = !SORTED && KOps<KeyT>::WORDS == 1;
  __shared__ unsigned long long s_l0base;
  extern __shared__ __align__(16) unsigned char cs_smem[];
  KeyT *S = reinterpret_cast<KeyT *>(cs_smem);                    // [CAP]
  uint32_t *hist = reinterpret_cast<uint32_t *>(S + CAP);         // [CS_BUCKETS]
  uint32_t *cur = hist + CS_BUCKETS;                              // [CS_BUCKETS]
  uint32_t *pstart = cur + CS_BUCKETS;                            // [CS_BUCKETS + 1]
  uint16_t *cb = reinterpret_cast<uint16_t *>(pstart + CS_BUCKETS + 1);  // [CS_BUCKETS + 1]
  uint32_t *SPw = reinterpret_cast<uint32_t *>(cb + CS_BUCKETS + 2);     // [CAP / 4] payloads, when TP
  __shared__ uint32_t sm[CS_BLOCK / 32];
  __shared__ int s_big, s_nchunks, s_bad;
  __shared__ uint32_t s_cnt;
  uint64_t j = blockIdx.x, jend = j + 1;
  if (jlist) {  // the sub-buckets the warp dedup left
    j = jlist[blockIdx.x];
    jend = j + 1;
  } else if (clist) {
    const uint32_t bin = upper_segment(coff, nbins, (uint64_t)blockIdx.x);
    const uint2 r = clist[((uint64_t)bin << P) + (blockIdx.x - coff[bin])];
    j = ((uint64_t)bin << P) + r.x;
    jend = ((uint64_t)bin << P) + r.y;
  }
  if (j >= nsub) return;
  const uint64_t a = sb_off[j], n = sb_off[jend] - a;
  const unsigned tid = threadIdx.x;
  // the sub-bucket's distinct keys end at T[a, a + result); ~0u: oversized
  auto body = [&]() -> uint32_t {
    if (n == 0) return 0;
    CsShared sh{hist, cur, sm, &s_big, TP ? reinterpret_cast<uint8_t *>(SPw) : nullptr};
    CsDigit plain{shift, bits, 0, 0, 0u};
    if (jend - j > 1) {  // a packed run: bucket = place of the sub-bucket in the run, then the next bits
      const uint32_t span = (uint32_t)(jend - j);
      if (span > CS_BUCKETS) return ~0u;  // the plan never makes one; refused (LSD path) rather than mis-bucketed
      int g = 0;
      while ((1u << g) < span) g++;
      const int rest = shift + bits;  // the sub-bucket prefix sits at bits [rest, rest + P)
      const int b2 = 10 - g < rest ? 10 - g : rest;
      plain = CsDigit{rest, P, rest - b2, b2, (uint32_t)(j & ((1ull << P) - 1))};
    }
    uint32_t m = (uint32_t)n;
    bool distinct = false;
    // 64-bit keys: one copy of each key first.  Repeats put hundreds of
    // copies of a k-mer in one bucket, where sorting copies would dominate.
    if ((!SORTED || n > CS_DEDUP_MIN) && KOps<KeyT>::WORDS == 1) {
      uint32_t d = cs_hash_dedup(reinterpret_cast<uint64_t *>(T), a, n, reinterpret_cast<uint64_t *>(S), CAP, &s_cnt, sm,
                                 TP, SPw);
      if (d != ~0u) {
        m = d;
        distinct = true;
        if (!SORTED) return d;  // distinct keys are all that is needed
      }
    }
    if (m <= CAP)
      return cs_sort_unique_range<KeyT>(T + a, m, plain, S, sh, T + a, distinct, TP ? TP + a : nullptr,
                                        TP ? TP + a : nullptr);
    // local split on the next `bits` bits into U[a, a+n)
    const uint32_t npieces = 1u << bits, pmask = npieces - 1;
    for (uint32_t i = tid; i <= CS_BUCKETS; i += CS_BLOCK) pstart[i] = 0;
    __syncthreads();
    for (uint64_t i = tid; i < n; i += CS_BLOCK) atomicAdd(&pstart[KOps<KeyT>::digit(T[a + i], shift, pmask)], 1u);
    __syncthreads();
    if (tid == 0) {
      uint32_t run = 0;
      for (uint32_t p = 0; p < npieces; p++) {
        uint32_t v = pstart[p];
        pstart[p] = run;
        run += v;
      }
      pstart[npieces] = run;
      // greedy runs of consecutive pieces up to CAP keys
      int nc = 0, bad = 0;
      uint32_t acc = 0;
      cb[0] = 0;
      for (uint32_t p = 0; p < npieces; p++) {
        uint32_t sz = pstart[p + 1] - pstart[p];
        if (sz > CAP) {  // a piece of its own, deduplicated before sorting (64-bit keys)
          if (KOps<KeyT>::WORDS != 1) bad = 1;
          if (acc > 0) cb[++nc] = (uint16_t)p;
          cb[++nc] = (uint16_t)(p + 1);
          acc = 0;
          continue;
        }
        if (acc + sz > CAP && acc > 0) {
          cb[++nc] = (uint16_t)p;
          acc = 0;
        }
        acc += sz;
      }
      if (acc == 0) nc--;  // the loop already closed the last run
      cb[++nc] = (uint16_t)npieces;
      s_nchunks = nc;
      s_bad = bad;
    }
    __syncthreads();
    if (s_bad) return ~0u;
    for (uint32_t p = tid; p < npieces; p += CS_BLOCK) cur[p] = pstart[p];
    __syncthreads();
    for (uint64_t i = tid; i < n; i += CS_BLOCK) {
      KeyT key = T[a + i];
      const uint32_t at = atomicAdd(&cur[KOps<KeyT>::digit(key, shift, pmask)], 1u);
      U[a + at] = key;
      if (TP) UP[a + at] = TP[a + i];
    }
    __syncthreads();
    uint32_t outc = 0;
    for (int c = 0; c < s_nchunks; c++) {
      uint32_t p0 = cb[c], p1 = cb[c + 1];
      uint32_t span = p1 - p0;
      int g = 0;
      while ((1u << g) < span) g++;
      int b2 = 10 - g;
      if (b2 > shift) b2 = shift;
      CsDigit dig{shift, bits, shift - b2, b2, p0};
      uint32_t len = pstart[p1] - pstart[p0];
      bool dd = false;
      if (len > CS_DEDUP_MIN && KOps<KeyT>::WORDS == 1) {
        uint32_t d = cs_hash_dedup(reinterpret_cast<uint64_t *>(U), a + pstart[p0], len,
                                   reinterpret_cast<uint64_t *>(S), CAP, &s_cnt, sm, TP ? UP : nullptr, SPw);
        if (d != ~0u) {  // (a failed pass leaves U untouched)
          len = d;
          dd = true;
        }
        if (len > CAP) return ~0u;
      }
      outc += cs_sort_unique_range<KeyT>(U + a + pstart[p0], len, dig, S, sh, T + a + outc, dd,
                                         TP ? UP + a + pstart[p0] : nullptr, TP ? TP + a + outc : nullptr);
    }
    return outc;
  };
  const uint32_t res = body();
  if (tid == 0) {
    cnt[j] = res == ~0u ? 0 : res;
    if (res == ~0u) atomicOr(oversize, 1u);
  }
  for (uint64_t q = j + 1 + tid; q < jend; q += CS_BLOCK) cnt[q] = 0;
  if constexpr (L0) {
    if (l0.AR && res != ~0u) {
      __syncthreads();
      unsigned long long *h64 = reinterpret_cast<unsigned long long *>(hist);
      l0_slice(reinterpret_cast<const uint64_t *>(T) + a, res, j, P, l0, h64, h64 + L0_SW_MAX,
               reinterpret_cast<uint16_t *>(S), CAP * sizeof(KeyT) / 2, sm, &s_l0base, TP ? TP + a : nullptr, a,
               SPw);
    }
  }
}

// ---------------------------------------------------------------- warp dedup
// The unsorted (BBHash) form's dedup, one warp per sub-bucket and no block
// barriers: sub-buckets of a few hundred keys (the split of key *
// KEY_SPREAD_MUL spreads them evenly), a private 512-slot open-addressing set
// per warp in shared memory, and, with level 0 on, the sub-bucket's slice of
// BBHash level 0 marked, written and ranked by the same warp.  A warp takes
// runs of WD_RUN consecutive sub-buckets from a work counter (their offsets,
// keys and bins are then read in order, and uneven bins still balance).  A
// sub-bucket with more than WD_MAXD distinct keys (or a slice
// above WD_SWMAX words) is left untouched and listed in ov for the block
// kernel.
constexpr int WD_WARPS = 8;                 // warps per CTA
constexpr uint32_t WD_TW = 512;             // set slots per warp
constexpr uint32_t WD_MAXD = WD_TW / 4 * 3; // distinct keys a warp's set takes
constexpr uint32_t WD_SWMAX = 64;           // level-0 slice words a warp takes
constexpr uint32_t WD_SW1MAX = (WD_SWMAX + 7) / 8;  // level-1 slice words (an eighth of level 0's)
constexpr int WD_U = 4;                     // key loads in flight per lane
constexpr uint32_t WD_RUN = 64;             // sub-buckets a warp takes at a time
struct WdSmem {
  unsigned long long tab[WD_TW];
  unsigned long long set[WD_SWMAX], col[WD_SWMAX];     // level-0 slice: bits set, bits set twice
  unsigned long long set1[WD_SW1MAX], col1[WD_SW1MAX]; // level-1 slice
  uint8_t tpay[WD_TW];
  uint16_t ins[WD_MAXD];                    // the distinct keys' slots in insertion order
  uint8_t dp[WD_MAXD];                      // the distinct keys' joined payloads
  uint16_t pw[WD_SWMAX], pw1[WD_SW1MAX];    // placed bits before each word of the slices
};
static_assert(sizeof(WdSmem) % 8 == 0, "per-warp areas stay 8-byte aligned");

// PK: T holds packed words of a first pass of p1 bits (see pay_code); the
// set then holds each key's h = key * MS_HASH_MUL without its top p1 bits,
// level 0's bit comes from h directly, and the keys written back (T, the
// level-2 list) are h * KEY_SPREAD_INV.  TP is only written.
template <bool PK>
__global__ void __launch_bounds__(WD_WARPS * 32, 4) wd_dedup_kernel(uint64_t *T, uint8_t *TP, const uint64_t *sb_off,
                                                                   uint64_t nsub, int P, uint32_t *cnt, Level0Out l0,
                                                                   uint32_t *ov, uint32_t *ov_cnt, uint32_t *queue,
                                                                   int p1) {
  extern __shared__ __align__(16) unsigned char wd_smem[];
  WdSmem &m = reinterpret_cast<WdSmem *>(wd_smem)[threadIdx.x >> 5];
  const unsigned lane = lane_id(), lt = lanemask_lt();
  const unsigned long long EMPTY = ~0ull;  // above every key (keys use at most 62 bits)
  const bool pay = TP != nullptr, lv0 = l0.AR != nullptr, lpay = lv0 && l0.with_pay && pay;
  for (uint32_t i = lane; i < WD_TW; i += 32) {
    m.tab[i] = EMPTY;
    m.tpay[i] = 0;
  }
  __syncwarp();
  const uint64_t nruns = (nsub + WD_RUN - 1) / WD_RUN;
  for (;;) {
    uint32_t run = 0;
    if (lane == 0) run = atomicAdd(queue, 1u);
    run = __shfl_sync(FULL, run, 0);
    if (run >= nruns) break;
    const uint64_t j0 = (uint64_t)run * WD_RUN, j1 = j0 + WD_RUN < nsub ? j0 + WD_RUN : nsub;
    for (uint64_t j = j0; j < j1; j++) {
      const uint64_t a = sb_off[j], n = sb_off[j + 1] - a;
      const uint32_t bin = (uint32_t)(j >> P), sub = (uint32_t)(j & ((1ull << P) - 1));
      uint64_t W = 0, first = 0;
      uint32_t sw = 0;
      if (lv0) {
        W = l0.woff[bin + 1] - l0.woff[bin];
        sw = (uint32_t)(W >> P);
        first = l0.woff[bin] + (uint64_t)sub * sw;
      }
      bool over = lv0 && sw > WD_SWMAX;
      // PK: the h bits the sub-bucket's first-pass digit gives; a set entry
      // id stands for the key whose h is hi | id
      const uint64_t hi = PK ? (uint64_t)(sub >> (P - p1)) << (64 - p1) : 0;
      auto key_of = [&](unsigned long long id) -> uint64_t { return PK ? (hi | id) * KEY_SPREAD_INV : id; };
      auto l0_bit = [&](unsigned long long id) -> uint64_t {
        return PK ? (((uint64_t)(uint32_t)((hi | id) >> 32) * (uint32_t)W) >> 26) : bb_pos(id, 0, (uint32_t)W);
      };
      // 1. one copy of each key, its copies' payloads ORed (WD_U keys per lane
      //    loaded before the first is inserted).  Double hashing: the probe
      //    step is odd (so a probe sequence visits every slot) and comes from
      //    other bits of the same product, which keeps the runs a warp waits
      //    for (the longest of its 32 lanes) short at the set's load.  The
      //    first probes of a lane's WD_U keys are issued back to back; only
      //    the keys whose first slot held another key then walk on, one key
      //    index at a time.  (A key can find the set full only after more
      //    than WD_MAXD keys were claimed, so the sub-bucket goes to the block
      //    kernel anyway.)
      uint32_t d = 0;
      for (uint64_t base = 0; base < n && !over; base += 32 * WD_U) {
        unsigned long long key[WD_U];
        uint32_t p[WD_U], h[WD_U], stp[WD_U];
        bool claimed[WD_U], pend[WD_U];
  #pragma unroll
        for (int u = 0; u < WD_U; u++) {
          const uint64_t i = base + u * 32 + lane;
          if constexpr (PK) {
            const uint64_t w = i < n ? T[a + i] : 0;
            key[u] = i < n ? w >> p1 : EMPTY;
            p[u] = i < n ? pay_byte((uint32_t)w) : 0u;
          } else {
            key[u] = i < n ? T[a + i] : EMPTY;
            p[u] = (pay && i < n) ? TP[a + i] : 0u;
          }
        }
  #pragma unroll
        for (int u = 0; u < WD_U; u++) {
          claimed[u] = pend[u] = false;
          h[u] = stp[u] = 0;
          if (key[u] != EMPTY) {
            const unsigned long long hk = key[u] * 0x9E3779B97F4A7C15ull;
            h[u] = (uint32_t)(hk >> 55);                                // top 9 bits: WD_TW = 512
            stp[u] = ((uint32_t)(hk >> 40) | 1u) & (WD_TW - 1);
            const unsigned long long old = atomicCAS(&m.tab[h[u]], EMPTY, key[u]);
            if (old == EMPTY || old == key[u]) {
              claimed[u] = old == EMPTY;
              if (pay) atomicOr(reinterpret_cast<uint32_t *>(m.tpay) + (h[u] >> 2), p[u] << (8 * (h[u] & 3)));
            } else {
              pend[u] = true;
              h[u] = (h[u] + stp[u]) & (WD_TW - 1);
            }
          }
        }
  #pragma unroll
        for (int u = 0; u < WD_U; u++) {
          if (over) break;  // the set stays below full: at most WD_MAXD + 32 * WD_U keys in it
          if (__any_sync(FULL, pend[u]) && pend[u]) {
            for (uint32_t probe = 1; probe < WD_TW; probe++) {
              const unsigned long long old = atomicCAS(&m.tab[h[u]], EMPTY, key[u]);
              if (old == EMPTY || old == key[u]) {
                claimed[u] = old == EMPTY;
                if (pay) atomicOr(reinterpret_cast<uint32_t *>(m.tpay) + (h[u] >> 2), p[u] << (8 * (h[u] & 3)));
                break;
              }
              h[u] = (h[u] + stp[u]) & (WD_TW - 1);
            }
          }
          const unsigned b = __ballot_sync(FULL, claimed[u]);
          const uint32_t r = d + __popc(b & lt);
          if (claimed[u] && r < WD_MAXD) m.ins[r] = (uint16_t)h[u];
          d += __popc(b);
          over = d > WD_MAXD;
        }
      }
      __syncwarp();
      if (over) {  // left to the block kernel: clear the whole set, list j
        for (uint32_t i = lane; i < WD_TW; i += 32) {
          m.tab[i] = EMPTY;
          m.tpay[i] = 0;
        }
        if (lane == 0) ov[atomicAdd(ov_cnt, 1u)] = (uint32_t)j;
        __syncwarp();
        continue;
      }
      const uint64_t lo_bit = (uint64_t)sub * sw * 64;
      if (lv0) {
        for (uint32_t w = lane; w < sw; w += 32) m.set[w] = m.col[w] = 0;
        __syncwarp();
      }
      // 2. the distinct keys (and bytes) to T[a, a + d); with level 0, each
      //    key's bit marked and its byte kept in dp, the key itself left in
      //    the set (ins[r] stays its slot) until step 5 empties it; a key's
      //    level-0 and level-1 bits are recomputed from it where needed
      bool bad = false;
      for (uint32_t r = lane; r < d; r += 32) {
        const uint32_t h = m.ins[r];
        const unsigned long long key = m.tab[h];
        const uint8_t pr = m.tpay[h];
        T[a + r] = key_of(key);
        if (pay) TP[a + r] = pr;
        m.tpay[h] = 0;
        if (lv0) {
          const uint64_t bpos = l0_bit(key) - lo_bit;
          if (bpos < (uint64_t)sw * 64) {
            const unsigned long long bit = 1ull << (bpos & 63);
            if (atomicOr(&m.set[bpos >> 6], bit) & bit) atomicOr(&m.col[bpos >> 6], bit);
          } else {
            bad = true;  // not this slice's key: cannot happen with the shared hash
          }
          m.dp[r] = pr;
        } else {
          m.tab[h] = EMPTY;
        }
      }
      if (lane == 0) cnt[j] = d;
      if (!lv0) {
        __syncwarp();
        continue;
      }
      if (__any_sync(FULL, bad) && lane == 0) atomicOr(l0.err, 1u);
      __syncwarp();
      // 3. the slice written; placed bits per word and their exclusive prefix
      //    (sw <= 64: two words a lane)
      const unsigned long long f0 = lane < sw ? m.set[lane] & ~m.col[lane] : 0ull;
      const unsigned long long f1 = lane + 32 < sw ? m.set[lane + 32] & ~m.col[lane + 32] : 0ull;
      const uint32_t c0 = (uint32_t)__popcll(f0), c1 = (uint32_t)__popcll(f1);
      const uint32_t i0 = warp_inclusive_scan(c0), i1 = warp_inclusive_scan(c1);
      const uint32_t t0 = __shfl_sync(FULL, i0, 31), placed = t0 + __shfl_sync(FULL, i1, 31);
      if (lane < sw) {
        m.pw[lane] = (uint16_t)(i0 - c0);
        l0.AR[first + lane] = make_ulonglong2(f0, (unsigned long long)(i0 - c0));
      }
      if (lane + 32 < sw) {
        m.pw[lane + 32] = (uint16_t)(t0 + i1 - c1);
        l0.AR[first + lane + 32] = make_ulonglong2(f1, (unsigned long long)(t0 + i1 - c1));
      }
      // 4. each key level 0 places: its byte to its rank, its slot emptied;
      //    each key it leaves marks its bit in the sub-bucket's level-1 slice
      //    (sw1 words, its bit from level 1's hash) and is moved to the front
      //    of ins / dp (nsv of them; a key's new index is never above its old
      //    one, and the warp reads a group before it writes it)
      const uint32_t sw1 = (uint32_t)((l0.woff1[bin + 1] - l0.woff1[bin]) >> P);
      const uint64_t first1 = l0.woff1[bin] + (uint64_t)sub * sw1;
      const bool l1ok = sw1 <= WD_SW1MAX;  // always: level 1 is sized from level 0
      if (lane < sw1 && l1ok) m.set1[lane] = m.col1[lane] = 0;
      __syncwarp();
      uint32_t nsv = 0;
      for (uint32_t r0 = 0; r0 < d; r0 += 32) {
        const uint32_t r = r0 + lane;
        bool lv = false;  // left by level 0
        uint32_t h = 0;
        uint8_t pr = 0;
        if (r < d) {
          h = m.ins[r];
          pr = m.dp[r];
          const unsigned long long key = m.tab[h];
          const uint64_t bpos = l0_bit(key) - lo_bit;
          if (bpos < (uint64_t)sw * 64) {
            const unsigned long long fin = m.set[bpos >> 6] & ~m.col[bpos >> 6], bit = 1ull << (bpos & 63);
            if (fin & bit) {
              if (lpay) l0.l0pay[a + m.pw[bpos >> 6] + (uint32_t)__popcll(fin & (bit - 1))] = pr;
              m.tab[h] = EMPTY;
            } else if (l1ok) {
              lv = true;
              const uint32_t q1 = bb_slice_pos(key_of(key), 1, sw1);
              const unsigned long long bit1 = 1ull << (q1 & 63);
              if (atomicOr(&m.set1[q1 >> 6], bit1) & bit1) atomicOr(&m.col1[q1 >> 6], bit1);
            } else {
              m.tab[h] = EMPTY;
            }
          } else {
            m.tab[h] = EMPTY;
          }
        }
        const unsigned lb = __ballot_sync(FULL, lv);
        __syncwarp();  // every lane's reads of this group before any lane's writes
        if (lv) {
          const uint32_t k = nsv + __popc(lb & lt);
          m.ins[k] = (uint16_t)h;
          m.dp[k] = pr;
        }
        nsv += __popc(lb);
        __syncwarp();
      }
      const unsigned long long g1 = (lane < sw1 && l1ok) ? m.set1[lane] & ~m.col1[lane] : 0ull;
      const uint32_t e1 = (uint32_t)__popcll(g1), k1 = warp_inclusive_scan(e1);
      const uint32_t placed1 = __shfl_sync(FULL, k1, 31);
      if (lane < sw1 && l1ok) {
        m.pw1[lane] = (uint16_t)(k1 - e1);
        l0.AR1[first1 + lane] = make_ulonglong2(g1, (unsigned long long)(k1 - e1));
      }
      if (lane == 0) {
        l0.placed[j] = placed;
        l0.placed1[j] = placed1;
      }
      // survivors of level 1: one reservation in the bin's list
      unsigned long long sbase = 0;
      const uint32_t nsurv = nsv - placed1;
      if (lane == 0 && (nsurv || !l1ok)) {
        if (l1ok) sbase = atomicAdd(&l0.surv_cnt[bin], (unsigned long long)nsurv);
        if (!l1ok || sbase + nsurv > l0.surv_off[bin + 1] - l0.surv_off[bin]) {
          atomicOr(l0.err, 1u);
          sbase = ~0ull;
        }
      }
      sbase = __shfl_sync(FULL, sbase, 0);
      __syncwarp();
      // 5. each key level 0 left: its byte to its level-1 rank or the key to
      //    level 2; the rest of the set emptied
      uint64_t so = l0.surv_off[bin] + sbase;
      for (uint32_t k0 = 0; k0 < nsv; k0 += 32) {
        const uint32_t k = k0 + lane;
        bool surv = false;
        unsigned long long key = 0;
        if (k < nsv) {
          const uint32_t h = m.ins[k];
          key = key_of(m.tab[h]);
          m.tab[h] = EMPTY;
          const uint32_t q1 = bb_slice_pos(key, 1, sw1);
          const unsigned long long fin1 = m.set1[q1 >> 6] & ~m.col1[q1 >> 6], bit1 = 1ull << (q1 & 63);
          if (fin1 & bit1) {
            if (lpay) l0.l0pay[a + placed + m.pw1[q1 >> 6] + (uint32_t)__popcll(fin1 & (bit1 - 1))] = m.dp[k];
          } else {
            surv = true;
          }
        }
        const unsigned sb = __ballot_sync(FULL, surv);
        if (surv && sbase != ~0ull) {
          const uint64_t at = so + __popc(sb & lt);
          l0.surv[at] = key;
          if (lpay) l0.surv_pay[at] = m.dp[k];
        }
        so += __popc(sb);
      }
      __syncwarp();
    }
  }
}

// Packed sub-buckets the warp dedup left to the block kernel, back to keys
// and payload bytes (one warp per listed sub-bucket).
__global__ void wd_unpack_kernel(uint64_t *T, uint8_t *TP, const uint64_t *sb_off, const uint32_t *ov,
                                 const uint32_t *ov_cnt, int P, int p1) {
  const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= *ov_cnt) return;
  const uint64_t j = ov[w], a = sb_off[j], n = sb_off[j + 1] - a;
  const uint32_t sub = (uint32_t)(j & ((1ull << P) - 1));
  const uint64_t hi = (uint64_t)(sub >> (P - p1)) << (64 - p1);
  for (uint64_t i = lane_id(); i < n; i += 32) {
    const uint64_t x = T[a + i];
    TP[a + i] = (uint8_t)pay_byte((uint32_t)x);
    T[a + i] = (hi | (x >> p1)) * KEY_SPREAD_INV;
  }
}

// Chunk plan of the sorted form: per bin (one thread), runs of consecutive
// sub-buckets packed greedily up to cap keys and at most CS_BUCKETS
// sub-buckets (the run's counting sort buckets a key by its sub-bucket's
// place in the run first; sparse stretches of the key space -- canonical
// k-mers starting with TTT... -- hold thousands of near-empty sub-buckets at
// wide splits), a sub-bucket above cap keys being a run of its own, written as
// (first, end) sub-bucket indices within the bin to clist[bin << P ...];
// ccount[bin] = the bin's runs.
__global__ void cs_plan_kernel(const uint64_t *sb_off, uint32_t nbins, int P, uint32_t cap, uint2 *clist,
                               uint32_t *ccount) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbins) return;
  const uint32_t per = 1u << P;
  const uint64_t *o = sb_off + ((uint64_t)b << P);
  uint2 *out = clist + ((uint64_t)b << P);
  uint32_t nc = 0, start = 0;
  uint64_t acc = 0;
  for (uint32_t q = 0; q < per; q++) {
    const uint64_t sz = o[q + 1] - o[q];
    if ((acc > 0 && acc + sz > cap) || q - start == CS_BUCKETS) {
      out[nc++] = make_uint2(start, q);
      start = q;
      acc = 0;
    }
    acc += sz;
  }
  out[nc++] = make_uint2(start, per);
  ccount[b] = nc;
}

// One warp per sub-bucket: copy its distinct keys to the dense array.
template <class KeyT>
__global__ void cs_compact_kernel(const KeyT *T, const uint64_t *sb_off, const uint32_t *cnt, const uint64_t *out_off,
                                  uint64_t nsub, KeyT *dist) {
  uint64_t j = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (j >= nsub) return;
  uint32_t c = cnt[j];
  uint64_t a = sb_off[j], o = out_off[j];
  for (uint32_t i = lane_id(); i < c; i += 32) dist[o + i] = T[a + i];
}

__global__ void cs_bin_off_kernel(const uint64_t *out_off, uint32_t nbins, uint64_t per_bin, uint64_t *dist_off) {
  uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b <= nbins) dist_off[b] = out_off[(uint64_t)b * per_bin];
}

template <class KeyT, int BITS>
void ms_pass(const KeyT *in, KeyT *out, uint64_t n, const uint64_t *seg_off, uint32_t nseg, int shift, bool hashed,
             MsdScratch &sc, cudaStream_t s, const uint8_t *pin, uint8_t *pout, int pack) {
  constexpr uint32_t DIG = 1u << BITS;
  uint32_t ub = (uint32_t)(ceil_div(n, MS_TILE) + nseg);
  uint32_t *tile_off = sc.tile_off.get<uint32_t>(nseg + 1);
  segment_tiles(seg_off, nseg, MS_TILE, tile_off, s);
  uint32_t *H = sc.hist.get<uint32_t>((uint64_t)ub * DIG);
  uint64_t *Hs = sc.hscan.get<uint64_t>((uint64_t)ub * DIG + 1);
  ms_hist_kernel<KeyT, BITS><<<ub, MS_BLOCK, 0, s>>>(in, seg_off, tile_off, nseg, shift, hashed, H);
  CF1_LAUNCH_CHECK();
  exclusive_scan_u32(H, Hs, (uint64_t)ub * DIG, sc.scan_tmp, s);
  size_t smem = MS_TILE * sizeof(KeyT) + (MS_NW + 1) * DIG * sizeof(uint32_t) + DIG * sizeof(uint64_t) +
                (pin ? MS_TILE : 0);
  auto kern = ms_scatter_kernel<KeyT, BITS, false>;
  if constexpr (KOps<KeyT>::WORDS == 1)
    if (pack) kern = ms_scatter_kernel<KeyT, BITS, true>;
  CF1_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<ub, MS_BLOCK, smem, s>>>(in, out, seg_off, tile_off, nseg, shift, hashed, Hs, pin, pout, pack);
  CF1_LAUNCH_CHECK();
}

template <class KeyT>
void ms_pass_bits(int bits, const KeyT *in, KeyT *out, uint64_t n, const uint64_t *seg_off, uint32_t nseg, int shift,
                  bool hashed, MsdScratch &sc, cudaStream_t s, const uint8_t *pin, uint8_t *pout, int pack = 0) {
  switch (bits) {
    case 1: ms_pass<KeyT, 1>(in, out, n, seg_off, nseg, shift, hashed, sc, s, pin, pout, pack); break;
    case 2: ms_pass<KeyT, 2>(in, out, n, seg_off, nseg, shift, hashed, sc, s, pin, pout, pack); break;
    case 3: ms_pass<KeyT, 3>(in, out, n, seg_off, nseg, shift, hashed, sc, s, pin, pout, pack); break;
    case 4: ms_pass<KeyT, 4>(in, out, n, seg_off, nseg, shift, hashed, sc, s, pin, pout, pack); break;
    case 5: ms_pass<KeyT, 5>(in, out, n, seg_off, nseg, shift, hashed, sc, s, pin, pout, pack); break;
    case 6: ms_pass<KeyT, 6>(in, out, n, seg_off, nseg, shift, hashed, sc, s, pin, pout, pack); break;
    case 7: ms_pass<KeyT, 7>(in, out, n, seg_off, nseg, shift, hashed, sc, s, pin, pout, pack); break;
    case 8: ms_pass<KeyT, 8>(in, out, n, seg_off, nseg, shift, hashed, sc, s, pin, pout, pack); break;
    default: throw Error(-1, "MSD pass width must be 1..8 bits");
  }
}

template <int BITS>
void subbuckets(const uint64_t *seg_off, const uint32_t *tile_off, uint32_t nseg, const uint64_t *Hs,
                uint64_t *sb_off, cudaStream_t s) {
  uint64_t nsub = (uint64_t)nseg << BITS;
  ms_subbucket_kernel<BITS><<<(unsigned)ceil_div(nsub + 1, 256), 256, 0, s>>>(seg_off, tile_off, nseg, Hs, sb_off);
  CF1_LAUNCH_CHECK();
}

void subbuckets_bits(int bits, const uint64_t *seg_off, const uint32_t *tile_off, uint32_t nseg, const uint64_t *Hs,
                     uint64_t *sb_off, cudaStream_t s) {
  switch (bits) {
    case 1: subbuckets<1>(seg_off, tile_off, nseg, Hs, sb_off, s); break;
    case 2: subbuckets<2>(seg_off, tile_off, nseg, Hs, sb_off, s); break;
    case 3: subbuckets<3>(seg_off, tile_off, nseg, Hs, sb_off, s); break;
    case 4: subbuckets<4>(seg_off, tile_off, nseg, Hs, sb_off, s); break;
    case 5: subbuckets<5>(seg_off, tile_off, nseg, Hs, sb_off, s); break;
    case 6: subbuckets<6>(seg_off, tile_off, nseg, Hs, sb_off, s); break;
    case 7: subbuckets<7>(seg_off, tile_off, nseg, Hs, sb_off, s); break;
    case 8: subbuckets<8>(seg_off, tile_off, nseg, Hs, sb_off, s); break;
    default: throw Error(-1, "MSD pass width must be 1..8 bits");
  }
}

}  // namespace

template <class KeyT>
void msd_compact(const KeyT *kept, uint64_t nsub, KeyT *dist, MsdScratch &sc, cudaStream_t s) {
  if (!nsub) return;
  cs_compact_kernel<KeyT><<<(unsigned)ceil_div(nsub * 32, 256), 256, 0, s>>>(
      kept, sc.sb_off.as<const uint64_t>(), sc.cnt.as<const uint32_t>(), sc.out_off.as<const uint64_t>(), nsub, dist);
  CF1_LAUNCH_CHECK();
}

template <class KeyT>
int msd_prefix_bits(uint64_t max_bin_keys, bool sorted) {
  // Split on the key's own top bits (sorted), sub-buckets of the average bin
  // size run several times over it (the first bases of canonical k-mers are
  // skewed ~5x), so 64-bit keys aim lower to stay within shared memory
  // (3.1 Gbp, k = 31: 14 bits instead of 12, phase 3 245 -> 230 ms).
  // The unsorted 64-bit form (a warp per sub-bucket, WD_MAXD distinct keys
  // at most) aims at a third of a warp's set for the largest bin.
  const uint64_t target = KOps<KeyT>::WORDS == 1 ? (sorted ? cs_cap<KeyT, true>() / 8 : WD_MAXD / 2)
                                                 : cs_cap_for(true, sorted) / 2;
  int p = 0;
  while (p < 16 && (max_bin_keys >> p) > target) p++;
  return p;
}

template <class KeyT>
bool msd_sort_unique(KeyT *keys, KeyT *alt, uint64_t n, const uint64_t *seg_off, uint32_t nbins, int key_bits, int P,
                     KeyT *dist, uint64_t *dist_off, MsdScratch &sc, cudaStream_t s, bool sorted,
                     const Level0Out *l0, KeyT **kept, uint8_t *pkeys, uint8_t *palt, uint8_t **kept_pay,
                     uint8_t **l0pay_buf) {
  uint8_t *PT = pkeys;  // payloads beside T (nullptr: keys carry none)
  // passes on the top P bits: P1 then P2 (P2 may be 0) -- of the key, or of
  // its hash when only distinct keys are wanted (64-bit keys)
  const bool hashed = !sorted && KOps<KeyT>::WORDS == 1;
  if (hashed) key_bits = 64;
  // packed passes (see pay_code): the hashed split of keys with payloads
  // whose dedup builds BBHash level 0, with a first pass of >= 6 bits
  const bool pk = hashed && pkeys && palt && l0 && l0->AR && l0->with_pay && P >= (int)PACK_MIN_BITS;
  int P1 = P > 8 ? (P + 1) / 2 : P;
  if (pk && P1 < (int)PACK_MIN_BITS) P1 = PACK_MIN_BITS;
  const int P2 = P - P1;
  KeyT *T = keys;
  uint64_t nsub = (uint64_t)nbins << P;
  uint64_t *sb_off = sc.sb_off.get<uint64_t>(nsub + 1);
  if (P == 0) {
    CF1_CUDA(cudaMemcpyAsync(sb_off, seg_off, (nbins + 1) * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
  } else if (n) {
    ms_pass_bits<KeyT>(P1, keys, alt, n, seg_off, nbins, key_bits - P1, hashed, sc, s, pkeys, pk ? nullptr : palt,
                       pk ? P1 : 0);
    const uint64_t *seg2 = seg_off;
    uint32_t nseg2 = nbins;
    if (P2) {
      // segments of pass 2: (bin, first digit), from pass 1's scanned histogram
      uint64_t *sb1 = sc.sb_off1.get<uint64_t>(((uint64_t)nbins << P1) + 1);
      subbuckets_bits(P1, seg_off, sc.tile_off.as<uint32_t>(), nbins, sc.hscan.as<uint64_t>(), sb1, s);
      nseg2 = (uint32_t)((uint64_t)nbins << P1);
      seg2 = sb1;
      if (pk)  // packed words: their own top bits are the next digit, the bytes travel inside
        ms_pass_bits<KeyT>(P2, alt, keys, n, seg2, nseg2, 64 - P2, false, sc, s, nullptr, nullptr);
      else
        ms_pass_bits<KeyT>(P2, alt, keys, n, seg2, nseg2, key_bits - P1 - P2, hashed, sc, s, palt, pkeys);
      T = keys;
      PT = pkeys;
    } else {
      T = alt;
      PT = palt;
    }
    subbuckets_bits(P2 ? P2 : P1, seg2, sc.tile_off.as<uint32_t>(), nseg2, sc.hscan.as<uint64_t>(), sb_off, s);
  } else {
    CF1_CUDA(cudaMemsetAsync(sb_off, 0, (nsub + 1) * sizeof(uint64_t), s));
  }
  uint32_t *cnt = sc.cnt.get<uint32_t>(nsub + 1);
  uint32_t *over = sc.flag.get<uint32_t>(1);
  CF1_CUDA(cudaMemsetAsync(over, 0, 4, s));
  int rest = key_bits - P;
  int bits = rest < CS_BITS ? rest : CS_BITS;
  int shift = rest - bits;
  if (bits <= 0) {
    bits = 1;  // every key of a sub-bucket is equal: one bucket
    shift = 0;
  }
  if (hashed) {  // the key's own bits: any bits split a sub-bucket into pieces
    bits = CS_BITS;
    shift = 0;
  }
  // S, hist, cur, pstart (u32) and the chunk bounds (u16)
  const uint32_t cap = cs_cap_for(KOps<KeyT>::WORDS == 2, sorted);
  size_t smem = cap * sizeof(KeyT) + (3 * CS_BUCKETS + 1) * sizeof(uint32_t) + (CS_BUCKETS + 2) * sizeof(uint16_t) +
                (pkeys ? cap : 0);
  auto kern = sorted ? cs_sort_unique_kernel<KeyT, true> : cs_sort_unique_kernel<KeyT, false>;
  CF1_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  KeyT *U = T == keys ? alt : keys;
  uint8_t *PU = pkeys ? (PT == pkeys ? palt : pkeys) : nullptr;
  if (l0pay_buf) *l0pay_buf = PU;
  if (nsub) {
    Level0Out lo;
    if (l0 && hashed) lo = *l0;
    lo.with_pay = lo.with_pay && PT != nullptr;
    lo.l0pay = PU;
    for (auto &e : sc.ev)
      if (!e) CF1_CUDA(cudaEventCreate(&e));
    // sorted form: consecutive small sub-buckets of a bin are packed into
    // one CTA's run (the top bits of canonical k-mers are skewed, so most
    // sub-buckets are far below the capacity the largest ones need)
    const uint2 *clist = nullptr;
    const uint64_t *coff = nullptr;
    uint64_t grid = nsub;
    if (sorted && P > 0) {
      uint2 *cl = sc.clist.get<uint2>(nsub);
      uint32_t *cc = sc.ccount.get<uint32_t>(nbins + 1);
      uint64_t *co = sc.coff.get<uint64_t>(nbins + 1);
      // runs of up to 2/3 of the capacity: the shared-memory set of the
      // dedup (a power of two >= 1.5 n slots, filled to 3/4 at most) then
      // always holds the run, so it never falls back to sorting copies
      cs_plan_kernel<<<(unsigned)ceil_div(nbins, 128), 128, 0, s>>>(sb_off, nbins, P, cap * 2 / 3, cl, cc);
      CF1_LAUNCH_CHECK();
      exclusive_scan_u32(cc, co, nbins, sc.scan_tmp, s);
      CF1_CUDA(cudaMemcpyAsync(&grid, co + nbins, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
      CF1_CUDA(cudaStreamSynchronize(s));
      clist = cl;
      coff = co;
    }
    CF1_CUDA(cudaEventRecord(sc.ev[0], s));
    if (hashed) {
      // the unsorted form: one warp per sub-bucket; the few it cannot hold
      // (more than WD_MAXD distinct keys) go to the block kernel after it
      uint32_t *ov = sc.ov.get<uint32_t>(nsub + 1);
      uint32_t *ovc = sc.ovc.get<uint32_t>(2);  // overflow count, work counter
      CF1_CUDA(cudaMemsetAsync(ovc, 0, 2 * sizeof(uint32_t), s));
      const size_t wsm = WD_WARPS * sizeof(WdSmem);
      auto wkern = pk ? wd_dedup_kernel<true> : wd_dedup_kernel<false>;
      CF1_CUDA(cudaFuncSetAttribute(wkern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsm));
      const unsigned wgrid = persistent_grid(wkern, WD_WARPS * 32, wsm, -1, ceil_div(nsub, WD_WARPS));
      wkern<<<wgrid, WD_WARPS * 32, wsm, s>>>(reinterpret_cast<uint64_t *>(T), PT, sb_off, nsub, P, cnt, lo, ov, ovc,
                                              ovc + 1, pk ? P1 : 0);
      CF1_LAUNCH_CHECK();
      uint32_t h_ov = 0;
      CF1_CUDA(cudaMemcpyAsync(&h_ov, ovc, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      CF1_CUDA(cudaStreamSynchronize(s));
      sc.last_overflow = h_ov;
      if (h_ov && pk) {  // the block kernel takes keys and bytes
        wd_unpack_kernel<<<(unsigned)ceil_div((uint64_t)h_ov * 32, 256), 256, 0, s>>>(
            reinterpret_cast<uint64_t *>(T), PT, sb_off, ov, ovc, P, P1);
        CF1_LAUNCH_CHECK();
      }
      if (h_ov) {
        kern<<<h_ov, CS_BLOCK, smem, s>>>(T, U, sb_off, nsub, shift, rest > 0 ? bits : 0, cnt, over, P, lo, PT, PU,
                                          nullptr, nullptr, nbins, ov);
        CF1_LAUNCH_CHECK();
      }
    } else {
      kern<<<(unsigned)grid, CS_BLOCK, smem, s>>>(T, U, sb_off, nsub, shift, rest > 0 ? bits : 0, cnt, over, P, lo, PT,
                                                  PU, clist, coff, nbins, nullptr);
      CF1_LAUNCH_CHECK();
    }
    CF1_CUDA(cudaEventRecord(sc.ev[1], s));
  }
  uint32_t h_over = 0;
  CF1_CUDA(cudaMemcpyAsync(&h_over, over, 4, cudaMemcpyDeviceToHost, s));
  CF1_CUDA(cudaStreamSynchronize(s));
  sc.ms_dedup = 0;
  if (nsub) CF1_CUDA(cudaEventElapsedTime(&sc.ms_dedup, sc.ev[0], sc.ev[1]));
  if (h_over) return false;
  uint64_t *out_off = sc.out_off.get<uint64_t>(nsub + 1);
  exclusive_scan_u32(cnt, out_off, nsub, sc.scan_tmp, s);
  if (kept) *kept = T;
  if (kept_pay) *kept_pay = PT;
  if (dist) msd_compact<KeyT>(T, nsub, dist, sc, s);
  cs_bin_off_kernel<<<(unsigned)ceil_div(nbins + 1, 256), 256, 0, s>>>(out_off, nbins, 1ull << P, dist_off);
  CF1_LAUNCH_CHECK();
  return true;
}

#define CF1_INST(KT)                                                                                              \
  template int msd_prefix_bits<KT>(uint64_t, bool);                                                                     \
  template bool msd_sort_unique<KT>(KT *, KT *, uint64_t, const uint64_t *, uint32_t, int, int, KT *, uint64_t *, \
                                    MsdScratch &, cudaStream_t, bool, const Level0Out *, KT **, uint8_t *,    \
                                    uint8_t *, uint8_t **, uint8_t **);                                       \
  template void msd_compact<KT>(const KT *, uint64_t, KT *, MsdScratch &, cudaStream_t);
CF1_INST(uint64_t)
CF1_INST(Key2)
#undef CF1_INST

}  // namespace cf1
