// Phases 1 and 2 on the device: input packing, canonical-minimizer histogram
// (src/minimizer.rs:27-110), greedy partition (src/minimizer.rs:116-172) and
// super k-mer routing into bins (src/superkmer.rs:21-153).
//
// The reference routes 2-bit-packed super k-mers to per-bin files
// (src/superkmer.rs:156-210).  Here the whole input stays resident in HBM as a
// 2-bit array, so a routed super k-mer is an 8-byte record (first position,
// k-mer count, bin) grouped by bin; phases 3 and 4 read the bases through it.
#include "cf1_device_util.cuh"
#include "cf1_internal.cuh"

namespace cf1 {

namespace {

// ---------------------------------------------------------------- pack ----
// Four threads per word of NM (64 input bytes): each loads its 16 bytes with
// one 16-byte load, so a warp reads 512 consecutive bytes; a pair of threads
// makes one word of W and a quad one word of NM (by shuffles), and the words
// are stored by the even / first lanes.  A byte is a base when (byte & 0xDF)
// is one of 'A' 'C' 'G' 'T' (upper- or lower-case, src/dna.rs:64-92); bits
// 1-2 of the upper-case letter give A0 C1 G3 T2, and one xor fixes G/T.
// Bytes past L read as placeholders.
__global__ void pack_kernel(const uint8_t *ascii, uint64_t L, uint64_t *W, uint64_t *NM, uint64_t t0, uint64_t n_nm) {
  const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t t = t0 + (g >> 2);  // the NM word this thread's 16 bases belong to
  const uint32_t q = (uint32_t)(g & 3);
  const bool live = t < n_nm;
  const uint64_t base = t * 64 + q * 16;
  uint32_t v[4];
  if (live && base + 16 <= L) {
    const uint4 x = *reinterpret_cast<const uint4 *>(ascii + base);
    v[0] = x.x;
    v[1] = x.y;
    v[2] = x.z;
    v[3] = x.w;
  } else {
#pragma unroll
    for (int i = 0; i < 4; i++) {
      uint32_t y = 0;
      for (int j = 0; j < 4; j++) {
        const uint64_t p = base + 4 * i + j;
        y |= (uint32_t)(live && p < L ? ascii[p] : (uint8_t)'N') << (8 * j);
      }
      v[i] = y;
    }
  }
  uint32_t w = 0, nm = 0;  // base i of the 16 at bits 30-2i of w, its placeholder bit at bit i of nm
#pragma unroll
  for (int i = 0; i < 16; i++) {
    const uint32_t c = (v[i >> 2] >> (8 * (i & 3))) & 0xFF;
    const uint32_t u = c & 0xDF;
    const bool ok = (u == 'A') | (u == 'C') | (u == 'G') | (u == 'T');
    uint32_t b = (u >> 1) & 3;
    b ^= b >> 1;
    w |= (ok ? b : 0u) << (30 - 2 * i);
    nm |= (uint32_t)(!ok) << i;
  }
  const uint32_t w_next = __shfl_down_sync(FULL, w, 1);
  const uint32_t pair = nm | (__shfl_down_sync(FULL, nm, 1) << 16);
  const uint32_t pair_next = __shfl_down_sync(FULL, pair, 2);
  if (live) {
    if ((q & 1) == 0) W[2 * t + (q >> 1)] = ((uint64_t)w << 32) | w_next;
    if (q == 0) NM[t] = pair | ((uint64_t)pair_next << 32);
  }
}

// -------------------------------------------------------------- super k-mers ----
// One CTA per tile of T = BLOCK*ITEMS k-mer start positions (or, in persistent
// mode, tiles pulled from an atomic counter).  The tile's bases span
// T + k - 1 positions, so consecutive tiles overlap by k-1 bases.
//   1. the 32-bit order values mix_order(c) of the T + w - 1 canonical m-mers
//      into shared memory (mix_order is a bijection, so they rank m-mers as
//      the spec's 64-bit order keys do);
//   2. sliding-window minimum over w by log2(w) doubling passes; a window
//      that holds a placeholder gets the value 0xFFFFFFFF, which no m-mer has;
//   3. each thread takes ITEMS consecutive k-mers: a segment starts where the
//      window minimum changes; one block scan numbers the segments, their
//      starts go to shared memory, and a segment's length is the distance to
//      the next start -- no thread walks a run;
//   4. each valid segment is a super k-mer: it counts once in the histogram of
//      its minimizer bucket (phase 1) and is written once, with its bucket, to
//      an unordered record list that phase 2 routes by bin (a tile reserves
//      its slots with one atomic add).
constexpr uint32_t SK_INVALID = 0xFFFFFFFFu;

template <int BLOCK, int ITEMS, int KC>
__global__ void __launch_bounds__(BLOCK) superkmer_kernel(SuperkmerArgs a) {
  constexpr uint32_t T = BLOCK * ITEMS;
  extern __shared__ __align__(16) uint32_t dyn32[];
  uint32_t *bufA = dyn32;
  uint32_t *bufB = dyn32 + T + 64;
  __shared__ uint32_t s_tile;
  __shared__ unsigned long long s_base;
  __shared__ uint32_t sm[BLOCK / 32];
  const int k = KC ? KC : a.k, m = KC ? M_FIXED : a.m, w = KC ? W_FIXED : a.w;
  const unsigned tid = threadIdx.x;
  const uint64_t NK = a.L - (uint64_t)k + 1;
  uint64_t tile = a.tile_begin + blockIdx.x;
  unsigned long long my_kmers = 0;
  for (;;) {
    if (a.tile_counter) {
      if (tid == 0) s_tile = atomicAdd(a.tile_counter, 1u);
      __syncthreads();
      tile = s_tile;
    }
    if (tile >= a.n_tiles) break;
    const uint64_t P0 = tile * T;
    const uint32_t nk = (uint32_t)min((uint64_t)T, NK - P0);
    const uint32_t nm = nk + w - 1;
    // thread tid owns k-mers [p0, p0 + ITEMS)
    const uint32_t p0 = tid * ITEMS;
    uint32_t zv[ITEMS];
    uint32_t prev = SK_INVALID;
    uint32_t *starts;     // segment starts, once the windows are taken
    const uint32_t *zrow;  // window minima by position (read at segment starts)
    if constexpr (KC != 0) {
      // k, m, w fixed: each thread rolls the m-mers of its ITEMS positions
      // (one extraction, then one base each) and takes its windows' minima
      // in registers; no doubling passes.
      static_assert(ITEMS % 4 == 0 && ITEMS <= W_FIXED, "window split needs ITEMS <= w");
      constexpr uint32_t MM = (1u << (2 * M_FIXED)) - 1;
      auto order_run = [&](uint32_t q0) {  // order values of m-mers q0 .. q0 + ITEMS - 1
        uint32_t fw = (uint32_t)KOps<uint64_t>::extract(a.W, P0 + q0, M_FIXED), r = mmer_rc(fw, M_FIXED);
        uint64_t nxt = KOps<uint64_t>::extract(a.W, P0 + q0 + M_FIXED, 32);  // the bases after, left-aligned
        uint32_t v[ITEMS];
        v[0] = mix_order(fw < r ? fw : r);
#pragma unroll
        for (int i = 1; i < ITEMS; i++) {
          const uint32_t b = (uint32_t)(nxt >> 62);
          nxt <<= 2;
          fw = ((fw << 2) | b) & MM;
          r = (r >> 2) | ((3u - b) << (2 * M_FIXED - 2));
          v[i] = mix_order(fw < r ? fw : r);
        }
#pragma unroll
        for (int i = 0; i < ITEMS; i += 4)
          *reinterpret_cast<uint4 *>(bufA + q0 + i) = make_uint4(v[i], v[i + 1], v[i + 2], v[i + 3]);
      };
      if (p0 < nm) order_run(p0);
      constexpr uint32_t TAIL = (W_FIXED - 1 + ITEMS - 1) / ITEMS;  // threads for the w - 1 m-mers past T
      if (tid < TAIL && T + tid * ITEMS < nm) order_run(T + tid * ITEMS);
      __syncthreads();
      // window i = A[i .. i + w - 1] (A = bufA + p0): the part left of the
      // shared middle A[ITEMS - 1 .. w - 1] by suffix minima, the part right
      // of it by prefix minima; window -1 (k-mer p0 - 1) for the segment test
      constexpr int NA = ITEMS + W_FIXED - 1, NV = (NA + 3) / 4;
      uint32_t A[NV * 4];
#pragma unroll
      for (int v = 0; v < NV; v++) {
        const uint4 x = *reinterpret_cast<const uint4 *>(bufA + p0 + 4 * v);
        A[4 * v] = x.x;
        A[4 * v + 1] = x.y;
        A[4 * v + 2] = x.z;
        A[4 * v + 3] = x.w;
      }
      uint32_t mid0 = A[ITEMS - 1];
#pragma unroll
      for (int j = ITEMS; j <= W_FIXED - 2; j++) mid0 = min(mid0, A[j]);
      const uint32_t mid = min(mid0, A[W_FIXED - 1]);
      uint32_t S = SK_INVALID, win[ITEMS];
#pragma unroll
      for (int i = ITEMS - 1; i >= 0; i--) {
        if (i < ITEMS - 1) S = min(S, A[i]);
        win[i] = min(S, mid);
      }
      uint32_t Pf = SK_INVALID;
#pragma unroll
      for (int i = 1; i < ITEMS; i++) {
        Pf = min(Pf, A[W_FIXED + i - 1]);
        win[i] = min(win[i], Pf);
      }
      // placeholders: the k bases of window i are bits i .. i + k - 1 of nmb
      uint64_t nmb = ~0ull;
      if (p0 <= nk) {
        const uint64_t bs = P0 + p0, wi = bs >> 6;
        const int sh = (int)(bs & 63);
        nmb = a.NM[wi] >> sh;
        if (sh) nmb |= a.NM[wi + 1] << (64 - sh);
      }
      constexpr uint64_t KMASK = (1ull << KC) - 1;
#pragma unroll
      for (int i = 0; i < ITEMS; i++) zv[i] = (p0 + i < nk && ((nmb >> i) & KMASK) == 0) ? win[i] : SK_INVALID;
      if (p0 > 0 && p0 <= nk && !is_n(a.NM, P0 + p0 - 1) && (nmb & (KMASK >> 1)) == 0) {
        const uint32_t am1 = bufA[p0 - 1];
        prev = min(am1, min(S, mid0));
      }
      starts = bufB;
      zrow = bufA;  // written at the segment starts after the scan below
    } else {
      for (uint32_t q = tid; q < nm; q += BLOCK) {
        uint32_t fw = (uint32_t)KOps<uint64_t>::extract(a.W, P0 + q, m);
        uint32_t r = mmer_rc(fw, m);
        bufA[q] = mix_order(fw < r ? fw : r);
      }
      __syncthreads();
      uint32_t *src = bufA, *dst = bufB;
      uint32_t len = nm, span = 1;
      while (span * 2 <= (uint32_t)w) {
        for (uint32_t q = tid; q + span < len; q += BLOCK) dst[q] = min(src[q], src[q + span]);
        __syncthreads();
        uint32_t *t2 = src;
        src = dst;
        dst = t2;
        len -= span;
        span *= 2;
      }
      for (uint32_t p = tid; p < nk; p += BLOCK) {
        uint32_t v = min(src[p], src[p + w - span]);
        dst[p] = window_clean(a.NM, P0 + p, k) ? v : SK_INVALID;
      }
      __syncthreads();
      const uint32_t *z = dst;
      starts = src;  // free now: segment starts
      zrow = z;
      prev = p0 > 0 && p0 <= nk ? z[p0 - 1] : SK_INVALID;
#pragma unroll
      for (int i = 0; i < ITEMS; i++) zv[i] = p0 + i < nk ? z[p0 + i] : SK_INVALID;
    }
    uint32_t bflags = 0, nb = 0, nv = 0;
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      const uint32_t p = p0 + i;
      const bool b = p < nk && (p == 0 || zv[i] != prev);
      bflags |= (uint32_t)b << i;
      nb += b;
      nv += b && zv[i] != SK_INVALID;
      prev = zv[i];
    }
    // one scan numbers both the segments (high half) and the valid ones (low)
    uint32_t tot;
    const uint32_t pre = block_exclusive_scan<BLOCK>((nb << 16) | nv, sm, tot);
    const uint32_t nseg = tot >> 16, nrec = tot & 0xFFFFu;
    // starts[s] = the segment's first position | its record number << 16
    // (0xFFFF: its window holds a placeholder, no record); then one thread
    // per segment writes the records, so the per-record work runs on full
    // warps instead of on the ~1 lane in 9 whose item starts a segment
    uint32_t seg = pre >> 16, vi = pre & 0xFFFFu;
#pragma unroll
    for (int i = 0; i < ITEMS; i++)
      if ((bflags >> i) & 1) {
        const bool valid = zv[i] != SK_INVALID;
        starts[seg++] = (p0 + i) | ((valid ? vi : 0xFFFFu) << 16);
        if constexpr (KC != 0)
          if (valid) bufA[p0 + i] = zv[i];
        vi += valid;
      }
    if (tid == 0) {
      starts[nseg] = nk;
      s_base = nrec ? atomicAdd(a.rec_count, (unsigned long long)nrec) : 0;
    }
    __syncthreads();
    for (uint32_t sg = tid; sg < nseg; sg += BLOCK) {
      const uint32_t st = starts[sg], rn = st >> 16;
      if (rn == 0xFFFFu) continue;
      const uint32_t p = st & 0xFFFFu, n = (starts[sg + 1] & 0xFFFFu) - p;
      const uint32_t bk = mix_bucket(mix_order_inv(zrow[p]));
      atomicAdd(&a.hist[bk], 1u);
      my_kmers += n;
      const uint64_t o = s_base + rn;
      if (o < a.rec_cap) {
        a.rec_tmp[o] = rec_pack(P0 + p, n, 0);
        a.rec_bucket[o] = (uint16_t)bk;
      }
    }
    __syncthreads();
    if (!a.tile_counter) break;
  }
  my_kmers = warp_sum(my_kmers);
  if (lane_id() == 0 && my_kmers) atomicAdd(a.n_kmers, my_kmers);
}

constexpr int SK_BLOCK = 256;

// Phase 2: every record of the unordered list goes to its bin's range
// (records of a bin end up in no particular order).  A CTA takes a tile of
// 4096 records: each record is ranked inside its bin by a shared-memory
// counter, each bin of the tile reserves its run of slots with one global
// atomic, the tile is staged in shared memory in bin order, and the runs are
// written out by consecutive threads on consecutive addresses (a tile gives
// each of 256 bins a run of ~16 records, which a direct store from the
// ranking thread would scatter over 32 sectors per warp store).
constexpr int BS_BLOCK = 256;
constexpr int BS_ITEMS = 16;
constexpr uint32_t BS_TILE = BS_BLOCK * BS_ITEMS;
__global__ void __launch_bounds__(BS_BLOCK, 3) bin_scatter_kernel(const uint64_t *rec_tmp, const uint16_t *rec_bucket,
                                                               uint64_t n, const uint16_t *lut, uint32_t num_bins,
                                                               const uint64_t *rec_off, uint32_t *cursor,
                                                               uint64_t *records, uint32_t *err) {
  extern __shared__ __align__(16) uint64_t bs_smem[];
  uint64_t *stage = bs_smem;                                           // [BS_TILE]
  uint32_t *s_cnt = reinterpret_cast<uint32_t *>(bs_smem + BS_TILE);  // [num_bins]
  uint32_t *s_start = s_cnt + num_bins;                                // [num_bins] tile-local
  uint32_t *s_base = s_start + num_bins;                               // [num_bins] in the bin's range
  __shared__ uint32_t sm[BS_BLOCK / 32];
  const unsigned tid = threadIdx.x;
  for (uint32_t b = tid; b < num_bins; b += BS_BLOCK) s_cnt[b] = 0;
  __syncthreads();
  const uint64_t r0 = (uint64_t)blockIdx.x * BS_TILE;
  const uint32_t nt = (uint32_t)(n - r0 < BS_TILE ? n - r0 : BS_TILE);
  uint32_t li[BS_ITEMS];  // rank inside the bin, ~0u past the tile's end
  uint64_t rec[BS_ITEMS];  // the routed record (its bin in the low bits)
#pragma unroll
  for (int i = 0; i < BS_ITEMS; i++) {
    const uint32_t j = (uint32_t)i * BS_BLOCK + tid;
    li[i] = 0xFFFFFFFFu;
    if (j < nt) {
      const uint64_t t = rec_tmp[r0 + j];
      const uint32_t b = rec_bucket ? lut[rec_bucket[r0 + j]] : rec_bin(t);  // no buckets: the records carry their bin
      rec[i] = rec_pack(rec_pos(t), rec_n(t), b);
      li[i] = atomicAdd(&s_cnt[b], 1u);
    }
  }
  __syncthreads();
  // tile-local starts: each thread scans a run of consecutive bins
  const uint32_t per = (num_bins + BS_BLOCK - 1) / BS_BLOCK, b0 = tid * per;
  uint32_t own = 0;
  for (uint32_t b = b0; b < b0 + per && b < num_bins; b++) own += s_cnt[b];
  uint32_t tot;
  uint32_t run = block_exclusive_scan<BS_BLOCK>(own, sm, tot);
  for (uint32_t b = b0; b < b0 + per && b < num_bins; b++) {
    const uint32_t c = s_cnt[b];
    s_start[b] = run;
    if (c) s_base[b] = atomicAdd(&cursor[b], c);
    run += c;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < BS_ITEMS; i++)
    if (li[i] != 0xFFFFFFFFu) stage[s_start[rec_bin(rec[i])] + li[i]] = rec[i];
  __syncthreads();
  for (uint32_t i = tid; i < nt; i += BS_BLOCK) {
    const uint64_t r = stage[i];
    const uint32_t b = rec_bin(r);
    const uint64_t idx = rec_off[b] + s_base[b] + (i - s_start[b]);
    if (idx < rec_off[b + 1]) records[idx] = r;
    else atomicOr(err, (uint32_t)DEV_OVERFLOW);
  }
}

void launch_sk(const SuperkmerArgs &a, int persistent_ctas, cudaStream_t s) {
  if (a.n_tiles <= a.tile_begin) return;
  size_t smem = 2 * (a.tile + 64) * sizeof(uint32_t);
  const bool fixed = a.k == K_FIXED && a.m == M_FIXED && a.w == W_FIXED;
  switch (a.tile) {
#define CF1_SK_CASE(IT)                                                                              \
  case SK_BLOCK * IT: {                                                                            \
    auto kern = fixed ? superkmer_kernel<SK_BLOCK, IT, K_FIXED> : superkmer_kernel<SK_BLOCK, IT, 0>; \
    CF1_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
    unsigned grid = persistent_ctas ? persistent_grid(kern, SK_BLOCK, smem, persistent_ctas, a.n_tiles) \
                                    : (unsigned)(a.n_tiles - a.tile_begin);                        \
    kern<<<grid, SK_BLOCK, smem, s>>>(a);                                                          \
    break;                                                                                         \
  }
    CF1_SK_CASE(4)
    CF1_SK_CASE(8)
    CF1_SK_CASE(16)
#undef CF1_SK_CASE
    default:
      throw Error(-1, "super k-mer tile must be 1024, 2048 or 4096");
  }
  CF1_LAUNCH_CHECK();
}

// -------------------------------------------------------------- partition ----
// One CTA.  Boundaries follow the reference's greedy walk: add the bucket,
// place a boundary when the running count reaches total/num_bins, carry the
// excess.  When no bucket exceeds the target the walk never lags, so the
// boundaries after bucket i number min(floor(C(i)/target), num_bins-1) with C
// the inclusive prefix sum; otherwise one thread walks the buckets.
__global__ void __launch_bounds__(1024) partition_kernel(const uint32_t *hist, uint32_t B, uint16_t *lut,
                                                         uint64_t *rec_off, uint32_t *n_bins_eff) {
  constexpr int BLK = 1024;
  constexpr int PER = NUM_BUCKETS / BLK;  // 64
  __shared__ uint64_t sm[BLK / 32];
  __shared__ unsigned long long s_bin[MAX_BINS];
  __shared__ uint32_t s_max;
  const unsigned tid = threadIdx.x;
  const uint32_t b0 = tid * PER;
  uint64_t lsum = 0;
  uint32_t lmax = 0;
  for (int i = 0; i < PER; i++) {
    uint32_t h = hist[b0 + i];
    lsum += h;
    lmax = h > lmax ? h : lmax;
  }
  if (tid == 0) s_max = 0;
  for (uint32_t b = tid; b < B; b += BLK) s_bin[b] = 0;
  __syncthreads();
  atomicMax(&s_max, lmax);
  uint64_t total;
  uint64_t pre = block_exclusive_scan<BLK>(lsum, sm, total);
  const uint64_t target = total / B;
  const uint32_t cap = B - 1;
  if (target == 0 || (uint64_t)s_max <= target) {
    uint64_t C = pre;
    uint64_t j_prev = target == 0 ? min((uint64_t)b0, (uint64_t)cap) : min(C / target, (uint64_t)cap);
    for (int i = 0; i < PER; i++) {
      uint32_t bucket = b0 + i;
      lut[bucket] = (uint16_t)j_prev;
      C += hist[bucket];
      j_prev = target == 0 ? min((uint64_t)bucket + 1, (uint64_t)cap) : min(C / target, (uint64_t)cap);
    }
  } else if (tid == 0) {
    uint64_t cur = 0, nb = 0;
    for (uint32_t bucket = 0; bucket < NUM_BUCKETS; bucket++) {
      lut[bucket] = (uint16_t)nb;
      cur += hist[bucket];
      if (cur >= target && nb < cap) {
        nb++;
        cur -= target;
      }
    }
  }
  __syncthreads();
  for (int i = 0; i < PER; i++) atomicAdd(&s_bin[lut[b0 + i]], (unsigned long long)hist[b0 + i]);
  __syncthreads();
  uint64_t carry = 0;
  for (uint32_t base = 0; base < B; base += BLK) {
    uint32_t b = base + tid;
    uint64_t c = b < B ? s_bin[b] : 0;
    uint64_t tot;
    uint64_t p = block_exclusive_scan<BLK>(c, sm, tot);
    if (b < B) rec_off[b] = carry + p;
    carry += tot;
  }
  if (tid == 0) {
    rec_off[B] = carry;
    *n_bins_eff = (uint32_t)lut[NUM_BUCKETS - 1] + 1;
  }
}

}  // namespace

void launch_pack(const uint8_t *ascii, uint64_t L, uint64_t *W, uint64_t *NM, cudaStream_t s) {
  launch_pack_words(ascii, L, W, NM, 0, ceil_div(L, 64), s);
}

void launch_pack_words(const uint8_t *ascii, uint64_t L, uint64_t *W, uint64_t *NM, uint64_t w0, uint64_t w1,
                       cudaStream_t s) {
  if (w1 <= w0) return;
  pack_kernel<<<(unsigned)ceil_div((w1 - w0) * 4, 256), 256, 0, s>>>(ascii, L, W, NM, w0, w1);
  CF1_LAUNCH_CHECK();
}

void launch_superkmer_scan(const SuperkmerArgs &a, int persistent_ctas, cudaStream_t s) {
  launch_sk(a, persistent_ctas, s);
}

void launch_bin_scatter(const uint64_t *rec_tmp, const uint16_t *rec_bucket, uint64_t n, const uint16_t *lut,
                        uint32_t num_bins, const uint64_t *rec_off, uint32_t *cursor, uint64_t *records, uint32_t *err,
                        cudaStream_t s) {
  if (n == 0) return;
  size_t smem = BS_TILE * sizeof(uint64_t) + 3 * num_bins * sizeof(uint32_t);
  CF1_CUDA(cudaFuncSetAttribute(bin_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  bin_scatter_kernel<<<(unsigned)ceil_div(n, (uint64_t)BS_TILE), BS_BLOCK, smem, s>>>(
      rec_tmp, rec_bucket, n, lut, num_bins, rec_off, cursor, records, err);
  CF1_LAUNCH_CHECK();
}

void launch_partition(const uint32_t *hist, uint32_t num_bins, uint16_t *lut, uint64_t *rec_off, uint32_t *n_bins_eff,
                      cudaStream_t s) {
  partition_kernel<<<1, 1024, 0, s>>>(hist, num_bins, lut, rec_off, n_bins_eff);
  CF1_LAUNCH_CHECK();
}

}  // namespace cf1
