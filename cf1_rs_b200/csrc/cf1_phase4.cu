// Phase 4 on the device: DFA vertex classification (src/classify.rs:34-601).
//
// The reference walks every placeholder-free run of every record and, per
// k-mer, queries the MPHF and compare-and-swaps the vertex state
// (src/classify.rs:106-118, 385-518; src/state_vector.rs:47-70).  Here the
// same per-occurrence step runs over the routed super k-mers, bin after bin,
// so one bin's MPHF blocks and state words are what the SMs touch at a time.
// Each occurrence reads its true neighbours from the resident sequence, so the
// k-mer's (front, back) contribution is exactly the reference's.  The DFA is
// a per-side join, so the final words do not depend on the order of the
// updates, and two update modes give the same words:
//   * side sets (default): each occurrence ORs its side-set byte into the
//     vertex's byte with a fire-and-forget atomic (no read, no retry); a
//     streaming pass then packs the bytes into the reference layout;
//   * CAS: a 64-bit atomicCAS loop directly on the reference layout (12 five-
//     bit states per word, LSB first), as src/state_vector.rs:47-70 does.
#include "cf1_device_util.cuh"
#include "cf1_internal.cuh"
#include "cf1_mphf.cuh"
#include "cf1_phase4.cuh"

namespace cf1 {

namespace {

// Threads per CTA: 256 for the learned form's kernel, 128 for the BBHash
// form's (0.7 ms faster at 3.1 Gbp than 256; 512 was 6 ms slower).
constexpr int CL_BLOCK = 256, CL_BLOCK_DEFER = 128;

// Joins contribution c into slot's state (src/state_vector.rs:47-70 CAS loop).
// Each failed CAS means another thread changed the word; a word changes at
// most 12 states x 3 steps, so 64 attempts always suffice.
CF1_D void state_join_cas(unsigned long long *states, uint64_t slot, uint32_t c, uint32_t *err, uint32_t &retries) {
  uint64_t wi = slot / 12;
  uint32_t sh = (uint32_t)(slot - wi * 12) * 5;
  unsigned long long *p = states + wi;
  unsigned long long old = *reinterpret_cast<volatile unsigned long long *>(p);
  for (int it = 0; it < 64; it++) {
    uint32_t cur = (uint32_t)(old >> sh) & 31u;
    uint32_t nv = join_state(cur, c);
    if (nv == cur) return;
    unsigned long long nw = (old & ~(31ull << sh)) | ((unsigned long long)nv << sh);
    unsigned long long prev = atomicCAS(p, old, nw);
    if (prev == old) return;
    old = prev;
    retries++;
  }
  atomicOr(err, (uint32_t)DEV_CAS_LIMIT);
}

// BBHash probes past level 0, deferred: a warp's lanes whose key is not placed
// at level 0 (~12%) park {hash, bin | contribution << 16} in the warp's queue,
// and once 32 wait, 32 lanes walk the deeper levels together.  Walking them
// in place would hold every lane of nearly every warp through level 1 (a
// warp waits for its deepest lane) for a few lanes' sake.
constexpr int CL_QCAP = 64;  // < 32 waiting + up to 32 parked by one step

template <class KeyT, bool SIDESET, bool MAY_DEFER>
__device__ __forceinline__ void classify_body(const ClassifyArgs<KeyT> &a) {
  __shared__ ulonglong2 deferred[MAY_DEFER ? CL_BLOCK_DEFER / 32 : 1][MAY_DEFER ? CL_QCAP : 1];
  const unsigned lane = lane_id();
  const uint64_t n_chunks = (a.n_rec + 31) / 32;
  uint64_t chunk = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint32_t retries = 0;
  const int k = a.k;
  const bool defer = MAY_DEFER && !a.mphf.learned;  // BBHash form (the learned form probes its own way)
  ulonglong2 *dq = deferred[MAY_DEFER ? threadIdx.x >> 5 : 0];
  uint32_t qn = 0;  // parked probes (the same in every lane)
  auto apply = [&](uint64_t slot, uint32_t c) {
    if (slot == SLOT_NONE) atomicOr(a.err, (uint32_t)DEV_MPHF_MISS);
    else if (SIDESET) atomicOr(a.sides + (slot >> 2), sideset_lookup(c) << (8 * (uint32_t)(slot & 3)));
    else state_join_cas(a.states, slot, c, a.err, retries);
  };
  auto drain = [&](uint32_t cnt) {  // lanes < cnt walk the last cnt parked probes
    if (lane < cnt) {
      const ulonglong2 e = dq[qn - cnt + lane];
      const uint32_t bin = (uint32_t)e.y & 0xFFFFu;
      const uint64_t local = bb_walk(a.mphf.bb, bin, e.x, 1, a.mphf.bb.levels);
      apply(local == SLOT_NONE ? SLOT_NONE : a.mphf.dist_off[bin] + local, (uint32_t)(e.y >> 16));
    }
    qn -= cnt;
    __syncwarp();
  };
  for (;;) {
    if (a.queue) {
      uint32_t c = 0;
      if (lane == 0) c = atomicAdd(a.queue, 1u);
      chunk = __shfl_sync(FULL, c, 0);
    }
    if (chunk >= n_chunks) break;
    uint64_t r = chunk * 32 + lane;
    bool valid = r < a.n_rec;
    uint64_t rec = valid ? a.records[r] : 0;
    uint32_t n = valid ? rec_n(rec) : 0;
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
      uint64_t orec = __shfl_sync(FULL, rec, lo);
      uint32_t oex = __shfl_sync(FULL, excl, lo);
      const uint32_t q = j - oex;  // k-mer q of the super k-mer
      uint64_t p = rec_pos(orec) + q;
      bool park = false;  // level 0 did not place the key: defer its probe
      uint64_t H = 0, pbin = 0;
      if (j < total && p + k > a.L) {
        atomicOr(a.err, (uint32_t)DEV_OVERFLOW);
      } else if (j < total) {
        uint32_t bin = rec_bin(orec);
        KeyT fw = KOps<KeyT>::extract(a.W, p, k);
        KeyT rc = KOps<KeyT>::rc(fw, k);
        // Inside a super k-mer the k-mers before and after are valid windows,
        // so only its first and last k-mers can lack a neighbour.
        bool hp = q > 0 || (p > 0 && !is_n(a.NM, p - 1));
        bool hn = q + 1 < rec_n(orec) || (p + k < a.L && !is_n(a.NM, p + k));
        uint32_t pb = hp ? base_at(a.W, p - 1) : 0;
        uint32_t nb = hn ? base_at(a.W, p + k) : 0;
        uint32_t c = contribution(fw, rc, hp, pb, hn, nb, k);
        const KeyT key = kmin(fw, rc);
        if (defer) {
          H = bb_key_hash(key);
          const uint64_t local = bb_walk(a.mphf.bb, bin, H, 0, 1);
          if (local != SLOT_NONE) apply(a.mphf.dist_off[bin] + local, c);
          else park = true, pbin = bin | c << 16;
        } else {
          apply(mphf_slot<KeyT, true>(a.mphf, bin, key), c);
        }
      }
      if (defer) {
        const uint32_t m = __ballot_sync(FULL, park);
        if (park) dq[qn + __popc(m & lanemask_lt())] = make_ulonglong2(H, pbin);
        qn += __popc(m);
        __syncwarp();
        if (qn >= 32) drain(32);
      }
    }
    if (!a.queue) break;
  }
  if (qn) drain(qn);
  retries = warp_sum(retries);
  if (lane == 0 && retries) atomicAdd(a.cas_retries, (unsigned long long)retries);
}

// The learned form's kernel, and the BBHash form's (deferred deep probes).
// The deferring one keeps the learned walk as a branch it never takes: that
// build measured 44.0 ms at 3.1 Gbp, one without it 47.7 ms (the register
// allocation differs).
template <class KeyT, bool SIDESET>
__global__ void __launch_bounds__(CL_BLOCK) classify_kernel(ClassifyArgs<KeyT> a) {
  classify_body<KeyT, SIDESET, false>(a);
}
template <class KeyT, bool SIDESET>
__global__ void __launch_bounds__(CL_BLOCK_DEFER) classify_defer_kernel(ClassifyArgs<KeyT> a) {
  classify_body<KeyT, SIDESET, true>(a);
}

// One warp per sub-bucket: each distinct key's side-set byte to its slot.
// A learned bin's slot is the key's rank, which the dense layout already
// gives; a BBHash bin probes level 0 first for PL_U keys per lane at once
// (independent loads in flight: one probe after another would leave the
// warp waiting on each), then walks the deeper levels for the ~12% level 0
// did not place.
constexpr int PL_U = 4;
template <class KeyT>
__global__ void __launch_bounds__(256) place_sides_kernel(MphfView<KeyT> m, const KeyT *kept, const KeyT *dense,
                                                          const uint8_t *kept_pay, const uint64_t *sb_off,
                                                          const uint32_t *cnt, const uint64_t *out_off, uint64_t j0,
                                                          uint64_t j1, int P, uint8_t *sides, uint32_t *err) {
  const uint64_t j = j0 + (((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (j >= j1) return;
  const uint32_t c = cnt[j], bin = (uint32_t)(j >> P);
  const uint64_t a = sb_off[j], o = out_off[j], base = m.dist_off[bin], end = m.dist_off[bin + 1];
  const bool ranked = m.learned && m.li.roots[bin].use_learned;
  const unsigned lane = lane_id();
  bool miss = false;
  if (ranked) {
    for (uint32_t i = lane; i < c; i += 32) sides[o + i] = kept_pay[a + i];
  } else {
    const BBMeta m0 = m.bb.levels ? m.bb.meta[bin] : BBMeta{};  // level 0 of this bin
    for (uint32_t i0 = 0; i0 < c; i0 += 32 * PL_U) {
      uint64_t H[PL_U];
      uint8_t pay[PL_U];
      ulonglong2 e[PL_U];
      uint32_t bit[PL_U];
#pragma unroll
      for (int u = 0; u < PL_U; u++) {
        const uint32_t i = i0 + u * 32 + lane;
        H[u] = 0;
        pay[u] = 0;
        if (i < c) {
          H[u] = bb_key_hash(dense ? dense[o + i] : kept[a + i]);
          pay[u] = kept_pay[a + i];
        }
      }
#pragma unroll
      for (int u = 0; u < PL_U; u++) {
        const uint32_t i = i0 + u * 32 + lane;
        e[u] = make_ulonglong2(0ull, 0ull);
        bit[u] = 0;
        if (i < c && m0.nwords) {
          const uint64_t pos = bb_pos(H[u], 0, m0.nwords);
          e[u] = m.bb.AR[m0.word_off + (pos >> 6)];
          bit[u] = (uint32_t)(pos & 63);
        }
      }
#pragma unroll
      for (int u = 0; u < PL_U; u++) {
        const uint32_t i = i0 + u * 32 + lane;
        if (i >= c) continue;
        uint64_t local;
        if ((e[u].x >> bit[u]) & 1) {
          local = (uint32_t)(m0.rank_adj + (uint32_t)e[u].y + (uint32_t)popc64(e[u].x & ((1ull << bit[u]) - 1)));
          if (m.bb.l1_slice_bits >= 0)  // sliced levels: the bin's slices before this one
            local = (uint32_t)(local + m.bb.srank[0][((uint64_t)bin << m.bb.l1_slice_bits) +
                                                     bb_slice(H[u], m.bb.l1_slice_bits)]);
        } else
          local = m0.nwords ? bb_walk(m.bb, bin, H[u], 1, m.bb.levels) : SLOT_NONE;
        const uint64_t slot = local == SLOT_NONE ? SLOT_NONE : base + local;
        if (slot < end && slot >= base) sides[slot] = pay[u];
        else miss = true;
      }
    }
  }
  if (__any_sync(FULL, miss) && lane == 0) atomicOr(err, (uint32_t)DEV_MPHF_MISS);
}

// One warp per PL_GROUP consecutive sub-buckets: the bytes of the keys
// levels 0 and 1 placed (placed[j] and placed1[j] of them), already in rank
// order, to the two slices' runs of slots (level 1's bytes follow level 0's
// in l0pay).  The group's counts and slot bases are loaded by one lane each,
// in parallel, then every sub-bucket's bytes are copied by the whole warp.
constexpr uint32_t PL_GROUP = 8;
__global__ void __launch_bounds__(256) place_l0_kernel(BBView bb, const uint64_t *dist_off, const uint64_t *sb_off,
                                                       const uint32_t *placed, const uint32_t *placed1,
                                                       const uint8_t *l0pay, uint64_t j0, uint64_t j1, int P,
                                                       uint8_t *sides, uint32_t *err) {
  const unsigned lane = lane_id();
  const uint64_t g0 = j0 + (((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * PL_GROUP;
  if (g0 >= j1) return;  // the same for the whole warp
  const uint64_t j = g0 + lane;
  uint32_t np0 = 0, np1 = 0;
  uint64_t src = 0, base0 = 0, base1 = 0;
  bool bad = false;
  if (lane < PL_GROUP && j < j1) {
    np0 = placed[j];
    np1 = placed1[j];
    if (np0 | np1) {
      if (bb.l1_slice_bits != P || bb.levels < 2) {
        bad = true;
      } else {
        // a slice's first slot: the bin's slots, the keys earlier levels
        // placed, the placed keys of the bin's slices before it
        const uint32_t bin = (uint32_t)(j >> P);
        const uint64_t lo = dist_off[bin], hi = dist_off[bin + 1];
        src = sb_off[j];
        base0 = lo + (uint32_t)(bb.meta[bin].rank_adj + bb.srank[0][j]);
        base1 = lo + (uint32_t)(bb.meta[bb.nbins + bin].rank_adj + bb.srank[1][j]);
        bad = (np0 && base0 + np0 > hi) || (np1 && base1 + np1 > hi);
      }
      if (bad) np0 = np1 = 0;
    }
  }
  if (__any_sync(FULL, bad) && lane == 0) atomicOr(err, (uint32_t)DEV_MPHF_MISS);
  for (uint32_t i = 0; i < PL_GROUP; i++) {
    const uint32_t a0 = __shfl_sync(FULL, np0, i), a1 = __shfl_sync(FULL, np1, i);
    if (!(a0 | a1)) continue;
    const uint64_t s0 = __shfl_sync(FULL, src, i), b0 = __shfl_sync(FULL, base0, i),
                   b1 = __shfl_sync(FULL, base1, i);
    const uint8_t *sp = l0pay + s0;
    for (uint32_t r = lane; r < a0; r += 32) sides[b0 + r] = sp[r];
    for (uint32_t r = lane; r < a1; r += 32) sides[b1 + r] = sp[a0 + r];
  }
}

// The keys levels 0 and 1 left: SV_CTAS CTAs per bin, each key walks from
// level 2.
constexpr uint32_t SV_CTAS = 32;
__global__ void __launch_bounds__(256) place_surv_kernel(BBView bb, const uint64_t *dist_off, const uint64_t *surv,
                                                         const uint8_t *surv_pay, const uint64_t *surv_off,
                                                         const unsigned long long *surv_cnt, uint32_t b0,
                                                         uint8_t *sides, uint32_t *err) {
  const uint32_t bin = b0 + blockIdx.x / SV_CTAS, part = blockIdx.x % SV_CTAS;
  const uint64_t n = surv_cnt[bin], s0 = surv_off[bin], base = dist_off[bin], end = dist_off[bin + 1];
  bool miss = false;
  for (uint64_t i = (uint64_t)part * blockDim.x + threadIdx.x; i < n; i += (uint64_t)SV_CTAS * blockDim.x) {
    const uint64_t local = bb_walk(bb, bin, bb_key_hash(surv[s0 + i]), 2, bb.levels);
    const uint64_t slot = local == SLOT_NONE ? SLOT_NONE : base + local;
    if (slot >= base && slot < end) sides[slot] = surv_pay[s0 + i];
    else miss = true;
  }
  if (__syncthreads_or(miss) && threadIdx.x == 0) atomicOr(err, (uint32_t)DEV_MPHF_MISS);
}

// Word w of the state vector from side-set bytes 12w .. 12w+11 (three u32).
constexpr int PK_BLOCK = 256;
__global__ void __launch_bounds__(PK_BLOCK) sideset_pack_kernel(const uint32_t *sides, uint64_t w0, uint64_t w1,
                                                                unsigned long long *states) {
  __shared__ uint8_t lut[256];  // side-set byte -> 5-bit state
  lut[threadIdx.x] = (uint8_t)state_of_sideset(threadIdx.x);
  __syncthreads();
  uint64_t w = w0 + (uint64_t)blockIdx.x * PK_BLOCK + threadIdx.x;
  if (w >= w1) return;
  const uint32_t *q = sides + 3 * w;
  uint32_t b[3] = {q[0], q[1], q[2]};
  unsigned long long out = 0;
#pragma unroll
  for (int j = 0; j < 12; j++) out |= (unsigned long long)lut[(b[j >> 2] >> (8 * (j & 3))) & 0xFFu] << (5 * j);
  states[w] = out;
}

template <class KeyT>
CF1_D KeyT load_key(const uint64_t *w, uint64_t i);
template <>
CF1_D uint64_t load_key<uint64_t>(const uint64_t *w, uint64_t i) { return w[i]; }
template <>
CF1_D Key2 load_key<Key2>(const uint64_t *w, uint64_t i) { return Key2{w[2 * i], w[2 * i + 1]}; }

template <class KeyT>
CF1_D void store_key(uint64_t *w, uint64_t i, const KeyT &k);
template <>
CF1_D void store_key<uint64_t>(uint64_t *w, uint64_t i, const uint64_t &k) { w[i] = k; }
template <>
CF1_D void store_key<Key2>(uint64_t *w, uint64_t i, const Key2 &k) {
  w[2 * i] = k.lo;
  w[2 * i + 1] = k.hi;
}

template <class KeyT>
__global__ void dump_kernel(MphfView<KeyT> m, uint32_t nbins, uint64_t n, const unsigned long long *states,
                            uint64_t *keys_out, uint8_t *states_out) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t bin = upper_segment(m.dist_off, nbins, i);
  KeyT key = m.keys[i];
  uint64_t slot = mphf_slot(m, bin, key);
  uint8_t st = 0xFF;
  if (slot != SLOT_NONE && slot < n) st = (uint8_t)((states[slot / 12] >> (5 * (slot % 12))) & 31);
  store_key<KeyT>(keys_out, i, key);
  states_out[i] = st;
}

template <class KeyT>
__global__ void verify_mark_kernel(MphfView<KeyT> m, uint32_t nbins, uint64_t n, uint32_t *seen, uint32_t *err) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t bin = upper_segment(m.dist_off, nbins, i);
  uint64_t slot = mphf_slot(m, bin, m.keys[i]);
  if (slot == SLOT_NONE || slot >= n) atomicOr(err, (uint32_t)DEV_BIJECTION);
  else atomicAdd(&seen[slot], 1u);
}

__global__ void verify_check_kernel(const uint32_t *seen, uint64_t n, uint32_t *err) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && seen[i] != 1u) atomicOr(err, (uint32_t)DEV_BIJECTION);
}

template <class KeyT>
__global__ void query_kernel(MphfView<KeyT> m, const uint16_t *lut, int k, int mlen, const uint64_t *in, uint64_t n,
                             uint64_t *out) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  KeyT key = load_key<KeyT>(in, i);
  uint64_t mz = kmer_minimizer(key, k, mlen);
  uint32_t bin = lut[mix_bucket((uint32_t)mz)];
  uint64_t slot = mphf_slot(m, bin, key);
  out[i] = slot == SLOT_NONE ? 0 : slot;  // absent keys: unwrap_or(0), src/mphf.rs:269
}

}  // namespace

template <class KeyT>
void launch_classify(const ClassifyArgs<KeyT> &a, int persistent_ctas, cudaStream_t s) {
  if (a.n_rec == 0) return;
  uint64_t warps = (a.n_rec + 31) / 32;
  // BBHash form: deep probes deferred; learned form: the plain walk
  const int block = a.mphf.learned ? CL_BLOCK : CL_BLOCK_DEFER;
  const uint64_t ctas = ceil_div(warps, (uint64_t)(block / 32));
  auto kern = a.sides ? (a.mphf.learned ? classify_kernel<KeyT, true> : classify_defer_kernel<KeyT, true>)
                      : (a.mphf.learned ? classify_kernel<KeyT, false> : classify_defer_kernel<KeyT, false>);
  kern<<<persistent_ctas ? persistent_grid(kern, block, 0, persistent_ctas, ctas) : (unsigned)ctas, block, 0, s>>>(a);
  CF1_LAUNCH_CHECK();
}

template <class KeyT>
void launch_place_sides(const MphfView<KeyT> &m, const KeyT *kept, const KeyT *dense, const uint8_t *kept_pay,
                        const uint64_t *sb_off, const uint32_t *cnt, const uint64_t *out_off, uint64_t j0, uint64_t j1,
                        int P, uint8_t *sides, uint32_t *err, cudaStream_t s) {
  if (j1 <= j0) return;
  place_sides_kernel<KeyT><<<(unsigned)ceil_div((j1 - j0) * 32, 256), 256, 0, s>>>(
      m, kept, dense, kept_pay, sb_off, cnt, out_off, j0, j1, P, sides, err);
  CF1_LAUNCH_CHECK();
}

void launch_place_l0(const BBView &bb, const uint64_t *dist_off, const uint64_t *sb_off, const uint32_t *placed,
                     const uint32_t *placed1, const uint8_t *l0pay, uint64_t j0, uint64_t j1, int P, uint8_t *sides,
                     uint32_t *err, cudaStream_t s) {
  if (j1 <= j0) return;
  place_l0_kernel<<<(unsigned)ceil_div(ceil_div(j1 - j0, (uint64_t)PL_GROUP) * 32, 256), 256, 0, s>>>(
      bb, dist_off, sb_off, placed, placed1, l0pay, j0, j1, P, sides, err);
  CF1_LAUNCH_CHECK();
}

void launch_place_surv(const BBView &bb, const uint64_t *dist_off, const uint64_t *surv, const uint8_t *surv_pay,
                       const uint64_t *surv_off, const unsigned long long *surv_cnt, uint32_t b0, uint32_t b1,
                       uint8_t *sides, uint32_t *err, cudaStream_t s) {
  if (b1 <= b0) return;
  place_surv_kernel<<<(b1 - b0) * SV_CTAS, 256, 0, s>>>(bb, dist_off, surv, surv_pay, surv_off, surv_cnt, b0, sides,
                                                        err);
  CF1_LAUNCH_CHECK();
}

void launch_sideset_pack(const uint32_t *sides, uint64_t w0, uint64_t w1, unsigned long long *states,
                         cudaStream_t s) {
  if (w1 <= w0) return;
  sideset_pack_kernel<<<(unsigned)ceil_div(w1 - w0, PK_BLOCK), PK_BLOCK, 0, s>>>(sides, w0, w1, states);
  CF1_LAUNCH_CHECK();
}

template <class KeyT>
void launch_dump(const MphfView<KeyT> &m, uint32_t nbins, uint64_t n, const unsigned long long *states, uint64_t *keys_out,
                 uint8_t *states_out, cudaStream_t s) {
  if (!n) return;
  dump_kernel<KeyT><<<(unsigned)ceil_div(n, 256), 256, 0, s>>>(m, nbins, n, states, keys_out, states_out);
  CF1_LAUNCH_CHECK();
}

template <class KeyT>
void launch_verify(const MphfView<KeyT> &m, uint32_t nbins, uint64_t n, uint32_t *seen, uint32_t *err, cudaStream_t s) {
  if (!n) return;
  CF1_CUDA(cudaMemsetAsync(seen, 0, n * 4, s));
  verify_mark_kernel<KeyT><<<(unsigned)ceil_div(n, 256), 256, 0, s>>>(m, nbins, n, seen, err);
  CF1_LAUNCH_CHECK();
  verify_check_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, s>>>(seen, n, err);
  CF1_LAUNCH_CHECK();
}

template <class KeyT>
void launch_query(const MphfView<KeyT> &m, const uint16_t *lut, int k, int mlen, const uint64_t *in, uint64_t n,
                  uint64_t *out, cudaStream_t s) {
  if (!n) return;
  query_kernel<KeyT><<<(unsigned)ceil_div(n, 256), 256, 0, s>>>(m, lut, k, mlen, in, n, out);
  CF1_LAUNCH_CHECK();
}

#define CF1_INST(KT)                                                                                             \
  template void launch_classify<KT>(const ClassifyArgs<KT> &, int, cudaStream_t);                               \
  template void launch_place_sides<KT>(const MphfView<KT> &, const KT *, const KT *, const uint8_t *,           \
                                       const uint64_t *, const uint32_t *, const uint64_t *, uint64_t, uint64_t, \
                                       int, uint8_t *, uint32_t *, cudaStream_t);                                \
  template void launch_dump<KT>(const MphfView<KT> &, uint32_t, uint64_t, const unsigned long long *, uint64_t *, \
                                uint8_t *, cudaStream_t);                                                       \
  template void launch_verify<KT>(const MphfView<KT> &, uint32_t, uint64_t, uint32_t *, uint32_t *, cudaStream_t); \
  template void launch_query<KT>(const MphfView<KT> &, const uint16_t *, int, int, const uint64_t *, uint64_t,   \
                                 uint64_t *, cudaStream_t);
CF1_INST(uint64_t)
CF1_INST(Key2)
#undef CF1_INST

}  // namespace cf1
