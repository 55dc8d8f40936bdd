// Slot queries: Mphf::hash (src/mphf.rs:268-270) for the two device backends.
//
// The key set is split into bins (phase 2); bin b owns slots
// [dist_off[b], dist_off[b+1]).  Inside a bin a key's local slot comes from
//   * BBHash (per bin): levels of bit arrays 8x the keys still unplaced
//     (ph::fmph's relative_level_size 200 would be 2x, src/mphf.rs:155-160);
//     the first level where the key's bit is set gives the level rank; or
//   * the learned index: a small MLP root picks a leaf, the leaf's linear
//     model predicts the rank, and a search in [pred - err, pred + err] of the
//     bin's sorted keys finds the exact rank, which is the local slot.
// Both evaluate identically on the host (cf1_export.cu), so every
// floating-point step is an explicitly rounded single operation.
#pragma once
#include "cf1_internal.cuh"

namespace cf1 {

constexpr uint64_t SLOT_NONE = ~0ull;

// BBHash hashing (multiply-shift, Dietzfelbinger et al. 1997): a 64-bit key
// H -- the k-mer itself for k <= 32, a mix of both words above -- and per
// level l the top 32 bits of H * BB_MUL[l] (odd, independent per level;
// level 0's is KEY_SPREAD_MUL), scaled to the block size.  Two keys that collide at one level differ in H,
// and the next level's multiplier spreads that difference afresh, so their
// next collision is as unlikely as a fresh one.
constexpr uint64_t BB_SEED = 0xD1B54A32D192ED03ull;
constexpr uint32_t BB_MAX_LEVELS = 64;
#define CF1_BB_MUL_TABLE                                                                       \
  {0xd6e8feb86659fd93ull, 0x358e91a8e48b97dbull, 0x970f24b9078ea7c7ull, 0x8f4bacefadb4bcb1ull, \
   0xa1802fdd5c8f452bull, 0xde85f58b25603303ull, 0x364762f470077587ull, 0x7f864ce0775a0c77ull, \
   0x73cc8629f782b791ull, 0x5b3cac1b3a1059edull, 0xf3f2d21e76f5d423ull, 0x5311b35a85f468b1ull, \
   0x9e88fd5a131be1adull, 0x9e9c01811d2017e5ull, 0x129062e2de60e9ffull, 0x56392910d55d4001ull, \
   0x369f3d3960628741ull, 0x07d07f6fa9535d11ull, 0xd28c09328db0b0b1ull, 0x1ae6162a1a4d4957ull, \
   0xb1210c3c3e2d9b4dull, 0x4f6d46e98e254fa1ull, 0x7769e3490c7cff51ull, 0xaa0e641aed9e44d9ull, \
   0x9af1b4f518c92531ull, 0xad08829c8b86913dull, 0x74b11bbb7c9b68b5ull, 0xf88c91c7a171ab17ull, \
   0x6f3ef252b55ad381ull, 0x4913fb1d991cf239ull, 0x08665c7e23c0234full, 0x680bd205a47aa7fbull, \
   0xab26a44018d9d3ebull, 0xf38a638278b6472dull, 0x96db61b024ebdb5bull, 0xa8a816634336b1e3ull, \
   0x6d4ee8af9b7d3935ull, 0x6996bb528191ecf1ull, 0xd9054779fe0087cdull, 0x225b83001770e169ull, \
   0xc2cdad46272294abull, 0xe3e791cdd9a11fbfull, 0x37378255f5fd2a7bull, 0xd2b93a15118fee2bull, \
   0x7db37ee48f069867ull, 0x09670f4e3d3e2fd9ull, 0xe9beb57f8493c53full, 0x47921d41eea996ebull, \
   0xdf3db336bee3959full, 0x9ed13e46eb4adfebull, 0x137132bc0e302887ull, 0xda532fced984988bull, \
   0x3939421e2266f117ull, 0x55db8408d8b43be9ull, 0x9b3c3b4a24da4965ull, 0x397e02be01aca861ull, \
   0x723c864e2ada4953ull, 0x533aa12154e09b8full, 0x516fa0ddd045e98bull, 0x8da77e07eff2b063ull, \
   0xe9b3bdcdc9c409cdull, 0x9b6df4ffc06e320full, 0x0550f8043685bb11ull, 0x42c2a6bcdd74430bull}
static __constant__ uint64_t c_bb_mul[BB_MAX_LEVELS] = CF1_BB_MUL_TABLE;
static constexpr uint64_t h_bb_mul[BB_MAX_LEVELS] = CF1_BB_MUL_TABLE;
static_assert(h_bb_mul[0] == KEY_SPREAD_MUL, "level 0 must hash like the unsorted phase-3 split");

CF1_HD uint64_t bb_key_hash(uint64_t key) { return key; }
CF1_HD uint64_t bb_key_hash(const Key2 &key) { return KOps<Key2>::hash(key, BB_SEED); }

// Bit of a key (hash H) in a block of nwords words at level l: a 32-bit hash
// scaled to [0, 64 nwords).
CF1_HD uint64_t bb_pos(uint64_t H, uint32_t l, uint32_t nwords) {
#ifdef __CUDA_ARCH__
  const uint64_t mul = c_bb_mul[l];
#else
  const uint64_t mul = h_bb_mul[l];
#endif
  const uint32_t t = (uint32_t)((H * mul) >> 32);
  return ((uint64_t)t * nwords) >> 26;
}

// Bit of a key (hash H) inside a slice of sw words at level l.
CF1_HD uint32_t bb_slice_pos(uint64_t H, uint32_t l, uint32_t sw) {
#ifdef __CUDA_ARCH__
  const uint64_t mul = c_bb_mul[l];
#else
  const uint64_t mul = h_bb_mul[l];
#endif
  const uint32_t t = (uint32_t)((H * mul) >> 32);
  return (uint32_t)(((uint64_t)t * sw) >> 26);
}

// Slice of a key among 2^P: the top P bits of its level-0 hash (its phase-3
// sub-bucket).
CF1_HD uint64_t bb_slice(uint64_t H, int P) {
  return P ? (uint64_t)((uint32_t)((H * KEY_SPREAD_MUL) >> 32) >> (32 - P)) : 0;
}

// Bit of a key at a sliced level l of nwords words in 2^P slices: its slice,
// and the bit inside it from level l's own hash.
CF1_HD uint64_t bb_pos_sliced(uint64_t H, uint32_t l, uint32_t nwords, int P) {
  const uint32_t sw = nwords >> P;
  return bb_slice(H, P) * 64 * sw + bb_slice_pos(H, l, sw);
}

// Levels [l0, l1) of a key's walk (hash H): the first level whose bit is set
// gives the local slot.
CF1_HD uint64_t bb_walk(const BBView &v, uint32_t bin, uint64_t H, uint32_t l0, uint32_t l1) {
  for (uint32_t l = l0; l < l1; l++) {
    const BBMeta mt = v.meta[(uint64_t)l * v.nbins + bin];
    if (mt.nwords == 0) return SLOT_NONE;
    const bool sliced = l < 2 && v.l1_slice_bits >= 0;
    const uint64_t pos = (sliced && l == 1) ? bb_pos_sliced(H, 1, mt.nwords, v.l1_slice_bits) : bb_pos(H, l, mt.nwords);
    const ulonglong2 e = v.AR[mt.word_off + (pos >> 6)];
    const uint32_t bit = (uint32_t)(pos & 63);
    if ((e.x >> bit) & 1) {
      uint32_t r = mt.rank_adj + (uint32_t)e.y + (uint32_t)popc64(e.x & ((1ull << bit) - 1));
      if (sliced)  // the placed keys of the bin's slices before this one
        r += v.srank[l][((uint64_t)bin << v.l1_slice_bits) + bb_slice(H, v.l1_slice_bits)];
      return r;
    }
  }
  return SLOT_NONE;
}

template <class KeyT>
CF1_HD uint64_t bb_local_slot(const BBView &v, uint32_t bin, const KeyT &key) {
  return bb_walk(v, bin, bb_key_hash(key), 0, v.levels);
}

// ---- learned index ----
CF1_HD float f_mul(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fmul_rn(a, b);
#else
  return a * b;
#endif
}
CF1_HD float f_fma(float a, float b, float c) {
#ifdef __CUDA_ARCH__
  return __fmaf_rn(a, b, c);
#else
  return fmaf(a, b, c);
#endif
}
CF1_HD float u64_to_f(uint64_t x) {
#ifdef __CUDA_ARCH__
  return __ull2float_rn(x);
#else
  return (float)x;
#endif
}
CF1_HD float f_sub(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fsub_rn(a, b);
#else
  return a - b;
#endif
}
CF1_HD int64_t f_round(float x) {
#ifdef __CUDA_ARCH__
  return (int64_t)__float2ll_rn(x);
#else
  return (int64_t)llrintf(x);
#endif
}

// Root input: the key's top 64 bits relative to the bin's smallest key,
// scaled to [0, 1].
CF1_HD float li_x(const LIRoot &r, uint64_t h) { return f_mul(u64_to_f(h - r.hmin), r.inv_range); }

// Hidden activation of the training network: clipped ReLU, clamp(z, 0, 1).
CF1_HD float li_act(float z) { return z > 0.f ? (z < 1.f ? z : 1.f) : 0.f; }

// The root on its piecewise-linear form: find the piece, one fma.
CF1_HD float li_root_eval(const LIRoot &r, float x) {
  uint32_t j = 0;
#pragma unroll
  for (int i = 1; i < LI_HIDDEN; i++) j += x >= r.knot[i] ? 1u : 0u;
  return f_fma(r.slope[j], f_sub(x, r.knot[j]), r.base[j]);
}

CF1_HD uint32_t li_leaf_of(const LIRoot &r, float y) {
  float t = f_mul(y, (float)r.n_leaves);
  if (!(t > 0.f)) return 0;
  if (t >= (float)r.n_leaves) return r.n_leaves - 1;
  uint32_t li = (uint32_t)t;
  return li < r.n_leaves ? li : r.n_leaves - 1;
}

// Predicted local rank of a key routed to leaf lf.
CF1_HD int64_t li_predict(const LILeaf &lf, uint64_t h) {
  float d = u64_to_f(h - lf.hfirst);
  float q = f_mul(d, lf.slope);
  if (!(q < 4.0e18f)) q = 4.0e18f;  // keys left of the leaf wrap around; keep the sum in range
  return (int64_t)lf.first_rank + f_round(q);
}

// The window [lo, hi] of local ranks a query for key searches: root, leaf,
// the leaf's line, +- its error bound, clamped to the bin.  False when the
// root sends the key to an empty leaf.
template <class KeyT>
CF1_HD bool li_window(const LIView &v, uint64_t n_bin, uint32_t bin, const KeyT &key, int64_t &lo, int64_t &hi) {
  const LIRoot &r = v.roots[bin];
  uint64_t h = KOps<KeyT>::high64(key, v.k);
  uint32_t leaf = li_leaf_of(r, li_root_eval(r, li_x(r, h)));
  const LILeaf lf = v.leaves[r.leaf_off + leaf];
  if (lf.n == 0) return false;
  int64_t p = li_predict(lf, h);
  lo = p - (int64_t)lf.err;
  hi = p + (int64_t)lf.err;
  if (lo < 0) lo = 0;
  if (hi > (int64_t)n_bin - 1) hi = (int64_t)n_bin - 1;
  return true;
}

template <class KeyT>
CF1_HD uint64_t li_local_slot(const LIView &v, const KeyT *bin_keys, uint64_t n_bin, uint32_t bin, const KeyT &key) {
  int64_t lo, hi;
  if (!li_window(v, n_bin, bin, key, lo, hi)) return SLOT_NONE;
  // lower_bound in [lo, hi]
  int64_t a = lo, b = hi + 1;
  while (a < b) {
    int64_t mid = (a + b) >> 1;
    if (bin_keys[mid] < key) a = mid + 1;
    else b = mid;
  }
  if (a <= hi && bin_keys[a] == key) return (uint64_t)a;
  return SLOT_NONE;
}

// MEMBER: the caller knows the key is in the set (phase 4 queries only keys
// of the input), so BBHash's slot needs no range check.
template <class KeyT, bool MEMBER = false>
CF1_HD uint64_t mphf_slot(const MphfView<KeyT> &v, uint32_t bin, const KeyT &key) {
  uint64_t base = v.dist_off[bin];
  if (MEMBER && !v.learned) {
    const uint64_t local = bb_local_slot(v.bb, bin, key);
    return local == SLOT_NONE ? SLOT_NONE : base + local;
  }
  uint64_t local;
  uint64_t n_bin = v.dist_off[bin + 1] - base;
  if (v.learned && v.li.roots[bin].use_learned)
    local = li_local_slot(v.li, v.keys + base, n_bin, bin, key);
  else
    local = bb_local_slot(v.bb, bin, key);
  return local < n_bin ? base + local : SLOT_NONE;
}

}  // namespace cf1
