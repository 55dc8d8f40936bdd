// Slot queries: Mphf::hash (src/mphf.rs:268-270) for the two device backends.
//
// The key set is split into bins (phase 2); bin b owns slots
// [dist_off[b], dist_off[b+1]).  Inside a bin a key's local slot comes from
//   * BBHash (per bin): levels of bit arrays 2x the keys still unplaced
//     (gamma 2, like ph::fmph's relative_level_size 200, src/mphf.rs:155-160);
//     the first level where the key's bit is set gives the level rank; or
//   * the learned index: a small MLP root picks a leaf, the leaf's linear
//     model predicts the rank, and a search in [pred - err, pred + err] of the
//     bin's sorted keys finds the exact rank, which is the local slot.
// Both evaluate identically on the host (cf1_host_query.cpp), so every
// floating-point step is an explicitly rounded single operation.
#pragma once
#include "cf1_internal.cuh"

namespace cf1 {

constexpr uint64_t SLOT_NONE = ~0ull;

CF1_HD uint64_t bb_seed(uint32_t level) { return 0x9E3779B97F4A7C15ull * (uint64_t)(level + 1) ^ 0xD1B54A32D192ED03ull; }

template <class KeyT>
CF1_HD uint64_t bb_local_slot(const BBView &v, uint32_t bin, const KeyT &key) {
  for (uint32_t l = 0; l < v.levels; l++) {
    const BBMeta mt = v.meta[(uint64_t)l * v.nbins + bin];
    if (mt.m_bits == 0) return SLOT_NONE;
    uint64_t pos = mulhi64(KOps<KeyT>::hash(key, bb_seed(l)), mt.m_bits);
    const ulonglong2 e = v.AR[l][mt.word_off + (pos >> 6)];
    uint32_t bit = (uint32_t)(pos & 63);
    if ((e.x >> bit) & 1) return mt.rank_adj + e.y + (uint64_t)popc64(e.x & ((1ull << bit) - 1));
  }
  return SLOT_NONE;
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

// Hidden activation: clipped ReLU, clamp(z, 0, 1).
CF1_HD float li_act(float z) { return z > 0.f ? (z < 1.f ? z : 1.f) : 0.f; }

CF1_HD float li_root_eval(const LIRoot &r, float x) {
  float y = r.b2;
  for (int j = 0; j < LI_HIDDEN; j++) y = f_fma(r.w2[j], li_act(f_fma(r.w1[j], x, r.b1[j])), y);
  return y;
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

template <class KeyT>
CF1_HD uint64_t li_local_slot(const LIView &v, const KeyT *bin_keys, uint64_t n_bin, uint32_t bin, const KeyT &key) {
  const LIRoot &r = v.roots[bin];
  uint64_t h = KOps<KeyT>::high64(key, v.k);
  uint32_t leaf = li_leaf_of(r, li_root_eval(r, li_x(r, h)));
  const LILeaf lf = v.leaves[r.leaf_off + leaf];
  if (lf.n == 0) return SLOT_NONE;
  int64_t p = li_predict(lf, h);
  int64_t lo = p - (int64_t)lf.err, hi = p + (int64_t)lf.err;
  if (lo < 0) lo = 0;
  if (hi > (int64_t)n_bin - 1) hi = (int64_t)n_bin - 1;
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

template <class KeyT>
CF1_HD uint64_t mphf_slot(const MphfView<KeyT> &v, uint32_t bin, const KeyT &key) {
  uint64_t base = v.dist_off[bin];
  uint64_t local;
  uint64_t n_bin = v.dist_off[bin + 1] - base;
  if (v.learned && v.li.roots[bin].use_learned)
    local = li_local_slot(v.li, v.keys + base, n_bin, bin, key);
  else
    local = bb_local_slot(v.bb, bin, key);
  return local < n_bin ? base + local : SLOT_NONE;
}

}  // namespace cf1
