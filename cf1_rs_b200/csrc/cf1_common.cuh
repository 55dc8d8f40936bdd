// Shared device/host definitions of the cf1 GPU path.
//
// Sequence layout in HBM (after the pack kernel):
//   * W  : 2-bit bases, 32 per u64 word, most significant first -- base i sits
//          at bits 62-2*(i%32)..63-2*(i%32) of word i/32 (A=0 C=1 G=2 T=3,
//          src/dna.rs:1-9).  Two zero words of padding follow.
//   * NM : placeholder mask, 64 bases per u64 word, bit i%64 of word i/64 set
//          when base i is not in ACGTacgt (src/dna.rs:40-44,81-92).
// All records are concatenated with one placeholder between them; a record
// boundary and a placeholder are the same thing to every phase
// (src/classify.rs:76-77, src/superkmer.rs:156-178).
//
// A k-mer is an integer with its first base in the most significant used bits
// (src/kmer.rs:377-382); k <= 32 uses one u64, 33 <= k <= 63 uses Key2
// (lo = bits 0..63, hi = the rest), compared high word first
// (src/kmer.rs:72-89).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define CF1_HD __host__ __device__ __forceinline__
#define CF1_D __device__ __forceinline__

namespace cf1 {

struct Key2 {
  uint64_t lo, hi;
};
CF1_HD bool operator<(const Key2 &a, const Key2 &b) { return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo); }
CF1_HD bool operator==(const Key2 &a, const Key2 &b) { return a.hi == b.hi && a.lo == b.lo; }
CF1_HD bool operator!=(const Key2 &a, const Key2 &b) { return !(a == b); }
CF1_HD bool operator<=(const Key2 &a, const Key2 &b) { return !(b < a); }

// ------------------------------------------------------------------ bits ----
CF1_HD uint64_t rev_bits64(uint64_t x) {
#ifdef __CUDA_ARCH__
  return __brevll(x);
#else
  x = ((x >> 1) & 0x5555555555555555ull) | ((x & 0x5555555555555555ull) << 1);
  x = ((x >> 2) & 0x3333333333333333ull) | ((x & 0x3333333333333333ull) << 2);
  x = ((x >> 4) & 0x0F0F0F0F0F0F0F0Full) | ((x & 0x0F0F0F0F0F0F0F0Full) << 4);
  x = ((x >> 8) & 0x00FF00FF00FF00FFull) | ((x & 0x00FF00FF00FF00FFull) << 8);
  x = ((x >> 16) & 0x0000FFFF0000FFFFull) | ((x & 0x0000FFFF0000FFFFull) << 16);
  return (x >> 32) | (x << 32);
#endif
}
// Reverses the order of the 2-bit groups of a word (each group keeps its bits).
CF1_HD uint64_t rev_bases64(uint64_t x) {
  uint64_t r = rev_bits64(x);
  return ((r >> 1) & 0x5555555555555555ull) | ((r & 0x5555555555555555ull) << 1);
}
CF1_HD int popc64(uint64_t x) {
#ifdef __CUDA_ARCH__
  return __popcll(x);
#else
  return __builtin_popcountll(x);
#endif
}
CF1_HD uint64_t mulhi64(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
  return __umul64hi(a, b);
#else
  return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

// --------------------------------------------------------- k-mer algebra ----
// KOps<KeyT> collects what the path needs of Kmer<K> (src/kmer.rs): extraction
// from the packed sequence, reverse complement (src/kmer.rs:161-200, computed
// here by bit reversal instead of the byte table), rolling
// (src/kmer.rs:240-262), ordering and the radix digits of the sort.
template <class KeyT>
struct KOps;

template <>
struct KOps<uint64_t> {
  static constexpr int WORDS = 1;
  // The k-mer whose first base is base p (k <= 32).
  static CF1_HD uint64_t extract(const uint64_t *W, uint64_t p, int k) {
    uint64_t i = p >> 5;
    int s = (int)(p & 31) * 2;
    uint64_t w0 = W[i], w1 = W[i + 1];
    uint64_t top = s ? ((w0 << s) | (w1 >> (64 - s))) : w0;
    return top >> (64 - 2 * k);
  }
  // The same, and from the words it reads the base after the k-mer (next,
  // base p + k); prev (base p - 1) needs one more word only when p starts a
  // word.  want_prev: the caller knows base p - 1 exists.
  static CF1_HD uint64_t extract_nb(const uint64_t *W, uint64_t p, int k, bool want_prev, uint32_t &prev,
                                    uint32_t &next) {
    uint64_t i = p >> 5;
    int s = (int)(p & 31) * 2;
    uint64_t w0 = W[i], w1 = W[i + 1];
    uint64_t top = s ? ((w0 << s) | (w1 >> (64 - s))) : w0;  // bases p .. p + 31
    next = (uint32_t)(top >> (62 - 2 * k)) & 3;               // k <= 31
    prev = want_prev ? (s ? (uint32_t)(w0 >> (64 - s)) & 3 : (uint32_t)W[i - 1] & 3) : 0;
    return top >> (64 - 2 * k);
  }
  static CF1_HD uint64_t rc(uint64_t x, int k) { return rev_bases64(~x) >> (64 - 2 * k); }
  static CF1_HD uint64_t mask(int k) { return k >= 32 ? ~0ull : ((1ull << (2 * k)) - 1); }
  static CF1_HD void roll(uint64_t &fw, uint64_t &rcv, uint32_t base, int k) {
    fw = ((fw << 2) | base) & mask(k);
    rcv = (rcv >> 2) | ((uint64_t)(3 - base) << (2 * k - 2));
  }
  static CF1_HD uint32_t digit(uint64_t x, int shift, uint32_t dmask) { return (uint32_t)(x >> shift) & dmask; }
  // 64-bit mix of key ^ seed (the fmix64 finalizer of MurmurHash3).
  static CF1_HD uint64_t hash(uint64_t x, uint64_t seed) {
    x ^= seed;
    x ^= x >> 33; x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
  }
  static CF1_HD uint64_t high64(uint64_t x, int k) { return x << (64 - 2 * k); }  // left-aligned
  static CF1_HD uint64_t sub_low(uint64_t a, uint64_t b) { return a - b; }
  static CF1_HD uint64_t lo(uint64_t x) { return x; }
  static CF1_HD uint64_t hi(uint64_t) { return 0; }
  static CF1_HD uint64_t make(uint64_t lo, uint64_t) { return lo; }
  static CF1_HD uint64_t max_key() { return ~0ull; }
};

template <>
struct KOps<Key2> {
  static constexpr int WORDS = 2;
  // The k-mer whose first base is base p (33 <= k <= 63).
  static CF1_HD Key2 extract(const uint64_t *W, uint64_t p, int k) {
    uint64_t i = p >> 5;
    int s = (int)(p & 31) * 2;
    uint64_t w0 = W[i], w1 = W[i + 1], w2 = W[i + 2];
    uint64_t t0 = s ? ((w0 << s) | (w1 >> (64 - s))) : w0;
    uint64_t t1 = s ? ((w1 << s) | (w2 >> (64 - s))) : w1;
    int sh = 128 - 2 * k;  // 2..62
    Key2 r;
    r.hi = t0 >> sh;
    r.lo = (t1 >> sh) | (t0 << (64 - sh));
    return r;
  }
  // The same, and the bases after (p + k) and before (p - 1) the k-mer, as
  // KOps<uint64_t>::extract_nb.
  static CF1_HD Key2 extract_nb(const uint64_t *W, uint64_t p, int k, bool want_prev, uint32_t &prev,
                                uint32_t &next) {
    uint64_t i = p >> 5;
    int s = (int)(p & 31) * 2;
    uint64_t w0 = W[i], w1 = W[i + 1], w2 = W[i + 2];
    uint64_t t0 = s ? ((w0 << s) | (w1 >> (64 - s))) : w0;  // bases p .. p + 31
    uint64_t t1 = s ? ((w1 << s) | (w2 >> (64 - s))) : w1;  // bases p + 32 .. p + 63
    next = (uint32_t)(t1 >> (62 - 2 * (k - 32))) & 3;       // 33 <= k <= 63
    prev = want_prev ? (s ? (uint32_t)(w0 >> (64 - s)) & 3 : (uint32_t)W[i - 1] & 3) : 0;
    int sh = 128 - 2 * k;  // 2..62
    Key2 r;
    r.hi = t0 >> sh;
    r.lo = (t1 >> sh) | (t0 << (64 - sh));
    return r;
  }
  static CF1_HD Key2 rc(Key2 x, int k) {
    uint64_t rhi = rev_bases64(~x.lo), rlo = rev_bases64(~x.hi);
    int sh = 128 - 2 * k;
    Key2 r;
    r.lo = (rlo >> sh) | (rhi << (64 - sh));
    r.hi = rhi >> sh;
    return r;
  }
  static CF1_HD void roll(Key2 &fw, Key2 &rcv, uint32_t base, int k) {
    uint64_t mhi = (1ull << (2 * k - 64)) - 1;
    fw.hi = ((fw.hi << 2) | (fw.lo >> 62)) & mhi;
    fw.lo = (fw.lo << 2) | base;
    rcv.lo = (rcv.lo >> 2) | (rcv.hi << 62);
    rcv.hi = (rcv.hi >> 2) | ((uint64_t)(3 - base) << (2 * k - 66));
  }
  static CF1_HD uint32_t digit(Key2 x, int shift, uint32_t dmask) {
    if (shift >= 64) return (uint32_t)(x.hi >> (shift - 64)) & dmask;
    uint64_t v = x.lo >> shift;
    if (shift > 0) v |= x.hi << (64 - shift);
    return (uint32_t)v & dmask;
  }
  static CF1_HD uint64_t hash(Key2 x, uint64_t seed) {
    return KOps<uint64_t>::hash(x.lo ^ KOps<uint64_t>::hash(x.hi, seed ^ 0x2545F4914F6CDD1Dull), seed);
  }
  static CF1_HD uint64_t high64(Key2 x, int k) {  // top 64 bits of the left-aligned key
    int sh = 128 - 2 * k;
    return (x.hi << sh) | (sh ? (x.lo >> (64 - sh)) : 0);
  }
  static CF1_HD uint64_t lo(Key2 x) { return x.lo; }
  static CF1_HD uint64_t hi(Key2 x) { return x.hi; }
  static CF1_HD Key2 make(uint64_t lo, uint64_t hi) { return Key2{lo, hi}; }
  static CF1_HD Key2 max_key() { return Key2{~0ull, ~0ull}; }
};

template <class KeyT>
CF1_HD KeyT kmin(KeyT a, KeyT b) { return b < a ? b : a; }

// Base at position p of the packed sequence.
CF1_HD uint32_t base_at(const uint64_t *W, uint64_t p) { return (uint32_t)(W[p >> 5] >> (62 - 2 * (p & 31))) & 3; }
CF1_HD bool is_n(const uint64_t *NM, uint64_t p) { return (NM[p >> 6] >> (p & 63)) & 1; }
// True when bases [p, p+k) hold no placeholder (k <= 63).
CF1_HD bool window_clean(const uint64_t *NM, uint64_t p, int k) {
  uint64_t i = p >> 6;
  int s = (int)(p & 63);
  uint64_t bits = NM[i] >> s;
  if (s) bits |= NM[i + 1] << (64 - s);
  return (bits & ((1ull << k) - 1)) == 0;
}

// ---------------------------------------------------------- binning spec ----
// Canonical minimizers (m odd, m <= 15): order key (mix_order(c) << 32) | c of
// the canonical m-mer c; a k-mer's minimizer is the least order key of its
// w = k-m+1 m-mers, equal for both strands.  Histogram bucket: top 16 bits of
// mix_bucket(c) (65,536 buckets as src/minimizer.rs:8).
CF1_HD uint32_t mix_order(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
  return x;
}
// Odd multiplier whose product's top bits spread 64-bit keys evenly.  The
// unsorted phase-3 split (sub-bucket = top bits of key * KEY_SPREAD_MUL) and
// BBHash level 0 (bit = top bits of key * KEY_SPREAD_MUL, scaled) use the same
// one, so the keys of one sub-bucket land in one stretch of level 0's bits.
constexpr uint64_t KEY_SPREAD_MUL = 0xD6E8FEB86659FD93ull;
// Its inverse mod 2^64 (Newton's iteration x <- x (2 - a x) doubles the
// correct low bits, from 3 for x = a): key = (key * KEY_SPREAD_MUL) *
// KEY_SPREAD_INV.
constexpr uint64_t inverse_mod64(uint64_t a) {
  uint64_t x = a;
  for (int i = 0; i < 6; i++) x *= 2 - a * x;
  return x;
}
constexpr uint64_t KEY_SPREAD_INV = inverse_mod64(KEY_SPREAD_MUL);
static_assert(KEY_SPREAD_MUL * KEY_SPREAD_INV == 1, "KEY_SPREAD_INV inverts KEY_SPREAD_MUL");

// Packed words of the phase-3 multisplit (hashed split of 64-bit keys with
// payload bytes, pass 1 of at least 6 bits): after the first pass a key's
// top p1 bits of h = key * KEY_SPREAD_MUL are its segment's, so the word
// keeps the other 64 - p1 bits of h, shifted up, and the payload byte's
// 6-bit code in the p1 bits freed.
// The next pass splits on the word's own top bits; the dedup rebuilds h from
// the sub-bucket's index and the key as h * KEY_SPREAD_INV.  A single
// occurrence's side-set byte has nibbles in {3, 5, 6, 9, F} (sideset_byte):
// each nibble is a 3-bit code (0 also has one; anything else, which no
// occurrence gives, reads as F).
constexpr uint64_t pay_nib_codes() {
  uint64_t t = 0;
  for (uint32_t v = 0; v < 16; v++) {
    const uint64_t c = v == 3 ? 0 : v == 5 ? 1 : v == 6 ? 2 : v == 9 ? 3 : v == 0 ? 5 : 4;
    t |= c << (3 * v);
  }
  return t;
}
constexpr uint64_t PAY_NIB_CODE = pay_nib_codes();  // nibble -> code, 3 bits each
constexpr uint32_t PAY_NIB_OF = 0x0F9653u;            // code -> nibble, 4 bits each (codes 0..5)
CF1_HD uint32_t pay_code(uint32_t byte) {
  return (uint32_t)((PAY_NIB_CODE >> (3 * (byte & 0xF))) & 7) | ((uint32_t)((PAY_NIB_CODE >> (3 * (byte >> 4))) & 7) << 3);
}
CF1_HD uint32_t pay_byte(uint32_t code) {
  return ((PAY_NIB_OF >> (4 * (code & 7))) & 0xF) | (((PAY_NIB_OF >> (4 * ((code >> 3) & 7))) & 0xF) << 4);
}
constexpr uint32_t PACK_MIN_BITS = 6;  // a packed word's payload code needs 6 of the freed bits

// Inverse of mix_order (the multipliers' inverses mod 2^32; x ^= x >> 15 is
// undone by x ^= (x >> 15) ^ (x >> 30)).  mix_order is a bijection, so the
// order key (mix_order(c) << 32) | c ranks m-mers exactly as mix_order(c)
// alone, and c = mix_order_inv(mix_order(c)).  No canonical m-mer (c < 2^30)
// has mix_order(c) = 0xFFFFFFFF (its preimage is 0xD5F9EFC4).
CF1_HD uint32_t mix_order_inv(uint32_t x) {
  x ^= x >> 16; x *= 0x43021123u; x ^= (x >> 15) ^ (x >> 30); x *= 0x1d69e2a5u; x ^= x >> 16;
  return x;
}
CF1_HD uint32_t mix_bucket(uint32_t x) {
  x ^= 0x5bd1e995u;
  x ^= x >> 16; x *= 0x21f0aaadu; x ^= x >> 15; x *= 0x735a2d97u; x ^= x >> 15;
  return x >> 16;
}
CF1_HD uint32_t mmer_rc(uint32_t x, int m) {
  return (uint32_t)(rev_bases64(~(uint64_t)x) >> (64 - 2 * m));
}
CF1_HD uint64_t mmer_order(uint32_t fw, int m) {
  uint32_t r = mmer_rc(fw, m);
  uint32_t c = fw < r ? fw : r;
  return ((uint64_t)mix_order(c) << 32) | c;
}
// Minimizer order key of a k-mer given as an integer (any strand).
template <class KeyT>
CF1_HD uint64_t kmer_minimizer(KeyT key, int k, int m) {
  uint64_t best = ~0ull;
  uint32_t mm = (1u << (2 * m)) - 1;
  for (int i = 0; i + m <= k; i++) {
    int sh = 2 * (k - m - i);  // m-mer i of the k-mer (from the front)
    uint32_t v;
    if (sh >= 64) v = (uint32_t)(KOps<KeyT>::hi(key) >> (sh - 64)) & mm;
    else {
      uint64_t x = KOps<KeyT>::lo(key) >> sh;
      if (sh > 0 && KOps<KeyT>::WORDS == 2) x |= KOps<KeyT>::hi(key) << (64 - sh);
      v = (uint32_t)x & mm;
    }
    uint64_t o = mmer_order(v, m);
    best = o < best ? o : best;
  }
  return best;
}

// ------------------------------------------------------------ super k-mers ----
// A routed super k-mer: first k-mer position (40 bits), k-mer count - 1
// (12 bits), bin (12 bits).
constexpr uint32_t MAX_TILE = 4096;
constexpr uint32_t MAX_BINS = 4096;
constexpr uint32_t NUM_BUCKETS = 65536;
CF1_HD uint64_t rec_pack(uint64_t pos, uint32_t n, uint32_t bin) {
  return (pos << 24) | ((uint64_t)(n - 1) << 12) | bin;
}
CF1_HD uint64_t rec_pos(uint64_t r) { return r >> 24; }
CF1_HD uint32_t rec_n(uint64_t r) { return (uint32_t)((r >> 12) & 0xFFF) + 1; }
CF1_HD uint32_t rec_bin(uint64_t r) { return (uint32_t)(r & 0xFFF); }

// ------------------------------------------------------------------ states ----
// 5-bit codes (src/state.rs:80-146): 0 unvisited, 3 MIMO, 4|b MISO(back b),
// 8|f SIMO(front f), 16|f<<2|b SISO(front f, back b).  In side form a state is
// a pair (front, back) over {A,C,G,T, M=4}, unvisited = (7,7).  Every
// transition of src/classify.rs:147-518 is the per-side join below, which is
// why final states do not depend on update order.
constexpr uint32_t SIDE_M = 4;
constexpr uint32_t SIDE_NONE = 7;
CF1_HD uint32_t encode_sides(uint32_t f, uint32_t b) {
  if (f == SIDE_M) return b == SIDE_M ? 3u : (4u | b);
  if (b == SIDE_M) return 8u | f;
  return 16u | (f << 2) | b;
}
CF1_HD void decode_sides(uint32_t s, uint32_t &f, uint32_t &b) {
  if (s == 0) { f = SIDE_NONE; b = SIDE_NONE; }
  else if (s == 3) { f = SIDE_M; b = SIDE_M; }
  else if (s < 8) { f = SIDE_M; b = s & 3; }
  else if (s < 12) { f = s & 3; b = SIDE_M; }
  else { f = (s >> 2) & 3; b = s & 3; }
}
CF1_HD uint32_t join_side(uint32_t a, uint32_t b) {
  return a == SIDE_NONE ? b : (b == SIDE_NONE ? a : (a == b ? a : SIDE_M));
}
CF1_HD uint32_t join_state(uint32_t s, uint32_t c) {
  if (s == 0) return c;
  if (s == 3 || s == c) return s;
  uint32_t f1, b1, f2, b2;
  decode_sides(s, f1, b1);
  decode_sides(c, f2, b2);
  return encode_sides(join_side(f1, f2), join_side(b1, b2));
}

// Side sets: the per-side join embedded in bitwise OR, so that a vertex's
// sides can be joined by fire-and-forget atomic ORs and turned into the
// 5-bit state afterwards.  A side is one nibble: base b is the weight-2 code
// 0x3, 0x5, 0x6 or 0x9, M is 0xF, unvisited is 0.  OR of a code with itself
// keeps it; OR of two different weight-2 codes, or of anything with 0xF, has
// weight >= 3, which reads back as M -- exactly join_side.  One byte per
// vertex: front nibble low, back nibble high.
CF1_HD uint32_t side_code(uint32_t side) { return side == SIDE_M ? 0xFu : (0x9653u >> (4 * side)) & 0xFu; }
CF1_HD uint32_t side_of_code(uint32_t nib) {
  if (popc64(nib) >= 3) return SIDE_M;
  return nib == 0x3u ? 0u : nib == 0x5u ? 1u : nib == 0x6u ? 2u : 3u;
}
CF1_HD uint32_t sideset_of_state(uint32_t c) {
  uint32_t f, b;
  decode_sides(c, f, b);
  return side_code(f) | (side_code(b) << 4);
}
// sideset_of_state of all 32 states, 8 bytes to a word, for a lookup by
// shift: (SIDESET_TABLE[c >> 3] >> 8 (c & 7)) & 0xFF.
constexpr uint32_t sideset_ce(uint32_t c) {
  // decode_sides / side_code in constant-expression form
  uint32_t f = SIDE_NONE, b = SIDE_NONE;
  if (c == 3) f = b = SIDE_M;
  else if (c >= 4 && c < 8) f = SIDE_M, b = c & 3;
  else if (c >= 8 && c < 12) f = c & 3, b = SIDE_M;
  else if (c >= 12) f = (c >> 2) & 3, b = c & 3;
  auto code = [](uint32_t side) -> uint32_t { return side == SIDE_M ? 0xFu : side == SIDE_NONE ? 0u : (0x9653u >> (4 * side)) & 0xFu; };
  return code(f) | (code(b) << 4);
}
constexpr uint64_t sideset_word_ce(uint32_t w) {
  uint64_t x = 0;
  for (uint32_t i = 0; i < 8; i++) x |= (uint64_t)sideset_ce(8 * w + i) << (8 * i);
  return x;
}
CF1_HD uint32_t sideset_lookup(uint32_t c) {
  constexpr uint64_t t0 = sideset_word_ce(0), t1 = sideset_word_ce(1), t2 = sideset_word_ce(2), t3 = sideset_word_ce(3);
  const uint64_t w = c < 16 ? (c < 8 ? t0 : t1) : (c < 24 ? t2 : t3);
  return (uint32_t)(w >> (8 * (c & 7))) & 0xFFu;
}
CF1_HD uint32_t state_of_sideset(uint32_t byte) {
  if (byte == 0) return 0;  // no occurrence reached the vertex
  return encode_sides(side_of_code(byte & 0xFu), side_of_code(byte >> 4));
}

// The (front, back) contribution of one k-mer occurrence in canonical
// orientation (src/classify.rs:65-518): isolated -> (M,M); rightmost ->
// fwd (prev,M) / bwd (M,~prev); self loop (canonical == next canonical,
// src/classify.rs:143-145,160-177): leftmost or direct repeat -> (M,M), inverted
// repeat -> as rightmost; leftmost -> fwd (M,next) / bwd (~next,M); internal ->
// fwd (prev,next) / bwd (~next,~prev).  Direction FWD means the k-mer equals
// its canonical form (src/directed_kmer.rs:26-35).
template <class KeyT>
CF1_HD uint32_t contribution(KeyT fw, KeyT rcv, bool has_prev, uint32_t prev, bool has_next, uint32_t next, int k) {
  KeyT can = kmin(fw, rcv);
  bool fwd = fw == can;
  if (!has_prev && !has_next) return 3u;
  uint32_t right = fwd ? encode_sides(prev, SIDE_M) : encode_sides(SIDE_M, 3 - prev);
  if (!has_next) return right;
  KeyT nf = fw, nr = rcv;
  KOps<KeyT>::roll(nf, nr, next, k);
  if (kmin(nf, nr) == can) {
    if (!has_prev || nf == fw) return 3u;
    return right;
  }
  if (!has_prev) return fwd ? encode_sides(SIDE_M, next) : encode_sides(3 - next, SIDE_M);
  return fwd ? encode_sides(prev, next) : encode_sides(3 - next, 3 - prev);
}

// sideset_lookup(contribution(...)) computed directly: the side-set byte of
// one occurrence (front nibble low, back nibble high; M = 0xF), from what it
// depends on: whether the k-mer is read forward (fwd), whether it has a base
// before / after it (and which), whether the next k-mer is the same vertex
// (next_same) and, if so, the same oriented k-mer (next_same_fw).  prev is
// not read without has_prev, nor next, next_same, next_same_fw without
// has_next.
CF1_HD uint32_t sideset_byte(bool fwd, bool has_prev, uint32_t prev, bool has_next, uint32_t next, bool next_same,
                             bool next_same_fw) {
  if (!has_prev && !has_next) return 0xFFu;
  const uint32_t cp = side_code(prev), cpc = side_code(3 - prev);
  const uint32_t right = fwd ? (cp | 0xF0u) : (0x0Fu | (cpc << 4));
  if (!has_next) return right;
  if (next_same) return (!has_prev || next_same_fw) ? 0xFFu : right;
  const uint32_t cn = side_code(next), cnc = side_code(3 - next);
  if (!has_prev) return fwd ? (0x0Fu | (cn << 4)) : (cnc | 0xF0u);
  return fwd ? (cp | (cn << 4)) : (cnc | (cpc << 4));
}

// The same from the k-mer's forward and reverse-complement values and the
// next k-mer's (nf, nr: the k-mer rolled by `next`), which a caller walking
// the sequence has already; with !has_next nf and nr are not read.
template <class KeyT>
CF1_HD uint32_t contribution_sideset_rolled(KeyT fw, KeyT rcv, KeyT nf, KeyT nr, bool has_prev, uint32_t prev,
                                            bool has_next, uint32_t next) {
  const KeyT can = kmin(fw, rcv);
  return sideset_byte(fw == can, has_prev, prev, has_next, next, has_next && kmin(nf, nr) == can,
                      has_next && nf == fw);
}

template <class KeyT>
CF1_HD uint32_t contribution_sideset(KeyT fw, KeyT rcv, bool has_prev, uint32_t prev, bool has_next, uint32_t next,
                                     int k) {
  KeyT nf = fw, nr = rcv;
  KOps<KeyT>::roll(nf, nr, next, k);
  return contribution_sideset_rolled(fw, rcv, nf, nr, has_prev, prev, has_next, next);
}

// ------------------------------------------------------------- error flags ----
enum DeviceError : uint32_t {
  DEV_OK = 0,
  DEV_CAS_LIMIT = 1u << 0,     // a CAS loop passed its iteration cap
  DEV_MPHF_MISS = 1u << 1,     // a queried key was not found
  DEV_OVERFLOW = 1u << 2,      // a buffer or queue bound was hit
  DEV_BIJECTION = 1u << 3,     // slot seen twice or never
  DEV_WAIT_LIMIT = 1u << 4,    // a bounded spin wait gave up
  DEV_FOREIGN = 1u << 5,       // a received record is not this shard's to process
};

}  // namespace cf1
