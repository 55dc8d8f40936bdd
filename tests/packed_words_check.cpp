// Host check of the packed multisplit words (cf1_common.cuh): the side-set
// byte's 6-bit code round-trips for every byte a single occurrence can have,
// KEY_SPREAD_INV inverts KEY_SPREAD_MUL, and a word packed the way the first
// multisplit pass packs it gives back, the way the second pass and the warp
// dedup read it, the next digit, the hash, the key and the byte.  Prints
// "ok" and exits 0, or names the first failure and exits 1.
#include <cstdio>
#include <random>

#include "cf1_common.cuh"

using namespace cf1;

int main() {
  const uint32_t nib[5] = {0x3, 0x5, 0x6, 0x9, 0xF};
  for (uint32_t a : nib)
    for (uint32_t b : nib) {
      const uint32_t byte = a | (b << 4), code = pay_code(byte);
      if (code >= 64 || pay_byte(code) != byte) {
        std::printf("byte %02x: code %u decodes to %02x\n", byte, code, pay_byte(code));
        return 1;
      }
    }
  if (KEY_SPREAD_MUL * KEY_SPREAD_INV != 1) {
    std::printf("KEY_SPREAD_INV does not invert KEY_SPREAD_MUL\n");
    return 1;
  }
  std::mt19937_64 rng(7);
  for (int P = (int)PACK_MIN_BITS; P <= 16; P++) {
    // the split of the multisplit: P1 bits first (at least PACK_MIN_BITS when packing), then P2
    int P1 = P > 8 ? (P + 1) / 2 : P;
    if (P1 < (int)PACK_MIN_BITS) P1 = PACK_MIN_BITS;
    const int P2 = P - P1;
    for (int it = 0; it < 200000; it++) {
      const uint64_t key = rng() >> 2;  // k = 31: 62 bits
      const uint32_t byte = nib[rng() % 5] | (nib[rng() % 5] << 4);
      const uint64_t h = key * KEY_SPREAD_MUL;
      const uint64_t w = (h << P1) | pay_code(byte);            // first pass's output word
      const uint32_t sub = (uint32_t)(h >> (64 - P));             // the key's sub-bucket in its bin
      const uint32_t d2 = P2 ? (uint32_t)(w >> (64 - P2)) : 0u;   // second pass's digit
      const uint64_t hi = (uint64_t)(sub >> (P - P1)) << (64 - P1);
      const uint64_t h2 = hi | (w >> P1);                          // the dedup's rebuilt hash
      if (d2 != (sub & ((1u << P2) - 1)) || h2 != h || h2 * KEY_SPREAD_INV != key ||
          pay_byte((uint32_t)w) != byte) {
        std::printf("P=%d key %llx byte %02x: packed word %llx reads back wrong\n", P, (unsigned long long)key,
                    byte, (unsigned long long)w);
        return 1;
      }
    }
  }
  std::printf("ok\n");
  return 0;
}
