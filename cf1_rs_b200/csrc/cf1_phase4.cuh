// Launchers of the phase-4 and MPHF-query kernels (cf1_phase4.cu).
#pragma once
#include "cf1_internal.cuh"

namespace cf1 {

template <class KeyT>
struct ClassifyArgs {
  const uint64_t *records;
  uint64_t n_rec;
  const uint64_t *W;
  const uint64_t *NM;
  uint64_t L;
  int k;
  MphfView<KeyT> mphf;
  unsigned long long *states;   // CAS mode: ceil(n_distinct/12) words, zeroed
  uint32_t *sides;              // side-set mode: 12 * ceil(n_distinct/12) bytes, zeroed; nullptr = CAS mode
  uint32_t *queue;              // persistent mode work counter (zeroed), else nullptr
  uint32_t *err;
  unsigned long long *cas_retries;
};

template <class KeyT>
void launch_classify(const ClassifyArgs<KeyT> &a, int persistent_ctas, cudaStream_t s);

// Packs side-set bytes (3 u32 per state word) into state words [w0, w1).
void launch_sideset_pack(const uint32_t *sides, uint64_t w0, uint64_t w1, unsigned long long *states,
                         cudaStream_t s);

template <class KeyT>
void launch_dump(const MphfView<KeyT> &m, uint32_t nbins, uint64_t n, const unsigned long long *states, uint64_t *keys_out,
                 uint8_t *states_out, cudaStream_t s);

template <class KeyT>
void launch_verify(const MphfView<KeyT> &m, uint32_t nbins, uint64_t n, uint32_t *seen, uint32_t *err, cudaStream_t s);

template <class KeyT>
void launch_query(const MphfView<KeyT> &m, const uint16_t *lut, int k, int mlen, const uint64_t *in, uint64_t n,
                  uint64_t *out, cudaStream_t s);

}  // namespace cf1
