// Prefix sums and segment tiling.
#include "cf1_device_util.cuh"
#include "cf1_internal.cuh"

namespace cf1 {

std::atomic<uint64_t> g_launches{0};

namespace {

constexpr int SCAN_BLOCK = 512;
constexpr int SCAN_ITEMS = 8;
constexpr uint64_t SCAN_CHUNK = (uint64_t)SCAN_BLOCK * SCAN_ITEMS;

template <class T>
__global__ void __launch_bounds__(SCAN_BLOCK) scan_reduce_kernel(const T *in, uint64_t n, uint64_t *sums) {
  __shared__ uint64_t sm[SCAN_BLOCK / 32];
  uint64_t base = (uint64_t)blockIdx.x * SCAN_CHUNK + (uint64_t)threadIdx.x * SCAN_ITEMS;
  uint64_t acc = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++)
    if (base + i < n) acc += (uint64_t)in[base + i];
  uint64_t tot = block_sum<SCAN_BLOCK>(acc, sm);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

template <class T>
__global__ void __launch_bounds__(SCAN_BLOCK) scan_down_kernel(const T *in, uint64_t n, const uint64_t *block_off,
                                                               uint64_t *out) {
  __shared__ uint64_t sm[SCAN_BLOCK / 32];
  uint64_t base = (uint64_t)blockIdx.x * SCAN_CHUNK + (uint64_t)threadIdx.x * SCAN_ITEMS;
  uint64_t v[SCAN_ITEMS];
  uint64_t acc = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++) {
    v[i] = (base + i < n) ? (uint64_t)in[base + i] : 0;
    acc += v[i];
  }
  uint64_t tot;
  uint64_t pre = block_exclusive_scan<SCAN_BLOCK>(acc, sm, tot);
  pre += block_off ? block_off[blockIdx.x] : 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++) {
    if (base + i < n) out[base + i] = pre;
    pre += v[i];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == SCAN_BLOCK - 1) out[n] = pre;
}

__global__ void zero_total_kernel(uint64_t *out) { out[0] = 0; }

template <class T>
void scan_impl(const T *in, uint64_t *out, uint64_t n, DevBuf &scratch, size_t scratch_off, cudaStream_t s) {
  if (n == 0) {
    zero_total_kernel<<<1, 1, 0, s>>>(out);
    CF1_LAUNCH_CHECK();
    return;
  }
  uint64_t nb = ceil_div(n, SCAN_CHUNK);
  if (nb == 1) {
    scan_down_kernel<T><<<1, SCAN_BLOCK, 0, s>>>(in, n, nullptr, out);
    CF1_LAUNCH_CHECK();
    return;
  }
  // scratch layout at scratch_off: sums[nb], sums_scan[nb+1], deeper levels after.
  uint64_t *sums = reinterpret_cast<uint64_t *>(static_cast<char *>(scratch.p) + scratch_off);
  uint64_t *sums_scan = sums + nb;
  scan_reduce_kernel<T><<<(unsigned)nb, SCAN_BLOCK, 0, s>>>(in, n, sums);
  CF1_LAUNCH_CHECK();
  scan_impl<uint64_t>(sums, sums_scan, nb, scratch, scratch_off + (2 * nb + 1) * sizeof(uint64_t), s);
  scan_down_kernel<T><<<(unsigned)nb, SCAN_BLOCK, 0, s>>>(in, n, sums_scan, out);
  CF1_LAUNCH_CHECK();
}

size_t scan_scratch_bytes(uint64_t n) {
  size_t bytes = 64;
  while (n > SCAN_CHUNK) {
    uint64_t nb = ceil_div(n, SCAN_CHUNK);
    bytes += (2 * nb + 1) * sizeof(uint64_t);
    n = nb;
  }
  return bytes;
}

// seg_off: offsets (segment b has seg_off[b+1] - seg_off[b] items) or, when
// counts is set, the item counts themselves.
__global__ void segment_tiles_kernel(const uint64_t *seg_off, uint32_t nseg, uint32_t tile, bool counts,
                                     uint32_t *tile_off) {
  constexpr int B = 1024;
  __shared__ uint32_t sm[B / 32];
  uint32_t carry = 0;
  for (uint32_t base = 0; base < nseg; base += B) {
    uint32_t b = base + threadIdx.x;
    uint32_t c = 0;
    if (b < nseg) c = (uint32_t)(((counts ? seg_off[b] : seg_off[b + 1] - seg_off[b]) + tile - 1) / tile);
    uint32_t tot;
    uint32_t pre = block_exclusive_scan<B>(c, sm, tot);
    if (b < nseg) tile_off[b] = carry + pre;
    carry += tot;
  }
  if (threadIdx.x == 0) tile_off[nseg] = carry;
}

}  // namespace

void exclusive_scan_u32(const uint32_t *in, uint64_t *out, uint64_t n, DevBuf &scratch, cudaStream_t s) {
  scratch.reserve(scan_scratch_bytes(n));
  scan_impl<uint32_t>(in, out, n, scratch, 0, s);
}
void exclusive_scan_u64(const uint64_t *in, uint64_t *out, uint64_t n, DevBuf &scratch, cudaStream_t s) {
  scratch.reserve(scan_scratch_bytes(n));
  scan_impl<uint64_t>(in, out, n, scratch, 0, s);
}

void segment_tiles(const uint64_t *seg_off, uint32_t nseg, uint32_t tile, uint32_t *tile_off, cudaStream_t s) {
  segment_tiles_kernel<<<1, 1024, 0, s>>>(seg_off, nseg, tile, false, tile_off);
  CF1_LAUNCH_CHECK();
}

void segment_tiles_counts(const uint64_t *cnt, uint32_t nseg, uint32_t tile, uint32_t *tile_off, cudaStream_t s) {
  segment_tiles_kernel<<<1, 1024, 0, s>>>(cnt, nseg, tile, true, tile_off);
  CF1_LAUNCH_CHECK();
}

}  // namespace cf1
