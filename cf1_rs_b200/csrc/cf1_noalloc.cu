// cf1gpu_distinct_kmers_noalloc: phase 3a (canonical k-mer extraction, LSD
// radix sort, adjacent-unique) for one record, with every byte of scratch in
// a fixed file-scope device array instead of memory allocated per call.
//
// Who needs this: code that must not allocate device memory while it runs --
// a host application that owns the whole device memory pool and hands the
// library only its input and output buffers, or a caller inside a section
// where cudaMalloc would synchronise the device or is forbidden.  Such a
// caller passes device pointers for the record and the outputs; the library
// uses only the array below.
//
// The array is sized for NA_MAX_BASES bases (1 Mi) and every GPU that loads
// this part of the library keeps it (17 MiB) until the process exits.
// All calls share it and it keeps the last call's contents, so each call
// first clears the counters it relies on.  Two calls whose work overlaps on
// the GPU (different streams, or different host threads on one device) race
// on the array and corrupt each other's results: serialise them.
//
// Host code never uses the array's name as an address (on the host it is only
// a stand-in symbol): the first call on each device, with that device
// current, looks up the device address with cudaGetSymbolAddress and caches
// it.  Make that first call before any stream capture on the device.
#include <mutex>

#include "../../include/cf1gpu.h"
#include "cf1_device_util.cuh"
#include "cf1_internal.cuh"

namespace cf1 {

namespace {

constexpr uint64_t NA_MAX_BASES = 1ull << 20;
constexpr int NA_BLOCK = 256;
constexpr int NA_ITEMS = 8;
constexpr uint32_t NA_TILE = NA_BLOCK * NA_ITEMS;            // 2048 keys
constexpr uint32_t NA_MAX_TILES = NA_MAX_BASES / NA_TILE;     // 512
constexpr uint32_t NA_DIGITS = 256;
constexpr int NA_NW = NA_BLOCK / 32;
// The histogram and scatter kernels index per-digit arrays by thread.
static_assert(NA_BLOCK == (int)NA_DIGITS, "one thread per radix digit");

// Scratch layout (byte offsets).
constexpr size_t NA_KEYS = 0;                                          // u64 [NA_MAX_BASES]
constexpr size_t NA_ALT = NA_KEYS + NA_MAX_BASES * 8;                  // u64 [NA_MAX_BASES]
constexpr uint32_t NA_HENTRIES = NA_DIGITS * NA_MAX_TILES;
constexpr size_t NA_HIST = NA_ALT + NA_MAX_BASES * 8;                  // u32 [NA_HENTRIES]
constexpr size_t NA_HSCAN = NA_HIST + NA_HENTRIES * 4;                 // u32 [NA_HENTRIES + 1]
constexpr size_t NA_TCNT = NA_HSCAN + NA_HENTRIES * 4 + 256;           // u32 [NA_MAX_TILES]
constexpr size_t NA_TOFF = NA_TCNT + NA_MAX_TILES * 4;                 // u32 [NA_MAX_TILES + 1]
constexpr size_t NA_COUNT = NA_TOFF + (NA_MAX_TILES + 1) * 4 + 252;    // u32 number of keys (256-aligned)
constexpr size_t NA_SCRATCH_BYTES = NA_COUNT + 256;                    // 17.0 MiB in all

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_SCRATCH_BYTES];

struct Scratch {
  uint64_t *keys, *alt;
  uint32_t *hist, *hscan, *tcnt, *toff, *count;
};

Scratch carve(unsigned char *base) {
  Scratch s;
  s.keys = reinterpret_cast<uint64_t *>(base + NA_KEYS);
  s.alt = reinterpret_cast<uint64_t *>(base + NA_ALT);
  s.hist = reinterpret_cast<uint32_t *>(base + NA_HIST);
  s.hscan = reinterpret_cast<uint32_t *>(base + NA_HSCAN);
  s.tcnt = reinterpret_cast<uint32_t *>(base + NA_TCNT);
  s.toff = reinterpret_cast<uint32_t *>(base + NA_TOFF);
  s.count = reinterpret_cast<uint32_t *>(base + NA_COUNT);
  return s;
}

// Canonical k-mer of every placeholder-free window [p, p+k) (src/mphf.rs:
// 334-343 decode + canonicalise); order does not matter, the sort follows.
__global__ void na_extract_kernel(const uint8_t *seq, uint64_t len, int k, uint64_t *keys, uint32_t *count) {
  uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool ok = p + (uint64_t)k <= len;
  uint64_t fw = 0;
  for (int j = 0; ok && j < k; j++) {
    uint32_t u = seq[p + j] & 0xDF;
    ok = (u == 'A') | (u == 'C') | (u == 'G') | (u == 'T');
    uint32_t b = (u >> 1) & 3;
    fw = (fw << 2) | (b ^ (b >> 1));
  }
  uint64_t can = 0;
  if (ok) {
    uint64_t rc = KOps<uint64_t>::rc(fw, k);
    can = fw < rc ? fw : rc;
  }
  unsigned m = __ballot_sync(FULL, ok);
  uint32_t base = 0;
  if (lane_id() == 0 && m) base = atomicAdd(count, (uint32_t)__popc(m));
  base = __shfl_sync(FULL, base, 0);
  if (ok) keys[base + __popc(m & lanemask_lt())] = can;
}

// Per tile digit counts, digit-major (digit d of tile t at d * ntiles + t).
// Launched over all ntiles tiles of the call's largest possible key count:
// tiles past the actual count write zeros, so every entry the scan reads was
// written by this call and nothing a previous call left reaches it.
__global__ void __launch_bounds__(NA_BLOCK) na_hist_kernel(const uint64_t *keys, const uint32_t *count, int shift,
                                                           uint32_t ntiles, uint32_t *H) {
  __shared__ uint32_t h[NA_DIGITS];
  const uint32_t t = blockIdx.x, n = *count;
  h[threadIdx.x] = 0;
  __syncthreads();
  uint64_t start = (uint64_t)t * NA_TILE, end = start + NA_TILE < n ? start + NA_TILE : n;
  for (uint64_t i = start + threadIdx.x; i < end; i += NA_BLOCK) atomicAdd(&h[(keys[i] >> shift) & 0xFF], 1u);
  __syncthreads();
  H[threadIdx.x * ntiles + t] = h[threadIdx.x];
}

// One CTA: exclusive scan of n u32 values (n <= NA_DIGITS * NA_MAX_TILES).
__global__ void __launch_bounds__(1024) na_scan_kernel(const uint32_t *in, uint32_t *out, uint32_t n) {
  __shared__ uint32_t sm[32];
  uint32_t carry = 0;
  for (uint32_t base = 0; base < n; base += 1024) {
    uint32_t i = base + threadIdx.x;
    uint32_t v = i < n ? in[i] : 0, tot;
    uint32_t pre = block_exclusive_scan<1024>(v, sm, tot);
    if (i < n) out[i] = carry + pre;
    carry += tot;
  }
  if (threadIdx.x == 0) out[n] = carry;
}

// Stable scatter of one tile (round-major order, warp ranks by match_any,
// per (round, warp, digit) counts turned into offsets per digit).
__global__ void __launch_bounds__(NA_BLOCK) na_scatter_kernel(const uint64_t *in, uint64_t *out, const uint32_t *count,
                                                              int shift, uint32_t ntiles, const uint32_t *Hs) {
  __shared__ uint16_t cnt[NA_ITEMS * NA_NW * NA_DIGITS];
  __shared__ uint32_t s_base[NA_DIGITS];
  const uint32_t t = blockIdx.x, n = *count;
  const unsigned tid = threadIdx.x, warp = tid >> 5;
  uint64_t start = (uint64_t)t * NA_TILE;
  if (start >= n) return;
  uint64_t end = start + NA_TILE < n ? start + NA_TILE : n;
  uint32_t *c32 = reinterpret_cast<uint32_t *>(cnt);
  for (uint32_t i = tid; i < NA_ITEMS * NA_NW * NA_DIGITS / 2; i += NA_BLOCK) c32[i] = 0;
  s_base[tid] = Hs[tid * ntiles + t];
  __syncthreads();
  uint64_t key[NA_ITEMS];
  uint32_t dg[NA_ITEMS], wr[NA_ITEMS];
  const unsigned lt = lanemask_lt();
#pragma unroll
  for (int r = 0; r < NA_ITEMS; r++) {
    uint64_t i = start + (uint64_t)r * NA_BLOCK + tid;
    bool act = i < end;
    key[r] = act ? in[i] : 0;
    dg[r] = act ? (uint32_t)(key[r] >> shift) & 0xFF : 0xFFFFFFFFu;
    unsigned peers = __match_any_sync(FULL, dg[r]);
    wr[r] = __popc(peers & lt);
    if (act && wr[r] == 0) cnt[(r * NA_NW + warp) * NA_DIGITS + dg[r]] = (uint16_t)__popc(peers);
  }
  __syncthreads();
  {
    uint32_t run = 0;
    for (int r = 0; r < NA_ITEMS; r++)
      for (int w = 0; w < NA_NW; w++) {
        uint16_t &c = cnt[(r * NA_NW + w) * NA_DIGITS + tid];
        uint32_t v = c;
        c = (uint16_t)run;
        run += v;
      }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < NA_ITEMS; r++)
    if (dg[r] != 0xFFFFFFFFu) out[s_base[dg[r]] + cnt[(r * NA_NW + warp) * NA_DIGITS + dg[r]] + wr[r]] = key[r];
}

__global__ void __launch_bounds__(NA_BLOCK) na_unique_count_kernel(const uint64_t *keys, const uint32_t *count,
                                                                   uint32_t *tcnt) {
  __shared__ uint32_t sm[NA_NW];
  const uint32_t t = blockIdx.x, n = *count;
  uint64_t start = (uint64_t)t * NA_TILE, end = start + NA_TILE < n ? start + NA_TILE : n;
  uint32_t c = 0;
  for (uint64_t i = start + threadIdx.x; i < end; i += NA_BLOCK) c += (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
  uint32_t tot = block_sum<NA_BLOCK>(c, sm);
  if (threadIdx.x == 0) tcnt[t] = tot;
}

__global__ void __launch_bounds__(NA_BLOCK) na_unique_write_kernel(const uint64_t *keys, const uint32_t *count,
                                                                   const uint32_t *toff, uint32_t ntiles,
                                                                   uint64_t *out, uint64_t *n_out) {
  __shared__ uint32_t sm[NA_NW];
  const uint32_t t = blockIdx.x, n = *count;
  uint64_t i0 = (uint64_t)t * NA_TILE + (uint64_t)threadIdx.x * NA_ITEMS;
  uint32_t flags = 0, c = 0;
#pragma unroll
  for (int j = 0; j < NA_ITEMS; j++) {
    uint64_t i = i0 + j;
    bool f = i < n && (i == 0 || keys[i] != keys[i - 1]);
    flags |= (uint32_t)f << j;
    c += f;
  }
  uint32_t tot;
  uint32_t pre = block_exclusive_scan<NA_BLOCK>(c, sm, tot);
  uint64_t o = toff[t] + pre;
#pragma unroll
  for (int j = 0; j < NA_ITEMS; j++)
    if ((flags >> j) & 1) out[o++] = keys[i0 + j];
  if (t == 0 && threadIdx.x == 0) *n_out = toff[ntiles];
}

std::mutex g_addr_mu;
void *g_addr[64] = {};

}  // namespace

}  // namespace cf1

extern "C" int cf1gpu_distinct_kmers_noalloc(int device, uint32_t k, const uint8_t *d_seq, size_t len,
                                             uint64_t *d_keys_out, size_t out_cap, uint64_t *d_n_out, void *stream) {
  using namespace cf1;
  if (len > NA_MAX_BASES) return CF1GPU_ERR_TOO_LARGE;
  if (k < 1 || k > 31 || k % 2 == 0) return CF1GPU_ERR_INVALID_ARG;
  uint64_t max_keys = len >= k ? len - k + 1 : 0;
  if ((len && !d_seq) || !d_keys_out || !d_n_out || out_cap < max_keys) return CF1GPU_ERR_INVALID_ARG;
  if (device < 0 || device >= 64) return CF1GPU_ERR_INVALID_ARG;
  (void)cudaGetLastError();  // an earlier call's error is not this call's
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (s) {  // the work goes to `device`: a stream of another device is refused
    int sdev = -1;
    if (cudaStreamGetDevice(s, &sdev) != cudaSuccess) return CF1GPU_ERR_INVALID_ARG;
    if (sdev != device) return CF1GPU_ERR_INVALID_ARG;
  }
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  if (cudaSetDevice(device) != cudaSuccess) return CF1GPU_ERR_CUDA;
  void *base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (!g_addr[device]) {
      // once per device, with the device current: the array's device address
      if (cudaGetSymbolAddress(&g_addr[device], g_noalloc_scratch) != cudaSuccess) {
        g_addr[device] = nullptr;
        if (prev >= 0) cudaSetDevice(prev);
        return CF1GPU_ERR_CUDA;
      }
    }
    base = g_addr[device];
  }
  Scratch sc = carve(static_cast<unsigned char *>(base));
  uint32_t ntiles = (uint32_t)((max_keys + NA_TILE - 1) / NA_TILE);
  cudaError_t e = cudaMemsetAsync(sc.count, 0, sizeof(uint32_t), s);
  if (e == cudaSuccess && max_keys) {
    na_extract_kernel<<<(unsigned)((max_keys + 255) / 256), 256, 0, s>>>(d_seq, len, (int)k, sc.keys, sc.count);
    uint64_t *src = sc.keys, *dst = sc.alt;
    for (int shift = 0; shift < 2 * (int)k; shift += 8) {
      na_hist_kernel<<<ntiles, NA_BLOCK, 0, s>>>(src, sc.count, shift, ntiles, sc.hist);
      na_scan_kernel<<<1, 1024, 0, s>>>(sc.hist, sc.hscan, NA_DIGITS * ntiles);
      na_scatter_kernel<<<ntiles, NA_BLOCK, 0, s>>>(src, dst, sc.count, shift, ntiles, sc.hscan);
      uint64_t *t = src;
      src = dst;
      dst = t;
    }
    na_unique_count_kernel<<<ntiles, NA_BLOCK, 0, s>>>(src, sc.count, sc.tcnt);
    na_scan_kernel<<<1, 1024, 0, s>>>(sc.tcnt, sc.toff, ntiles);
    na_unique_write_kernel<<<ntiles, NA_BLOCK, 0, s>>>(src, sc.count, sc.toff, ntiles, d_keys_out, d_n_out);
    e = cudaGetLastError();
  } else if (e == cudaSuccess) {
    e = cudaMemsetAsync(d_n_out, 0, sizeof(uint64_t), s);
  }
  if (prev >= 0) cudaSetDevice(prev);
  return e == cudaSuccess ? CF1GPU_OK : CF1GPU_ERR_CUDA;
}
