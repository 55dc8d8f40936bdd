// A bin's super k-mers in the reference's on-disk bin record format.
//
// route_superkmers writes every super k-mer of bin b to cf1_bin_%05d.bin
// (src/superkmer.rs:181-202, 224-226) as a little-endian u16 base count
// followed by the bases 2-bit packed, four per byte, the first base in the
// top two bits (A0 C1 G2 T3); BinReader::read_packed_superkmer reads them
// back (src/superkmer.rs:283-298).  Here a routed super k-mer is a record
// (first position, k-mer count, bin) over the resident 2-bit input, so a bin's
// file is produced on demand: one warp per record writes its header and
// packed bytes at the record's offset in the bin's image.
#include <vector>

#include "cf1_context.cuh"
#include "cf1_device_util.cuh"
#include "cf1_pipeline.cuh"

namespace cf1 {

namespace {

__global__ void bin_sizes_kernel(const uint64_t *records, uint64_t n, int k, uint64_t *size) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) size[i] = 2 + ((uint64_t)rec_n(records[i]) + k - 1 + 3) / 4;
}

// The 4 bases starting at base q, first base in the top two bits.
CF1_D uint32_t four_bases(const uint64_t *W, uint64_t q) {
  uint64_t i = q >> 5;
  int s = (int)(q & 31) * 2;
  uint64_t top = s ? ((W[i] << s) | (W[i + 1] >> (64 - s))) : W[i];
  return (uint32_t)(top >> 56);
}

__global__ void bin_pack_kernel(const uint64_t *records, uint64_t n, const uint64_t *off, const uint64_t *W, int k,
                                uint8_t *out) {
  const uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (r >= n) return;
  const uint64_t rec = records[r];
  const uint64_t pos = rec_pos(rec);
  const uint32_t len = rec_n(rec) + k - 1;  // bases of the super k-mer
  uint8_t *o = out + off[r];
  const uint32_t nbytes = 2 + (len + 3) / 4;
  for (uint32_t j = lane_id(); j < nbytes; j += 32) {
    uint32_t v;
    if (j < 2) {
      v = (len >> (8 * j)) & 0xFF;  // u16 little-endian base count
    } else {
      const uint32_t b = 4 * (j - 2);  // first base of this byte
      v = four_bases(W, pos + b);
      if (b + 4 > len) v &= 0xFFu << (2 * (b + 4 - len));  // bases past the end are 0
    }
    o[j] = (uint8_t)v;
  }
}

}  // namespace

size_t export_bin(cf1gpu_ctx *c, uint32_t bin, uint8_t *dst, size_t cap) {
  cudaStream_t s = c->stream;
  uint64_t r[2];
  CF1_CUDA(cudaMemcpyAsync(r, c->d_rec_off.as<uint64_t>() + bin, 2 * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  CF1_CUDA(cudaStreamSynchronize(s));
  const uint64_t n = r[1] - r[0];
  if (n == 0) return 0;
  const uint64_t *records = c->d_records.as<const uint64_t>() + r[0];
  uint64_t *size = c->d_binfile.get<uint64_t>(2 * n + 2);
  uint64_t *off = size + n + 1;
  bin_sizes_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, s>>>(records, n, c->k, size);
  CF1_LAUNCH_CHECK();
  exclusive_scan_u64(size, off, n, c->d_scan, s);
  uint64_t total = 0;
  CF1_CUDA(cudaMemcpyAsync(&total, off + n, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  CF1_CUDA(cudaStreamSynchronize(s));
  if (!dst) return total;
  if (cap < total) throw Error(CF1GPU_ERR_INVALID_ARG, "bin buffer too small: need " + std::to_string(total));
  uint8_t *img = c->d_binimg.get<uint8_t>(total);
  bin_pack_kernel<<<(unsigned)ceil_div(n * 32, 256), 256, 0, s>>>(records, n, off, c->d_W.as<const uint64_t>(), c->k,
                                                                 img);
  CF1_LAUNCH_CHECK();
  CF1_CUDA(cudaMemcpyAsync(dst, img, total, cudaMemcpyDeviceToHost, s));
  CF1_CUDA(cudaStreamSynchronize(s));
  return total;
}

}  // namespace cf1
