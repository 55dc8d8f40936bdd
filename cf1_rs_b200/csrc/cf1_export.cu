// Flat host image of the device MPHF and Mphf::hash over it on the CPU.
//
// Phase 5 (src/output.rs) calls Mphf::hash / bucket_id for every k-mer from
// many host threads (src/directed_kmer.rs:81-109, src/output.rs:728-731).
// The image holds everything a query needs: the bucket -> bin table, the
// per-bin slot offsets, the BBHash levels and, in learned mode, the roots,
// leaves and the sorted distinct keys.  The query code is the device code
// (cf1_mphf.cuh), compiled for the host.  Image layout version 5: the BBHash
// levels are one array of 16-byte {bit word, level rank} entries addressed
// through the 16-byte per-(level, bin) metadata, so the image and every
// section in it start on a 16-byte boundary; the header says whether levels 0
// and 1 are sliced (and on how many bits), whose per-slice start ranks follow
// the entries.
#include <cstring>
#include <vector>

#include "cf1_context.cuh"
#include "cf1_mphf.cuh"
#include "cf1_pipeline.cuh"

namespace cf1 {

namespace {

constexpr uint64_t IMAGE_MAGIC = 0x3146485048504D43ull;  // "CMPHPHF1"

struct ImageHeader {
  uint64_t magic;
  uint32_t version, k, m, nbins, levels, learned, key_words;
  int32_t l1_slice_bits;  // BBView::l1_slice_bits
  uint64_t n_distinct, n_leaves;
  uint64_t lut_off, dist_off_off, meta_off, ar_off, ar_words, roots_off, leaves_off, keys_off, total;
  uint64_t srank_off, srank_words;  // sliced levels 0 and 1: their per-slice start ranks, one table each
};

constexpr uint32_t IMAGE_VERSION = 5;
inline uint64_t align16(uint64_t x) { return (x + 15) & ~15ull; }  // sections are 16-byte aligned

template <class KeyT>
size_t export_impl(cf1gpu_ctx *c, void *dst, size_t cap) {
  Backend<KeyT> &be = ctx_backend<KeyT>(c);
  const bool learned = c->opts.mphf_mode == CF1GPU_MPHF_LEARNED;
  const uint32_t B = c->nbins, NL = be.bb.levels;
  const uint64_t nleaves = learned ? be.li.stats.leaves : 0;
  ImageHeader h;
  std::memset(&h, 0, sizeof(h));
  h.magic = IMAGE_MAGIC;
  h.version = IMAGE_VERSION;
  h.k = c->k;
  h.m = c->m;
  h.nbins = B;
  h.levels = NL;
  h.learned = learned;
  h.key_words = KOps<KeyT>::WORDS;
  h.l1_slice_bits = be.bb.l1_slice_bits;
  h.n_distinct = c->n_distinct;
  h.n_leaves = nleaves;
  uint64_t off = align16(sizeof(ImageHeader));
  h.lut_off = off;
  off = align16(off + NUM_BUCKETS * sizeof(uint16_t));
  h.dist_off_off = off;
  off = align16(off + (B + 1) * sizeof(uint64_t));
  h.meta_off = off;
  off = align16(off + (uint64_t)NL * B * sizeof(BBMeta));
  h.ar_off = off;
  h.ar_words = be.bb.total_words;
  off = align16(off + h.ar_words * sizeof(ulonglong2));
  h.srank_off = off;
  h.srank_words = h.l1_slice_bits >= 0 ? be.bb.srank_words : 0;
  off = align16(off + 2 * h.srank_words * sizeof(uint32_t));
  h.roots_off = off;
  off = align16(off + (learned ? B * sizeof(LIRoot) : 0));
  h.leaves_off = off;
  off = align16(off + nleaves * sizeof(LILeaf));
  h.keys_off = off;
  off = align16(off + (learned ? c->n_distinct * sizeof(KeyT) : 0));
  h.total = off;
  if (!dst) return off;
  if (cap < off) throw Error(CF1GPU_ERR_INVALID_ARG, "export buffer too small");
  if (reinterpret_cast<uintptr_t>(dst) % 16)
    throw Error(CF1GPU_ERR_INVALID_ARG, "export buffer must be 16-byte aligned");
  char *d = static_cast<char *>(dst);
  cudaStream_t s = c->stream;
  std::memcpy(d, &h, sizeof(h));
  CF1_CUDA(cudaMemcpyAsync(d + h.lut_off, c->d_lut.p, NUM_BUCKETS * 2, cudaMemcpyDeviceToHost, s));
  CF1_CUDA(cudaMemcpyAsync(d + h.dist_off_off, c->d_dist_off.p, (B + 1) * 8, cudaMemcpyDeviceToHost, s));
  if (NL)
    CF1_CUDA(cudaMemcpyAsync(d + h.meta_off, be.bb.meta_device(), (size_t)NL * B * sizeof(BBMeta), cudaMemcpyDeviceToHost, s));
  if (h.ar_words)
    CF1_CUDA(cudaMemcpyAsync(d + h.ar_off, be.bb.entries_device(), h.ar_words * sizeof(ulonglong2),
                             cudaMemcpyDeviceToHost, s));
  for (int l = 0; l < 2 && h.srank_words; l++)
    CF1_CUDA(cudaMemcpyAsync(d + h.srank_off + l * h.srank_words * sizeof(uint32_t), be.bb.srank_device(l),
                             h.srank_words * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  if (learned) {
    CF1_CUDA(cudaMemcpyAsync(d + h.roots_off, be.li.roots_device(), B * sizeof(LIRoot), cudaMemcpyDeviceToHost, s));
    CF1_CUDA(cudaMemcpyAsync(d + h.leaves_off, be.li.leaves_device(), nleaves * sizeof(LILeaf), cudaMemcpyDeviceToHost, s));
    CF1_CUDA(cudaMemcpyAsync(d + h.keys_off, c->d_dist.p, c->n_distinct * sizeof(KeyT), cudaMemcpyDeviceToHost, s));
  }
  CF1_CUDA(cudaStreamSynchronize(s));
  return off;
}

template <class KeyT>
void host_query_impl(const ImageHeader &h, const char *img, const uint64_t *keys, size_t n, uint64_t *slots) {
  MphfView<KeyT> v;
  v.keys = reinterpret_cast<const KeyT *>(img + h.keys_off);
  v.dist_off = reinterpret_cast<const uint64_t *>(img + h.dist_off_off);
  v.bb.AR = reinterpret_cast<const ulonglong2 *>(img + h.ar_off);
  v.bb.meta = reinterpret_cast<const BBMeta *>(img + h.meta_off);
  v.bb.levels = h.levels;
  v.bb.nbins = h.nbins;
  v.bb.l1_slice_bits = h.l1_slice_bits;
  v.bb.pad = 0;
  v.bb.srank[0] = reinterpret_cast<const uint32_t *>(img + h.srank_off);
  v.bb.srank[1] = v.bb.srank[0] + h.srank_words;
  v.li.roots = reinterpret_cast<const LIRoot *>(img + h.roots_off);
  v.li.leaves = reinterpret_cast<const LILeaf *>(img + h.leaves_off);
  v.li.k = (int)h.k;
  v.learned = (int)h.learned;
  const uint16_t *lut = reinterpret_cast<const uint16_t *>(img + h.lut_off);
  for (size_t i = 0; i < n; i++) {
    KeyT key = KOps<KeyT>::make(keys[i * KOps<KeyT>::WORDS], KOps<KeyT>::WORDS == 2 ? keys[i * 2 + 1] : 0);
    uint64_t mz = kmer_minimizer(key, (int)h.k, (int)h.m);
    uint32_t bin = lut[mix_bucket((uint32_t)mz)];
    uint64_t s = mphf_slot(v, bin, key);
    slots[i] = s == SLOT_NONE ? 0 : s;  // unwrap_or(0), src/mphf.rs:269
  }
}

}  // namespace

size_t export_mphf(cf1gpu_ctx *c, void *dst, size_t cap) {
  if (c->wide) return export_impl<Key2>(c, dst, cap);
  return export_impl<uint64_t>(c, dst, cap);
}

void host_query(const void *image, size_t bytes, const uint64_t *keys, size_t n, uint64_t *slots) {
  if (bytes < sizeof(ImageHeader) || reinterpret_cast<uintptr_t>(image) % 16)
    throw Error(CF1GPU_ERR_INVALID_ARG, "MPHF image too small or not 16-byte aligned");
  ImageHeader h;
  std::memcpy(&h, image, sizeof(h));
  if (h.magic != IMAGE_MAGIC || h.version != IMAGE_VERSION || h.total > bytes)
    throw Error(CF1GPU_ERR_INVALID_ARG, "not a cf1 MPHF image");
  const char *img = static_cast<const char *>(image);
  if (h.key_words == 2) host_query_impl<Key2>(h, img, keys, n, slots);
  else host_query_impl<uint64_t>(h, img, keys, n, slots);
}

}  // namespace cf1
