// Internal entry points behind the C ABI (cf1_pipeline.cu, cf1_export.cu).
#pragma once
#include <cstddef>
#include <cstdint>

struct cf1gpu_ctx;

namespace cf1 {
void add_record(cf1gpu_ctx *c, const char *name, size_t name_len, const uint8_t *seq, size_t len);
void add_records(cf1gpu_ctx *c, const uint8_t *seqs, const uint64_t *off, size_t n);
void add_fasta(cf1gpu_ctx *c, const char *path);
void upload(cf1gpu_ctx *c);
void run_resident(cf1gpu_ctx *c);
size_t run_streamed(cf1gpu_ctx *c, const uint8_t *seqs, const uint64_t *off, size_t n, uint64_t *words, size_t cap);
void xshard_scan(cf1gpu_ctx *c, uint32_t *hist, uint64_t *n_local);
void xshard_route(cf1gpu_ctx *c, const uint32_t *hist, uint64_t *send, size_t cap, uint64_t *counts);
void xshard_finish(cf1gpu_ctx *c, const uint64_t *recv, size_t n);
void dump_states(cf1gpu_ctx *c, uint64_t *keys, uint8_t *states);
void verify_bijection(cf1gpu_ctx *c);
void query(cf1gpu_ctx *c, const uint64_t *keys, size_t n, uint64_t *slots);
void learned_summary(const cf1gpu_ctx *c, double out5[5]);
size_t export_mphf(cf1gpu_ctx *c, void *dst, size_t cap);
size_t export_bin(cf1gpu_ctx *c, uint32_t bin, uint8_t *dst, size_t cap);
void host_query(const void *image, size_t bytes, const uint64_t *keys, size_t n, uint64_t *slots);
}  // namespace cf1
