// The C ABI (include/cf1gpu.h): argument checks, status codes, messages.
#include <cstring>
#include <new>
#include <string>

#include "cf1_context.cuh"
#include "cf1_learned.cuh"
#include "cf1_pipeline.cuh"

namespace {

thread_local std::string g_create_error;

template <class F>
int guard(cf1gpu_ctx *c, F f) {
  try {
    f();
    return CF1GPU_OK;
  } catch (const cf1::Error &e) {
    if (c) c->last_error = e.what();
    else g_create_error = e.what();
    return e.status;
  } catch (const std::bad_alloc &) {
    if (c) c->last_error = "host allocation failed";
    return CF1GPU_ERR_OOM;
  } catch (const std::exception &e) {
    if (c) c->last_error = e.what();
    return CF1GPU_ERR_INVALID_ARG;
  }
}

int minimizer_len(int k) {  // src/params.rs:221-228
  int m = k / 2 < 15 ? k / 2 : 15;
  if (m % 2 == 0) m = m - 1 < 1 ? 1 : m - 1;
  return m;
}

}  // namespace

extern "C" {

void cf1gpu_default_opts(cf1gpu_opts *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->k = 31;
  o->num_bins = 128;
  o->device = 0;
  o->mphf_mode = CF1GPU_MPHF_BBHASH;
}

int cf1gpu_create(const cf1gpu_opts *opts, cf1gpu_ctx **out) {
  if (!opts || !out) return CF1GPU_ERR_INVALID_ARG;
  *out = nullptr;
  if (opts->k < 1 || opts->k > 63 || opts->k % 2 == 0) {
    g_create_error = "k must be odd and in [1, 63], got " + std::to_string(opts->k);
    return CF1GPU_ERR_INVALID_ARG;
  }
  if (opts->num_bins < 1 || opts->num_bins > cf1::MAX_BINS) {
    g_create_error = "num_bins must be in [1, 4096]";
    return CF1GPU_ERR_INVALID_ARG;
  }
  if (opts->mphf_mode > CF1GPU_MPHF_LEARNED) {
    g_create_error = "unknown mphf_mode";
    return CF1GPU_ERR_INVALID_ARG;
  }
  if (opts->sk_tile && opts->sk_tile != 1024 && opts->sk_tile != 2048 && opts->sk_tile != 4096) {
    g_create_error = "sk_tile must be 1024, 2048 or 4096";
    return CF1GPU_ERR_INVALID_ARG;
  }
  if (opts->sort_mode > 1) {
    g_create_error = "sort_mode must be 0 (MSD) or 1 (LSD)";
    return CF1GPU_ERR_INVALID_ARG;
  }
  if (opts->state_update > 2) {
    g_create_error = "state_update must be 0 (side sets joined in phase 3), 1 (CAS) or 2 (side-set classification)";
    return CF1GPU_ERR_INVALID_ARG;
  }
  if (opts->shard_count > cf1::MAX_BINS || (opts->shard_count > 1 && opts->shard_index >= opts->shard_count) ||
      (opts->shard_count <= 1 && opts->shard_index != 0)) {
    g_create_error = "shard_index must be below shard_count (at most 4096 shards)";
    return CF1GPU_ERR_INVALID_ARG;
  }
  cf1gpu_ctx *c = new (std::nothrow) cf1gpu_ctx();
  if (!c) return CF1GPU_ERR_OOM;
  int st = guard(nullptr, [&] {
    c->opts = *opts;
    c->opts.tuner_cache_path = nullptr;
    if (opts->tuner_cache_path) c->tuner_path = opts->tuner_cache_path;
    c->k = (int)opts->k;
    c->m = minimizer_len(c->k);
    c->w = c->k - c->m + 1;
    c->wide = c->k > 32;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
      throw cf1::Error(CF1GPU_ERR_CUDA, "no CUDA device: the cf1 GPU path has no CPU fallback");
    if (opts->device < 0 || opts->device >= ndev) throw cf1::Error(CF1GPU_ERR_INVALID_ARG, "device ordinal out of range");
    CF1_CUDA(cudaSetDevice(opts->device));
    cudaDeviceProp prop;
    CF1_CUDA(cudaGetDeviceProperties(&prop, opts->device));
    c->num_sms = prop.multiProcessorCount;
    CF1_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CF1_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    for (auto &e : c->ev) CF1_CUDA(cudaEventCreate(&e));
    for (auto &e : c->stage_ev) CF1_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    if (opts->sk_tile) c->tune.sk_tile = opts->sk_tile;
    if (opts->learned_max_err) c->learned.max_err = opts->learned_max_err;
    if (opts->learned_train_steps > 0) c->learned.train_steps = opts->learned_train_steps;
    if (opts->learned_train_steps < 0) c->learned.train_steps = -1;
    if (opts->learned_leaf_size) c->learned.leaf_size = opts->learned_leaf_size;
    c->force_lsd = opts->sort_mode == 1;
  });
  if (st != CF1GPU_OK) {
    delete c;
    return st;
  }
  *out = c;
  return CF1GPU_OK;
}

int cf1gpu_add_record(cf1gpu_ctx *c, const char *name, size_t name_len, const uint8_t *seq, size_t len) {
  if (!c || (!seq && len)) return CF1GPU_ERR_INVALID_ARG;
  return guard(c, [&] { cf1::add_record(c, name, name_len, seq, len); });
}

int cf1gpu_add_records(cf1gpu_ctx *c, const uint8_t *seqs, const uint64_t *offsets, size_t n) {
  if (!c || (n && (!seqs || !offsets))) return CF1GPU_ERR_INVALID_ARG;
  for (size_t i = 0; i < n; i++)
    if (offsets[i + 1] < offsets[i]) return CF1GPU_ERR_INVALID_ARG;
  return guard(c, [&] { cf1::add_records(c, seqs, offsets, n); });
}

int cf1gpu_add_fasta(cf1gpu_ctx *c, const char *path) {
  if (!c || !path) return CF1GPU_ERR_INVALID_ARG;
  return guard(c, [&] { cf1::add_fasta(c, path); });
}

int cf1gpu_reset_input(cf1gpu_ctx *c) {
  if (!c) return CF1GPU_ERR_INVALID_ARG;
  c->L = 0;
  c->dev_valid = 0;
  c->ms_intake = 0;
  c->n_records = 0;
  c->n_bases = 0;
  c->short_seqs.clear();
  c->uploaded = false;
  c->ran = false;
  c->x_step = 0;
  return CF1GPU_OK;
}

int cf1gpu_upload(cf1gpu_ctx *c) {
  if (!c) return CF1GPU_ERR_INVALID_ARG;
  return guard(c, [&] { cf1::upload(c); });
}

int cf1gpu_run_resident(cf1gpu_ctx *c) {
  if (!c) return CF1GPU_ERR_INVALID_ARG;
  return guard(c, [&] { cf1::run_resident(c); });
}

int cf1gpu_run_phases_1_4(cf1gpu_ctx *c) {
  if (!c) return CF1GPU_ERR_INVALID_ARG;
  return guard(c, [&] {
    cf1::upload(c);
    cf1::run_resident(c);
  });
}

int cf1gpu_get_stats(const cf1gpu_ctx *c, cf1gpu_stats *out) {
  if (!c || !out) return CF1GPU_ERR_INVALID_ARG;
  *out = c->stats;
  return CF1GPU_OK;
}

uint64_t cf1gpu_total_kmers(const cf1gpu_ctx *c) { return (c && c->ran) ? c->n_distinct : 0; }

int cf1gpu_run_streamed(cf1gpu_ctx *c, const uint8_t *seqs, const uint64_t *offsets, size_t n_records,
                        uint64_t *state_words, size_t words_cap, size_t *n_words) {
  if (!c || !n_words || (n_records && (!seqs || !offsets)) || (words_cap && !state_words))
    return CF1GPU_ERR_INVALID_ARG;
  for (size_t i = 0; i < n_records; i++)
    if (offsets[i + 1] < offsets[i]) return CF1GPU_ERR_INVALID_ARG;
  return guard(c, [&] { *n_words = cf1::run_streamed(c, seqs, offsets, n_records, state_words, words_cap); });
}

int cf1gpu_export_bin(cf1gpu_ctx *c, uint32_t bin, uint8_t *dst, size_t *bytes) {
  if (!c || !bytes) return CF1GPU_ERR_INVALID_ARG;
  if (!c->ran) {
    c->last_error = "no results: run phases 1-4 first";
    return CF1GPU_ERR_STATE;
  }
  if (bin >= c->opts.num_bins) {
    c->last_error = "bin must be below num_bins = " + std::to_string(c->opts.num_bins);
    return CF1GPU_ERR_INVALID_ARG;
  }
  return guard(c, [&] { *bytes = cf1::export_bin(c, bin, dst, dst ? *bytes : 0); });
}

int cf1gpu_bin_distinct_counts(const cf1gpu_ctx *c, uint64_t *counts, size_t nbins) {
  if (!c || (nbins && !counts)) return CF1GPU_ERR_INVALID_ARG;
  cf1gpu_ctx *m = const_cast<cf1gpu_ctx *>(c);
  if (!c->ran) {
    m->last_error = "no results: run phases 1-4 first";
    return CF1GPU_ERR_STATE;
  }
  if (nbins != c->opts.num_bins) {
    m->last_error = "nbins must be num_bins = " + std::to_string(c->opts.num_bins);
    return CF1GPU_ERR_INVALID_ARG;
  }
  return guard(m, [&] {
    std::vector<uint64_t> off(nbins + 1);
    CF1_CUDA(cudaMemcpyAsync(off.data(), c->d_dist_off.p, (nbins + 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                             c->stream));
    CF1_CUDA(cudaStreamSynchronize(c->stream));
    for (size_t b = 0; b < nbins; b++) counts[b] = off[b + 1] - off[b];
  });
}

int cf1gpu_xshard_scan(cf1gpu_ctx *c, uint32_t *hist, uint64_t *n_records) {
  if (!c || !hist || !n_records) return CF1GPU_ERR_INVALID_ARG;
  return guard(c, [&] { cf1::xshard_scan(c, hist, n_records); });
}

int cf1gpu_xshard_route(cf1gpu_ctx *c, const uint32_t *hist, uint64_t *records, size_t records_cap, uint64_t *counts) {
  if (!c || !hist || !counts || (records_cap && !records)) return CF1GPU_ERR_INVALID_ARG;
  return guard(c, [&] { cf1::xshard_route(c, hist, records, records_cap, counts); });
}

int cf1gpu_xshard_finish(cf1gpu_ctx *c, const uint64_t *records, size_t n) {
  if (!c || (n && !records)) return CF1GPU_ERR_INVALID_ARG;
  return guard(c, [&] { cf1::xshard_finish(c, records, n); });
}

int cf1gpu_copy_states(cf1gpu_ctx *c, uint64_t *dst, size_t n_words) {
  if (!c || (!dst && n_words)) return CF1GPU_ERR_INVALID_ARG;
  if (!c->ran) {
    c->last_error = "no results: run phases 1-4 first";
    return CF1GPU_ERR_STATE;
  }
  uint64_t nw = (c->n_distinct + 11) / 12;
  if (n_words != nw) {
    c->last_error = "n_words must be ceil(total_kmers / 12) = " + std::to_string(nw);
    return CF1GPU_ERR_INVALID_ARG;
  }
  return guard(c, [&] {
    if (nw) CF1_CUDA(cudaMemcpyAsync(dst, c->d_states.p, nw * 8, cudaMemcpyDeviceToHost, c->stream));
    CF1_CUDA(cudaStreamSynchronize(c->stream));
  });
}

int cf1gpu_query(cf1gpu_ctx *c, const uint64_t *keys, size_t n, uint64_t *slots) {
  if (!c || (n && (!keys || !slots))) return CF1GPU_ERR_INVALID_ARG;
  if (!c->ran) {
    c->last_error = "no MPHF: run phases 1-4 first";
    return CF1GPU_ERR_STATE;
  }
  return guard(c, [&] { cf1::query(c, keys, n, slots); });
}

int cf1gpu_dump_states(cf1gpu_ctx *c, uint64_t *keys, uint8_t *states, size_t n) {
  if (!c || (n && (!keys || !states))) return CF1GPU_ERR_INVALID_ARG;
  if (!c->ran) {
    c->last_error = "no results: run phases 1-4 first";
    return CF1GPU_ERR_STATE;
  }
  if (n != c->n_distinct) {
    c->last_error = "n must be total_kmers";
    return CF1GPU_ERR_INVALID_ARG;
  }
  return guard(c, [&] { cf1::dump_states(c, keys, states); });
}

int cf1gpu_verify_bijection(cf1gpu_ctx *c) {
  if (!c) return CF1GPU_ERR_INVALID_ARG;
  if (!c->ran) {
    c->last_error = "no MPHF: run phases 1-4 first";
    return CF1GPU_ERR_STATE;
  }
  return guard(c, [&] { cf1::verify_bijection(c); });
}

size_t cf1gpu_short_seq_count(const cf1gpu_ctx *c) { return c ? c->short_seqs.size() : 0; }

int cf1gpu_short_seq(const cf1gpu_ctx *c, size_t i, char *name_buf, size_t name_cap, uint64_t *len) {
  if (!c || i >= c->short_seqs.size()) return CF1GPU_ERR_INVALID_ARG;
  const auto &e = c->short_seqs[i];
  if (len) *len = e.second;
  if (name_buf && name_cap) {
    size_t n = e.first.size() < name_cap - 1 ? e.first.size() : name_cap - 1;
    std::memcpy(name_buf, e.first.data(), n);
    name_buf[n] = 0;
  }
  return CF1GPU_OK;
}

int cf1gpu_export_mphf(cf1gpu_ctx *c, void *dst, size_t *bytes) {
  if (!c || !bytes) return CF1GPU_ERR_INVALID_ARG;
  if (!c->ran) {
    c->last_error = "no MPHF: run phases 1-4 first";
    return CF1GPU_ERR_STATE;
  }
  return guard(c, [&] {
    size_t need = cf1::export_mphf(c, nullptr, 0);
    if (dst) {
      if (*bytes < need) throw cf1::Error(CF1GPU_ERR_INVALID_ARG, "export buffer too small");
      cf1::export_mphf(c, dst, *bytes);
    }
    *bytes = need;
  });
}

int cf1gpu_mphf_host_query(const void *image, size_t bytes, const uint64_t *keys, size_t n, uint64_t *slots) {
  if (!image || (n && (!keys || !slots))) return CF1GPU_ERR_INVALID_ARG;
  try {
    cf1::host_query(image, bytes, keys, n, slots);
    return CF1GPU_OK;
  } catch (const cf1::Error &e) {
    g_create_error = e.what();
    return e.status;
  }
}

int cf1gpu_learned_stats(const cf1gpu_ctx *c, double out5[5]) {
  if (!c || !out5) return CF1GPU_ERR_INVALID_ARG;
  cf1::learned_summary(c, out5);
  return CF1GPU_OK;
}

int cf1gpu_learned_grad_q(int device, const float *q, const float *x, const float *t, size_t n, float *grad_q,
                          float *loss) {
  if (!q || !grad_q || !loss || (n && (!x || !t))) return CF1GPU_ERR_INVALID_ARG;
  try {
    CF1_CUDA(cudaSetDevice(device));
    cf1::learned_grad_q_host(q, x, t, n, grad_q, loss);
    return CF1GPU_OK;
  } catch (const cf1::Error &e) {
    g_create_error = e.what();
    return e.status;
  }
}

int cf1gpu_learned_grad(int device, const float *params, const float *x, const float *t, size_t n, float *grad,
                        float *loss) {
  if (!params || !grad || !loss || (n && (!x || !t))) return CF1GPU_ERR_INVALID_ARG;
  try {
    CF1_CUDA(cudaSetDevice(device));
    cf1::learned_grad_host(params, x, t, n, grad, loss);
    return CF1GPU_OK;
  } catch (const cf1::Error &e) {
    g_create_error = e.what();
    return e.status;
  }
}

const char *cf1gpu_last_error(const cf1gpu_ctx *c) { return c ? c->last_error.c_str() : g_create_error.c_str(); }

void cf1gpu_destroy(cf1gpu_ctx *c) {
  if (!c) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
  for (auto &e : c->ev)
    if (e) cudaEventDestroy(e);
  for (auto &e : c->stage_ev)
    if (e) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  delete c;
}

const char *cf1gpu_version(void) { return "cf1gpu 0.1 sm_100a"; }

}  // extern "C"
