/*
 * cf1gpu.h -- C ABI of the B200 (sm_100a) k-mer state path of cf1-rs
 * (phases 1-4: minimizer histogram, super k-mer routing into bins, per-bin
 * dedup + minimal perfect hash, DFA vertex classification into the packed
 * 5-bit state vector).
 *
 * All paths cited below are files of the cf1-rs reference crate.
 *
 * The seam this replaces is `run_pipeline::<K>` (src/pipeline.rs:66-118),
 * lines 76-105: count_minimizer_histogram (src/minimizer.rs:27-98),
 * partition_minimizers (src/minimizer.rs:116-144), route_superkmers
 * (src/superkmer.rs:21-101), Mphf::<K>::build (src/mphf.rs:32-43),
 * AtomicStateVector::new (src/state_vector.rs:17-26) and classify_vertices
 * (src/classify.rs:524-601).  What phase 5 (src/output.rs) needs afterwards is
 * (1) Mphf::hash / bucket_id / total_kmers (src/mphf.rs:268-280), served here
 * by cf1gpu_query on the device and by cf1gpu_export_mphf +
 * cf1gpu_mphf_host_query on the host; (2) the AtomicStateVector words in the
 * reference bit layout (12 five-bit states per u64, LSB first,
 * src/state_vector.rs:36-70), served by cf1gpu_copy_states; (3) the
 * short-sequence list (src/classify.rs:550-561), served by
 * cf1gpu_short_seq_count / cf1gpu_short_seq.
 *
 * Ownership: the context owns all device memory and pinned staging buffers.
 * Output buffers are caller-allocated.  Input bytes are copied during the
 * call, so the caller may free them on return.  Keys of k > 32 pass as
 * (lo, hi) u64 pairs, the order of KmerBits::word(.., 0/1)
 * (src/kmer.rs:426-432); keys of k <= 32 pass as one u64.
 *
 * Errors: every int-returning call returns CF1GPU_OK (0) or a negative
 * status; cf1gpu_last_error gives the message.  No call aborts the process
 * or traps the device.  A context is not thread-safe for mutation; after a
 * run, cf1gpu_query / cf1gpu_copy_states may be called from one thread at a
 * time, and exported MPHF images are immutable and may be queried from any
 * number of host threads.
 */
#ifndef CF1GPU_H
#define CF1GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CF1GPU_OK 0
#define CF1GPU_ERR_INVALID_ARG (-1)   /* bad k, bins, null pointer, size mismatch */
#define CF1GPU_ERR_OOM (-2)           /* device or pinned host allocation failed */
#define CF1GPU_ERR_CUDA (-3)          /* a CUDA runtime call failed */
#define CF1GPU_ERR_DEVICE_TIMEOUT (-4) /* a bounded device wait gave up */
#define CF1GPU_ERR_BIJECTION (-5)     /* MPHF is not a bijection onto [0, n) */
#define CF1GPU_ERR_QUEUE_OVERRUN (-6) /* a device work queue or buffer overflowed */
#define CF1GPU_ERR_STATE (-7)         /* call made in the wrong order */
#define CF1GPU_ERR_IO (-8)            /* input file could not be read */
#define CF1GPU_ERR_TOO_LARGE (-9)     /* input exceeds a fixed-capacity entry point's limit */

/* MPHF backends (the reference uses ph::fmph, src/mphf.rs:16). */
#define CF1GPU_MPHF_BBHASH 0   /* per-bin GPU BBHash (gamma 2) */
#define CF1GPU_MPHF_LEARNED 1  /* per-bin learned index, BBHash fallback */

typedef struct cf1gpu_ctx cf1gpu_ctx;

typedef struct cf1gpu_opts {
  uint32_t k;                 /* odd, 1..63 (src/params.rs:167-170) */
  uint32_t num_bins;          /* --num-bins (src/params.rs:58-59), 1..4096 */
  int32_t device;             /* CUDA device ordinal */
  uint32_t mphf_mode;         /* CF1GPU_MPHF_* */
  uint32_t batched;           /* 1: persistent work-queue kernels (one full-occupancy wave per phase kernel
                                 pulling fixed-size chunks from an atomic queue) */
  uint32_t track_short_seqs;  /* --track-short-seqs (src/params.rs:45-47) */
  const char *tuner_cache_path; /* autotuner cache file, NULL = built-in defaults.  With a path, the first run
                                 of each (k <= 32 or not, sorted bins or not, batched or not, log2 input
                                 bases) measures the phase-1 tile (1024/2048/4096, unless sk_tile is set)
                                 and the phase-3 MSD split width (-1..+2 bits), keeps the fastest and
                                 writes them to the file; later runs and contexts read them back */
  uint32_t learned_max_err;   /* learned index: per-bin error bound above which the bin falls back to BBHash (0 = default 1024) */
  int32_t learned_train_steps; /* learned index root training steps: 0 = default (300), < 0 = no training (identity root) */
  uint32_t learned_leaf_size; /* learned index target keys per leaf (0 = default 32) */
  uint32_t sk_tile;           /* k-mer positions per minimizer tile: 1024, 2048 or 4096 (0 = tuner / default) */
  uint32_t sort_mode;         /* phase-3 sort: 0 = per-bin MSD + shared-memory sort (LSD when a sub-bucket
                                 overflows), 1 = segmented LSD radix sort only */
  uint32_t state_update;      /* how the vertex states are formed, all giving the same words:
                                 0 = each k-mer occurrence's side-set byte travels with its key through the
                                 phase-3 sort, whose dedup ORs a vertex's occurrences together; phase 4 then
                                 puts each distinct key's byte in its slot and packs the words (with the LSD
                                 sort, which carries no bytes, phase 4 falls back to mode 2);
                                 1 = phase 4 classifies every occurrence with an atomicCAS loop on the
                                 packed words (src/state_vector.rs:47-70);
                                 2 = phase 4 classifies every occurrence into side-set bytes by atomic OR,
                                 then packs them */
  uint32_t shard_index;       /* bin sharding over shard_count devices: this context keeps the bins b with
                                 b % shard_count == shard_index for phases 3-4 (phases 1-2 still route the
                                 whole input, so every shard sees the same partition); slots, states and
                                 total_kmers are then those of its own bins */
  uint32_t shard_count;       /* 0 or 1 = no sharding */
} cf1gpu_opts;

typedef struct cf1gpu_stats {
  uint64_t n_bases;            /* bases added (all records) */
  uint64_t n_records;          /* records added */
  uint64_t n_short;            /* records shorter than k */
  uint64_t n_superkmers;       /* phase-1/2 super k-mers */
  uint64_t n_kmer_occurrences; /* valid k-mer windows */
  uint64_t n_distinct;         /* distinct canonical k-mers (Mphf::total_kmers) */
  uint64_t n_bins;             /* bins after partitioning (src/minimizer.rs:137-141) */
  uint64_t n_state_words;      /* ceil(n_distinct / 12) */
  uint64_t mphf_bytes;         /* device bytes of the MPHF */
  uint64_t bbhash_levels;      /* deepest BBHash level used */
  uint64_t learned_bins;       /* bins served by the learned index */
  uint64_t fallback_bins;      /* bins served by BBHash in learned mode */
  uint64_t learned_max_err;    /* largest leaf error bound among learned bins */
  uint64_t classify_cas_retries; /* failed CAS attempts in phase 4 */
  uint64_t n_kernel_launches;  /* kernels this library launched during the last run */
  uint64_t sort_msd_bits;      /* top bits the MSD sort split bins on; UINT64_MAX when the LSD path ran */
  uint64_t tuner_state;        /* 0 no autotuner, 1 parameters from the cache, 2 measured in this run */
  uint64_t sk_tile;            /* phase-1 tile this run used */
  uint64_t state_path;         /* how the last run formed the states: 0 joined in phase 3, 1 CAS classification,
                                  2 side-set classification (state_update, or 2 when the LSD sort ran) */
  uint64_t dedup_overflow;     /* sub-buckets the warp dedup left to the block kernel (BBHash form) */
  double ms_h2d;               /* host->device copy of the input */
  double ms_phase1;            /* pack + minimizer histogram + partition */
  double ms_phase2;            /* super k-mer routing */
  double ms_phase3_sort;       /* k-mer expansion + per-bin sort + unique */
  double ms_phase3_mphf;       /* MPHF construction (+ bijection check) */
  double ms_phase4;            /* classification */
  double ms_total;             /* device time of phases 1-4 (excludes h2d) */
  double ms_classify_kernel;   /* the phase-4 kernel alone: classification, or the placing of joined side sets */
  double ms_dedup_kernel;      /* the phase-3 shared-memory sort / dedup kernel alone (0 when the LSD path ran) */
  double reserved_d[3];
} cf1gpu_stats;

/* Fills defaults: k 31, 128 bins, device 0, BBHash, not batched. */
void cf1gpu_default_opts(cf1gpu_opts *opts);

/* Params::from_resolved checks (src/params.rs:154-197) + device set-up. */
int cf1gpu_create(const cf1gpu_opts *opts, cf1gpu_ctx **out);

/* One input record in input order (the host parses FASTA/FASTQ, as needletail
 * does at src/classify.rs:541-546).  `name` may be NULL; its first
 * whitespace-delimited token is kept for short-sequence tracking. */
int cf1gpu_add_record(cf1gpu_ctx *ctx, const char *name, size_t name_len, const uint8_t *seq, size_t len);

/* Many records at once: record i is seqs[offsets[i] .. offsets[i+1]). */
int cf1gpu_add_records(cf1gpu_ctx *ctx, const uint8_t *seqs, const uint64_t *offsets, size_t n_records);

/* Reads every record of a FASTA/FASTQ file (plain or gzip). */
int cf1gpu_add_fasta(cf1gpu_ctx *ctx, const char *path);

/* Drops all added records and results (keeps device buffers for reuse). */
int cf1gpu_reset_input(cf1gpu_ctx *ctx);

/* Copies the added records to the device (part of cf1gpu_run_phases_1_4). */
int cf1gpu_upload(cf1gpu_ctx *ctx);

/* Phases 1-4 over the records already on the device (no host copies). */
int cf1gpu_run_resident(cf1gpu_ctx *ctx);

/* cf1gpu_upload + cf1gpu_run_resident: pipeline.rs:76-105 in one call. */
int cf1gpu_run_phases_1_4(cf1gpu_ctx *ctx);

/* cf1gpu_reset_input + cf1gpu_add_records + cf1gpu_run_phases_1_4 +
 * cf1gpu_copy_states in one call, with the copies overlapped: the record
 * bytes go to the device in chunks while phase 1 scans the part already
 * there, and phase 4 runs in stages of whole bins while the state words of
 * finished stages come back.  Give seqs and state_words in page-locked host
 * memory (cudaHostAlloc / cudaHostRegister) for the overlap; pageable buffers
 * work, with the copies in series.  words_cap is state_words' size in words;
 * *n_words receives ceil(total_kmers / 12).  A buffer too small is an error
 * after the run (the results stay on the device for cf1gpu_copy_states). */
int cf1gpu_run_streamed(cf1gpu_ctx *ctx, const uint8_t *seqs, const uint64_t *offsets, size_t n_records,
                        uint64_t *state_words, size_t words_cap, size_t *n_words);

int cf1gpu_get_stats(const cf1gpu_ctx *ctx, cf1gpu_stats *out);

/* Mphf::total_kmers (src/mphf.rs:278-280). */
uint64_t cf1gpu_total_kmers(const cf1gpu_ctx *ctx);

/* Distinct k-mers of every bin (counts[b], b < nbins = num_bins; 0 for the
 * bins of other shards): bin b owns the slots from the sum of the counts
 * before it.  Across shards these give the global slot offsets -- the one
 * exchange bin sharding needs (no counterpart in the reference, which runs
 * on one host). */
int cf1gpu_bin_distinct_counts(const cf1gpu_ctx *ctx, uint64_t *counts, size_t nbins);

/* Exchange-based bin sharding: the alternative to cf1gpu_run_phases_1_4 for
 * shard_count contexts (one per device) that all hold the whole input.  Each
 * scans only its slice of the input, and the shards swap their super k-mer
 * records once:
 *   1. cf1gpu_xshard_scan: phase 1 over this shard's share of the minimizer
 *      tiles; hist receives the share's 65,536-bucket histogram,
 *      *n_records the share's super k-mer records.
 *   2. caller: sum hist over the shards (an all-reduce).
 *   3. cf1gpu_xshard_route: the partition of the summed histogram (the same on
 *      every shard), then the share's records, each tagged with its bin, into
 *      records[0 .. *n_records) grouped by owner shard (bin % shard_count):
 *      counts[r] records for shard r, r < shard_count.
 *   4. caller: send group r to shard r (an all-to-all).
 *   5. cf1gpu_xshard_finish: phases 2-4 on the n records this shard received,
 *      in any order.  Records of another shard's bin, or reaching past the
 *      input, are refused (CF1GPU_ERR_INVALID_ARG).
 * Afterwards the context holds its bins' results exactly as after a
 * replicated-routing run (cf1gpu_bin_distinct_counts, cf1gpu_copy_states).
 * The reference routes on one host (src/superkmer.rs:21-210); this split of
 * its phase 1-2 work over devices has no counterpart there.  Buffers may be
 * host memory or device memory of the context's device (cudaMemcpyDefault),
 * so an NCCL all-reduce and all-to-all can run on them in place. */
int cf1gpu_xshard_scan(cf1gpu_ctx *ctx, uint32_t *hist, uint64_t *n_records);
int cf1gpu_xshard_route(cf1gpu_ctx *ctx, const uint32_t *hist, uint64_t *records, size_t records_cap,
                        uint64_t *counts);
int cf1gpu_xshard_finish(cf1gpu_ctx *ctx, const uint64_t *records, size_t n);

/* The state vector words (src/state_vector.rs:7-71 layout); n_words must be
 * ceil(total_kmers / 12). */
int cf1gpu_copy_states(cf1gpu_ctx *ctx, uint64_t *dst, size_t n_words);

/* Mphf::hash for a batch of canonical k-mers (src/mphf.rs:268-270): the
 * slot in [0, total_kmers); absent keys give 0, like unwrap_or(0). */
int cf1gpu_query(cf1gpu_ctx *ctx, const uint64_t *keys, size_t n, uint64_t *slots);

/* Every distinct canonical k-mer with its state (for parity checks): keys in
 * storage order (bins in order; each bin sorted in learned mode and with
 * sort_mode 1, otherwise in no particular order), n must be total_kmers. */
int cf1gpu_dump_states(cf1gpu_ctx *ctx, uint64_t *keys, uint8_t *states, size_t n);

/* Verification pass: queries every distinct key on the device and checks that
 * the slots form a bijection onto [0, total_kmers).  0 when they do. */
int cf1gpu_verify_bijection(cf1gpu_ctx *ctx);

/* Short sequences (src/classify.rs:550-561), in input order. */
size_t cf1gpu_short_seq_count(const cf1gpu_ctx *ctx);
int cf1gpu_short_seq(const cf1gpu_ctx *ctx, size_t i, char *name_buf, size_t name_cap, uint64_t *len);

/* Flat host image of the MPHF.  Call with dst NULL to get the size; dst must
 * be 16-byte aligned. */
int cf1gpu_export_mphf(cf1gpu_ctx *ctx, void *dst, size_t *bytes);

/* Bin `bin`'s super k-mers in the reference's on-disk bin record format
 * (src/superkmer.rs:181-202: per super k-mer a little-endian u16 base count,
 * then the bases 2-bit packed four per byte, first base in the top bits --
 * the bytes route_superkmers writes to cf1_bin_%05d.bin, superkmer.rs:224-226,
 * and BinReader::read_packed_superkmer reads, superkmer.rs:283-298).  Super
 * k-mers in this library's routing order.  Call with dst NULL to get the size
 * in *bytes; otherwise *bytes is the buffer's size and receives the size
 * written. */
int cf1gpu_export_bin(cf1gpu_ctx *ctx, uint32_t bin, uint8_t *dst, size_t *bytes);

/* Mphf::hash on the host over an exported image (thread-safe, no device);
 * image must be 16-byte aligned. */
int cf1gpu_mphf_host_query(const void *image, size_t bytes, const uint64_t *keys, size_t n, uint64_t *slots);

/* Learned-index statistics of the last run (learned mode): out5 =
 * {mean leaf error bound and mean search window over the keys of learned
 * bins, mean final training loss over bins, largest leaf error over all
 * bins, bins where verification found a key outside its window}. */
int cf1gpu_learned_stats(const cf1gpu_ctx *ctx, double out5[5]);

/* Diagnostics: full-batch MSE loss and gradient of a learned-index root
 * (1 -> 16 clipped-ReLU clamp(w1 x + b1, 0, 1) -> 1, params = w1[16] b1[16]
 * w2[16] b2) over n samples, computed on `device` by the code the training
 * kernel runs. */
int cf1gpu_learned_grad(int device, const float *params, const float *x, const float *t, size_t n, float *grad,
                        float *loss);

/* Gradient the learned-index trainer applies: dL/dq of one training step for
 * the trained parameters q = knot logits theta[16], output weights w2[16],
 * output bias b2 (33 floats).  The first layer is derived from the knots --
 * widths d = softmax(theta), knots t_j = d_0 + ... + d_{j-1}, w1_j = 1/d_j,
 * b1_j = -t_j/d_j -- so grad_q carries the chain rule through the softmax and
 * the knot sums on top of cf1gpu_learned_grad's dL/dP.  Same loss (mean
 * squared error over the n samples (x_i, t_i)).  Diagnostic: no counterpart in
 * the reference (its MPHF has no trained part, src/mphf.rs:155-160). */
int cf1gpu_learned_grad_q(int device, const float *q, const float *x, const float *t, size_t n, float *grad_q,
                          float *loss);

/* Distinct canonical k-mers of one record, for callers that must not
 * allocate device memory.  No counterpart in the reference (it has no
 * device memory at all): this exists for host applications that own the
 * device memory pool and give the library only their buffers, and for code
 * running where a cudaMalloc would synchronise the device or is not allowed.
 * It allocates nothing: its scratch is a fixed array inside the library
 * (17 MiB, kept by every GPU that loads it until the process exits).
 *
 * d_seq: the record's ASCII bases in device memory, len <= 1048576 (1 Mi)
 * bases -- longer records return CF1GPU_ERR_TOO_LARGE without running.
 * k: odd, 1..31.  d_keys_out: device buffer of out_cap u64, out_cap >=
 * len - k + 1; receives the distinct canonical k-mers of the record's
 * placeholder-free windows, ascending (the phase-3 key set of
 * src/mphf.rs:323-363 for this record).  d_n_out: device u64, their count.
 * Work is queued on `stream` (a cudaStream_t, NULL = the default stream
 * of `device`); a stream must belong to `device` -- the call makes `device`
 * current before launching, and a stream of another device returns
 * CF1GPU_ERR_INVALID_ARG.  Outputs are valid once the stream has run it.
 *
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with the device current; make that first call
 * before any stream capture.  Calls share the array and it keeps the last
 * call's contents (each call clears what it needs): calls that overlap on
 * the GPU race and corrupt each other, so serialise them. */
int cf1gpu_distinct_kmers_noalloc(int device, uint32_t k, const uint8_t *d_seq, size_t len, uint64_t *d_keys_out,
                                  size_t out_cap, uint64_t *d_n_out, void *stream);

const char *cf1gpu_last_error(const cf1gpu_ctx *ctx);
void cf1gpu_destroy(cf1gpu_ctx *ctx);

/* Library build identification (e.g. "sm_100a"). */
const char *cf1gpu_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CF1GPU_H */
