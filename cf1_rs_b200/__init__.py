"""B200 (sm_100a) k-mer state path of cf1-rs, phases 1-4.

Thin ctypes binding of the C ABI in ``include/cf1gpu.h`` (``libcf1gpu.so``,
built in-tree by ``python -m cf1_rs_b200.build``).  There is no CPU fallback:
creating a context without a CUDA device, or importing without the built
library, raises.

    from cf1_rs_b200 import Cf1Gpu
    g = Cf1Gpu(k=31, num_bins=128, mode="bbhash")
    g.add_records(seq_u8, offsets_u64)      # or add_record / add_fasta
    g.run()                                 # phases 1-4 (src/pipeline.rs:76-105)
    words = g.states()                      # AtomicStateVector words
    slots = g.query(canonical_keys)         # Mphf::hash
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcf1gpu.so")
SYNTH_PATH = os.path.join(_HERE, "libcf1synth.so")

OK = 0
ERR_INVALID_ARG, ERR_OOM, ERR_CUDA, ERR_DEVICE_TIMEOUT, ERR_BIJECTION, ERR_QUEUE_OVERRUN, ERR_STATE, ERR_IO, \
    ERR_TOO_LARGE = range(-1, -10, -1)
NOALLOC_MAX_BASES = 1 << 20
MPHF_BBHASH, MPHF_LEARNED = 0, 1


class Cf1Error(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"cf1gpu error {status}: {msg}")
        self.status = status


class Opts(C.Structure):
    _fields_ = [
        ("k", C.c_uint32), ("num_bins", C.c_uint32), ("device", C.c_int32), ("mphf_mode", C.c_uint32),
        ("batched", C.c_uint32), ("track_short_seqs", C.c_uint32), ("tuner_cache_path", C.c_char_p),
        ("learned_max_err", C.c_uint32), ("learned_train_steps", C.c_int32), ("learned_leaf_size", C.c_uint32),
        ("sk_tile", C.c_uint32), ("sort_mode", C.c_uint32), ("state_update", C.c_uint32),
        ("shard_index", C.c_uint32), ("shard_count", C.c_uint32),
    ]


_STAT_U = ["n_bases", "n_records", "n_short", "n_superkmers", "n_kmer_occurrences", "n_distinct", "n_bins",
           "n_state_words", "mphf_bytes", "bbhash_levels", "learned_bins", "fallback_bins", "learned_max_err",
           "classify_cas_retries", "n_kernel_launches", "sort_msd_bits", "tuner_state", "sk_tile", "state_path", "dedup_overflow"]
_STAT_D = ["ms_h2d", "ms_phase1", "ms_phase2", "ms_phase3_sort", "ms_phase3_mphf", "ms_phase4", "ms_total",
           "ms_classify_kernel", "ms_dedup_kernel"]


class Stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in _STAT_U] + \
               [(n, C.c_double) for n in _STAT_D] + [("reserved_d", C.c_double * 3)]


_lib = None
_synth = None

u8p = C.POINTER(C.c_uint8)
u64p = C.POINTER(C.c_uint64)
f32p = C.POINTER(C.c_float)

# Every symbol include/cf1gpu.h declares.
EXPORTED = [
    "cf1gpu_default_opts", "cf1gpu_create", "cf1gpu_add_record", "cf1gpu_add_records", "cf1gpu_add_fasta",
    "cf1gpu_reset_input", "cf1gpu_upload", "cf1gpu_run_resident", "cf1gpu_run_phases_1_4", "cf1gpu_run_streamed",
    "cf1gpu_get_stats",
    "cf1gpu_total_kmers", "cf1gpu_bin_distinct_counts", "cf1gpu_copy_states", "cf1gpu_query", "cf1gpu_dump_states", "cf1gpu_verify_bijection",
    "cf1gpu_short_seq_count", "cf1gpu_short_seq", "cf1gpu_export_mphf", "cf1gpu_export_bin", "cf1gpu_mphf_host_query",
    "cf1gpu_learned_stats", "cf1gpu_learned_grad", "cf1gpu_learned_grad_q", "cf1gpu_last_error", "cf1gpu_destroy", "cf1gpu_version",
    "cf1gpu_distinct_kmers_noalloc", "cf1gpu_xshard_scan", "cf1gpu_xshard_route", "cf1gpu_xshard_finish",
]


def lib():
    """The loaded libcf1gpu.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m cf1_rs_b200.build` "
                          "(the cf1 GPU path has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.cf1gpu_default_opts.argtypes = [C.POINTER(Opts)]
    L.cf1gpu_default_opts.restype = None
    L.cf1gpu_create.argtypes = [C.POINTER(Opts), C.POINTER(vp)]
    L.cf1gpu_add_record.argtypes = [vp, C.c_char_p, C.c_size_t, u8p, C.c_size_t]
    L.cf1gpu_add_records.argtypes = [vp, u8p, u64p, C.c_size_t]
    L.cf1gpu_add_fasta.argtypes = [vp, C.c_char_p]
    for n in ("cf1gpu_reset_input", "cf1gpu_upload", "cf1gpu_run_resident", "cf1gpu_run_phases_1_4",
              "cf1gpu_verify_bijection"):
        getattr(L, n).argtypes = [vp]
    L.cf1gpu_get_stats.argtypes = [vp, C.POINTER(Stats)]
    L.cf1gpu_run_streamed.argtypes = [vp, u8p, u64p, C.c_size_t, u64p, C.c_size_t, C.POINTER(C.c_size_t)]
    L.cf1gpu_total_kmers.argtypes = [vp]
    L.cf1gpu_total_kmers.restype = C.c_uint64
    L.cf1gpu_bin_distinct_counts.argtypes = [vp, u64p, C.c_size_t]
    L.cf1gpu_copy_states.argtypes = [vp, u64p, C.c_size_t]
    L.cf1gpu_query.argtypes = [vp, u64p, C.c_size_t, u64p]
    L.cf1gpu_dump_states.argtypes = [vp, u64p, u8p, C.c_size_t]
    L.cf1gpu_short_seq_count.argtypes = [vp]
    L.cf1gpu_short_seq_count.restype = C.c_size_t
    L.cf1gpu_short_seq.argtypes = [vp, C.c_size_t, C.c_char_p, C.c_size_t, u64p]
    L.cf1gpu_export_mphf.argtypes = [vp, vp, C.POINTER(C.c_size_t)]
    L.cf1gpu_mphf_host_query.argtypes = [vp, C.c_size_t, u64p, C.c_size_t, u64p]
    L.cf1gpu_export_bin.argtypes = [vp, C.c_uint32, u8p, C.POINTER(C.c_size_t)]
    L.cf1gpu_learned_stats.argtypes = [vp, C.POINTER(C.c_double)]
    L.cf1gpu_learned_grad.argtypes = [C.c_int, f32p, f32p, f32p, C.c_size_t, f32p, f32p]
    L.cf1gpu_learned_grad_q.argtypes = [C.c_int, f32p, f32p, f32p, C.c_size_t, f32p, f32p]
    L.cf1gpu_last_error.argtypes = [vp]
    L.cf1gpu_last_error.restype = C.c_char_p
    L.cf1gpu_destroy.argtypes = [vp]
    L.cf1gpu_destroy.restype = None
    L.cf1gpu_version.restype = C.c_char_p
    L.cf1gpu_distinct_kmers_noalloc.argtypes = [C.c_int, C.c_uint32, vp, C.c_size_t, vp, C.c_size_t, vp, vp]
    L.cf1gpu_xshard_scan.argtypes = [vp, vp, u64p]
    L.cf1gpu_xshard_route.argtypes = [vp, vp, vp, C.c_size_t, vp]
    L.cf1gpu_xshard_finish.argtypes = [vp, vp, C.c_size_t]
    _lib = L
    return L


def distinct_kmers_noalloc(d_seq: int, length: int, k: int, d_keys_out: int, out_cap: int, d_n_out: int,
                           stream: int = 0, device: int = 0) -> int:
    """Distinct canonical k-mers of one device-resident record without any
    device allocation by the library (cf1gpu_distinct_kmers_noalloc).  All
    pointers are device addresses the caller owns; returns the status code."""
    return lib().cf1gpu_distinct_kmers_noalloc(device, k, d_seq, length, d_keys_out, out_cap, d_n_out,
                                               stream or None)


def _p(a, t):
    return a.ctypes.data_as(t)


def _addr(a) -> int:
    """Address of a numpy array (host) or a torch tensor (host or device)."""
    return a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data


def learned_grad(params: np.ndarray, x: np.ndarray, t: np.ndarray, device: int = 0):
    """(loss, grad) of a learned-index root MLP, computed on the GPU."""
    params = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    t = np.ascontiguousarray(t, np.float32)
    g = np.zeros(len(params), np.float32)
    loss = C.c_float()
    st = lib().cf1gpu_learned_grad(device, _p(params, f32p), _p(x, f32p), _p(t, f32p), len(x), _p(g, f32p),
                                   C.byref(loss))
    if st != OK:
        raise Cf1Error(st, lib().cf1gpu_last_error(None).decode())
    return float(loss.value), g


def learned_grad_q(q: np.ndarray, x: np.ndarray, t: np.ndarray, device: int = 0):
    """(loss, dL/dq) of one learned-index training step on the GPU: q = knot
    logits[16], output weights[16], output bias (cf1gpu_learned_grad_q)."""
    q = np.ascontiguousarray(q, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    t = np.ascontiguousarray(t, np.float32)
    g = np.zeros(len(q), np.float32)
    loss = C.c_float()
    st = lib().cf1gpu_learned_grad_q(device, _p(q, f32p), _p(x, f32p), _p(t, f32p), len(x), _p(g, f32p),
                                     C.byref(loss))
    if st != OK:
        raise Cf1Error(st, lib().cf1gpu_last_error(None).decode())
    return float(loss.value), g


def host_query(image: np.ndarray, keys: np.ndarray) -> np.ndarray:
    """Mphf::hash on the CPU over an exported image (see Cf1Gpu.export_mphf)."""
    keys = np.ascontiguousarray(keys, np.uint64)
    n = keys.shape[0]
    out = np.empty(n, np.uint64)
    st = lib().cf1gpu_mphf_host_query(image.ctypes.data, image.nbytes, _p(keys, u64p), n, _p(out, u64p))
    if st != OK:
        raise Cf1Error(st, lib().cf1gpu_last_error(None).decode())
    return out


class Cf1Gpu:
    """One phases-1-4 context on one GPU (the C ABI's cf1gpu_ctx)."""

    def __init__(self, k: int = 31, num_bins: int = 128, device: int = 0, mode: str = "bbhash",
                 batched: bool = False, track_short_seqs: bool = False, learned_max_err: int = 0,
                 learned_train_steps: int = 0, learned_leaf_size: int = 0, sk_tile: int = 0,
                 sort_mode: str = "msd", state_update: str = "phase3", shard_index: int = 0,
                 shard_count: int = 1, tuner_cache: str | None = None):
        L = lib()
        o = Opts()
        L.cf1gpu_default_opts(C.byref(o))
        o.k, o.num_bins, o.device = k, num_bins, device
        o.mphf_mode = {"bbhash": MPHF_BBHASH, "learned": MPHF_LEARNED}[mode]
        o.batched = int(batched)
        o.track_short_seqs = int(track_short_seqs)
        o.learned_max_err = learned_max_err
        o.learned_train_steps = learned_train_steps
        o.learned_leaf_size = learned_leaf_size
        o.sk_tile = sk_tile
        o.sort_mode = {"msd": 0, "lsd": 1}[sort_mode]
        o.state_update = {"phase3": 0, "cas": 1, "sideset": 2}[state_update]
        o.shard_index, o.shard_count = shard_index, shard_count
        self._tuner_path = tuner_cache.encode() if tuner_cache else None  # kept alive for the call
        o.tuner_cache_path = self._tuner_path
        h = C.c_void_p()
        st = L.cf1gpu_create(C.byref(o), C.byref(h))
        if st != OK:
            raise Cf1Error(st, L.cf1gpu_last_error(None).decode())
        self.h = h
        self.k = k
        self.num_bins = num_bins
        self.shard_index, self.shard_count = shard_index, max(shard_count, 1)
        self.kw = 1 if k <= 32 else 2

    def _check(self, st):
        if st != OK:
            raise Cf1Error(st, lib().cf1gpu_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            lib().cf1gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- input
    def add_record(self, seq: bytes, name: bytes = b""):
        buf = np.frombuffer(seq, np.uint8) if len(seq) else np.zeros(1, np.uint8)
        self._check(lib().cf1gpu_add_record(self.h, name, len(name), _p(buf, u8p), len(seq)))

    def add_records(self, seq: np.ndarray, offsets: np.ndarray):
        seq = np.ascontiguousarray(seq, np.uint8)
        offsets = np.ascontiguousarray(offsets, np.uint64)
        if seq.size == 0:
            seq = np.zeros(1, np.uint8)
        self._check(lib().cf1gpu_add_records(self.h, _p(seq, u8p), _p(offsets, u64p), len(offsets) - 1))

    def add_fasta(self, path: str):
        self._check(lib().cf1gpu_add_fasta(self.h, path.encode()))

    def reset_input(self):
        self._check(lib().cf1gpu_reset_input(self.h))

    # ---- run
    def upload(self):
        self._check(lib().cf1gpu_upload(self.h))

    def run_resident(self):
        self._check(lib().cf1gpu_run_resident(self.h))

    def run(self):
        self._check(lib().cf1gpu_run_phases_1_4(self.h))

    # ---- results
    def stats(self) -> dict:
        s = Stats()
        self._check(lib().cf1gpu_get_stats(self.h, C.byref(s)))
        return {n: getattr(s, n) for n in _STAT_U + _STAT_D}

    def learned_stats(self) -> dict:
        out = (C.c_double * 5)()
        self._check(lib().cf1gpu_learned_stats(self.h, out))
        return dict(mean_err=out[0], mean_window=out[1], train_loss=out[2], max_err_all=int(out[3]),
                    verify_miss_bins=int(out[4]))

    def total_kmers(self) -> int:
        return int(lib().cf1gpu_total_kmers(self.h))

    def bin_distinct_counts(self) -> np.ndarray:
        """Distinct k-mers of every bin (0 for the bins of other shards)."""
        out = np.empty(self.num_bins, np.uint64)
        self._check(lib().cf1gpu_bin_distinct_counts(self.h, _p(out, u64p), self.num_bins))
        return out

    # ---- exchange-based sharding (cf1gpu_xshard_*): buffers are numpy
    # arrays or torch tensors on the host or on this context's device
    def xshard_scan(self, hist=None):
        """Phase 1 over this shard's share of the input: (the share's 65,536
        bucket histogram, its number of super k-mer records)."""
        if hist is None:
            hist = np.zeros(65536, np.uint32)
        n = C.c_uint64(0)
        self._check(lib().cf1gpu_xshard_scan(self.h, _addr(hist), C.byref(n)))
        return hist, n.value

    def xshard_route(self, hist, n_records: int, records=None, counts=None):
        """The share's records grouped by owner shard, from the summed
        histogram: (records [n_records] u64, counts [shard_count] u64)."""
        if records is None:
            records = np.empty(max(n_records, 1), np.uint64)
        if counts is None:
            counts = np.zeros(max(self.shard_count, 1), np.uint64)
        self._check(lib().cf1gpu_xshard_route(self.h, _addr(hist), _addr(records), n_records, _addr(counts)))
        return records[:n_records], counts

    def xshard_finish(self, records, n: int | None = None):
        """Phases 2-4 on the records this shard received."""
        n = len(records) if n is None else n
        self._check(lib().cf1gpu_xshard_finish(self.h, _addr(records) if n else None, n))

    def run_streamed(self, seq: np.ndarray, offsets: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
        """Input in, state words out, copies overlapped with phases 1 and 4
        (see cf1gpu_run_streamed).  `out` (u64) must hold the words; by
        default it is sized for every k-mer window being distinct."""
        seq = np.ascontiguousarray(seq, np.uint8)
        offsets = np.ascontiguousarray(offsets, np.uint64)
        if seq.size == 0:
            seq = np.zeros(1, np.uint8)
        if out is None:
            out = np.empty(int(offsets[-1]) // 12 + 2 if len(offsets) else 1, np.uint64)
        nw = C.c_size_t(0)
        self._check(lib().cf1gpu_run_streamed(self.h, _p(seq, u8p), _p(offsets, u64p), len(offsets) - 1,
                                              _p(out, u64p), out.size, C.byref(nw)))
        return out[: nw.value]

    def states(self, out: np.ndarray | None = None) -> np.ndarray:
        nw = (self.total_kmers() + 11) // 12
        if out is None:
            out = np.empty(nw, np.uint64)
        self._check(lib().cf1gpu_copy_states(self.h, _p(out, u64p), nw))
        return out

    def dump_states(self):
        n = self.total_kmers()
        keys = np.empty(n * self.kw, np.uint64)
        st = np.empty(n, np.uint8)
        self._check(lib().cf1gpu_dump_states(self.h, _p(keys, u64p), _p(st, u8p), n))
        return (keys if self.kw == 1 else keys.reshape(n, 2)), st

    def query(self, keys: np.ndarray) -> np.ndarray:
        keys = np.ascontiguousarray(keys, np.uint64)
        n = keys.shape[0]
        out = np.empty(n, np.uint64)
        self._check(lib().cf1gpu_query(self.h, _p(keys, u64p), n, _p(out, u64p)))
        return out

    def verify_bijection(self):
        self._check(lib().cf1gpu_verify_bijection(self.h))

    def short_seqs(self):
        n = lib().cf1gpu_short_seq_count(self.h)
        out = []
        buf = C.create_string_buffer(4096)
        ln = C.c_uint64()
        for i in range(n):
            self._check(lib().cf1gpu_short_seq(self.h, i, buf, 4096, C.byref(ln)))
            out.append((buf.value.decode(), ln.value))
        return out

    def export_bin(self, b: int) -> bytes:
        """Bin b's super k-mers in the reference's on-disk bin record format."""
        need = C.c_size_t(0)
        self._check(lib().cf1gpu_export_bin(self.h, b, None, C.byref(need)))
        buf = np.empty(max(1, need.value), np.uint8)
        size = C.c_size_t(need.value)
        self._check(lib().cf1gpu_export_bin(self.h, b, _p(buf, u8p), C.byref(size)))
        return buf[: size.value].tobytes()

    def write_bin_files(self, work_dir: str) -> None:
        """cf1_bin_%05d.bin for every bin, as route_superkmers names them."""
        for b in range(self.num_bins):
            with open(os.path.join(work_dir, f"cf1_bin_{b:05d}.bin"), "wb") as f:
                f.write(self.export_bin(b))

    def mphf_image_bytes(self) -> int:
        """Size of the host image export_mphf would copy."""
        need = C.c_size_t(0)
        self._check(lib().cf1gpu_export_mphf(self.h, None, C.byref(need)))
        return int(need.value)

    def export_mphf(self) -> np.ndarray:
        need = C.c_size_t(0)
        self._check(lib().cf1gpu_export_mphf(self.h, None, C.byref(need)))
        raw = np.empty((need.value + 31) // 8, np.uint64)
        skip = (-raw.ctypes.data % 16) // 8  # the image is 16-byte aligned
        img = raw[skip:skip + (need.value + 7) // 8]
        size = C.c_size_t(img.nbytes)
        self._check(lib().cf1gpu_export_mphf(self.h, img.ctypes.data, C.byref(size)))
        return img


# ---------------------------------------------------------------- synthetic inputs
def _synth_lib():
    global _synth
    if _synth is None:
        if not os.path.exists(SYNTH_PATH):
            raise ImportError(f"{SYNTH_PATH} is missing: build it with `python -m cf1_rs_b200.build`")
        S = C.CDLL(SYNTH_PATH)
        S.cf1synth_generate.restype = C.c_void_p
        S.cf1synth_generate.argtypes = [C.c_int, C.c_double, C.c_uint64, C.c_int]
        for n in ("cf1synth_len", "cf1synth_nrec"):
            getattr(S, n).restype = C.c_uint64
            getattr(S, n).argtypes = [C.c_void_p]
        S.cf1synth_seq.restype = C.c_void_p
        S.cf1synth_seq.argtypes = [C.c_void_p]
        S.cf1synth_offsets.restype = C.c_void_p
        S.cf1synth_offsets.argtypes = [C.c_void_p]
        S.cf1synth_name.restype = C.c_size_t
        S.cf1synth_name.argtypes = [C.c_void_p, C.c_uint64, C.c_char_p, C.c_size_t]
        S.cf1synth_write_fasta.argtypes = [C.c_void_p, C.c_char_p]
        S.cf1synth_free.argtypes = [C.c_void_p]
        _synth = S
    return _synth


class SynthInput:
    """A seeded synthetic workload (1-5, see csrc/cf1_synth.cpp) held in host memory."""

    def __init__(self, config: int, scale: float = 1.0, seed: int = 0, nthreads: int = 0):
        S = _synth_lib()
        self.h = S.cf1synth_generate(config, scale, seed, nthreads or (os.cpu_count() or 1))
        if not self.h:
            raise ValueError(f"unknown synthetic workload {config}")
        n = S.cf1synth_len(self.h)
        r = S.cf1synth_nrec(self.h)
        self.seq = np.ctypeslib.as_array(C.cast(S.cf1synth_seq(self.h), u8p), shape=(max(n, 1),))[:n]
        self.offsets = np.ctypeslib.as_array(C.cast(S.cf1synth_offsets(self.h), u64p), shape=(r + 1,))
        self.config, self.scale = config, scale

    @property
    def n_records(self) -> int:
        return len(self.offsets) - 1

    def name(self, i: int) -> str:
        buf = C.create_string_buffer(256)
        _synth_lib().cf1synth_name(self.h, i, buf, 256)
        return buf.value.decode()

    def write_fasta(self, path: str):
        if _synth_lib().cf1synth_write_fasta(self.h, path.encode()) != 0:
            raise OSError(f"cannot write {path}")

    def __del__(self):
        if getattr(self, "h", None):
            _synth_lib().cf1synth_free(self.h)
            self.h = None
