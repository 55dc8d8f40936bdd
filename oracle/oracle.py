"""ctypes wrapper over the CPU oracle (test infrastructure only).

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline / reference arm
of ``bench.py`` import this module.  It restates the cf1-rs phases 1-4
semantics on the CPU (see ``cf1_oracle.cpp`` for the reference citations);
the product library never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libcf1oracle.so")
_lib = None

u8p = C.POINTER(C.c_uint8)
u64p = C.POINTER(C.c_uint64)
u32p = C.POINTER(C.c_uint32)
u16p = C.POINTER(C.c_uint16)


def build() -> None:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.cfo_mapped_base.restype = C.c_uint8
        L.cfo_mapped_base.argtypes = [C.c_uint8]
        L.cfo_is_placeholder.argtypes = [C.c_uint8]
        L.cfo_complement_base.restype = C.c_uint8
        L.cfo_complement_base.argtypes = [C.c_uint8]
        L.cfo_rc_byte.restype = C.c_uint8
        L.cfo_rc_byte.argtypes = [C.c_uint8]
        for name in ("cfo_kmer_reverse_complement", "cfo_kmer_canonical"):
            getattr(L, name).argtypes = [C.c_int, u64p, u64p]
        L.cfo_kmer_from_ascii.argtypes = [C.c_int, C.c_char_p, C.c_uint64, u64p]
        L.cfo_kmer_front.argtypes = [C.c_int, u64p]
        L.cfo_kmer_back.argtypes = [C.c_int, u64p]
        L.cfo_kmer_roll.argtypes = [C.c_int, u64p, u64p, C.c_uint8]
        L.cfo_kmer_label.argtypes = [C.c_int, u64p, C.c_char_p]
        L.cfo_kmer_cmp.argtypes = [C.c_int, u64p, u64p]
        L.cfo_kmer_from_packed_2bit.argtypes = [C.c_int, C.c_char_p, C.c_uint64, u64p]
        L.cfo_kmer_from_packed_2bit_reference_arith.argtypes = [C.c_int, C.c_char_p, C.c_uint64, u64p]
        L.cfo_state_from_vertex.restype = C.c_uint8
        L.cfo_state_from_vertex.argtypes = [C.c_int] * 5
        L.cfo_state_decode.argtypes = [C.c_uint8, C.POINTER(C.c_int)]
        L.cfo_state_class.argtypes = [C.c_uint8]
        L.cfo_state_is_dead_end.argtypes = [C.c_uint8]
        L.cfo_state_outputted.restype = C.c_uint8
        L.cfo_state_outputted.argtypes = [C.c_uint8]
        L.cfo_state_join.restype = C.c_uint8
        L.cfo_state_join.argtypes = [C.c_uint8, C.c_uint8]
        L.cfo_asv_new.restype = C.c_void_p
        L.cfo_asv_new.argtypes = [C.c_uint64]
        L.cfo_asv_free.argtypes = [C.c_void_p]
        L.cfo_asv_get.restype = C.c_uint8
        L.cfo_asv_get.argtypes = [C.c_void_p, C.c_uint64]
        L.cfo_asv_cas.argtypes = [C.c_void_p, C.c_uint64, C.c_uint8, C.c_uint8]
        L.cfo_asv_word.restype = C.c_uint64
        L.cfo_asv_word.argtypes = [C.c_void_p, C.c_uint64]
        L.cfo_asv_num_words.restype = C.c_uint64
        L.cfo_asv_num_words.argtypes = [C.c_void_p]
        L.cfo_run.restype = C.c_void_p
        L.cfo_run.argtypes = [C.c_int, u8p, u64p, C.c_uint64, C.c_int, C.c_int]
        L.cfo_free.argtypes = [C.c_void_p]
        for name in ("cfo_n_distinct", "cfo_n_occ", "cfo_num_state_words", "cfo_n_short"):
            getattr(L, name).restype = C.c_uint64
            getattr(L, name).argtypes = [C.c_void_p]
        L.cfo_copy_keys.argtypes = [C.c_void_p, u64p]
        L.cfo_copy_states.argtypes = [C.c_void_p, u8p]
        L.cfo_copy_state_words.argtypes = [C.c_void_p, u64p]
        L.cfo_copy_short.argtypes = [C.c_void_p, u64p, u64p]
        L.cfo_times.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.cfo_minimizer_len.argtypes = [C.c_int]
        L.cfo_mix_order.restype = C.c_uint32
        L.cfo_mix_order.argtypes = [C.c_uint32]
        L.cfo_mix_bucket.restype = C.c_uint32
        L.cfo_mix_bucket.argtypes = [C.c_uint32]
        L.cfo_superkmers.restype = C.c_uint64
        L.cfo_superkmers.argtypes = [u8p, C.c_uint64, C.c_int, C.c_uint32, u64p, u32p, u32p, C.c_uint64]
        L.cfo_partition.argtypes = [u64p, C.c_uint32, C.c_uint32, u16p, u32p]
        f32p = C.POINTER(C.c_float)
        f64p = C.POINTER(C.c_double)
        L.cfo_mlp_grad.argtypes = [f32p, f32p, f32p, C.c_uint64, f64p, f64p]
        L.cfo_learned_grad_q.argtypes = [f64p, f32p, f32p, C.c_uint64, f64p, f64p]
        L.cfo_learned_loss_q.restype = C.c_double
        L.cfo_learned_loss_q.argtypes = [f64p, f32p, f32p, C.c_uint64]
        L.cfo_part_index_new.restype = C.c_void_p
        L.cfo_part_index_new.argtypes = [C.c_int, u8p, u64p, C.c_uint64, C.c_uint32, C.c_int]
        L.cfo_part_index_free.argtypes = [C.c_void_p]
        L.cfo_part_index_n_occ.restype = C.c_uint64
        L.cfo_part_index_n_occ.argtypes = [C.c_void_p]
        L.cfo_part_index_seconds.restype = C.c_double
        L.cfo_part_index_seconds.argtypes = [C.c_void_p]
        L.cfo_part_run.restype = C.c_void_p
        L.cfo_part_run.argtypes = [C.c_void_p, C.c_uint32, C.c_int]
        L.cfo_part_free.argtypes = [C.c_void_p]
        for name in ("cfo_part_n_distinct", "cfo_part_n_occ"):
            getattr(L, name).restype = C.c_uint64
            getattr(L, name).argtypes = [C.c_void_p]
        L.cfo_part_times.argtypes = [C.c_void_p, f64p]
        L.cfo_part_copy.argtypes = [C.c_void_p, u64p, u8p]
        L.cfo_list_parts.argtypes = [u64p, C.c_uint64, C.c_int, C.c_uint32, C.c_int, u8p]
        L.cfo_part_compare.argtypes = [C.c_void_p, u64p, u8p, u8p, C.c_uint64, C.c_int, u64p]
        L.cfo_part_of.restype = C.c_uint32
        L.cfo_part_of.argtypes = [u64p, C.c_uint32]
        _lib = L
    return _lib


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(t)


# ---------------------------------------------------------------- k-mer ops
class Kmer:
    """A k-mer as the reference stores it: an integer, first base in the MSBs."""

    def __init__(self, k: int, value: int):
        self.k = k
        self.value = value

    def _arr(self):
        return (C.c_uint64 * 2)(self.value & (2**64 - 1), self.value >> 64)

    @staticmethod
    def _from(k, arr):
        return Kmer(k, int(arr[0]) | (int(arr[1]) << 64))

    @staticmethod
    def from_ascii(k: int, seq: bytes, offset: int = 0) -> "Kmer":
        out = (C.c_uint64 * 2)()
        lib().cfo_kmer_from_ascii(k, seq, offset, out)
        return Kmer._from(k, out)

    @staticmethod
    def from_packed_2bit(k: int, packed: bytes, offset: int, reference_arith: bool = False) -> "Kmer":
        out = (C.c_uint64 * 2)()
        fn = lib().cfo_kmer_from_packed_2bit_reference_arith if reference_arith else lib().cfo_kmer_from_packed_2bit
        fn(k, packed, offset, out)
        return Kmer._from(k, out)

    def reverse_complement(self) -> "Kmer":
        out = (C.c_uint64 * 2)()
        lib().cfo_kmer_reverse_complement(self.k, self._arr(), out)
        return Kmer._from(self.k, out)

    def canonical(self) -> "Kmer":
        out = (C.c_uint64 * 2)()
        lib().cfo_kmer_canonical(self.k, self._arr(), out)
        return Kmer._from(self.k, out)

    def front(self) -> int:
        return lib().cfo_kmer_front(self.k, self._arr())

    def back(self) -> int:
        return lib().cfo_kmer_back(self.k, self._arr())

    def label(self) -> str:
        buf = C.create_string_buffer(self.k + 1)
        lib().cfo_kmer_label(self.k, self._arr(), buf)
        return buf.value.decode()

    def __eq__(self, o):
        return self.k == o.k and self.value == o.value

    def __lt__(self, o):
        return lib().cfo_kmer_cmp(self.k, self._arr(), o._arr()) < 0


def roll(kmer: Kmer, rc: Kmer, base: int):
    a, b = kmer._arr(), rc._arr()
    lib().cfo_kmer_roll(kmer.k, a, b, base)
    return Kmer._from(kmer.k, a), Kmer._from(kmer.k, b)


# ---------------------------------------------------------------- states
SISO, MISO, SIMO, MIMO = 0, 1, 2, 3


def state_from_vertex(cls, front=0, back=0, visited=True, outputted=False) -> int:
    return lib().cfo_state_from_vertex(cls, front, back, int(visited), int(outputted))


def state_decode(code: int):
    out = (C.c_int * 5)()
    lib().cfo_state_decode(code, out)
    return dict(cls=out[0], front=out[1], back=out[2], visited=bool(out[3]), outputted=bool(out[4]))


class StateVector:
    """The reference's 12-per-u64 atomic state vector (src/state_vector.rs)."""

    def __init__(self, n: int):
        self.h = lib().cfo_asv_new(n)

    def __del__(self):
        if getattr(self, "h", None):
            lib().cfo_asv_free(self.h)

    def get(self, i):
        return lib().cfo_asv_get(self.h, i)

    def compare_and_swap(self, i, expected, new):
        return bool(lib().cfo_asv_cas(self.h, i, expected, new))

    def words(self):
        n = lib().cfo_asv_num_words(self.h)
        return [lib().cfo_asv_word(self.h, w) for w in range(n)]


# ---------------------------------------------------------------- pipeline
class OracleResult:
    def __init__(self, k, keys, states, state_words, short_idx, short_len, n_occ, times):
        self.k = k
        self.keys = keys          # uint64 [n] (k<=32) or [n,2] (lo, hi), sorted
        self.states = states      # uint8 [n]
        self.state_words = state_words
        self.short_idx = short_idx
        self.short_len = short_len
        self.n_occ = n_occ
        self.times = times        # (collect, sort, classify) seconds


def run(k: int, seq: np.ndarray, rec_off: np.ndarray, nthreads: int = 1, method: int = 0) -> OracleResult:
    """Phases 1-4 on the CPU. method 0 = classify.rs restatement, 1 = side-join fold."""
    seq = np.ascontiguousarray(seq, dtype=np.uint8)
    rec_off = np.ascontiguousarray(rec_off, dtype=np.uint64)
    L = lib()
    h = L.cfo_run(k, _p(seq, u8p), _p(rec_off, u64p), len(rec_off) - 1, nthreads, method)
    if not h:
        raise ValueError(f"k must be odd and in [1, 63], got {k}")
    try:
        n = L.cfo_n_distinct(h)
        kw = 1 if k <= 32 else 2
        keys = np.empty(n * kw, dtype=np.uint64)
        L.cfo_copy_keys(h, _p(keys, u64p))
        if kw == 2:
            keys = keys.reshape(n, 2)
        states = np.empty(n, dtype=np.uint8)
        L.cfo_copy_states(h, _p(states, u8p))
        nw = L.cfo_num_state_words(h)
        words = np.empty(nw, dtype=np.uint64)
        L.cfo_copy_state_words(h, _p(words, u64p))
        ns = L.cfo_n_short(h)
        si = np.empty(ns, dtype=np.uint64)
        sl = np.empty(ns, dtype=np.uint64)
        L.cfo_copy_short(h, _p(si, u64p), _p(sl, u64p))
        t = (C.c_double * 3)()
        L.cfo_times(h, t)
        return OracleResult(k, keys, states, words, si, sl, L.cfo_n_occ(h), tuple(t))
    finally:
        L.cfo_free(h)


# ---------------------------------------------------------------- partitioned run
class PartIndex:
    """Partition (part_of) of the canonical k-mer of every window of an input,
    for classify.rs restatements that run one hash partition at a time
    (cfo_part_index_new): inputs whose distinct k-mers do not fit in memory
    at once.  Keeps references to the input arrays while it lives."""

    def __init__(self, k: int, seq: np.ndarray, rec_off: np.ndarray, nparts: int, nthreads: int = 1):
        self.k, self.nparts = k, nparts
        self._seq = np.ascontiguousarray(seq, dtype=np.uint8)
        self._off = np.ascontiguousarray(rec_off, dtype=np.uint64)
        self.h = lib().cfo_part_index_new(k, _p(self._seq, u8p), _p(self._off, u64p), len(self._off) - 1, nparts,
                                          nthreads)
        if not self.h:
            raise ValueError(f"bad k ({k}) or partition count ({nparts})")

    def close(self):
        if getattr(self, "h", None):
            lib().cfo_part_index_free(self.h)
            self.h = None

    __del__ = close

    @property
    def n_occ(self) -> int:
        return lib().cfo_part_index_n_occ(self.h)

    @property
    def seconds(self) -> float:
        return lib().cfo_part_index_seconds(self.h)


class PartResult:
    """Per-k-mer states of one hash partition (cfo_part_run): the classify.rs
    step applied to every window whose canonical k-mer is in the partition.
    The union over all partitions equals run(method=0)."""

    def __init__(self, index: PartIndex, part: int, nthreads: int = 1):
        self.k, self.part, self.nparts = index.k, part, index.nparts
        self.h = lib().cfo_part_run(index.h, part, nthreads)
        if not self.h:
            raise ValueError(f"bad partition {part} of {index.nparts}")

    def close(self):
        if getattr(self, "h", None):
            lib().cfo_part_free(self.h)
            self.h = None

    __del__ = close

    @property
    def n_distinct(self) -> int:
        return lib().cfo_part_n_distinct(self.h)

    @property
    def n_occ(self) -> int:
        return lib().cfo_part_n_occ(self.h)

    @property
    def times(self):
        t = (C.c_double * 3)()
        lib().cfo_part_times(self.h, t)
        return tuple(t)

    def keys_states(self):
        n = self.n_distinct
        kw = 1 if self.k <= 32 else 2
        keys = np.empty(n * kw, dtype=np.uint64)
        st = np.empty(n, dtype=np.uint8)
        lib().cfo_part_copy(self.h, _p(keys, u64p), _p(st, u8p))
        return (keys if kw == 1 else keys.reshape(n, 2)), st

    def compare(self, keys: np.ndarray, states: np.ndarray, ids: np.ndarray, nthreads: int = 1) -> dict:
        """Lines a (key, state) list (any order; ids = list_parts of its keys)
        up with this partition."""
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        states = np.ascontiguousarray(states, dtype=np.uint8)
        ids = np.ascontiguousarray(ids, dtype=np.uint8)
        out = np.zeros(10, dtype=np.uint64)
        lib().cfo_part_compare(self.h, _p(keys, u64p), _p(states, u8p), _p(ids, u8p), len(states), nthreads,
                               _p(out, u64p))
        none = 2**64 - 1
        first = None
        if int(out[6]) != none or int(out[7]) != none:
            first = {"key": int(out[6]) | (int(out[7]) << 64), "state": int(out[8]),
                     "oracle_state": None if int(out[9]) == none else int(out[9])}
        return {"in_part": int(out[0]), "equal": int(out[1]), "state_diff": int(out[2]), "extra": int(out[3]),
                "dup": int(out[4]), "missing": int(out[5]), "first": first}


def list_parts(keys: np.ndarray, k: int, nparts: int, nthreads: int = 1) -> np.ndarray:
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    n = keys.shape[0]
    ids = np.empty(n, dtype=np.uint8)
    lib().cfo_list_parts(_p(keys, u64p), n, k, nparts, nthreads, _p(ids, u8p))
    return ids


def part_of(key: int, nparts: int) -> int:
    arr = (C.c_uint64 * 2)(key & (2**64 - 1), key >> 64)
    return lib().cfo_part_of(arr, nparts)


def check_lists(k: int, seq: np.ndarray, rec_off: np.ndarray, lists: dict, nparts: int = 8, nthreads: int = 1,
                log=None) -> dict:
    """Full check of (canonical k-mer, state) lists -- {name: (keys, states)},
    each in any order -- against the classify.rs restatement, run one hash
    partition at a time.  Per list, mismatches counts differing states,
    listed keys the oracle lacks, keys listed twice and oracle keys the list
    lacks."""
    import time
    t0 = time.perf_counter()
    names = list(lists)
    tot = {n: {"in_part": 0, "equal": 0, "state_diff": 0, "extra": 0, "dup": 0, "missing": 0} for n in names}
    first = {n: None for n in names}
    ids = {n: list_parts(lists[n][0], k, nparts, nthreads) for n in names}
    n_dist = n_occ = 0
    index = PartIndex(k, seq, rec_off, nparts, nthreads)
    try:
        for p in range(nparts):
            r = PartResult(index, p, nthreads)
            try:
                n_dist += r.n_distinct
                n_occ += r.n_occ
                for n in names:
                    c = r.compare(lists[n][0], lists[n][1], ids[n], nthreads)
                    for key in tot[n]:
                        tot[n][key] += c[key]
                    if first[n] is None and c["first"] is not None:
                        first[n] = c["first"]
                if log:
                    log(f"partition {p + 1}/{nparts}: {r.n_distinct} distinct, "
                        f"collect/sort/classify {[round(t, 1) for t in r.times]} s")
            finally:
                r.close()
    finally:
        index.close()
    out = {"checked": True, "method": "classify.rs restatement, hash-partitioned", "nparts": nparts,
           "n_distinct": n_dist, "n_occ": n_occ, "seconds": round(time.perf_counter() - t0, 1),
           "threads": nthreads, "lists": {}}
    for n in names:
        t = tot[n]
        out["lists"][n] = {"n_listed": int(len(lists[n][1])),
                           "mismatches": t["state_diff"] + t["extra"] + t["dup"] + t["missing"],
                           **{key: t[key] for key in ("state_diff", "extra", "dup", "missing")},
                           "first_mismatch": first[n]}
    return out


def check_states(k: int, seq: np.ndarray, rec_off: np.ndarray, keys: np.ndarray, states: np.ndarray,
                 nparts: int = 8, nthreads: int = 1, log=None) -> dict:
    """check_lists for one list: the result's counts at the top level."""
    r = check_lists(k, seq, rec_off, {"list": (keys, states)}, nparts, nthreads, log)
    one = r.pop("lists")["list"]
    r.update(one)
    return r


# ---------------------------------------------------------------- binning spec
def minimizer_len(k: int) -> int:
    return lib().cfo_minimizer_len(k)


def superkmers(seq: np.ndarray, k: int, tile: int):
    """Super k-mers (pos, n_kmers, bucket) of the concatenated sequence."""
    seq = np.ascontiguousarray(seq, dtype=np.uint8)
    L = lib()
    cap = max(1, len(seq))
    pos = np.empty(cap, dtype=np.uint64)
    n = np.empty(cap, dtype=np.uint32)
    b = np.empty(cap, dtype=np.uint32)
    cnt = L.cfo_superkmers(_p(seq, u8p), len(seq), k, tile, _p(pos, u64p), _p(n, u32p), _p(b, u32p), cap)
    return pos[:cnt], n[:cnt], b[:cnt]


def partition(hist: np.ndarray, num_bins: int):
    hist = np.ascontiguousarray(hist, dtype=np.uint64)
    lut = np.empty(len(hist), dtype=np.uint16)
    nb = C.c_uint32()
    lib().cfo_partition(_p(hist, u64p), len(hist), num_bins, _p(lut, u16p), C.byref(nb))
    return lut, nb.value


def mlp_grad(params: np.ndarray, x: np.ndarray, t: np.ndarray):
    """(loss, grad) of the learned-index root MLP in double precision."""
    params = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    t = np.ascontiguousarray(t, np.float32)
    g = np.zeros(len(params), np.float64)
    loss = C.c_double()
    lib().cfo_mlp_grad(_p(params, C.POINTER(C.c_float)), _p(x, C.POINTER(C.c_float)), _p(t, C.POINTER(C.c_float)),
                       len(x), _p(g, C.POINTER(C.c_double)), C.byref(loss))
    return loss.value, g


def learned_grad_q(q: np.ndarray, x: np.ndarray, t: np.ndarray):
    """(loss, dL/dq) of the learned-index root in its trained
    parameterisation (knot logits, output weights, output bias), in double
    precision."""
    q = np.ascontiguousarray(q, np.float64)
    x = np.ascontiguousarray(x, np.float32)
    t = np.ascontiguousarray(t, np.float32)
    g = np.zeros(len(q), np.float64)
    loss = C.c_double()
    lib().cfo_learned_grad_q(_p(q, C.POINTER(C.c_double)), _p(x, C.POINTER(C.c_float)), _p(t, C.POINTER(C.c_float)),
                             len(x), _p(g, C.POINTER(C.c_double)), C.byref(loss))
    return loss.value, g


def learned_loss_q(q: np.ndarray, x: np.ndarray, t: np.ndarray) -> float:
    q = np.ascontiguousarray(q, np.float64)
    x = np.ascontiguousarray(x, np.float32)
    t = np.ascontiguousarray(t, np.float32)
    return lib().cfo_learned_loss_q(_p(q, C.POINTER(C.c_double)), _p(x, C.POINTER(C.c_float)),
                                    _p(t, C.POINTER(C.c_float)), len(x))


def concat_records(records, sep: bytes = b"N"):
    """Concatenate records into one buffer with offsets (records are bytes)."""
    off = np.zeros(len(records) + 1, dtype=np.uint64)
    total = 0
    for i, r in enumerate(records):
        total += len(r)
        off[i + 1] = total
    buf = np.frombuffer(b"".join(records), dtype=np.uint8) if records else np.zeros(0, np.uint8)
    return buf, off
