"""Helpers for the GPU parity tests: run the C ABI path and the oracle on the
same input and line their per-k-mer states up by canonical k-mer."""
import numpy as np

from cf1_rs_b200 import Cf1Gpu
from oracle import oracle as o


def sort_by_key(keys, states):
    if keys.ndim == 1:
        order = np.argsort(keys, kind="stable")
    else:
        order = np.lexsort((keys[:, 0], keys[:, 1]))
    return keys[order], states[order]


def gpu_run(seq, off, k, **kw):
    g = Cf1Gpu(k=k, **kw)
    g.add_records(seq, off)
    g.run()
    return g


def assert_parity(seq, off, k, oracle_threads=8, **kw):
    """Per canonical k-mer states of the GPU path equal the oracle's."""
    ref = o.run(k, seq, off, nthreads=oracle_threads, method=0)
    g = gpu_run(seq, off, k, **kw)
    try:
        assert g.total_kmers() == len(ref.states)
        keys, st = g.dump_states()
        keys, st = sort_by_key(keys, st)
        assert np.array_equal(keys, ref.keys), "distinct canonical k-mer sets differ"
        bad = np.nonzero(st != ref.states)[0]
        assert bad.size == 0, f"{bad.size} states differ, first at {bad[:5]}: gpu {st[bad[:5]]} ref {ref.states[bad[:5]]}"
        s = g.stats()
        assert s["n_kmer_occurrences"] == ref.n_occ
        g.verify_bijection()
        return g, ref
    except Exception:
        g.close()
        raise
