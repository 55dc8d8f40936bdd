"""The two independent CPU oracles agree on per-k-mer states (CPU only)."""
import numpy as np
import pytest

from oracle import oracle as o
from tests.inputs import random_records


@pytest.mark.parametrize("k", [1, 3, 5, 7, 11, 15, 21, 31, 33, 47, 63])
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_direct_vs_join(k, seed):
    recs = random_records(seed * 100 + k, k, n_records=30, max_len=1500)
    seq, off = o.concat_records(recs)
    a = o.run(k, seq, off, nthreads=4, method=0)
    b = o.run(k, seq, off, nthreads=2, method=1)
    assert np.array_equal(a.keys, b.keys)
    assert np.array_equal(a.states, b.states)
    assert np.array_equal(a.state_words, b.state_words)
    assert np.array_equal(a.short_idx, b.short_idx) and np.array_equal(a.short_len, b.short_len)
    assert a.n_occ == b.n_occ
    # every visited state is a valid code: 3, 4-11, 16-31 (never 0, 1, 2, 12-15)
    assert a.states.size == 0 or (set(np.unique(a.states)) <= set([3] + list(range(4, 12)) + list(range(16, 32))))


def test_direct_is_schedule_independent():
    k = 31
    recs = random_records(99, k, n_records=60, max_len=4000)
    seq, off = o.concat_records(recs)
    ref = o.run(k, seq, off, nthreads=1, method=0)
    for nt in (2, 5, 8):
        r = o.run(k, seq, off, nthreads=nt, method=0)
        assert np.array_equal(r.state_words, ref.state_words)


def test_chunked_long_record():
    # A record longer than CHUNK_KMERS (4M) takes the chunked path of
    # classify.rs:576-594; chunk edges must not change any state.
    rng = np.random.default_rng(5)
    k = 31
    L = 4_000_000 + 5000
    s = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, L)].copy()
    s[4_000_010:4_000_020] = ord("N")
    s[3_999_990:4_000_000] = s[100:110]
    seq, off = s, np.array([0, L], dtype=np.uint64)
    a = o.run(k, seq, off, nthreads=8, method=0)
    b = o.run(k, seq, off, nthreads=8, method=1)
    assert np.array_equal(a.states, b.states) and np.array_equal(a.keys, b.keys)


def test_invalid_k():
    with pytest.raises(ValueError):
        o.run(32, np.zeros(10, np.uint8), np.array([0, 10], np.uint64))
