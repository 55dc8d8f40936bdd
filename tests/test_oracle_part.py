"""The hash-partitioned oracle (cfo_part_*): the classify.rs restatement run
one partition of the canonical k-mers at a time, used to check inputs whose
distinct k-mers do not fit in memory at once (the 3.1 Gbp genome).  Its union
over partitions must equal the whole-run oracle (which walks every run of
every record, src/classify.rs:34-141), and its comparison must count every
kind of mistake planted in a (key, state) list."""
import numpy as np
import pytest

from oracle import oracle as o
from tests.inputs import random_records


def _sorted(keys, states):
    order = np.argsort(keys, kind="stable") if keys.ndim == 1 else np.lexsort((keys[:, 0], keys[:, 1]))
    return keys[order], states[order]


@pytest.mark.parametrize("k", [1, 3, 15, 31, 33, 63])
@pytest.mark.parametrize("nparts", [1, 3, 7])
def test_partition_union_equals_whole_run(k, nparts):
    recs = random_records(11 + k, k, n_records=50, max_len=3000)
    seq, off = o.concat_records(recs)
    ref = o.run(k, seq, off, nthreads=4, method=0)
    index = o.PartIndex(k, seq, off, nparts, 3)
    assert index.n_occ == ref.n_occ
    keys, states, occ = [], [], 0
    for p in range(nparts):
        r = o.PartResult(index, p, 3)
        kk, ss = r.keys_states()
        keys.append(kk)
        states.append(ss)
        occ += r.n_occ
        r.close()
    index.close()
    kk, ss = _sorted(np.concatenate(keys), np.concatenate(states))
    assert occ == ref.n_occ
    assert np.array_equal(kk, ref.keys)
    assert np.array_equal(ss, ref.states)


def test_chunked_records_match():
    """Records above the 4M-k-mer chunk size (src/classify.rs:565-594) are cut
    into chunks; the partitioned run steps windows on their own and must agree
    with the chunked walk across chunk ends."""
    rng = np.random.default_rng(5)
    L = 4_000_000 + 5000
    s = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, L)].copy()
    s[4_000_010:4_000_020] = ord("N")
    s[3_999_990:4_000_000] = s[100:110]
    seq, off = o.concat_records([s.tobytes(), b"ACGTACGTAC" * 10])
    ref = o.run(31, seq, off, nthreads=8, method=0)
    res = o.check_states(31, seq, off, ref.keys, ref.states, nparts=2, nthreads=8)
    assert res["mismatches"] == 0 and res["n_distinct"] == len(ref.states) and res["n_occ"] == ref.n_occ


@pytest.mark.parametrize("k", [15, 31, 63])
def test_compare_counts_planted_mistakes(k):
    recs = random_records(21 + k, k, n_records=40, max_len=2000)
    seq, off = o.concat_records(recs)
    ref = o.run(k, seq, off, nthreads=4, method=0)
    keys, st = ref.keys.copy(), ref.states.copy()
    n = len(st)
    rng = np.random.default_rng(k)
    perm = rng.permutation(n)  # any order
    keys, st = keys[perm], st[perm]
    st[3] ^= 1                                   # one state differs
    keys = np.concatenate([keys[:-1], keys[5:6]])  # last key dropped, key 5 listed twice
    st = np.concatenate([st[:-1], st[5:6]])
    extra = keys[:1].copy()                      # a key that is not in the set: all ones
    extra[...] = np.uint64(2**64 - 1) if k <= 32 else np.uint64(2**64 - 1)
    keys = np.concatenate([keys, extra])
    st = np.concatenate([st, st[:1]])
    res = o.check_lists(k, seq, off, {"good": (ref.keys, ref.states), "bad": (keys, st)}, nparts=4, nthreads=4)
    good, bad = res["lists"]["good"], res["lists"]["bad"]
    assert good["mismatches"] == 0
    assert bad["state_diff"] == 1
    assert bad["missing"] == 1
    assert bad["dup"] == 1
    assert bad["extra"] == 1
    assert bad["mismatches"] == 4
    assert res["n_distinct"] == n and res["n_occ"] == ref.n_occ
