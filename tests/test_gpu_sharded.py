"""Bin sharding on the device: the shards of one input, run one after another
on one GPU, cover the unsharded run exactly.

Each shard keeps the bins b with b % world == rank.  A bin's slots depend
only on its own keys (BBHash levels and learned leaves are built per bin), so
the shards' state runs laid end to end in bin order must be the unsharded
run's state vector word for word, and their per-k-mer states the oracle's."""
import numpy as np
import pytest

from cf1_rs_b200 import sharded
from oracle import oracle as o
from tests.gpu_util import gpu_run, sort_by_key
from tests.inputs import random_records

pytestmark = pytest.mark.gpu

BINS = 16


@pytest.mark.parametrize("mode", ["bbhash", "learned"])
@pytest.mark.parametrize("k,world", [(31, 2), (31, 3), (63, 2), (15, 5)])
def test_shards_cover_the_unsharded_run(k, world, mode):
    recs = random_records(700 + k + world, k, n_records=80, max_len=6000)
    seq, off = o.concat_records(recs)
    ref = o.run(k, seq, off, nthreads=8)
    counts, codes, keys, states = [], [], [], []
    for r in range(world):
        be = sharded.GpuShardBackend(k, BINS, r, world, mode=mode)
        try:
            c, s = be.run(seq, off)
            be.ctx.verify_bijection()  # the shard's slots are a bijection onto its own range
            kk, ss = be.ctx.dump_states()
        finally:
            be.close()
        counts.append(c)
        codes.append(s)
        keys.append(kk)
        states.append(ss)
    counts = np.stack(counts)
    goff = sharded.global_offsets(counts)  # raises if two shards hold keys of one bin
    assert int(goff[-1]) == len(ref.states)
    # per k-mer: the shards' union is the oracle's result
    kk, ss = sort_by_key(np.concatenate(keys), np.concatenate(states))
    assert np.array_equal(kk, ref.keys)
    assert np.array_equal(ss, ref.states)
    # laid end to end: the unsharded run's words and per-bin counts
    g = gpu_run(seq, off, k, mode=mode, num_bins=BINS)
    try:
        assert np.array_equal(counts.sum(axis=0), g.bin_distinct_counts())
        assert np.array_equal(sharded.pack_states(sharded.assemble_states(codes, counts)), g.states())
    finally:
        g.close()


def test_bin_counts_match_total():
    recs = random_records(5150, 31, n_records=40, max_len=4000)
    seq, off = o.concat_records(recs)
    g = gpu_run(seq, off, 31, num_bins=BINS)
    try:
        c = g.bin_distinct_counts()
        assert c.shape == (BINS,) and int(c.sum()) == g.total_kmers()
    finally:
        g.close()
