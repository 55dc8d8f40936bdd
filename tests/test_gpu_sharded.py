"""Bin sharding on the device: the shards of one input, run one after another
on one GPU, cover the unsharded run exactly.

Each shard keeps the bins b with b % world == rank and numbers its bins'
slots itself (BBHash levels and learned leaves are built per bin).  The
shards' state runs laid end to end in bin order are the global state vector:
every key's global slot -- its bin's global offset plus its place in the
owner's run of the bin -- holds its state, the global slots are a
permutation, and the per-k-mer states are the oracle's.  (Slots inside a bin
also depend on the run's sub-bucket split width, which follows the largest
bin a context holds, so they need not equal the unsharded run's.)"""
import numpy as np
import pytest

from cf1_rs_b200 import sharded
from oracle import oracle as o
from tests.gpu_util import gpu_run, sort_by_key
from tests.inputs import random_records

pytestmark = pytest.mark.gpu

BINS = 16


def check_assembly(counts, codes, states, slots):
    """The shards' state runs laid end to end hold every key's state at the
    key's global slot, and the global slots are a permutation."""
    goff = sharded.global_offsets(counts)
    assembled = sharded.assemble_states(codes, counts)
    gslots = []
    for r in range(len(codes)):
        own = np.concatenate([[0], np.cumsum(counts[r])]).astype(np.int64)
        local = slots[r].astype(np.int64)
        b = np.searchsorted(own, local, side="right") - 1
        g = goff[b].astype(np.int64) + (local - own[b])
        assert np.array_equal(assembled[g], states[r])
        gslots.append(g)
    assert np.array_equal(np.sort(np.concatenate(gslots)), np.arange(int(goff[-1])))


@pytest.mark.parametrize("mode", ["bbhash", "learned"])
@pytest.mark.parametrize("k,world", [(31, 2), (31, 3), (63, 2), (15, 5)])
def test_shards_cover_the_unsharded_run(k, world, mode):
    recs = random_records(700 + k + world, k, n_records=80, max_len=6000)
    seq, off = o.concat_records(recs)
    ref = o.run(k, seq, off, nthreads=8)
    counts, codes, keys, states, slots = [], [], [], [], []
    for r in range(world):
        be = sharded.GpuShardBackend(k, BINS, r, world, mode=mode)
        try:
            c, s = be.run(seq, off)
            be.ctx.verify_bijection()  # the shard's slots are a bijection onto its own range
            kk, ss = be.ctx.dump_states()
            slots.append(be.ctx.query(kk))
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
    check_assembly(counts, codes, states, slots)
    # and the per-bin counts are the unsharded run's
    g = gpu_run(seq, off, k, mode=mode, num_bins=BINS)
    try:
        assert np.array_equal(counts.sum(axis=0), g.bin_distinct_counts())
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


def exchange_emulated(seq, off, k, world, **opts):
    """An exchange-sharded run of `world` shards, one after another on one
    GPU: every shard scans its share, the histograms are summed and each
    shard's routed groups are handed to their owners on the host."""
    from cf1_rs_b200 import Cf1Gpu

    ctxs = [Cf1Gpu(k=k, num_bins=BINS, shard_index=r, shard_count=world, **opts) for r in range(world)]
    for g in ctxs:
        g.add_records(seq, off)
    scans = [g.xshard_scan() for g in ctxs]
    hist = np.sum([h.astype(np.uint64) for h, _ in scans], axis=0).astype(np.uint32)
    routed = [g.xshard_route(hist, n) for g, (_, n) in zip(ctxs, scans)]
    for d, g in enumerate(ctxs):
        parts = []
        for rec, cnt in routed:
            o_ = np.concatenate([[0], np.cumsum(cnt.astype(np.int64))])
            parts.append(rec[o_[d]: o_[d + 1]])
        g.xshard_finish(np.concatenate(parts))
    return ctxs, scans, routed


@pytest.mark.parametrize("mode", ["bbhash", "learned"])
@pytest.mark.parametrize("k,world", [(31, 2), (31, 3), (63, 2), (21, 4)])
def test_exchange_shards_cover_the_unsharded_run(k, world, mode):
    recs = random_records(900 + k + world, k, n_records=80, max_len=6000)
    seq, off = o.concat_records(recs)
    ref = o.run(k, seq, off, nthreads=8)
    ctxs, scans, routed = exchange_emulated(seq, off, k, world, mode=mode)
    try:
        counts = np.stack([g.bin_distinct_counts() for g in ctxs])
        goff = sharded.global_offsets(counts)  # raises if two shards hold keys of one bin
        assert int(goff[-1]) == len(ref.states)
        for g in ctxs:
            g.verify_bijection()
        keys, states = zip(*[g.dump_states() for g in ctxs])
        kk, ss = sort_by_key(np.concatenate(keys), np.concatenate(states))
        assert np.array_equal(kk, ref.keys)
        assert np.array_equal(ss, ref.states)
        codes = [sharded.unpack_states(g.states(), g.total_kmers()) for g in ctxs]
        check_assembly(counts, codes, states, [g.query(kk_) for g, kk_ in zip(ctxs, keys)])
        g1 = gpu_run(seq, off, k, mode=mode, num_bins=BINS)
        try:
            # the shares split the unsharded run's records; every group is its owner's
            assert sum(n for _, n in scans) == g1.stats()["n_superkmers"]
            for rec, cnt in routed:
                o_ = np.concatenate([[0], np.cumsum(cnt.astype(np.int64))])
                for d in range(world):
                    assert np.all((rec[o_[d]: o_[d + 1]] & np.uint64(0xFFF)) % np.uint64(world) == d)
            assert np.array_equal(counts.sum(axis=0), g1.bin_distinct_counts())
        finally:
            g1.close()
    finally:
        for g in ctxs:
            g.close()


def test_exchange_refuses_foreign_records_and_runs_again():
    from cf1_rs_b200 import Cf1Error

    recs = random_records(4242, 31, n_records=30, max_len=4000)
    seq, off = o.concat_records(recs)
    ctxs, scans, routed = exchange_emulated(seq, off, 31, 2)
    try:
        g = ctxs[0]
        with pytest.raises(Cf1Error):  # finish before a new scan and route
            g.xshard_finish(routed[0][0])
        hist = scans[0][0] + scans[1][0]
        _, n = g.xshard_scan()
        rec, cnt = g.xshard_route(hist, n)
        c0 = int(cnt[0])
        assert 0 < c0 < n
        with pytest.raises(Cf1Error) as e:  # shard 1's group handed to shard 0
            g.xshard_finish(rec[c0:])
        assert "not this shard" in str(e.value)
        past = rec[:1].copy()
        past[0] = (np.uint64(len(seq) + 10**6) << np.uint64(24)) | (past[0] & np.uint64(0xFFFFFF))
        _, n = g.xshard_scan()
        g.xshard_route(hist, n)
        with pytest.raises(Cf1Error):  # a record reaching past the input
            g.xshard_finish(past)
        g.run()  # the context still runs
        assert g.total_kmers() > 0
    finally:
        for g in ctxs:
            g.close()
