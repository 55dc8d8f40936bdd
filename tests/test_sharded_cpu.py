"""Bin sharding's host side (cf1_rs_b200.sharded) on the CPU: two gloo ranks
exchange per-bin counts and states, rank 0 assembles the global state vector.

The device part is played by an oracle backend: the super k-mers and the
partition of the oracle's restatement of the binning spec give every k-mer
its bin, and the oracle's classification gives its state.  The assembled
vector must equal the same data laid out in one process (bins in order, keys
sorted inside a bin), and shards that disagree on the partition must be
refused."""
import os
import socket
import tempfile

import numpy as np
import pytest

from cf1_rs_b200 import sharded
from oracle import oracle as o
from tests.inputs import random_records

K, BINS, TILE = 31, 16, 2048
LUT2 = np.zeros(256, np.uint8)
for _c, _v in zip(b"ACGTacgt", [0, 1, 2, 3, 0, 1, 2, 3]):
    LUT2[_c] = _v


def device_sequence(recs, k):
    """The device's concatenation: records of >= k bases, one placeholder after each."""
    return np.frombuffer(b"".join(r + b"N" for r in recs if len(r) >= k), np.uint8)


def canonical_windows(cat, k):
    """Canonical k-mer of every window start of the concatenation."""
    bb = LUT2[cat].astype(np.uint64)
    nw = len(cat) - k + 1
    fw = np.zeros(nw, np.uint64)
    rc = np.zeros(nw, np.uint64)
    for i in range(k):
        fw = (fw << np.uint64(2)) | bb[i: i + nw]
        rc = rc | ((np.uint64(3) - bb[i: i + nw]) << np.uint64(2 * i))
    return np.minimum(fw, rc)


def occurrence_positions(pos, n):
    """Window start of every k-mer occurrence of super k-mers (pos, n)."""
    n = n.astype(np.int64)
    starts = np.repeat(pos.astype(np.int64), n)
    within = np.arange(len(starts)) - np.repeat(np.cumsum(n) - n, n)
    return starts + within


def window_bins_and_keys(recs, k, num_bins):
    """(canonical key, bin) of every k-mer occurrence, bins from the spec."""
    cat = device_sequence(recs, k)
    pos, n, bucket = o.superkmers(cat, k, TILE)
    hist = np.bincount(bucket.astype(np.int64), minlength=65536).astype(np.uint64)
    lut, _ = o.partition(hist, num_bins)
    can = canonical_windows(cat, k)
    bins = np.repeat(lut[bucket].astype(np.int64), n.astype(np.int64))
    return can[occurrence_positions(pos, n)], bins


class OracleShardBackend:
    """Stand-in for one GPU shard: its bins' distinct keys sorted, with the
    oracle's states.  `stray` makes it also claim a bin it does not own."""

    def __init__(self, k, num_bins, rank, world, stray=None):
        self.k, self.nb, self.rank, self.world, self.stray = k, num_bins, rank, world, stray

    def run(self, recs, _offsets=None):
        seq, off = o.concat_records(recs)
        ref = o.run(self.k, seq, off, nthreads=2)
        keys, bins = window_bins_and_keys(recs, self.k, self.nb)
        counts = np.zeros(self.nb, np.uint64)
        codes = []
        for b in range(self.nb):
            if b % self.world != self.rank and b != self.stray:
                continue
            kb = np.unique(keys[bins == b])
            counts[b] = len(kb)
            codes.append(ref.states[np.searchsorted(ref.keys, kb)])
        return counts, (np.concatenate(codes).astype(np.uint8) if codes else np.zeros(0, np.uint8))


class OracleExchangeBackend:
    """Stand-in for one GPU's share of an exchange-sharded run: its slice of
    the minimizer tiles' super k-mers, routing by the summed histogram's
    partition, and the oracle's states for the bins it owns.  Records travel
    in the device's 64-bit layout (position << 24 | (n - 1) << 12 | bin)."""

    def __init__(self, k, num_bins, rank, world, misroute=False):
        self.k, self.nb, self.rank, self.world, self.misroute = k, num_bins, rank, world, misroute

    def load(self, recs, _offsets=None):
        self.recs = recs
        self.cat = device_sequence(recs, self.k)

    def scan(self):
        import torch

        pos, n, bucket = o.superkmers(self.cat, self.k, TILE)
        nt = -(-(len(self.cat) - self.k + 1) // TILE)
        t = pos.astype(np.int64) // TILE
        sel = (t >= nt * self.rank // self.world) & (t < nt * (self.rank + 1) // self.world)
        self.pos, self.n, self.bucket = pos[sel], n[sel], bucket[sel]
        hist = np.bincount(self.bucket.astype(np.int64), minlength=65536).astype(np.int32)
        return torch.from_numpy(hist), int(sel.sum())

    def route(self, hist, n_local):
        import torch

        lut, _ = o.partition(hist.numpy().astype(np.uint32).astype(np.uint64), self.nb)
        bins = lut[self.bucket].astype(np.uint64)
        owner = (bins + np.uint64(1 if self.misroute else 0)) % np.uint64(self.world)
        order = np.argsort(owner, kind="stable")
        rec = (self.pos.astype(np.uint64) << np.uint64(24)) | ((self.n.astype(np.uint64) - np.uint64(1)) << np.uint64(12)) | bins
        counts = np.bincount(owner.astype(np.int64), minlength=self.world).astype(np.int64)
        assert len(rec) == n_local
        return torch.from_numpy(rec[order].view(np.int64).copy()), torch.from_numpy(counts)

    def finish(self, recv):
        r = recv.numpy().view(np.uint64)
        pos, n, bins = r >> np.uint64(24), ((r >> np.uint64(12)) & np.uint64(0xFFF)) + np.uint64(1), r & np.uint64(0xFFF)
        if np.any(bins % np.uint64(self.world) != np.uint64(self.rank)):
            raise ValueError(f"rank {self.rank} received a record of a bin it does not own")
        keys = canonical_windows(self.cat, self.k)[occurrence_positions(pos, n)]
        kb_bins = np.repeat(bins.astype(np.int64), n.astype(np.int64))
        seq, off = o.concat_records(self.recs)
        ref = o.run(self.k, seq, off, nthreads=2)
        counts = np.zeros(self.nb, np.uint64)
        codes = []
        for b in range(self.rank, self.nb, self.world):
            kb = np.unique(keys[kb_bins == b])
            counts[b] = len(kb)
            codes.append(ref.states[np.searchsorted(ref.keys, kb)])
        self._codes = np.concatenate(codes).astype(np.uint8) if codes else np.zeros(0, np.uint8)
        return counts

    def codes(self):
        return self._codes


def _exchange_main(rank, world, port, out_path, misroute):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        recs = random_records(2025, K, n_records=30, max_len=3000)
        backend = OracleExchangeBackend(K, BINS, rank, world, misroute=misroute and rank == 1)
        backend.load(recs)
        try:
            goff, words = sharded.run_exchange(backend)
            if rank == 0:
                np.savez(out_path, goff=goff, words=words, n_local=len(backend.pos))
        except ValueError as e:
            with open(out_path + f".err{rank}", "w") as f:
                f.write(str(e))
            raise
    finally:
        dist.destroy_process_group()


def _rank_main(rank, world, port, out_path, stray):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        recs = random_records(2024, K, n_records=30, max_len=3000)
        backend = OracleShardBackend(K, BINS, rank, world, stray=stray if rank == 1 else None)
        try:
            goff, words = sharded.run_sharded(backend, recs, None)
            if rank == 0:
                np.savez(out_path, goff=goff, words=words)
        except ValueError as e:
            if rank == 0:
                with open(out_path + ".err", "w") as f:
                    f.write(str(e))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _spawn(world, stray=None):
    import torch.multiprocessing as mp

    d = tempfile.mkdtemp()
    out = os.path.join(d, "r.npz")
    mp.spawn(_rank_main, args=(world, _free_port(), out, stray), nprocs=world, join=True)
    return out


def test_pack_unpack_round_trip():
    rng = np.random.default_rng(3)
    codes = rng.integers(0, 32, 1000).astype(np.uint8)
    for n in (0, 1, 11, 12, 13, 1000):
        assert np.array_equal(sharded.unpack_states(sharded.pack_states(codes[:n]), n), codes[:n])


def test_global_offsets_and_assembly_in_one_process():
    counts = np.array([[3, 0, 2, 0], [0, 1, 0, 4]], np.uint64)  # bins 0, 2 on rank 0; 1, 3 on rank 1
    goff = sharded.global_offsets(counts)
    assert goff.tolist() == [0, 3, 4, 6, 10]
    codes = [np.array([1, 2, 3, 4, 5], np.uint8), np.array([6, 7, 8, 9, 10], np.uint8)]
    assert sharded.assemble_states(codes, counts).tolist() == [1, 2, 3, 6, 4, 5, 7, 8, 9, 10]
    bad = counts.copy()
    bad[1, 0] = 1  # rank 1 claims a key of rank 0's bin
    with pytest.raises(ValueError):
        sharded.global_offsets(bad)


def test_two_gloo_ranks_assemble_the_global_vector():
    out = _spawn(2)
    r = np.load(out)
    recs = random_records(2024, K, n_records=30, max_len=3000)
    # the same data laid out in one process
    counts, codes = OracleShardBackend(K, BINS, 0, 1).run(recs)
    goff = np.zeros(BINS + 1, np.uint64)
    np.cumsum(counts, out=goff[1:])
    assert np.array_equal(r["goff"], goff)
    assert np.array_equal(r["words"], sharded.pack_states(codes))
    # and every state is the oracle's
    seq, off = o.concat_records(recs)
    ref = o.run(K, seq, off, nthreads=2)
    assert int(goff[-1]) == len(ref.states)
    assert np.array_equal(np.sort(sharded.unpack_states(r["words"], len(ref.states))), np.sort(ref.states))


def test_two_gloo_ranks_refuse_overlapping_shards():
    out = _spawn(2, stray=0)  # rank 1 also claims bin 0
    assert os.path.exists(out + ".err") and "does not own" in open(out + ".err").read()


def _spawn_exchange(world, misroute=False):
    import torch.multiprocessing as mp

    d = tempfile.mkdtemp()
    out = os.path.join(d, "x.npz")
    try:
        mp.spawn(_exchange_main, args=(world, _free_port(), out, misroute), nprocs=world, join=True)
    except Exception:
        pass  # a rank that refused its records ends the job; the test reads its message
    return out, d


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_ranks_assemble_the_global_vector(world):
    out, _ = _spawn_exchange(world)
    r = np.load(out)
    recs = random_records(2025, K, n_records=30, max_len=3000)
    # the same data laid out in one process: the replicated-routing result
    counts, codes = OracleShardBackend(K, BINS, 0, 1).run(recs)
    goff = np.zeros(BINS + 1, np.uint64)
    np.cumsum(counts, out=goff[1:])
    assert np.array_equal(r["goff"], goff)
    assert np.array_equal(r["words"], sharded.pack_states(codes))
    assert 0 < int(r["n_local"])  # rank 0 scanned a share of the input, not all of it
    cat = device_sequence(recs, K)
    assert int(r["n_local"]) < len(o.superkmers(cat, K, TILE)[0])


def test_exchange_refuses_misrouted_records():
    out, d = _spawn_exchange(2, misroute=True)  # rank 1 sends every record to the wrong owner
    errs = [open(os.path.join(d, f)).read() for f in os.listdir(d) if ".err" in f]
    assert not os.path.exists(out)
    assert any("does not own" in e for e in errs)
