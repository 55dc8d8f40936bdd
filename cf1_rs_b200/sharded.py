"""Phases 1-4 sharded by bin over several GPUs, one process per GPU.

Canonical minimizers put every canonical k-mer in exactly one bin
(src/mphf.rs:27-28), so once the super k-mers are routed, the keys, the MPHF
and the states of different bins share nothing.  Every rank routes the whole
input (phases 1-2 are a small share of the work and give every rank the same
minimizer histogram, hence the same partition), keeps the bins b with
``b % world == rank`` and runs phases 3-4 on them alone.  The one exchange
is an all-gather of the per-bin distinct counts: bin b's global slots start
at the sum of the counts of the bins before it, and the global state vector
is the owners' per-bin state runs laid end to end in bin order.

Exchange-based sharding (:func:`run_exchange`) splits phases 1-2 as well:
every rank scans only its share of the input's minimizer tiles, the ranks
sum their minimizer histograms (all-reduce; every rank then derives the same
partition), route their records to the bins' owners (one all-to-all of
8-byte records: the input itself is resident on every rank), and each owner
runs phases 2-4 on what it received.

The device part sits behind a small backend interface (``run`` returning the
per-bin counts and the local 5-bit states; ``scan``/``route``/``finish`` for
the exchange), so the collective plumbing and the assembly below are the
same code whether the states come from the GPUs (:class:`GpuShardBackend`,
:class:`GpuExchangeBackend`) or from a stand-in in a CPU test.
"""
from __future__ import annotations

import numpy as np


def owner(b: int, world: int) -> int:
    """Rank that keeps bin b."""
    return b % world


# ------------------------------------------------------------ state codes ----
def unpack_states(words: np.ndarray, n: int) -> np.ndarray:
    """5-bit states of slots [0, n) from state-vector words (12 per u64, LSB
    first, src/state_vector.rs:36-42)."""
    words = np.asarray(words, np.uint64)
    j = np.arange(12, dtype=np.uint64) * np.uint64(5)
    codes = ((words[:, None] >> j[None, :]) & np.uint64(31)).astype(np.uint8).reshape(-1)
    return codes[:n]


def pack_states(codes: np.ndarray) -> np.ndarray:
    """State-vector words holding `codes` (the inverse of unpack_states)."""
    codes = np.asarray(codes, np.uint8)
    nw = (len(codes) + 11) // 12
    pad = np.zeros(nw * 12, np.uint64)
    pad[: len(codes)] = codes
    j = np.arange(12, dtype=np.uint64) * np.uint64(5)
    return np.bitwise_or.reduce(pad.reshape(nw, 12) << j[None, :], axis=1) if nw else np.zeros(0, np.uint64)


# ------------------------------------------------------------- assembly ----
def global_offsets(counts_all: np.ndarray) -> np.ndarray:
    """Global slot offsets [B+1] from every rank's per-bin counts [world, B].

    Raises ValueError when a bin has keys on a rank that does not own it:
    the shards disagree on the partition, and their slots would overlap."""
    counts_all = np.asarray(counts_all, np.uint64)
    world, nb = counts_all.shape
    own = np.arange(nb) % world
    stray = counts_all.copy()
    stray[own, np.arange(nb)] = 0
    if stray.any():
        r, b = np.argwhere(stray)[0]
        raise ValueError(f"bin {b} has keys on rank {r}, which does not own it")
    counts = counts_all[own, np.arange(nb)]
    off = np.zeros(nb + 1, np.uint64)
    np.cumsum(counts, out=off[1:])
    return off


def assemble_states(codes_per_rank, counts_all: np.ndarray) -> np.ndarray:
    """Global 5-bit states in global slot order from each rank's local states
    (its bins in order, each bin's slots as that rank's MPHF numbers them)."""
    counts_all = np.asarray(counts_all, np.uint64)
    world, nb = counts_all.shape
    goff = global_offsets(counts_all)
    out = np.zeros(int(goff[-1]), np.uint8)
    for r in range(world):
        codes = np.asarray(codes_per_rank[r], np.uint8)
        loff = np.zeros(nb + 1, np.uint64)
        np.cumsum(counts_all[r], out=loff[1:])
        if len(codes) != int(loff[-1]):
            raise ValueError(f"rank {r} sent {len(codes)} states for {int(loff[-1])} slots")
        for b in range(r, nb, world):
            n = int(counts_all[r, b])
            if n:
                out[int(goff[b]): int(goff[b]) + n] = codes[int(loff[b]): int(loff[b]) + n]
    return out


# --------------------------------------------------------- collectives ----
def allgather_counts(counts: np.ndarray, device=None) -> np.ndarray:
    """All ranks' per-bin counts [world, B] (torch.distributed all-gather)."""
    import torch
    import torch.distributed as dist

    t = torch.from_numpy(np.asarray(counts, np.uint64).astype(np.int64))
    if device is not None:
        t = t.to(device)
    parts = [torch.empty_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(parts, t)
    return np.stack([p.cpu().numpy() for p in parts]).astype(np.uint64)


def gather_codes(codes: np.ndarray, device=None):
    """Every rank's local states, on every rank (sizes first, then one padded
    all-gather; each rank's states are a few bytes per k-mer)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size()
    n = torch.tensor([len(codes)], dtype=torch.int64, device=device)
    sizes = [torch.empty_like(n) for _ in range(world)]
    dist.all_gather(sizes, n)
    sizes = [int(x.item()) for x in sizes]
    m = max(sizes) if sizes else 0
    buf = torch.zeros(m, dtype=torch.uint8, device=device)
    if len(codes):
        buf[: len(codes)] = torch.from_numpy(np.asarray(codes, np.uint8)).to(buf.device)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    return [p[:s].cpu().numpy() for p, s in zip(parts, sizes)]


# ------------------------------------------------------------- backends ----
class GpuShardBackend:
    """This rank's shard on its GPU through the C ABI."""

    def __init__(self, k: int, num_bins: int, rank: int, world: int, device: int = 0, **opts):
        from cf1_rs_b200 import Cf1Gpu

        self.ctx = Cf1Gpu(k=k, num_bins=num_bins, device=device, shard_index=rank, shard_count=world, **opts)

    def run(self, seq: np.ndarray, offsets: np.ndarray):
        g = self.ctx
        g.reset_input()
        g.add_records(seq, offsets)
        g.run()
        return g.bin_distinct_counts(), unpack_states(g.states(), g.total_kmers())

    def close(self):
        self.ctx.close()


def run_sharded(backend, seq: np.ndarray, offsets: np.ndarray, device=None, assemble: bool = True):
    """Runs this rank's shard and the exchange.  Returns (global slot offsets,
    global packed state words or None).  Every rank must call it (it holds
    collectives); with assemble=False the states stay on their ranks."""
    counts, codes = backend.run(seq, offsets)
    counts_all = allgather_counts(counts, device)
    goff = global_offsets(counts_all)
    if not assemble:
        return goff, None
    codes_all = gather_codes(codes, device)
    return goff, pack_states(assemble_states(codes_all, counts_all))


# ------------------------------------------------ exchange-based sharding ----
def exchange_records(send, counts):
    """All-to-all of routed records: `send` (int64 tensor) holds counts[r]
    records for rank r, in rank order; returns the records sent to this rank
    by every rank (int64 tensor on send's device)."""
    import torch
    import torch.distributed as dist

    recv_counts = torch.empty_like(counts)
    dist.all_to_all_single(recv_counts, counts)
    in_splits = [int(x) for x in counts.tolist()]
    out_splits = [int(x) for x in recv_counts.tolist()]
    recv = torch.empty(sum(out_splits), dtype=torch.int64, device=send.device)
    dist.all_to_all_single(recv, send, out_splits, in_splits)
    return recv


class GpuExchangeBackend:
    """This rank's share of an exchange-sharded run on its GPU (the
    cf1gpu_xshard_* entry points).  Buffers are torch tensors on the GPU, so
    the all-reduce and the all-to-all run on them in place (NCCL)."""

    def __init__(self, k: int, num_bins: int, rank: int, world: int, device: int = 0, **opts):
        import torch

        from cf1_rs_b200 import Cf1Gpu

        self.dev = torch.device("cuda", device)
        self.world = world
        self.ctx = Cf1Gpu(k=k, num_bins=num_bins, device=device, shard_index=rank, shard_count=world, **opts)

    def _settle(self):
        # torch's stream (its allocations and collectives) before the library's
        import torch

        torch.cuda.current_stream(self.dev).synchronize()

    def load(self, seq: np.ndarray, offsets: np.ndarray):
        self.ctx.reset_input()
        self.ctx.add_records(seq, offsets)

    def scan(self):
        import torch

        hist = torch.zeros(65536, dtype=torch.int32, device=self.dev)  # u32 counts (sums wrap alike)
        self._settle()
        _, n = self.ctx.xshard_scan(hist)
        return hist, n

    def route(self, hist, n_local: int):
        import torch

        records = torch.empty(max(n_local, 1), dtype=torch.int64, device=self.dev)
        counts = torch.zeros(self.world, dtype=torch.int64, device=self.dev)
        self._settle()
        self.ctx.xshard_route(hist, n_local, records, counts)
        return records[:n_local], counts

    def finish(self, recv):
        self._settle()
        self.ctx.xshard_finish(recv, recv.numel())
        return self.ctx.bin_distinct_counts()

    def codes(self):
        g = self.ctx
        return unpack_states(g.states(), g.total_kmers())

    def close(self):
        self.ctx.close()


def run_exchange(backend, device=None, assemble: bool = True):
    """Runs this rank's share of an exchange-sharded run (the backend holds
    the input already).  Returns (global slot offsets, global packed state
    words or None); every rank must call it (it holds collectives)."""
    import torch.distributed as dist

    hist, n_local = backend.scan()
    dist.all_reduce(hist)  # the input's minimizer histogram, on every rank
    send, counts = backend.route(hist, n_local)
    recv = exchange_records(send, counts)
    bin_counts = backend.finish(recv)
    counts_all = allgather_counts(bin_counts, device)
    goff = global_offsets(counts_all)
    if not assemble:
        return goff, None
    codes_all = gather_codes(backend.codes(), device)
    return goff, pack_states(assemble_states(codes_all, counts_all))
