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

The device part sits behind a small backend interface (``run`` returning the
per-bin counts and the local 5-bit states), so the collective plumbing and
the assembly below are the same code whether the states come from the GPUs
(:class:`GpuShardBackend`) or from a stand-in in a CPU test.
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
