"""Bit-exact parity at full size: the transcriptome (100k transcripts,
--track-short-seqs) and the 200 Mbp repetitive genome, both MPHF forms,
every canonical k-mer's state against the CPU oracle's classify.rs
restatement (hash-partitioned so the whole key set is checked at once)."""
import os

import numpy as np
import pytest

import cf1_rs_b200 as cg
from oracle import oracle as o

FULL = {
    2: dict(k=31, num_bins=128, track_short_seqs=True),
    3: dict(k=31, num_bins=128),
}


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", sorted(FULL))
def test_full_size_workload(cfg):
    x = cg.SynthInput(cfg)  # scale 1.0: the whole configuration
    kw = dict(FULL[cfg])
    k = kw.pop("k")
    dumps, distinct = {}, {}
    for mode in ("bbhash", "learned"):
        g = cg.Cf1Gpu(k=k, mode=mode, batched=mode == "learned", **kw)
        try:
            g.add_records(x.seq, x.offsets)
            g.run()
            g.verify_bijection()
            dumps[mode] = g.dump_states()
            distinct[mode] = g.total_kmers()
            if kw.get("track_short_seqs"):
                lens = np.diff(x.offsets.astype(np.int64))
                want = [int(n) for n in lens if n < k]
                assert [n for _, n in g.short_seqs()] == want
        finally:
            g.close()
    res = o.check_lists(k, x.seq, x.offsets, dumps, nparts=2, nthreads=os.cpu_count() or 1)
    for mode in dumps:
        r = res["lists"][mode]
        assert r["mismatches"] == 0, (mode, r)
        assert distinct[mode] == res["n_distinct"] == r["n_listed"]
