"""Phase 5 (unitig extraction, GFA-reduced .cf_seg / .cf_seq) on the
structures phases 1-4 hand over.

The reference's phase 5 (src/output.rs) is Rust and stays as it is; it reads
only Mphf::hash / bucket_id and the state vector.  `oracle.phase5` restates
it; these tests check the restatement against itself on the CPU (every
distinct k-mer in exactly one segment, every record spelled back by its
tiling, output independent of the slot numbering after canonicalisation)
and then run it on the GPU path's exported MPHF image and state words: the
canonical output must equal the one from the oracle's own structures."""
import numpy as np
import pytest

import cf1_rs_b200 as cg
from oracle import oracle as o
from oracle import phase5 as p5
from tests.gpu_util import gpu_run
from tests.inputs import random_records


def named(recs):
    return [(f"seq{i}", r) for i, r in enumerate(recs)]


def oracle_slot_of(ref):
    """The oracle's MPHF: a key's rank among the sorted distinct keys."""
    keys = ref.keys

    def slot_of(q):
        if keys.ndim == 1:
            return np.searchsorted(keys, q)
        kk = [(int(h) << 64) | int(lo) for lo, h in keys]
        qq = [(int(h) << 64) | int(lo) for lo, h in q]
        return np.searchsorted(np.array(kk, dtype=object), np.array(qq, dtype=object))

    return slot_of


def kmers_of(s, k):
    for i in range(len(s) - k + 1):
        w = s[i:i + k]
        yield min(w, p5.revcomp(w))


def check_self_consistent(out, recs, k, ref):
    spell = dict(out.segs)
    assert len(spell) == len(out.segs), "a unitig was written twice"
    # every distinct canonical k-mer lies in exactly one segment
    seen = []
    for s in spell.values():
        seen.extend(kmers_of(s, k))
    assert len(seen) == len(set(seen)) == len(ref.states)
    # each occurrence spells its stretch of the record, in its direction
    for (name, rec), units in zip([r for r in named(recs) if len(r[1]) >= k], out.unitigs):
        for uid, fwd, a, b in units:
            text = rec[a:b + k].decode().upper()
            assert (text if fwd else p5.revcomp(text)) == spell[uid], (name, uid)
        # unitigs tile the record's placeholder-free stretches end to end
        for (_, _, _, b0), (_, _, a1, _) in zip(units, units[1:]):
            gap = rec[b0 + 1:a1 + k - 1]
            assert a1 == b0 + 1 or any(p5.is_placeholder(c) for c in gap)


@pytest.mark.parametrize("k,poly_n", [(31, False), (31, True), (15, True), (33, False)])
def test_phase5_restatement_is_self_consistent(k, poly_n):
    recs = random_records(77 + k, k, n_records=25, max_len=1500)
    seq, off = o.concat_records(recs)
    ref = o.run(k, seq, off, nthreads=2)
    out = p5.extract_and_output(named(recs), k, oracle_slot_of(ref), ref.state_words, poly_n_stretch=poly_n)
    check_self_consistent(out, recs, k, ref)
    assert out.meta["kmer_count"] == len(ref.states)
    if poly_n:
        assert any("N" in t for _, t in out.tilings)


def test_phase5_output_is_free_of_slot_numbering():
    k = 31
    recs = random_records(4711, k, n_records=25, max_len=1500)
    seq, off = o.concat_records(recs)
    ref = o.run(k, seq, off, nthreads=2)
    a = p5.extract_and_output(named(recs), k, oracle_slot_of(ref), ref.state_words)
    # another bijection onto the same slots, with the states moved along
    perm = np.random.default_rng(5).permutation(len(ref.states)).astype(np.uint64)
    from cf1_rs_b200 import sharded
    moved = np.zeros(len(ref.states), np.uint8)
    moved[perm] = ref.states
    slot_of = oracle_slot_of(ref)
    b = p5.extract_and_output(named(recs), k, lambda q: perm[slot_of(q)], sharded.pack_states(moved))
    assert [u for u, _ in a.segs] != [u for u, _ in b.segs]
    assert p5.canonical(a) == p5.canonical(b)


@pytest.mark.gpu
@pytest.mark.parametrize("queries", ["host_image", "device_batches"])
@pytest.mark.parametrize("mode", ["bbhash", "learned"])
@pytest.mark.parametrize("k", [31, 63])
def test_phase5_on_gpu_structures_matches_oracle(k, mode, queries):
    """Phase 5's MPHF queries answered either by the exported host image
    (cf1gpu_mphf_host_query) or by cf1gpu_query on the device, one call per
    batch of a record's k-mers, the MPHF never leaving the GPU."""
    recs = random_records(9000 + k, k, n_records=40, max_len=3000)
    seq, off = o.concat_records(recs)
    ref = o.run(k, seq, off, nthreads=8)
    g = gpu_run(seq, off, k, mode=mode, num_bins=16)
    try:
        words = g.states()
        if queries == "host_image":
            image = g.export_mphf()
            gpu = p5.extract_and_output(named(recs), k, lambda q: cg.host_query(image, q), words,
                                        poly_n_stretch=True)
        else:
            gpu = p5.extract_and_output(named(recs), k, g.query, words, poly_n_stretch=True)
    finally:
        g.close()
    cpu = p5.extract_and_output(named(recs), k, oracle_slot_of(ref), ref.state_words, poly_n_stretch=True)
    assert len(gpu.segs) == len(cpu.segs)
    assert p5.canonical(gpu) == p5.canonical(cpu)
    assert gpu.meta == cpu.meta
