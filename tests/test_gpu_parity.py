"""GPU parity: per-k-mer states of the CUDA path (through the C ABI) equal the
oracle's, bit for bit, keyed by canonical k-mer."""
import os
import tempfile

import numpy as np
import pytest

import cf1_rs_b200 as cg
from oracle import oracle as o
from tests.gpu_util import assert_parity, gpu_run, sort_by_key
from tests.inputs import random_records

pytestmark = pytest.mark.gpu

KS = [1, 3, 5, 7, 9, 15, 21, 31, 33, 45, 61, 63]


@pytest.mark.parametrize("mode", ["bbhash", "learned"])
@pytest.mark.parametrize("k", KS)
def test_edge_case_records(k, mode):
    recs = random_records(1000 + k, k, n_records=60, max_len=4000)
    seq, off = o.concat_records(recs)
    g, _ = assert_parity(seq, off, k, mode=mode, num_bins=16, track_short_seqs=True)
    g.close()


@pytest.mark.parametrize("k", [31, 63])
@pytest.mark.parametrize("mode", ["bbhash", "learned"])
def test_batched_mode(k, mode):
    recs = random_records(77 + k, k, n_records=200, max_len=6000)
    seq, off = o.concat_records(recs)
    assert_parity(seq, off, k, mode=mode, batched=True, num_bins=64)[0].close()


@pytest.mark.parametrize("bins", [1, 2, 7, 128, 4096])
def test_bin_counts(bins):
    recs = random_records(5, 31, n_records=80, max_len=5000)
    seq, off = o.concat_records(recs)
    g, _ = assert_parity(seq, off, 31, num_bins=bins)
    assert 1 <= g.stats()["n_bins"] <= bins
    g.close()


@pytest.mark.parametrize("sort_mode", ["msd", "lsd"])
@pytest.mark.parametrize("k", [15, 31, 33, 63])
def test_sort_modes(k, sort_mode):
    recs = random_records(300 + k, k, n_records=80, max_len=6000)
    seq, off = o.concat_records(recs)
    g, _ = assert_parity(seq, off, k, num_bins=8, sort_mode=sort_mode)
    bits = g.stats()["sort_msd_bits"]
    assert (bits == 2**64 - 1) if sort_mode == "lsd" else (bits < 64)
    g.close()


@pytest.mark.parametrize("mode", ["bbhash", "learned"])
@pytest.mark.parametrize("k", [5, 31, 33, 63])
def test_state_update_modes(k, mode):
    # side sets joined by the phase-3 dedup, side-set OR per occurrence + pack,
    # and the CAS loop on packed words all give the same words
    recs = random_records(900 + k, k, n_records=120, max_len=5000)
    seq, off = o.concat_records(recs)
    words = {}
    for upd in ("phase3", "sideset", "cas"):
        g, _ = assert_parity(seq, off, k, mode=mode, num_bins=16, state_update=upd)
        words[upd] = g.states()
        if upd != "cas":
            assert g.stats()["classify_cas_retries"] == 0
        g.close()
    assert np.array_equal(words["phase3"], words["cas"])
    assert np.array_equal(words["sideset"], words["cas"])


def test_sorted_runs_over_sparse_key_ranges(tmp_path):
    """One bin of ~12M k-mer occurrences; the autotuner's first run tries
    split widths up to 16 bits (65,536 sub-buckets).  Canonical k-mers are
    rare at the top of the key space (starting TTG.., TTT..: a few keys per
    sub-bucket), so there the sorted dedup's packed runs are limited by their
    1,024-sub-bucket bucket range rather than by their key capacity."""
    rng = np.random.default_rng(404)
    s = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 12_000_000)].tobytes()
    seq, off = o.concat_records([s[:7_000_000], s[7_000_000:]])
    cache = str(tmp_path / "tuner.txt")
    g, _ = assert_parity(seq, off, 31, mode="learned", num_bins=1, tuner_cache=cache)
    assert g.stats()["tuner_state"] == 2  # this run measured the widths
    g.close()


@pytest.mark.parametrize("n_bases,bits", [(24_540, 6), (392_600, 10)])
def test_packed_words_with_subbuckets_left_to_block_kernel(tmp_path, n_bases, bits):
    """BBHash form, one bin of random sequence.  The tuner line sets the split
    one bit below the default, so sub-buckets average ~383 distinct keys and
    about half pass the warp dedup's 384: those go to the block kernel, whose
    input is unpacked first.  With a split of 6 bits (one pass) or 10 (6 + 4)
    the multisplit runs on packed words."""
    rng = np.random.default_rng(n_bases)
    s = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, n_bases)].tobytes()
    seq, off = o.concat_records([s])
    size_class = (n_bases + 1).bit_length() - 1  # floor(log2) of the input with its record separator
    cache = tmp_path / "tuner.txt"
    cache.write_text(f"cf1tune 1 wide=0 sorted=0 batched=0 size={size_class} sk_tile=2048 msd_delta=-1 "
                     "p1_ms=1.000 p3_ms=1.000\n")
    g, _ = assert_parity(seq, off, 31, mode="bbhash", num_bins=1, tuner_cache=str(cache))
    st = g.stats()
    assert st["tuner_state"] == 1 and st["sort_msd_bits"] == bits
    assert st["dedup_overflow"] > 0
    g.close()


@pytest.mark.parametrize("mode", ["bbhash", "learned"])
def test_phase3_join_with_lsd_fallback_and_oversized_subbuckets(mode):
    # The LSD sort carries no side-set bytes: phase 4 then classifies the
    # occurrences.  Long homopolymers and tandem repeats put thousands of
    # copies of a few keys in one sub-bucket, where the dedup's joins and the
    # sorted path's runs of equal keys do the work.
    rng = np.random.default_rng(77)
    recs = [b"A" * 20000, b"AT" * 9000, (b"ACGTTGCA" * 3000), bytes(np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 50000)])]
    recs.append(recs[-1][1000:9000][::-1].translate(bytes.maketrans(b"ACGT", b"TGCA")))
    seq, off = o.concat_records(recs)
    for sort_mode in ("msd", "lsd"):
        g, _ = assert_parity(seq, off, 31, mode=mode, num_bins=4, sort_mode=sort_mode)
        g.close()


def _pinned_copy(a):
    import torch

    t = torch.empty(max(1, a.nbytes), dtype=torch.uint8, pin_memory=True)
    v = t.numpy()[: a.nbytes].view(a.dtype)
    v[:] = a
    return t, v


@pytest.mark.parametrize("k", [21, 33])
def test_page_locked_intake(k):
    # records in page-locked memory are DMA'd to the device directly; mixed
    # with staged (pageable) calls the result equals one staged run
    recs = random_records(4242 + k, k, n_records=90, max_len=9000)
    seq, off = o.concat_records(recs)
    ref, _ = assert_parity(seq, off, k, num_bins=8)
    want = ref.states()
    ref.close()
    a, b = len(recs) // 3, 2 * len(recs) // 3
    parts = [o.concat_records(recs[:a]), o.concat_records(recs[a:b]), o.concat_records(recs[b:])]
    for pinned in ([True, False, True], [True, True, True], [False, True, True]):
        g = cg.Cf1Gpu(k=k, num_bins=8)
        keep = []
        for (ps, po), pin in zip(parts, pinned):
            if pin:
                t, ps = _pinned_copy(ps)
                keep.append(t)
            g.add_records(ps, po)
        g.run()
        assert np.array_equal(g.states(), want)
        g.close()


@pytest.mark.parametrize("k", [31, 63])
def test_oversized_subbucket(k):
    # a long homopolymer and a tandem repeat put tens of thousands of copies of
    # a few k-mers in one sub-bucket, beyond the shared-memory sort's capacity:
    # 64-bit keys are deduplicated through a shared-memory set first and stay
    # on the MSD path; 128-bit keys fall back to the LSD path
    recs = random_records(9, k, n_records=20, max_len=3000) + [b"A" * 30000, b"ACGT" * 9000]
    seq, off = o.concat_records(recs)
    g, _ = assert_parity(seq, off, k, num_bins=4)
    bits = g.stats()["sort_msd_bits"]
    assert (bits < 64) if k <= 32 else (bits == 2**64 - 1)
    g.close()


@pytest.mark.parametrize("bins", [1, 2])
def test_msd_two_passes(bins):
    # 5 M keys in one or two bins: the MSD split takes two multisplit passes
    x = cg.SynthInput(1)
    g, _ = assert_parity(x.seq, x.offsets, 31, num_bins=bins)
    assert g.stats()["sort_msd_bits"] > 8
    g.close()


@pytest.mark.parametrize("tile", [1024, 2048, 4096])
def test_superkmers_match_spec(tile):
    k = 31
    recs = random_records(11, k, n_records=50, max_len=8000)
    seq, off = o.concat_records(recs)
    g, ref = assert_parity(seq, off, k, sk_tile=tile, num_bins=32)
    # the device concatenates records of >= k bases, one placeholder after each
    cat = b"".join(r + b"N" for r in recs if len(r) >= k)
    pos, n, _ = o.superkmers(np.frombuffer(cat, np.uint8), k, tile)
    s = g.stats()
    assert s["n_superkmers"] == len(pos)
    assert s["n_kmer_occurrences"] == int(n.sum()) == ref.n_occ
    g.close()


@pytest.mark.parametrize("mode", ["bbhash", "learned"])
@pytest.mark.parametrize("k", [31, 63])
def test_query_state_words_and_host_image(k, mode):
    recs = random_records(21, k, n_records=40, max_len=5000)
    seq, off = o.concat_records(recs)
    g, ref = assert_parity(seq, off, k, mode=mode, num_bins=32)
    keys, st = g.dump_states()
    slots = g.query(keys)
    n = g.total_kmers()
    assert np.array_equal(np.sort(slots), np.arange(n, dtype=np.uint64))
    words = g.states()
    assert len(words) == (n + 11) // 12
    from_words = (words[slots // 12] >> (5 * (slots % 12)).astype(np.uint64)) & np.uint64(31)
    assert np.array_equal(from_words.astype(np.uint8), st)
    img = g.export_mphf()
    assert np.array_equal(cg.host_query(img, keys), slots)
    g.close()


def test_short_seqs_and_fasta():
    k = 31
    recs = [b"ACGT" * 5, b"ACGTTGCA" * 10, b"A" * 30, b"", b"GATTACA" * 20]
    names = ["short1 desc", "long1", "short2\tx", "empty", "long2"]
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "in.fa")
        with open(p, "w") as f:
            for nm, r in zip(names, recs):
                f.write(">" + nm + "\n")
                s = r.decode()
                for i in range(0, len(s), 7):
                    f.write(s[i:i + 7] + "\n")
        g = cg.Cf1Gpu(k=k, track_short_seqs=True)
        g.add_fasta(p)
        g.run()
        assert g.short_seqs() == [("short1", 20), ("short2", 30), ("empty", 0)]
        seq, off = o.concat_records(recs)
        ref = o.run(k, seq, off)
        keys, st = sort_by_key(*g.dump_states())
        assert np.array_equal(keys, ref.keys) and np.array_equal(st, ref.states)
        g.close()


@pytest.mark.parametrize("mode,batched", [("bbhash", False), ("learned", True)])
def test_autotuner_cache(mode, batched):
    # the first run of an input class measures the tile and the MSD width and
    # writes them to the cache; a second context reads them back; results
    # stay bit-exact either way
    recs = random_records(808, 31, n_records=120, max_len=9000)
    seq, off = o.concat_records(recs)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "tune.txt")
        with open(path, "w") as f:
            f.write("not a tuner line\ncf1tune 1 wide=0 sorted=0 size=3\n")  # ignored
        g, _ = assert_parity(seq, off, 31, mode=mode, batched=batched, num_bins=16, tuner_cache=path)
        s1 = g.stats()
        assert s1["tuner_state"] == 2 and s1["sk_tile"] in (1024, 2048, 4096)
        g.upload()
        g.run_resident()
        assert g.stats()["tuner_state"] == 1
        g.close()
        lines = [l for l in open(path).read().splitlines() if l.startswith("cf1tune 1 ")]
        assert len(lines) == 1 and f"sk_tile={s1['sk_tile']}" in lines[0]
        g2, _ = assert_parity(seq, off, 31, mode=mode, batched=batched, num_bins=16, tuner_cache=path)
        s2 = g2.stats()
        assert s2["tuner_state"] == 1 and s2["sk_tile"] == s1["sk_tile"]
        assert s2["sort_msd_bits"] == s1["sort_msd_bits"]
        g2.close()


@pytest.mark.parametrize("mode,batched,k,pinned", [("bbhash", False, 31, True), ("learned", True, 31, True),
                                                    ("bbhash", False, 63, False), ("bbhash", True, 21, True)])
def test_streamed_run_matches_staged(mode, batched, k, pinned):
    # several 1 MB input chunks (5 Mbp) and eight phase-4 stages; the words
    # equal those of the usual calls, and a second streamed run reuses the
    # context
    x = cg.SynthInput(1)
    ref = gpu_run(x.seq, x.offsets, k, mode=mode, batched=batched, num_bins=64)
    want = ref.states().copy()
    ref.close()
    g = cg.Cf1Gpu(k=k, mode=mode, batched=batched, num_bins=64)
    seq = x.seq
    keep = []
    if pinned:
        t, seq = _pinned_copy(np.asarray(x.seq, np.uint8))
        keep.append(t)
    for _ in range(2):
        out = None
        if pinned:
            t, out = _pinned_copy(np.zeros(len(want) + 3, np.uint64))
            keep.append(t)
        w = g.run_streamed(seq, x.offsets, out)
        assert np.array_equal(w, want)
    s = g.stats()
    assert s["ms_h2d"] > 0 and s["n_distinct"] == g.total_kmers()
    g.close()


def test_streamed_run_small_inputs_and_short_buffer():
    recs = random_records(2718, 31, n_records=50, max_len=4000)
    seq, off = o.concat_records(recs)
    g, ref = assert_parity(seq, off, 31, num_bins=8, track_short_seqs=True)
    want = g.states().copy()
    shorts = g.short_seqs()
    g.close()
    g = cg.Cf1Gpu(k=31, num_bins=8, track_short_seqs=True)
    assert np.array_equal(g.run_streamed(seq, off), want)
    assert [n for _, n in g.short_seqs()] == [n for _, n in shorts]
    with pytest.raises(cg.Cf1Error):
        g.run_streamed(seq, off, np.zeros(1, np.uint64))  # too small: an error after the run
    assert np.array_equal(g.states(), want)  # the results stay on the device
    keys, st = sort_by_key(*g.dump_states())
    assert np.array_equal(keys, ref.keys) and np.array_equal(st, ref.states)
    g.close()


def _read_bin_records(data: bytes):
    """Super k-mers of a bin file (the reader of src/superkmer.rs:283-298)."""
    out, i = [], 0
    while i < len(data):
        n = data[i] | (data[i + 1] << 8)
        nb = (n + 3) // 4
        packed = data[i + 2: i + 2 + nb]
        out.append("".join("ACGT"[(packed[j // 4] >> (6 - 2 * (j % 4))) & 3] for j in range(n)))
        i += 2 + nb
    assert i == len(data)
    return out


def _canon(kmer: str) -> str:
    rc = kmer.translate(str.maketrans("ACGT", "TGCA"))[::-1]
    return min(kmer, rc)


@pytest.mark.parametrize("k", [21, 31, 45])
def test_bin_files_match_routing(k):
    # every k-mer occurrence is in exactly one exported super k-mer, and a
    # bin file's k-mers are the distinct k-mers the device put in that bin
    recs = random_records(31337 + k, k, n_records=40, max_len=3000)
    seq, off = o.concat_records(recs)
    g, ref = assert_parity(seq, off, k, num_bins=8, mode="learned")
    keys, _ = g.dump_states()
    counts = g.bin_distinct_counts()
    ends = np.cumsum(counts)
    occ = 0
    with tempfile.TemporaryDirectory() as d:
        g.write_bin_files(d)
        for b in range(8):
            data = open(os.path.join(d, f"cf1_bin_{b:05d}.bin"), "rb").read()
            assert data == g.export_bin(b)
            kmers = set()
            for sk in _read_bin_records(data):
                assert len(sk) >= k
                occ += len(sk) - k + 1
                for i in range(len(sk) - k + 1):
                    kmers.add(_canon(sk[i: i + k]))
            lo = int(ends[b] - counts[b])
            want = set()
            for kk in keys[lo: int(ends[b])]:
                if keys.ndim == 1:
                    v = int(kk)
                else:
                    v = int(kk[0]) | (int(kk[1]) << 64)
                want.add("".join("ACGT"[(v >> (2 * (k - 1 - j))) & 3] for j in range(k)))
            assert kmers == want, f"bin {b}"
    assert occ == ref.n_occ
    g.close()


def test_deterministic_repeat_runs():
    recs = random_records(3, 31, n_records=100, max_len=8000)
    seq, off = o.concat_records(recs)
    g = gpu_run(seq, off, 31, num_bins=64)
    w1 = g.states().copy()
    g.upload()
    g.run_resident()
    w2 = g.states()
    assert np.array_equal(w1, w2)
    g.close()


@pytest.mark.parametrize("mode", ["bbhash", "learned"])
def test_workload1_full_size(mode):
    x = cg.SynthInput(1)
    g, _ = assert_parity(x.seq, x.offsets, 31, mode=mode, num_bins=128)
    g.close()


@pytest.mark.parametrize("cfg,scale,k,flags", [
    (2, 0.05, 31, dict(track_short_seqs=True)),
    (3, 0.1, 31, dict()),
    (4, 0.01, 63, dict()),
    (5, 0.005, 31, dict(num_bins=256)),
])
@pytest.mark.parametrize("mode", ["bbhash", "learned"])
def test_scaled_workloads(cfg, scale, k, flags, mode):
    x = cg.SynthInput(cfg, scale=scale)
    kw = dict(num_bins=128)
    kw.update(flags)
    g, _ = assert_parity(x.seq, x.offsets, k, mode=mode, **kw)
    g.close()


# ---- learned index: gradients against the CPU oracle, gain of the network ----
def test_learned_gradients_match_cpu():
    rng = np.random.default_rng(0)
    for trial in range(5):
        params = rng.normal(0, 0.7, 49).astype(np.float32)
        n = int(rng.integers(1, 3000))
        x = rng.random(n).astype(np.float32)
        t = np.sort(rng.random(n)).astype(np.float32)
        loss_g, grad_g = cg.learned_grad(params, x, t)
        loss_c, grad_c = o.mlp_grad(params, x, t)
        # fp32 device accumulation vs fp64 CPU: relative 1e-4 of the gradient scale
        scale = max(1e-6, float(np.abs(grad_c).max()))
        assert abs(loss_g - loss_c) <= 1e-4 * max(1.0, loss_c)
        assert np.abs(grad_g - grad_c).max() <= 1e-4 * scale


def test_learned_grad_q_matches_cpu():
    """The gradient the trainer applies -- through the softmax knot widths,
    w1 = 1/d and b1 = -t/d -- against the double-precision oracle."""
    rng = np.random.default_rng(3)
    for trial in range(8):
        if trial == 0:  # the trainer's starting point: the identity root
            q = np.concatenate([np.zeros(16), np.full(16, 1 / 16), [0.0]])
        else:
            q = np.concatenate([rng.normal(0, 0.8, 16), np.abs(rng.normal(1 / 16, 0.05, 16)), [rng.normal(0, 0.1)]])
        q = q.astype(np.float32)
        n = int(rng.integers(1, 4097))
        x = rng.random(n).astype(np.float32)
        t = np.sort(rng.random(n)).astype(np.float32)
        loss_g, grad_g = cg.learned_grad_q(q, x, t)
        loss_c, grad_c = o.learned_grad_q(q.astype(np.float64), x, t)
        scale = max(1e-6, float(np.abs(grad_c).max()))
        assert abs(loss_g - loss_c) <= 1e-4 * max(1.0, loss_c)
        # fp32 device arithmetic vs the fp64 oracle: 1e-4 of the gradient scale, logits included
        assert np.abs(grad_g - grad_c).max() <= 1e-4 * scale, (trial, np.abs(grad_g - grad_c).argmax())


def test_learned_network_gain():
    """The trained root shrinks the search windows of the index without it."""
    x = cg.SynthInput(5, scale=0.005)
    res = {}
    for steps in (-1, 0):  # -1: identity root (no network), 0: default training
        g = cg.Cf1Gpu(k=31, num_bins=64, mode="learned", learned_train_steps=steps, learned_max_err=1 << 30)
        g.add_records(x.seq, x.offsets)
        g.run()
        g.verify_bijection()
        res[steps] = (g.learned_stats(), sort_by_key(*g.dump_states()), g.stats())
        g.close()
    untrained, trained = res[-1][0], res[0][0]
    assert trained["train_loss"] < untrained["train_loss"]
    assert trained["mean_window"] < untrained["mean_window"]
    assert np.array_equal(res[-1][1][0], res[0][1][0]) and np.array_equal(res[-1][1][1], res[0][1][1])
