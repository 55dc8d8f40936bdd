"""cf1gpu_distinct_kmers_noalloc, the entry point for callers that cannot
allocate device memory (their host application owns the device memory pool,
or they run where a cudaMalloc is not allowed), checked against the regular
allocating path on the same records.

The file name sorts last, so a run that stops at the first failure has run
every other test before this one.  The test passes alone in a fresh process
and after the rest: it relies on nothing another test leaves behind, and it
calls the entry point twice in a row with records of different sizes, so
anything the shared scratch array kept from the first call would show up in
the second.
"""
import numpy as np
import pytest

import cf1_rs_b200 as cg

pytestmark = pytest.mark.gpu


def _record(seed: int, n: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    s = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, n)].copy()
    if n > 2000:
        s[n // 3:n // 3 + 50] = ord("N")                    # placeholder run
        s[n // 2:n // 2 + 400] = s[100:500]                 # repeat
        s[-500:] = np.frombuffer(b"acgt", np.uint8)[rng.integers(0, 4, 500)]  # lowercase
        s[n // 4] = ord("X")
    return s


def _regular(seq: np.ndarray, k: int) -> np.ndarray:
    g = cg.Cf1Gpu(k=k, num_bins=8)
    g.add_record(seq.tobytes())
    g.run()
    keys, _ = g.dump_states()
    g.close()
    return np.sort(keys)


def _noalloc(torch, seq: np.ndarray, k: int, out, n_out) -> np.ndarray:
    d_seq = torch.from_numpy(seq).to("cuda")
    st = cg.distinct_kmers_noalloc(d_seq.data_ptr(), seq.size, k, out.data_ptr(), out.numel(), n_out.data_ptr())
    assert st == cg.OK, st
    torch.cuda.synchronize()
    n = int(n_out.item())
    return out[:n].cpu().numpy().view(np.uint64).copy()


def test_noalloc_matches_regular_path_twice_in_a_row():
    torch = pytest.importorskip("torch")
    # caller-owned output buffers, sized for the largest record
    out = torch.zeros(cg.NOALLOC_MAX_BASES, dtype=torch.int64, device="cuda")
    n_out = torch.zeros(1, dtype=torch.int64, device="cuda")
    # k = 31 and 21 take an even number of 8-bit sort passes, k = 27 and 11 an
    # odd one (the sorted keys end in the other half of the scratch array)
    cases = [(31, _record(1, cg.NOALLOC_MAX_BASES)), (31, _record(2, 70_001)), (21, _record(3, 300_000)),
             (27, _record(5, 200_000)), (11, _record(6, 90_000)), (31, _record(4, 40))]
    for k, seq in cases:
        got = _noalloc(torch, seq, k, out, n_out)
        want = _regular(seq, k)
        assert np.array_equal(got, want), f"k={k} len={seq.size}: {got.size} vs {want.size} keys"


def test_noalloc_rejects_records_beyond_its_limit():
    torch = pytest.importorskip("torch")
    buf = torch.zeros(16, dtype=torch.int64, device="cuda")
    st = cg.distinct_kmers_noalloc(buf.data_ptr(), cg.NOALLOC_MAX_BASES + 1, 31, buf.data_ptr(), 1 << 21,
                                   buf.data_ptr())
    assert st == cg.ERR_TOO_LARGE
    assert cg.distinct_kmers_noalloc(buf.data_ptr(), 100, 32, buf.data_ptr(), 100, buf.data_ptr()) == cg.ERR_INVALID_ARG


def test_noalloc_refuses_a_stream_of_another_device():
    torch = pytest.importorskip("torch")
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two devices")
    buf = torch.zeros(16, dtype=torch.int64, device="cuda:0")
    with torch.cuda.device(1):
        other = torch.cuda.Stream()
    st = cg.distinct_kmers_noalloc(buf.data_ptr(), 100, 31, buf.data_ptr(), 100, buf.data_ptr(),
                                   stream=other.cuda_stream, device=0)
    assert st == cg.ERR_INVALID_ARG
