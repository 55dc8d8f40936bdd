"""The committed golden fixtures (tests/golden, written by make_golden.py):
the oracle and the GPU path must still produce exactly the frozen per-k-mer
states, and the phase-5 restatement the frozen canonical output."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as o
from oracle import phase5 as p5
from tests.gpu_util import gpu_run, sort_by_key

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
K_VALUES = (15, 31, 63)


def load(k):
    with np.load(os.path.join(GOLDEN, f"states_k{k}.npz")) as z:
        return {n: z[n] for n in z.files}


def records_of(seq, off):
    return [bytes(seq[int(off[i]):int(off[i + 1])]) for i in range(len(off) - 1)]


@pytest.mark.parametrize("k", K_VALUES)
def test_oracle_reproduces_golden_states(k):
    g = load(k)
    for method in (0, 1):
        ref = o.run(k, g["seq"], g["offsets"], nthreads=2, method=method)
        assert np.array_equal(ref.keys, g["keys"])
        assert np.array_equal(ref.states, g["states"])
        assert ref.n_occ == int(g["n_occ"])


def test_phase5_reproduces_golden_output():
    with open(os.path.join(GOLDEN, "phase5_k31.json")) as f:
        doc = json.load(f)
    k = doc["k"]
    g = load(k)
    ref = o.run(k, g["seq"], g["offsets"], nthreads=2)
    named = [(f"seq{i}", r) for i, r in enumerate(records_of(g["seq"], g["offsets"]))]
    out = p5.extract_and_output(named, k, lambda q: np.searchsorted(ref.keys, q), ref.state_words, poly_n_stretch=True)
    segs, tilings = p5.canonical(out)
    assert segs == doc["segments"]
    assert [[n, [t if isinstance(t, str) else list(t) for t in toks]] for n, toks in tilings] == doc["tilings"]
    assert out.meta == doc["meta"]


@pytest.mark.gpu
@pytest.mark.parametrize("k", K_VALUES)
@pytest.mark.parametrize("mode,update", [("bbhash", "phase3"), ("learned", "phase3"), ("bbhash", "sideset"),
                                         ("learned", "sideset"), ("bbhash", "cas")])
def test_gpu_reproduces_golden_states(k, mode, update):
    g = load(k)
    run = gpu_run(g["seq"], g["offsets"], k, mode=mode, state_update=update, num_bins=16)
    try:
        assert run.total_kmers() == len(g["states"])
        keys, states = sort_by_key(*run.dump_states())
        assert np.array_equal(keys, g["keys"])
        assert np.array_equal(states, g["states"])
    finally:
        run.close()
