"""Writes the committed golden fixtures of this directory (test data only).

    python tests/golden/make_golden.py

For each k in K_VALUES: a small seeded input with every edge case of
``tests/inputs.random_records`` (placeholder runs, lowercase, records shorter
than k and of exactly k bases, homopolymers, dinucleotide repeats, repeats on
both strands), its distinct canonical k-mers in increasing order and their
5-bit states.  The states come from the CPU oracle and are written only when
its two methods -- the restatement of src/classify.rs and the independent
per-side join fold -- agree on every k-mer.  ``phase5_k31.json`` holds the
canonicalised phase-5 output (src/output.rs, restated in oracle/phase5.py)
of the k = 31 input over the oracle's structures, with poly-N gaps.

The fixtures freeze these results: tests compare the oracle and the GPU path
with them, so a change to either shows against data that no longer depends
on the code under test.  The cf1-rs reference itself cannot be run here (no
Rust toolchain), and its own tests hold no such vectors.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as o  # noqa: E402
from oracle import phase5 as p5  # noqa: E402
from tests.inputs import random_records  # noqa: E402

K_VALUES = (15, 31, 63)
SEED = 20260101
N_RECORDS, MAX_LEN = 30, 1500


def records(k):
    return random_records(SEED + k, k, n_records=N_RECORDS, max_len=MAX_LEN)


def main():
    for k in K_VALUES:
        recs = records(k)
        seq, off = o.concat_records(recs)
        a = o.run(k, seq, off, nthreads=4, method=0)
        b = o.run(k, seq, off, nthreads=4, method=1)
        if not (np.array_equal(a.keys, b.keys) and np.array_equal(a.states, b.states)):
            raise SystemExit(f"k={k}: the two oracle methods disagree; no fixture written")
        np.savez_compressed(os.path.join(HERE, f"states_k{k}.npz"), seq=seq, offsets=off, keys=a.keys,
                            states=a.states, n_occ=np.uint64(a.n_occ))
        print(f"k={k}: {len(seq)} bytes, {len(a.states)} distinct k-mers")
    k = 31
    recs = records(k)
    seq, off = o.concat_records(recs)
    ref = o.run(k, seq, off, nthreads=4)
    named = [(f"seq{i}", r) for i, r in enumerate(recs)]
    out = p5.extract_and_output(named, k, lambda q: np.searchsorted(ref.keys, q), ref.state_words, poly_n_stretch=True)
    segs, tilings = p5.canonical(out)
    doc = {"k": k, "segments": segs,
           "tilings": [[name, [t if isinstance(t, str) else [t[0], t[1]] for t in toks]] for name, toks in tilings],
           "meta": out.meta}
    with open(os.path.join(HERE, "phase5_k31.json"), "w") as f:
        json.dump(doc, f, indent=0)
    print(f"phase 5, k=31: {len(segs)} segments")


if __name__ == "__main__":
    main()
