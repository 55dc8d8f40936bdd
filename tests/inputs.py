"""Small seeded test inputs with the edge cases the classifier must handle.

Records mix: i.i.d. bases, lowercase, placeholder runs (N and other letters),
records shorter than k, homopolymers (direct-repeat self loops), dinucleotide
repeats (inverted-repeat self loops), exact repeats on both strands (shared
k-mers with conflicting neighbours) and records of exactly k bases.
"""
import numpy as np

ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)


def _rc(s: bytes) -> bytes:
    return s.translate(bytes.maketrans(b"ACGTacgt", b"TGCAtgca"))[::-1]


def random_records(seed: int, k: int, n_records: int = 40, max_len: int = 3000, edge_cases: bool = True):
    rng = np.random.default_rng(seed)
    recs = []
    pool = []
    for i in range(n_records):
        kind = rng.integers(0, 10) if edge_cases else 0
        L = int(rng.integers(1, max_len))
        s = bytearray(ACGT[rng.integers(0, 4, L)].tobytes())
        if kind == 1 and L > 10:  # placeholder runs
            for _ in range(int(rng.integers(1, 5))):
                a = int(rng.integers(0, L))
                b = min(L, a + int(rng.integers(1, 2 * k + 3)))
                s[a:b] = b"N" * (b - a)
            if L > 3:
                s[int(rng.integers(0, L))] = b"XRn"[int(rng.integers(0, 3))]
        elif kind == 2:  # lowercase stretch
            a = int(rng.integers(0, L))
            s[a:] = bytes(s[a:]).lower()
        elif kind == 3:  # short record
            s = s[: int(rng.integers(0, max(1, k)))]
        elif kind == 4:  # homopolymer inside
            a = int(rng.integers(0, L))
            s[a:a] = bytes([ACGT[rng.integers(0, 4)]]) * int(rng.integers(k, 3 * k + 5))
        elif kind == 5:  # dinucleotide repeat inside (AT / CG are their own rc)
            a = int(rng.integers(0, L))
            unit = [b"AT", b"TA", b"CG", b"GC", b"AC"][int(rng.integers(0, 5))]
            s[a:a] = unit * int(rng.integers(k, 2 * k + 5))
        elif kind == 6 and pool:  # copy of an earlier piece, possibly rc, with a mutation
            src = pool[int(rng.integers(0, len(pool)))]
            piece = bytearray(src if rng.integers(0, 2) else _rc(src))
            if len(piece) > 2 and rng.integers(0, 2):
                j = int(rng.integers(0, len(piece)))
                piece[j] = ACGT[rng.integers(0, 4)]
            a = int(rng.integers(0, L))
            s[a:a] = piece
        elif kind == 7:  # exactly k bases
            s = s[:k] if len(s) >= k else s + bytes(ACGT[rng.integers(0, 4, k - len(s))].tobytes())
        elif kind == 8:  # exact k+1 / isolated k-mers between Ns
            s = bytearray()
            for _ in range(int(rng.integers(1, 6))):
                s += bytes(ACGT[rng.integers(0, 4, k + int(rng.integers(0, 2)))].tobytes()) + b"N"
        if len(s) > 2 * k:
            a = int(rng.integers(0, len(s) - k))
            pool.append(bytes(s[a:a + k + int(rng.integers(0, 3 * k))]).upper().replace(b"N", b"A"))
        recs.append(bytes(s))
    return recs
