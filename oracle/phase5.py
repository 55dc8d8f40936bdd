"""Phase 5 of cf1-rs (unitig extraction and the GFA-reduced output) restated
on the CPU -- test infrastructure only, like the rest of ``oracle/``.

The reference's phase 5 (src/output.rs) reads the input again and, over the
MPHF and the state vector that phases 1-4 built, walks every record's k-mers,
cuts them into maximal unitigs, claims each unitig once through the state
vector's "outputted" states, and writes

* ``.cf_seg``: one line per unitig, ``<id>\\t<sequence>`` (output.rs:740-760),
* ``.cf_seq``: one line per record of k bases or more,
  ``Reference:<file>_Sequence:<name>\\t<id><+|-> ...`` (output.rs:206-258).

It does not run here (it is Rust and cargo is absent), so this module
restates it, function by function, to show that the structures the GPU path
hands over -- the host image of the MPHF (``cf1gpu_export_mphf`` +
``cf1gpu_mphf_host_query``) and the state words (``cf1gpu_copy_states``) --
drive it to the same output as the oracle's own structures.  Unitig ids are
MPHF slots, so two runs compare after canonicalisation (:func:`canonical`):
each id becomes its segment's canonical spelling (the smaller of the
sequence and its reverse complement); the +/- directions compare k-mers, not
slots, and must match as they are.

The walk is serial: the reference spreads records (and chunks of records of
4 Mbp or more) over threads, and its own comments (output.rs:280-289, 384-399)
state that the chunked tiling equals the serial one.  With several threads
the order of the ``.cf_seq`` lines and which occurrence of a unitig claims it
first can vary; the canonical form does not depend on either.
"""
from __future__ import annotations

import numpy as np

# StateClass (src/state.rs:6-11)
SISO, MISO, SIMO, MIMO = 0, 1, 2, 3

# STATE_CLASS_TABLE (src/state.rs:250-270): the class of every 5-bit code
_CLASS = [SISO] * 32
_CLASS[3] = MIMO
for _c in (4, 5, 6, 7, 13):
    _CLASS[_c] = MISO
for _c in (8, 9, 10, 11, 14):
    _CLASS[_c] = SIMO
_CLASS[15] = MIMO

# OUTPUTTED_TABLE (src/state.rs:274-297)
_OUTPUTTED = [0] * 32
_OUTPUTTED[3] = 0b01111
for _c in (4, 5, 6, 7):
    _OUTPUTTED[_c] = 0b01101
for _c in (8, 9, 10, 11):
    _OUTPUTTED[_c] = 0b01110
_OUTPUTTED[12], _OUTPUTTED[13], _OUTPUTTED[14], _OUTPUTTED[15] = 0b01100, 0b01101, 0b01110, 0b01111
for _c in range(16, 32):
    _OUTPUTTED[_c] = 0b01100

_BASE = {ord(c): v for c, v in zip("ACGTacgt", (0, 1, 2, 3, 0, 1, 2, 3))}  # dna.rs:64-78
_COMP = {ord(c): v for c, v in zip("ACGTacgt", "TGCATGCA")}  # dna.rs:93-104 (else 'N')


def is_placeholder(b: int) -> bool:
    """dna.rs:40-44: anything but ACGTacgt."""
    return b not in _BASE


def to_upper(b: int) -> str:
    """dna.rs:46-54."""
    return chr(b if b <= ord("T") else b - (ord("a") - ord("A")))


def revcomp(s: str) -> str:
    return s[::-1].translate(str.maketrans("ACGTacgt", "TGCAtgca"))


def is_unipath_start(cls, fwd, prev_cls, prev_fwd) -> bool:
    """output.rs:79-112."""
    if cls == MIMO:
        return True
    if fwd:
        if cls == MISO:
            return True
    elif cls == SIMO:
        return True
    if prev_cls == MIMO:
        return True
    if prev_fwd:
        if prev_cls == SIMO:
            return True
    elif prev_cls == MISO:
        return True
    return False


def is_unipath_end(cls, fwd, next_cls, next_fwd) -> bool:
    """output.rs:114-148."""
    if cls == MIMO:
        return True
    if fwd:
        if cls == SIMO:
            return True
    elif cls == MISO:
        return True
    if next_cls == MIMO:
        return True
    if next_fwd:
        if next_cls == MISO:
            return True
    elif next_cls == SIMO:
        return True
    return False


class _States:
    """The state vector's get / compare-and-swap (state_vector.rs:36-70) over
    a copy of the words, single-threaded."""

    def __init__(self, words):
        self.w = [int(x) for x in np.asarray(words, np.uint64)]

    def get(self, i: int) -> int:
        return (self.w[i // 12] >> (5 * (i % 12))) & 31

    def set(self, i: int, code: int):
        sh = 5 * (i % 12)
        self.w[i // 12] = (self.w[i // 12] & ~(31 << sh)) | (code << sh)


class Phase5Out:
    def __init__(self):
        self.segs = []      # (unitig id, sequence) in claim order: the .cf_seg lines
        self.tilings = []   # (record name, tiling text): the .cf_seq lines
        self.unitigs = []   # per tiled record: [(id, fwd, start k-mer, end k-mer)]
        self.meta = dict(unipath_count=0, kmer_count=0, max_len=0, min_len=None, sum_len=0)

    def seg_text(self) -> str:
        return "".join(f"{i}\t{s}\n" for i, s in self.segs)

    def seq_text(self) -> str:
        return "".join(f"Reference:1_Sequence:{n}\t{t}\n" for n, t in self.tilings)


def _windows(seq: bytes, k: int):
    """Per window start: (fw, rc) as integers (first base in the top bits,
    kmer.rs:110-131, 161-210) and whether the window holds no placeholder."""
    n = len(seq)
    mask = (1 << (2 * k)) - 1
    fw = rc = 0
    run = 0  # valid bases ending here
    out_fw, out_rc, ok = [0] * (n - k + 1), [0] * (n - k + 1), [False] * (n - k + 1)
    for i, b in enumerate(seq):
        v = _BASE.get(b, 0)
        run = run + 1 if b in _BASE else 0
        fw = ((fw << 2) | v) & mask
        rc = (rc >> 2) | ((3 - v) << (2 * k - 2))
        s = i - k + 1
        if s >= 0:
            out_fw[s], out_rc[s], ok[s] = fw, rc, run >= k
    return out_fw, out_rc, ok


def _key_array(keys, k):
    if k <= 32:
        return np.array(keys, dtype=np.uint64)
    m = (1 << 64) - 1
    return np.array([[x & m, x >> 64] for x in keys], dtype=np.uint64).reshape(-1, 2)


def extract_and_output(records, k: int, slot_of, state_words, poly_n_stretch: bool = False) -> Phase5Out:
    """Phase 5 over `records` (a list of (name, bytes)), an MPHF given as
    ``slot_of(keys) -> slots`` (canonical keys as uint64 [n], or (lo, hi)
    pairs [n, 2] for k > 32) and the state vector's words (output.rs:152-354,
    358-404, 485-782)."""
    st = _States(state_words)
    out = Phase5Out()
    for name, seq in records:
        seq = bytes(seq)
        n = len(seq)
        if n < k:  # output.rs:186-188
            continue
        fw, rc, ok = _windows(seq, k)
        idx = [i for i, v in enumerate(ok) if v]
        can = {i: min(fw[i], rc[i]) for i in idx}
        slots = {}
        if idx:
            s = np.asarray(slot_of(_key_array([can[i] for i in idx], k)), dtype=np.uint64)
            slots = {i: int(x) for i, x in zip(idx, s)}

        def ann(i):  # AnnotatedKmer::new (directed_kmer.rs:80-97): class and direction
            return _CLASS[st.get(slots[i])], fw[i] == can[i]

        unitigs = []

        def output_unitig(a, b):  # output_gfa_unitig, output.rs:714-782
            uid = slots[a] if can[a] <= can[b] else slots[b]  # bucket_id of the smaller flanking k-mer
            fwd = fw[a] < rc[b]
            unitigs.append((uid, fwd, a, b))
            code = st.get(uid)
            if not 12 <= code <= 15:  # not outputted: claim it
                st.set(uid, _OUTPUTTED[code])
                ln = b - a + k
                if fwd:
                    text = "".join(to_upper(seq[a + o]) for o in range(ln))
                else:
                    text = "".join(_COMP.get(seq[b + k - 1 - o], "N") for o in range(ln))
                out.segs.append((uid, text))
                m = out.meta
                m["unipath_count"] += 1
                m["kmer_count"] += b - a + 1
                m["max_len"] = max(m["max_len"], ln)
                m["min_len"] = ln if m["min_len"] is None else min(m["min_len"], ln)
                m["sum_len"] += ln

        def contiguous(start, right_end):  # output_unitigs_contiguous, output.rs:506-712
            i = start
            cur = ann(i)
            no_left = i == 0 or is_placeholder(seq[i - 1])
            no_right = i + k == n or is_placeholder(seq[i + k])
            if no_left and no_right:
                output_unitig(i, i)
                return i + k
            if no_right:  # (both sides missing was handled above)
                if is_unipath_start(*cur, *ann(i - 1)):
                    output_unitig(i, i)
                return i + k
            nxt = ann(i + 1)
            on, ustart = False, i
            if no_left:
                on, ustart = True, i
            elif is_unipath_start(*cur, *ann(i - 1)):
                on, ustart = True, i
            if on and is_unipath_end(*cur, *nxt):
                output_unitig(ustart, i)
                on = False
            i += 1
            while True:
                if not on and i > right_end:
                    break
                prev, cur = cur, nxt
                if is_unipath_start(*cur, *prev):
                    on, ustart = True, i
                if i + k == n or is_placeholder(seq[i + k]):
                    if on:
                        output_unitig(ustart, i)
                    return i + k
                nxt = ann(i + 1)
                if on and is_unipath_end(*cur, *nxt):
                    output_unitig(ustart, i)
                    on = False
                i += 1
            return i + k

        right_end = n - k  # extract_unitigs_from_seq, output.rs:358-404
        i = 0
        while i <= right_end:
            while i <= right_end and not ok[i]:  # search_valid_kmer, output.rs:485-504
                i += 1
            if i > right_end:
                break
            i = contiguous(i, right_end)

        tokens = []  # the tiling line, output.rs:206-258
        for j, (uid, fwd, a, b) in enumerate(unitigs):
            if j == 0:
                if poly_n_stretch and a > 0:
                    tokens.append(f"N{a}")
            elif poly_n_stretch and unitigs[j - 1][3] + 1 != a:
                gap = a - unitigs[j - 1][3]
                if gap >= k + 1:
                    tokens.append(f"N{gap - k}")
            tokens.append(f"{uid}{'+' if fwd else '-'}")
        out.tilings.append((name, " ".join(tokens)))
        out.unitigs.append(unitigs)
    return out


def canonical(out: Phase5Out):
    """The slot-free form of a phase-5 output: the sorted canonical segment
    spellings, and per record its tiling with each id replaced by its
    segment's canonical spelling (directions and N gaps kept)."""
    spell = {}
    for uid, s in out.segs:
        if uid in spell:
            raise ValueError(f"unitig {uid} written twice")
        spell[uid] = min(s, revcomp(s))
    segs = sorted(spell.values())
    tilings = []
    for name, t in out.tilings:
        toks = []
        for tok in t.split():
            if tok.startswith("N"):
                toks.append(tok)
            else:
                toks.append((spell[int(tok[:-1])], tok[-1]))
        tilings.append((name, toks))
    return segs, tilings
