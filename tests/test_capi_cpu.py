"""CPU-only checks of the C ABI library: it loads, exports every symbol the
header declares, rejects bad options, and fails loudly without a GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import cf1_rs_b200 as cg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "cf1gpu.h")).read()
    return sorted(set(re.findall(r"\b(cf1gpu_\w+)\s*\(", text)))


def test_header_symbols_exported():
    L = cg.lib()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    assert sorted(cg.EXPORTED) == syms


def test_version():
    assert b"sm_100a" in cg.lib().cf1gpu_version()


def test_struct_sizes_match_header():
    # cf1gpu_opts: 6 u32, a pointer, 4 u32 + 4 reserved
    assert C.sizeof(cg.Opts) == 6 * 4 + 8 + 8 * 4
    assert C.sizeof(cg.Stats) == 20 * 8 + 12 * 8


@pytest.mark.parametrize("k", [0, 2, 32, 64, 65])
def test_invalid_k_rejected(k):
    L = cg.lib()
    o = cg.Opts()
    L.cf1gpu_default_opts(C.byref(o))
    o.k = k
    h = C.c_void_p()
    assert L.cf1gpu_create(C.byref(o), C.byref(h)) == cg.ERR_INVALID_ARG
    assert b"k must be odd" in L.cf1gpu_last_error(None)


def test_invalid_bins_rejected():
    L = cg.lib()
    o = cg.Opts()
    L.cf1gpu_default_opts(C.byref(o))
    for nb in (0, 4097):
        o.num_bins = nb
        h = C.c_void_p()
        assert L.cf1gpu_create(C.byref(o), C.byref(h)) == cg.ERR_INVALID_ARG


def test_invalid_state_update_rejected():
    L = cg.lib()
    o = cg.Opts()
    L.cf1gpu_default_opts(C.byref(o))
    assert o.state_update == 0  # side sets joined in phase 3 by default
    o.state_update = 3
    h = C.c_void_p()
    assert L.cf1gpu_create(C.byref(o), C.byref(h)) == cg.ERR_INVALID_ARG
    assert b"state_update" in L.cf1gpu_last_error(None)


def test_null_arguments():
    L = cg.lib()
    assert L.cf1gpu_create(None, None) == cg.ERR_INVALID_ARG
    assert L.cf1gpu_run_phases_1_4(None) == cg.ERR_INVALID_ARG
    assert L.cf1gpu_mphf_host_query(None, 0, None, 0, None) == cg.ERR_INVALID_ARG


def test_host_query_rejects_garbage_image():
    img = np.zeros(64, np.uint64)
    with pytest.raises(cg.Cf1Error):
        cg.host_query(img, np.zeros(3, np.uint64))


def test_no_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(cg.Cf1Error) as e:
        cg.Cf1Gpu(k=31)
    assert e.value.status == cg.ERR_CUDA


def test_synthetic_inputs_deterministic():
    a = cg.SynthInput(3, scale=0.002, nthreads=3)
    b = cg.SynthInput(3, scale=0.002, nthreads=7)
    assert np.array_equal(a.seq, b.seq) and np.array_equal(a.offsets, b.offsets)
    assert a.n_records == 24
    # poly-N stretches present, GC near 41%
    s = a.seq
    acgt = s[s != ord("N")]
    gc = np.isin(acgt, np.frombuffer(b"CG", np.uint8)).mean()
    assert 0.38 < gc < 0.44
    assert (s == ord("N")).sum() >= 1000


def test_synthetic_transcriptome_shape():
    t = cg.SynthInput(2, scale=0.01)
    lens = np.diff(t.offsets)
    assert t.n_records == 1000
    assert lens.min() >= 200 and lens.max() <= 100000
    assert 600 < np.median(lens) < 3000
