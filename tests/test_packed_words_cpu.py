"""Packed multisplit words on the host: tests/packed_words_check.cpp is built
against the library's cf1_common.cuh (the same pay_code / pay_byte /
KEY_SPREAD_INV the kernels use) and run; it checks that every side-set byte
of a single occurrence survives its 6-bit code and that a packed word gives
back the next digit, the key's hash, the key and the byte."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "cf1_rs_b200", "csrc")


def test_packed_words_round_trip(tmp_path):
    cxx = shutil.which("g++")
    inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    if not cxx or not os.path.exists(os.path.join(inc, "cuda_runtime.h")):
        pytest.skip("needs g++ and the CUDA runtime headers")
    exe = str(tmp_path / "packed_words_check")
    subprocess.run([cxx, "-std=c++17", "-O1", f"-I{inc}", f"-I{CSRC}", os.path.join(HERE, "packed_words_check.cpp"),
                    "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
