"""The C++ API (include/turbo_b200.hpp) with the reference's own test cases: tests/cpp/test_api.cpp
compiled with g++ against the header, libturbo_b200.so and the oracle (the reference's CPU
decoder restated), then run: codec cases on the CPU, decoder cases on the GPU."""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(ROOT, "turbo_cpp_b200", "lib")
ORACLE_DIR = os.path.join(ROOT, "oracle")
REF_LIB = os.path.join(ORACLE_DIR, "_ref", "libturbo_ref.so")


@pytest.fixture(scope="module")
def test_api(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ is not available")
    exe = str(tmp_path_factory.mktemp("cpp") / "test_api")
    cmd = ["g++", "-std=c++20", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "test_api.cpp"), "-o", exe,
           "-L", LIB_DIR, "-lturbo_b200", f"-Wl,-rpath,{LIB_DIR}",
           os.path.join(ORACLE_DIR, "liboracle.so"), f"-Wl,-rpath,{ORACLE_DIR}", "-ldl"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe


def _run(exe, mode):
    args = [exe, mode] + ([REF_LIB] if os.path.exists(REF_LIB) else [])
    r = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.stdout + r.stderr)[-3000:]
    assert "checks passed" in r.stdout


def test_cpp_api_codec_cases(test_api):
    _run(test_api, "cpu")


@pytest.mark.gpu
def test_cpp_api_decoder_cases(test_api):
    _run(test_api, "gpu")
