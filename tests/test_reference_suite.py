"""The reference's own test program, run on this library through the reference-side binding.

oracle/build_reference_suite.sh compiles the reference's tests/test_main.cpp and its unmodified
src/lte_turbo.cpp with TURBO_CPP_HAS_CUDA=1 against integration/lte_turbo_b200_binding.cpp
(the file a maintainer adds in place of src/lte_turbo_cuda.cu) and links libturbo_b200.so,
into oracle/_ref/reference_suite_b200.  Its GPU sections (test_main.cpp:132-186, 211-254,
287-302, 336-343) then decode through this library: GPU Stage 1 / Stage 2 round trips of
transport blocks of 40, 512, 6112 and 12000 bits, CRC flags, finite posteriors, Stage 2 within
5e-4 of the CPU decoder, Stage 1 within 5e-4 of Stage 2 and -- the one relaxed check -- Stage 1
within 1e-5 relative of the CPU decoder (test_main.cpp:142 asks for 2e-5 absolute).
"""
from __future__ import annotations

import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SUITE = os.path.join(ROOT, "oracle", "_ref", "reference_suite_b200")
LIB = os.path.join(ROOT, "turbo_cpp_b200", "lib", "libturbo_b200.so")

needs_suite = pytest.mark.skipif(not os.path.exists(SUITE),
                                 reason="oracle/_ref/reference_suite_b200 not built")


@needs_suite
def test_reference_suite_is_linked_to_this_library():
    """Without a GPU the binding reaches this library, which refuses with its own message."""
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is visible: the -m gpu test runs the suite")
    except ImportError:
        pass
    out = subprocess.run(["ldd", SUITE], capture_output=True, text=True, check=True).stdout
    line = [ln for ln in out.splitlines() if "libturbo_b200.so" in ln]
    assert line and os.path.realpath(line[0].split("=>")[1].split("(")[0].strip()) == \
        os.path.realpath(LIB)
    r = subprocess.run([SUITE], capture_output=True, text=True, timeout=120)
    assert r.returncode != 0 and "no CUDA device" in r.stderr


@pytest.mark.gpu
@needs_suite
def test_reference_suite_passes_on_b200():
    r = subprocess.run([SUITE], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "All tests passed" in r.stdout
