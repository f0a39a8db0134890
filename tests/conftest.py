"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on the CPU."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")
if GOLDEN_DIR not in sys.path:
    sys.path.insert(0, GOLDEN_DIR)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def golden():
    import make_golden

    return make_golden.load()


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle import Reference, reference_available

    if not reference_available():
        pytest.skip("oracle/_ref (the compiled reference) is not built here")
    return Reference()


@pytest.fixture(scope="session")
def tc():
    import turbo_cpp_b200

    turbo_cpp_b200.load_library()
    return turbo_cpp_b200


@pytest.fixture(scope="session")
def decoder(tc):
    return tc.Decoder(0)


def llr_close(gpu: np.ndarray, ref: np.ndarray, rtol: float = 1e-3):
    """Posterior parity: |gpu - ref| <= rtol * max(|ref|, 1) elementwise (relative for |LLR|
    >= 1, absolute rtol below), and identical hard decisions except where |ref| < 1e-4."""
    gpu = np.asarray(gpu, np.float64)
    ref = np.asarray(ref, np.float64)
    err = np.abs(gpu - ref) / np.maximum(np.abs(ref), 1.0)
    hard_bad = ((gpu >= 0) != (ref >= 0)) & (np.abs(ref) >= 1e-4)
    return float(err.max()) if err.size else 0.0, int(hard_bad.sum())


def awgn_blocks(tc, ks, ebn0_db, seed, fillers=None, crc24b=False):
    """Seeded BPSK/AWGN code blocks from the product's encoder and channel
    (tc_awgn_code_blocks).  Returns (LLRs [d0|d1|d2] per block back to back, info bits per
    block as a list)."""
    ks = [int(k) for k in ks]
    bits, llr = tc.awgn_code_blocks(seed, ks, ebn0_db, fillers, crc24b)
    out, pos = [], 0
    for k in ks:
        out.append(bits[pos:pos + k])
        pos += k
    return llr, out


def schedule_window(k, persistent):
    """The window each schedule cuts block size k into (guard 96): plain 128 steps; persistent
    at most 32 windows of at least 192 steps, of equal length rounded up to 8 (decoder.cu,
    decode_persistent)."""
    if not persistent:
        return min(128, k)
    nwin = max(1, min(32, k // 192))
    wlen = -(-(-(-k // nwin)) // 8) * 8
    if nwin > 1 and wlen < 96:
        nwin = max(1, k // 96)
        wlen = -(-(-(-k // nwin)) // 8) * 8
    return min(wlen, k)


def wilson(k: int, n: int, z: float = 1.96):
    """95% Wilson score interval of a binomial proportion k/n."""
    if n == 0:
        return 0.0, 1.0
    p = k / n
    d = 1 + z * z / n
    c = (p + z * z / (2 * n)) / d
    h = z * np.sqrt(p * (1 - p) / n + z * z / (4 * n * n)) / d
    return max(0.0, c - h), min(1.0, c + h)
