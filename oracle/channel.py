"""TEST INFRASTRUCTURE ONLY: the seeded BPSK/AWGN channel restated in numpy.

The product generates its synthetic code blocks with ``tc_awgn_code_blocks``
(``turbo_cpp_b200/csrc/lte_codec.cpp``: SplitMix64 finaliser over (seed, index) counters,
one Box-Muller draw per coded bit, LLR = 2y/sigma^2 with sigma^2 = 1/(2 R Eb/N0) and
R = K/(3(K+4))).  This module draws the same info bits and the same noise without loading the
product library, and encodes with the reference's own encoder (``turbo_encode_code_block``,
``src/lte_turbo.cpp:624-688``, through ``oracle/_ref``) or with the oracle's restatement of it
(``or_turbo_encode``).  The benchmark's reference arm uses it so that the reference decoder runs
on exactly the code blocks the GPU decodes, with only the reference's code loaded.

Only uncoded info bits without filler or CRC24B are generated here (the K=6144 benchmark
workload); the product's generator handles fillers and CRC24B payloads as well.
"""
from __future__ import annotations

import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def mix64(x):
    """SplitMix64 finaliser, elementwise on uint64 (wrapping arithmetic)."""
    x = np.asarray(x, np.uint64)
    with np.errstate(over="ignore"):
        x = x + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def _add(a, b):
    with np.errstate(over="ignore"):
        return np.asarray(a, np.uint64) + np.asarray(b, np.uint64)


def _unit(x):
    return ((x >> np.uint64(11)).astype(np.float64) + 0.5) * 2.0 ** -53


def block_seed(seed: int, i: int) -> np.uint64:
    """Per-block counter key of block i of a batch drawn with `seed`."""
    with np.errstate(over="ignore"):
        return mix64(np.uint64(seed & 0xFFFFFFFFFFFFFFFF)
                     + np.uint64(0x51ED270B27) * np.uint64(i + 1))


def random_bits(s: np.uint64, n: int) -> np.ndarray:
    key = mix64(np.uint64(s) ^ np.uint64(0x6A09E667F3BCC909))
    return (mix64(_add(key, np.arange(n, dtype=np.uint64))) >> np.uint64(63)).astype(np.uint8)


def awgn_llr(s: np.uint64, coded: np.ndarray, sigma2: float) -> np.ndarray:
    key = mix64(np.uint64(s) ^ np.uint64(0xBB67AE8584CAA73B))
    c = np.arange(coded.size, dtype=np.uint64)
    with np.errstate(over="ignore"):
        u1 = _unit(mix64(key + np.uint64(2) * c))
        u2 = _unit(mix64(key + np.uint64(2) * c + np.uint64(1)))
    z = np.sqrt(-2.0 * np.log(u1)) * np.cos(6.283185307179586 * u2)
    y = np.where(coded != 0, 1.0, -1.0) + np.sqrt(sigma2) * z
    return (2.0 / sigma2 * y).astype(np.float32)


def awgn_code_blocks(encoder, seed: int, k: int, ebn0_db, first: int = 0, count: int = 1):
    """Blocks first..first+count-1 of the batch that ``tc_awgn_code_blocks(seed, [k]*n, ebn0)``
    draws (any n > first+count-1): returns (bits uint8[count*k], llr float32[count*3(k+4)]).
    `encoder(k, filler, bits)` returns the [d0|d1|d2] code bits; `ebn0_db` is one value or one
    per block of the whole batch."""
    # the product takes Eb/N0 as float32 and widens it to double
    eb = np.broadcast_to(np.asarray(ebn0_db, np.float32).astype(np.float64), (first + count,))
    bits = np.empty(count * k, np.uint8)
    llr = np.empty(count * 3 * (k + 4), np.float32)
    rate = k / (3.0 * (k + 4))
    for j in range(count):
        i = first + j
        s = block_seed(seed, i)
        b = random_bits(s, k)
        d = np.asarray(encoder(k, 0, b), np.uint8)
        sigma2 = 1.0 / (2.0 * rate * 10.0 ** (float(eb[i]) / 10.0))
        bits[j * k:(j + 1) * k] = b
        llr[j * 3 * (k + 4):(j + 1) * 3 * (k + 4)] = awgn_llr(s ^ np.uint64(0x2545F4914F6CDD1D),
                                                               d, sigma2)
    return bits, llr
