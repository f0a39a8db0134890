"""Seeded synthetic workloads of the benchmark configurations (no dataset is involved).

Each generator returns host arrays built with the library's own encoder, rate matcher and
channel (C++); the same arrays feed the GPU decoder and, in the tests, the oracle.

* config 1: K=1024 blocks, rate 1/3, BPSK/AWGN 0.5 dB.
* config 2: K=6144 blocks, rate 1/3, BPSK/AWGN at Eb/N0 0.0..1.2 dB.
* config 3: transport blocks of uneven size through the whole chain.  The 3GPP TS 36.213 TBS
  table is not available here, so TBS is drawn uniformly from the multiples of 8 in
  [1000, 97896] (every table entry in that range is such a multiple; segmentation accepts any
  size).  CRC24A, segmentation into K+/K- blocks with filler and CRC24B, encoding, rate
  matching to G = TBS / r (r ~ U[0.3, 0.9], rounded up to a multiple of NL*Qm = 2, rv 0),
  BPSK/AWGN at Eb/N0 ~ U[0.5, 3.0] dB per transport block with rate TBS/G.
* config 5: code blocks of all 188 sizes with P ~ K, payload K-24 + CRC24B, per-block Eb/N0
  ~ U[0, 2] dB.
"""
from __future__ import annotations

import numpy as np

from . import (LteTurboCodecParams, awgn_code_blocks, awgn_llr, encode_transport_block,
               qpp_interleaver_table, random_bits)


def config3_transport_blocks(n_tb: int, seed: int, llr_seed: int | None = None):
    """Returns (tbs list of (TBS, C), blocks list of (K, F, E, rv), rate-matched LLRs, info bits
    per TB, Eb/N0 per TB).  `llr_seed` draws other channel noise for the same blocks."""
    rng = np.random.default_rng(seed)
    tbs, blocks, llrs, bits_out, ebs = [], [], [], [], []
    for t in range(n_tb):
        tbs_bits = int(rng.integers(1000 // 8, 97896 // 8 + 1)) * 8
        r = float(rng.uniform(0.3, 0.9))
        g = int(np.ceil(tbs_bits / r / 2.0)) * 2
        eb = float(rng.uniform(0.5, 3.0))
        bits = random_bits(seed * 100003 + t, tbs_bits)
        p = LteTurboCodecParams(transport_block_bits=tbs_bits, g_total=g, rv=0)
        enc = encode_transport_block(p, bits)
        rm = np.concatenate([b.rate_matched_bits for b in enc.code_blocks])
        sigma2 = 1.0 / (2.0 * (tbs_bits / g) * 10 ** (eb / 10.0))
        llrs.append(awgn_llr((seed if llr_seed is None else llr_seed) * 7919 + t, rm, sigma2))
        for b in enc.code_blocks:
            d = b.descriptor
            blocks.append((d.k_r, d.filler_count, d.e_r, 0))
        tbs.append((tbs_bits, len(enc.code_blocks)))
        bits_out.append(bits)
        ebs.append(eb)
    return tbs, blocks, np.concatenate(llrs), bits_out, np.array(ebs)


def config5_code_blocks(n: int, seed: int, ebn0_range=(0.0, 2.0)):
    """(K per block, LLRs [d0|d1|d2] back to back, info bits, Eb/N0 per block)."""
    rng = np.random.default_rng(seed)
    table = np.array([e.k for e in qpp_interleaver_table()])
    ks = rng.choice(table, size=n, p=table / table.sum())
    eb = rng.uniform(*ebn0_range, size=n).astype(np.float32)
    bits, llr = awgn_code_blocks(seed, ks, eb, None, True)
    return ks, llr, bits, eb


def rate_matched_bpsk(bits, g_total: int, info_bits: int, ebn0_db: float, seed: int):
    """BPSK/AWGN LLRs of rate-matched bits at code rate info_bits / g_total."""
    sigma2 = 1.0 / (2.0 * (info_bits / g_total) * 10 ** (ebn0_db / 10.0))
    return awgn_llr(seed, bits, sigma2)
