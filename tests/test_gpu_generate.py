"""Test-vector generation on the device (generate.cu) against the host codec: seeded bits with
CRC24B and the encoded streams bit for bit, the rate matcher bit for bit, the channel's LLRs
equal up to the last bit of double log/cos (device library against the host C library)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mixed(tc, n, seed):
    rng = np.random.default_rng(seed)
    table = np.array([e.k for e in tc.qpp_interleaver_table()])
    ks = rng.choice(table, n)
    fillers = np.where(rng.random(n) < 0.3, 8 * rng.integers(1, 4, n), 0)
    fillers = np.where(ks > fillers + 32, fillers, 0)
    ebn0 = rng.uniform(-1.0, 3.0, n).astype(np.float32)
    return ks, fillers, ebn0


@pytest.mark.parametrize("crc24b", [False, True])
def test_device_generator_matches_host_generator(tc, decoder, crc24b):
    ks, fillers, ebn0 = _mixed(tc, 400, 5 + crc24b)
    hb, hl = tc.awgn_code_blocks(99, ks, ebn0, fillers, crc24b)
    db, dl = decoder.awgn_code_blocks_device(99, ks, ebn0, fillers, crc24b)
    db, dl = db.cpu().numpy(), dl.cpu().numpy()
    assert np.array_equal(db, hb)
    diff = np.abs(dl - hl)
    assert diff.max() <= 1e-6 * max(1.0, float(np.abs(hl).max())), diff.max()
    assert np.mean(dl == hl) > 0.99999
    if crc24b:  # every block is a CRC24B codeword over [filler, K)
        pos = 0
        for k, f in zip(ks, fillers):
            assert tc.check_crc24b(db[pos + f:pos + k])
            pos += k


def test_device_encoder_and_rate_matcher_match_host(tc, decoder):
    import torch

    ks, fillers, _ = _mixed(tc, 150, 11)
    bits = np.concatenate([tc.random_bits(200 + i, k) for i, k in enumerate(ks)])
    pos = 0
    for k, f in zip(ks, fillers):
        bits[pos:pos + f] = 0
        pos += k
    d = decoder.turbo_encode_device(ks, torch.from_numpy(bits).cuda(), fillers).cpu().numpy()
    host, pos = [], 0
    for k, f in zip(ks, fillers):
        e = tc.turbo_encode_code_block(tc.CodeBlockDescriptor(k_r=int(k), filler_count=int(f)),
                                       bits[pos:pos + k])
        host.append(np.concatenate([e.systematic, e.parity0, e.parity1]))
        pos += k
    host = np.concatenate(host)
    assert np.array_equal(d, host)
    rng = np.random.default_rng(12)
    blocks = [(int(k), int(f), int(rng.integers(k // 3, 4 * k)), int(rng.integers(0, 4)))
              for k, f in zip(ks, fillers)]
    out = decoder.rate_match_device(blocks, torch.from_numpy(host).cuda()).cpu().numpy()
    ref, pos = [], 0
    for (k, f, e, rv) in blocks:
        ref.append(tc.rate_match(k, f, host[pos:pos + 3 * (k + 4)], e, rv))
        pos += 3 * (k + 4)
    assert np.array_equal(out, np.concatenate(ref))


def test_generation_argument_errors(tc, decoder):
    import torch

    with pytest.raises(tc.OutOfRange):
        decoder.awgn_code_blocks_device(1, [44], 1.0)
    with pytest.raises(tc.InvalidArgument):  # no room for the CRC24B after the filler
        decoder.awgn_code_blocks_device(1, [40], 1.0, [24], crc24b=True)
    with pytest.raises(tc.InvalidArgument):  # rate-matched output outside the buffer
        decoder.rate_match_device([(40, 0, -1, 0)], torch.zeros(132, dtype=torch.uint8).cuda())
