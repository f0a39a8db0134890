"""The product's host codec chain (libturbo_b200.so via turbo_cpp_b200) is bit-exact with the
reference: golden vectors from the reference, random cases against the oracle.  CPU only."""
from __future__ import annotations

import numpy as np
import pytest


def test_qpp(tc, golden, oracle):
    table = [(e.k, e.f1, e.f2) for e in tc.qpp_interleaver_table()]
    assert np.array_equal(np.array(table, np.int32), golden["qpp_table"])
    assert tc.qpp_entry_for_k(6144) == tc.qpp_interleaver_table()[-1]
    for k, _, _ in table:
        p = tc.qpp_permutation(k)
        assert np.array_equal(p, oracle.qpp_perm(k))
        inv = tc.qpp_inverse_permutation(k)
        assert np.array_equal(inv[p], np.arange(k))
    with pytest.raises(tc.OutOfRange):
        tc.qpp_permutation(41)
    with pytest.raises(tc.OutOfRange):
        tc.qpp_entry_for_k(6152)


def test_crc(tc, golden):
    off, data = golden["crc_off"], golden["crc_in"]
    fns = [(tc.append_crc24a, tc.check_crc24a, 24), (tc.append_crc24b, tc.check_crc24b, 24),
           (tc.append_crc16, tc.check_crc16, 16), (tc.append_crc8, tc.check_crc8, 8)]
    for kind, (app, chk, L) in enumerate(fns):
        out = golden[f"crc_out_{kind}"]
        for i in range(off.size - 1):
            b = data[off[i]:off[i + 1]]
            got = app(b)
            assert np.array_equal(got[b.size:], out[i * L:(i + 1) * L])
            assert chk(got)
            if got.size:
                bad = got.copy()
                bad[-1] ^= 1
                assert not chk(bad)
    # reference test_crc (test_main.cpp:25-35)
    bits = [1, 0, 1, 1, 0, 1, 0, 0, 1, 1, 0, 1]
    assert tc.check_crc24a(tc.append_crc24a(bits)) and tc.check_crc8(tc.append_crc8(bits))
    assert not tc.check_crc24b(np.zeros(10, np.uint8) + 1)  # shorter than the CRC


def test_segmentation(tc, golden):
    pos_in = pos_out = 0
    for row in golden["seg_info"]:
        b = int(row[0])
        bits = golden["seg_in"][pos_in:pos_in + b]
        pos_in += b
        s = tc.segment_transport_block(bits)
        assert [s.c, s.c_plus, s.c_minus, s.k_plus, s.k_minus, s.filler_bits, s.l] == \
            [int(x) for x in row[1:8]]
        n = int(row[8])
        assert np.array_equal(np.concatenate(s.code_blocks), golden["seg_out"][pos_out:pos_out + n])
        pos_out += n
    # reference test_segmentation (test_main.cpp:46-56)
    s40 = tc.segment_transport_block(np.ones(40, np.uint8))
    assert s40.c == 1 and s40.code_blocks[0].size == 40
    s = tc.segment_transport_block(np.zeros(6145, np.uint8))
    assert s.c > 1 and s.filler_bits > 0
    with pytest.raises(tc.InvalidArgument):
        tc.segment_transport_block(np.zeros(0, np.uint8))


def test_encoder(tc, golden):
    pos_in = pos_out = 0
    for k, f in golden["enc_cases"]:
        k, f = int(k), int(f)
        cb = golden["enc_in"][pos_in:pos_in + k]
        pos_in += k
        enc = tc.turbo_encode_code_block(tc.CodeBlockDescriptor(k_r=k, filler_count=f), cb)
        d = np.concatenate([enc.systematic, enc.parity0, enc.parity1])
        assert np.array_equal(d, golden["enc_out"][pos_out:pos_out + 3 * (k + 4)])
        pos_out += 3 * (k + 4)
        assert enc.descriptor.d_r == k + 4


def test_transport_block_encode_and_derate(tc, golden):
    pos_in = pos_rm = pos_der = 0
    rows = golden["tb_cb"]
    r = 0
    for tbs, gt, rv in golden["tb_cases"]:
        tbs, gt, rv = int(tbs), int(gt), int(rv)
        bits = golden["tb_in"][pos_in:pos_in + tbs]
        pos_in += tbs
        p = tc.LteTurboCodecParams(transport_block_bits=tbs, g_total=gt, rv=rv)
        enc = tc.encode_transport_block(p, bits)
        for blk in enc.code_blocks:
            _, _, _, k, f, e = (int(x) for x in rows[r])
            r += 1
            d = blk.descriptor
            assert (d.k_r, d.filler_count, d.e_r) == (k, f, e)
            assert np.array_equal(blk.rate_matched_bits, golden["tb_rm"][pos_rm:pos_rm + e])
            pos_rm += e
            der = tc.derate_match_code_block(p, d, blk.rate_matched_bits)
            assert np.array_equal(der, golden["tb_derate"][pos_der:pos_der + 3 * (k + 4)])
            pos_der += 3 * (k + 4)
    assert r == rows.shape[0]


def test_derate_llr_reduces_to_bits(tc, oracle):
    """The LLR-domain de-rate matcher equals the +-8 one when fed +-8, and the oracle's LLR
    walk in general (repetition combining, <NULL> and filler handling)."""
    rng = np.random.default_rng(3)
    for k, f, e, rv in [(40, 0, 500, 0), (40, 16, 60, 1), (1024, 0, 2000, 2), (6144, 32, 30000, 3),
                        (6144, 0, 9000, 0), (528, 8, 1585, 1)]:
        bits = rng.integers(0, 2, e).astype(np.uint8)
        a = tc.derate_match_code_block(tc.LteTurboCodecParams(rv=rv),
                                       tc.CodeBlockDescriptor(k_r=k, filler_count=f), bits)
        b = tc.derate_match_llr(k, f, np.where(bits == 1, 8.0, -8.0).astype(np.float32), rv)
        assert np.array_equal(a, b)
        x = rng.normal(0, 3, e).astype(np.float32)
        assert np.array_equal(tc.derate_match_llr(k, f, x, rv), oracle.derate_llr(k, f, x, rv))


def test_random_codec_against_oracle(tc, oracle):
    rng = np.random.default_rng(11)
    table = oracle.qpp_table()
    for _ in range(25):
        k = table[int(rng.integers(0, 188))][0]
        f = int(rng.integers(0, k // 2 + 1)) if rng.random() < 0.5 else 0
        cb = rng.integers(0, 2, k).astype(np.uint8)
        cb[:f] = 0
        enc = tc.turbo_encode_code_block(tc.CodeBlockDescriptor(k_r=k, filler_count=f), cb)
        d = np.concatenate([enc.systematic, enc.parity0, enc.parity1])
        assert np.array_equal(d, oracle.turbo_encode(k, f, cb))
        rv = int(rng.integers(0, 4))
        e = int(rng.integers(1, 5 * k))
        assert np.array_equal(tc.rate_match(k, f, d, e, rv), oracle.rate_match(k, f, d, e, rv))


def test_channel_is_seeded(tc):
    a = tc.random_bits(5, 1000)
    assert np.array_equal(a, tc.random_bits(5, 1000))
    assert np.array_equal(a[10:], tc.random_bits(5, 990, first=10))
    assert 400 < a.sum() < 600
    x = tc.awgn_llr(9, np.ones(20000, np.uint8), 0.5)
    assert abs(x.mean() - 4.0) < 0.1 and abs(x.std() - 2.0 / np.sqrt(0.5)) < 0.1
