"""The oracle (oracle/turbo_oracle.c) pinned against the reference: golden vectors produced by
the reference itself (tests/golden/make_golden.py), and the live reference when it is built.
CPU only."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import llr_close


def test_qpp_table_matches_golden(oracle, golden):
    # reference test_qpp_table (test_main.cpp:37-44): 188 entries, first (40,3,10), last
    # (6144,263,480); here every entry
    table = np.array(oracle.qpp_table(), np.int32)
    assert table.shape == (188, 3)
    assert tuple(table[0]) == (40, 3, 10) and tuple(table[-1]) == (6144, 263, 480)
    assert np.array_equal(table, golden["qpp_table"])
    for k in (40, 1024, 6144):
        assert np.array_equal(oracle.qpp_perm(k), golden[f"qpp_perm_{k}"])


def test_crc_matches_golden(oracle, golden):
    off = golden["crc_off"]
    data = golden["crc_in"]
    for kind, L in ((0, 24), (1, 24), (2, 16), (3, 8)):
        out = golden[f"crc_out_{kind}"]
        for i in range(off.size - 1):
            b = data[off[i]:off[i + 1]]
            got = oracle.crc_append(kind, b)
            assert np.array_equal(got[:b.size], b)
            assert np.array_equal(got[b.size:], out[i * L:(i + 1) * L]), (kind, b.size)
            assert oracle.crc_check(kind, got)


def test_segmentation_matches_golden(oracle, golden):
    info = golden["seg_info"]
    pos_in = pos_out = 0
    for row in info:
        b = int(row[0])
        bits = golden["seg_in"][pos_in:pos_in + b]
        pos_in += b
        got, cbs = oracle.segment(bits)
        assert [got[n] for n in ("c", "c_plus", "c_minus", "k_plus", "k_minus", "filler", "l")] \
            == [int(x) for x in row[1:8]]
        n = int(row[8])
        assert np.array_equal(cbs, golden["seg_out"][pos_out:pos_out + n])
        pos_out += n


def test_encoder_matches_golden(oracle, golden):
    pos_in = pos_out = 0
    for k, f in golden["enc_cases"]:
        cb = golden["enc_in"][pos_in:pos_in + k]
        pos_in += k
        d = oracle.turbo_encode(int(k), int(f), cb)
        assert np.array_equal(d, golden["enc_out"][pos_out:pos_out + 3 * (k + 4)]), (k, f)
        pos_out += 3 * (k + 4)


def test_rate_matching_matches_golden(oracle, golden):
    """CRC24A + segmentation + encode + rate matching per block, and the +-8 de-rate matcher."""
    pos_in = pos_rm = pos_der = 0
    cbrows = golden["tb_cb"]
    r = 0
    for tbs, gt, rv in golden["tb_cases"]:
        bits = golden["tb_in"][pos_in:pos_in + tbs]
        pos_in += tbs
        with_crc = oracle.crc_append(0, bits)
        seg, cbs = oracle.segment(with_crc)
        pos_cb = 0
        for j in range(seg["c"]):
            _, _, _, k, f, e = (int(x) for x in cbrows[r])
            r += 1
            assert k == (seg["k_minus"] if j < seg["c_minus"] else seg["k_plus"])
            assert f == (seg["filler"] if j == 0 else 0)
            assert e == oracle.compute_e(j, int(gt), seg["c"], 1, 2)
            d = oracle.turbo_encode(k, f, cbs[pos_cb:pos_cb + k])
            pos_cb += k
            rm = oracle.rate_match(k, f, d, e, int(rv))
            assert np.array_equal(rm, golden["tb_rm"][pos_rm:pos_rm + e])
            pos_rm += e
            der = oracle.derate_bits(k, f, rm, int(rv))
            assert np.array_equal(der, golden["tb_derate"][pos_der:pos_der + 3 * (k + 4)])
            pos_der += 3 * (k + 4)
    assert r == cbrows.shape[0]


def test_decoder_matches_golden_bitwise(oracle, golden):
    """The C restatement is bitwise identical to turbo_decode_code_block_cpu."""
    pos_l = pos_p = 0
    for k, f, it, es, ok, used, _eb in golden["dec_meta"]:
        llr = golden["dec_llr"][pos_l:pos_l + 3 * (k + 4)]
        pos_l += 3 * (k + 4)
        ref = golden["dec_post"][pos_p:pos_p + k]
        pos_p += k
        post, got_ok, got_used = oracle.decode_cb(int(k), int(f), llr, int(it), bool(es))
        assert np.array_equal(post.view(np.uint32), ref.view(np.uint32)), (k, f)
        assert (got_ok, got_used) == (bool(ok), int(used))


def test_windowed_schedule_reduces_to_full_trellis(oracle, golden):
    """window >= K is the full trellis, bit for bit, whatever the guard."""
    pos_l = pos_p = 0
    for k, f, it, es, ok, used, _eb in golden["dec_meta"][:8]:
        llr = golden["dec_llr"][pos_l:pos_l + 3 * (k + 4)]
        pos_l += 3 * (k + 4)
        ref = golden["dec_post"][pos_p:pos_p + k]
        pos_p += k
        for guard in (0, 64):
            post, _, _ = oracle.decode_cb(int(k), int(f), llr, int(it), bool(es), window=int(k),
                                          guard=guard)
            assert np.array_equal(post.view(np.uint32), ref.view(np.uint32))


def test_windowed_schedule_with_guard_tracks_full_trellis(oracle, golden):
    """With NII and a 96-step guard (the GPU's default schedule) the windowed schedule stays
    within 1e-3 of the full trellis on the golden blocks."""
    pos_l = pos_p = 0
    for k, f, it, es, ok, used, _eb in golden["dec_meta"]:
        llr = golden["dec_llr"][pos_l:pos_l + 3 * (k + 4)]
        pos_l += 3 * (k + 4)
        ref = golden["dec_post"][pos_p:pos_p + k]
        pos_p += k
        post, _, _ = oracle.decode_cb(int(k), int(f), llr, int(it), bool(es), window=128, guard=96)
        err, hard = llr_close(post, ref)
        assert err < 1e-3 and hard == 0, (k, err, hard)


def test_reference_roundtrips_recorded(golden):
    # the reference's own roundtrip tests (test_main.cpp:58-344) pass in the fixture
    for row in golden["roundtrip"]:
        assert row[5] == 1 and row[7] == 1, row


def test_oracle_matches_live_reference_random(oracle, reference):
    """Fresh random cases against the compiled reference (skipped when oracle/_ref is absent)."""
    rng = np.random.default_rng(7)
    table = oracle.qpp_table()
    for _ in range(12):
        k = table[int(rng.integers(0, 188))][0]
        f = int(rng.integers(0, min(k // 4, 64) + 1)) // 8 * 8
        cb = rng.integers(0, 2, k).astype(np.uint8)
        cb[:f] = 0
        d = oracle.turbo_encode(k, f, cb)
        assert np.array_equal(d, reference.turbo_encode(k, f, cb))
        llr = ((2.0 * d - 1) * 2.0 + rng.normal(0, 1.5, d.size)).astype(np.float32)
        a = oracle.decode_cb(k, f, llr, 4, True)
        b = reference.decode_cb(k, f, llr, 4, True)
        assert np.array_equal(a[0].view(np.uint32), b[0].view(np.uint32))
        assert a[1:] == b[1:]
        for rv in range(4):
            e = int(rng.integers(k // 3, 4 * k))
            rm = oracle.rate_match(k, f, d, e, rv)
            assert np.array_equal(oracle.derate_bits(k, f, rm, rv), reference.derate_bits(k, f, rm, rv))
