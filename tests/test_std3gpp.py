"""The TS 36.212 code (CONVENTION_3GPP; no reference counterpart), CPU side.

The oracle's 36.212 restatement is pinned by the published check values of the four CRCs
(catalogued as CRC-24/LTE-A, CRC-24/LTE-B, CRC-16/XMODEM and CRC-8/LTE: the CRC of ASCII
"123456789", most significant bit first) and by an RSC written here from the generator
polynomials; the product codec is then compared with the oracle bit for bit.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

MSG = np.unpackbits(np.frombuffer(b"123456789", np.uint8))
CHECK = {0: (24, 0xCDE703), 1: (24, 0x23EF52), 2: (16, 0x31C3), 3: (8, 0xEA)}
KS = (40, 48, 512, 1056, 4096, 6144)


def _value(bits, n):
    return int("".join(str(int(b)) for b in bits[-n:]), 2)


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_oracle_crc_check_values(oracle, kind):
    n, value = CHECK[kind]
    out = oracle.std_crc_append(kind, MSG)
    assert _value(out, n) == value
    assert oracle.std_crc_check(kind, out)


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_product_crc_matches_oracle(tc, oracle, kind):
    n, value = CHECK[kind]
    app = (tc.append_crc24a, tc.append_crc24b, tc.append_crc16, tc.append_crc8)[kind]
    chk = (tc.check_crc24a, tc.check_crc24b, tc.check_crc16, tc.check_crc8)[kind]
    assert _value(app(MSG, tc.CONVENTION_3GPP), n) == value
    rng = np.random.default_rng(kind)
    for size in (0, 1, 7, 100, 6120):
        bits = rng.integers(0, 2, size, dtype=np.uint8)
        out = app(bits, tc.CONVENTION_3GPP)
        assert np.array_equal(out, oracle.std_crc_append(kind, bits))
        assert chk(out, tc.CONVENTION_3GPP)
        bad = out.copy()
        bad[rng.integers(0, bad.size)] ^= 1
        assert not chk(bad, tc.CONVENTION_3GPP)
    # the reference's generator arrays are other polynomials for all four kinds
    assert not np.array_equal(app(MSG), app(MSG, tc.CONVENTION_3GPP))


def _spec_rsc_encode(bits):
    """TS 36.212 5.1.3.2.1 straight from the polynomials: g0 = 1 + D^2 + D^3 (feedback),
    g1 = 1 + D + D^3 (output); then three termination steps whose input is the feedback.
    Returns (parity of the info bits, tail systematic [3], tail parity [3])."""
    reg = [0, 0, 0]  # contents delayed by D, D^2, D^3
    par = []
    for u in bits:
        a = int(u) ^ reg[1] ^ reg[2]
        par.append(a ^ reg[0] ^ reg[2])
        reg = [a, reg[0], reg[1]]
    xs, zs = [], []
    for _ in range(3):
        x = reg[1] ^ reg[2]
        a = x ^ reg[1] ^ reg[2]  # 0
        zs.append(a ^ reg[0] ^ reg[2])
        xs.append(x)
        reg = [a, reg[0], reg[1]]
    assert reg == [0, 0, 0]
    return np.array(par, np.uint8), xs, zs


@pytest.mark.parametrize("k", KS)
def test_encoder_from_the_polynomials(tc, oracle, k):
    rng = np.random.default_rng(k)
    filler = 16 if k >= 512 else 0
    cb = rng.integers(0, 2, k, dtype=np.uint8)
    cb[:filler] = 0
    desc = tc.CodeBlockDescriptor(0, k, k + 4, 0, filler, tc.qpp_index(k))
    enc = tc.turbo_encode_code_block(desc, cb, tc.CONVENTION_3GPP)
    d = np.concatenate([enc.systematic, enc.parity0, enc.parity1])
    assert np.array_equal(d, oracle.std_turbo_encode(k, filler, cb))
    d0, d1, d2 = d[:k + 4], d[k + 4:2 * k + 8], d[2 * k + 8:]
    z, x_t, z_t = _spec_rsc_encode(cb)
    zp, xp_t, zp_t = _spec_rsc_encode(cb[tc.qpp_permutation(k)])
    assert np.array_equal(d0[filler:k], cb[filler:]) and not d0[:filler].any()
    assert np.array_equal(d1[filler:k], z[filler:]) and not d1[:filler].any()
    assert np.array_equal(d2[:k], zp)
    # 5.1.3.2.2 tail multiplexing
    assert [d0[k], d0[k + 1], d0[k + 2], d0[k + 3]] == [x_t[0], z_t[1], xp_t[0], zp_t[1]]
    assert [d1[k], d1[k + 1], d1[k + 2], d1[k + 3]] == [z_t[0], x_t[2], zp_t[0], xp_t[2]]
    assert [d2[k], d2[k + 1], d2[k + 2], d2[k + 3]] == [x_t[1], z_t[2], xp_t[1], zp_t[2]]
    # the reference's code is a different one
    ref = tc.turbo_encode_code_block(desc, cb)
    assert not np.array_equal(ref.parity0, enc.parity0)


@pytest.mark.parametrize("conv", [0, 1])
def test_encoder_is_linear(tc, conv):
    """Both codes are linear over GF(2), tails included: enc(a ^ b) = enc(a) ^ enc(b)."""
    rng = np.random.default_rng(5 + conv)
    for k in (40, 1024, 6144):
        desc = tc.CodeBlockDescriptor(0, k, k + 4, 0, 0, tc.qpp_index(k))
        a, b = (rng.integers(0, 2, k, dtype=np.uint8) for _ in range(2))

        def enc(x):
            e = tc.turbo_encode_code_block(desc, x, conv)
            return np.concatenate([e.systematic, e.parity0, e.parity1])
        assert np.array_equal(enc(a ^ b), enc(a) ^ enc(b))


def test_segmentation_attaches_36212_crc24b(tc):
    rng = np.random.default_rng(9)
    b = rng.integers(0, 2, 20000, dtype=np.uint8)
    with_crc = tc.append_crc24a(b, tc.CONVENTION_3GPP)
    assert tc.check_crc24a(with_crc, tc.CONVENTION_3GPP)
    std = tc.segment_transport_block(with_crc, tc.CONVENTION_3GPP)
    ref = tc.segment_transport_block(with_crc)
    assert std.c == ref.c > 1 and std.filler_bits == ref.filler_bits
    for s, r in zip(std.code_blocks, ref.code_blocks):
        assert np.array_equal(s[:-24], r[:-24])  # same data, different CRC24B
        assert tc.check_crc24b(s[std.filler_bits if s is std.code_blocks[0] else 0:],
                               tc.CONVENTION_3GPP)
    assert any(not np.array_equal(s, r) for s, r in zip(std.code_blocks, ref.code_blocks))


def test_unknown_convention_is_refused(tc):
    lib = tc.load_library()
    bits = np.zeros(8, np.uint8)
    out = np.zeros(32, np.uint8)
    ok = C.c_int()
    assert lib.tc_crc_append_conv(2, 0, bits.ctypes.data, 8, out.ctypes.data) == 1
    assert lib.tc_crc_check_conv(-1, 0, out.ctypes.data, 32, C.addressof(ok)) == 1
    d = np.zeros(3 * 44, np.uint8)
    assert lib.tc_turbo_encode_conv(7, 40, 0, bits.ctypes.data, d.ctypes.data) == 1
    # the allocation-free decoder takes the reference convention only (refused before any
    # device work, so this runs without a GPU)
    opt = tc._Options()
    lib.tc_decode_options_init(C.addressof(opt))
    opt.convention = tc.CONVENTION_3GPP
    assert lib.tc_decode_noalloc(0, None, 0, None, 0, None, None, None, C.addressof(opt),
                                 None) == 1
    assert b"reference convention" in lib.tc_last_error()


H = 1e-4


def _std_block(tc, k, ebn0, seed):
    """LLRs [d0|d1|d2] (float64) of one 36.212 code block and its bits."""
    cb = tc.random_bits(seed, k)
    desc = tc.CodeBlockDescriptor(0, k, k + 4, 0, 0, tc.qpp_index(k))
    e = tc.turbo_encode_code_block(desc, cb, tc.CONVENTION_3GPP)
    d = np.concatenate([e.systematic, e.parity0, e.parity1])
    sigma2 = 1.0 / (2.0 * (k / (3.0 * (k + 4))) * 10 ** (ebn0 / 10.0))
    return tc.awgn_llr(seed + 1, d, sigma2).astype(np.float64), cb.astype(np.float64)


@pytest.mark.parametrize("window,guard", [(0, 0), (64, 32)])
def test_std_fp64_forward_is_the_std_decoder(tc, oracle, window, guard):
    """The oracle's FP64 differentiable decoder on the 36.212 code, unit scales, equals its float
    36.212 decoder (same schedule) within 1e-4."""
    from conftest import llr_close

    for k in (40, 1024):
        llr, _ = _std_block(tc, k, 0.8, 7 + k)
        post, _, _, _ = oracle.adj_vjp(k, llr, np.ones(8), window, guard, std=True)
        ref, _, _ = oracle.std_decode_cb(k, 0, llr.astype(np.float32), 4, False, window=window,
                                         guard=guard)
        err, hard = llr_close(post.astype(np.float32), ref)
        assert err <= 1e-4 and hard == 0, (k, err)
        # and it is not the reference code's decoder
        other, _, _, _ = oracle.adj_vjp(k, llr, np.ones(8), window, guard)
        assert np.abs(other - post).max() > 1.0


def test_std_fp64_adjoint_matches_finite_differences(tc, oracle):
    """K=40, full trellis, 6 iterations, 12 scales, a noisy block (-3 dB, so that the gradients
    are well above the finite differences' rounding): the hand-written FP64 adjoint on the
    36.212 code against FP64 central differences (h = 1e-4) of the mean BCE, every LLR and
    scale."""
    k, iters = 40, 6
    llr, bits = _std_block(tc, k, -3.0, 21)
    scales = np.random.default_rng(3).uniform(0.6, 1.2, 2 * iters)

    def bce(post):
        return (float(np.mean(np.logaddexp(0.0, post) - bits * post)),
                (1.0 / (1.0 + np.exp(-post)) - bits) / post.size)

    post, _, _, _ = oracle.adj_vjp(k, llr, scales, std=True)
    _, gp = bce(post)
    _, _, g_llr, g_s = oracle.adj_vjp(k, llr, scales, grad_post=gp, std=True)

    def loss(l, s):
        return bce(oracle.adj_vjp(k, l, s, std=True)[0])[0]

    fd_s = np.array([(loss(llr, scales + H * e) - loss(llr, scales - H * e)) / (2 * H)
                     for e in np.eye(scales.size)])
    fd_l = np.array([(loss(llr + H * e, scales) - loss(llr - H * e, scales)) / (2 * H)
                     for e in np.eye(llr.size)])
    assert np.abs(fd_s - g_s).max() <= 1e-6 * np.abs(fd_s).max()
    assert np.abs(fd_l - g_llr).max() <= 1e-6 * np.abs(fd_l).max()
    # the tail LLRs (all twelve carry information in the 36.212 multiplexing) get gradients
    tails = [k, k + 1, k + 2, k + 3]
    for base in (0, k + 4, 2 * (k + 4)):
        assert np.all(np.abs(g_llr[[base + t for t in tails]]) > 0)
