"""GPU decoder parity (B200).  Every decode goes through the C ABI (libturbo_b200.so) and is
checked against the reference's own outputs (golden vectors) or the oracle restatement on the
same seeded inputs.

Tolerance (from the task's parity rule, written here once): posterior LLRs within 1e-3
relative, |gpu - cpu| <= 1e-3 * max(|cpu|, 1); hard decisions identical except where
|cpu LLR| < 1e-4; BER/BLER inside the 95% Wilson interval of the CPU run.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import awgn_blocks, llr_close, wilson

pytestmark = pytest.mark.gpu
RTOL = 1e-3


def _golden_cases(golden):
    cases, pos_l, pos_p = [], 0, 0
    for k, f, it, es, ok, used, eb in golden["dec_meta"]:
        llr = golden["dec_llr"][pos_l:pos_l + 3 * (k + 4)]
        pos_l += 3 * (k + 4)
        post = golden["dec_post"][pos_p:pos_p + k]
        pos_p += k
        cases.append(dict(k=int(k), f=int(f), it=int(it), es=bool(es), ok=bool(ok),
                          used=int(used), llr=llr, post=post))
    return cases


@pytest.mark.parametrize("window,guard", [(0, -1), (6144, 0), (128, 96), (256, 128)])
def test_golden_vectors(tc, decoder, golden, window, guard):
    """Reference posteriors, CRC flags and iteration counts; default schedule, full trellis and
    other windows.  Blocks with equal (iterations, early stop) go in one call."""
    cases = _golden_cases(golden)
    groups = {}
    for c in cases:
        groups.setdefault((c["it"], c["es"]), []).append(c)
    for (it, es), cs in groups.items():
        post, ok, used = decoder.decode([c["k"] for c in cs], np.concatenate([c["llr"] for c in cs]),
                                        [c["f"] for c in cs],
                                        tc.DecodeOptions(it, es, window, guard))
        pos = 0
        for j, c in enumerate(cs):
            err, hard = llr_close(post[pos:pos + c["k"]], c["post"])
            pos += c["k"]
            assert err <= RTOL and hard == 0, (c["k"], it, es, window, err, hard)
            assert bool(ok[j]) == c["ok"] and int(used[j]) == c["used"]


def test_full_trellis_is_tight(tc, decoder, golden):
    """window >= K: the reference's full trellis; only float rounding differs (MUFU ex2/lg2,
    log-sum order), so the agreement is far inside the 1e-3 bar."""
    worst = 0.0
    for c in _golden_cases(golden):
        post, _, _ = decoder.decode([c["k"]], c["llr"], [c["f"]],
                                    tc.DecodeOptions(c["it"], c["es"], 6144, 0))
        worst = max(worst, llr_close(post, c["post"])[0])
    assert worst < 2e-4, worst


@pytest.mark.parametrize("window,guard", [(32, 0), (32, 32), (64, 16), (128, 64), (256, 0)])
def test_matches_windowed_oracle(tc, decoder, oracle, window, guard):
    """Same window schedule on GPU and in the oracle (or_decode_cb_windowed)."""
    rng = np.random.default_rng(window * 100 + guard)
    table = [e.k for e in tc.qpp_interleaver_table()]
    ks = [table[i] for i in rng.integers(0, 188, 24)] + [40, 6144, 1024]
    fillers = [int(rng.integers(0, 3)) * 8 for _ in ks]
    llr, _ = awgn_blocks(tc, ks, 0.8, seed=window + guard, fillers=fillers)
    post, _, _ = decoder.decode(ks, llr, fillers, tc.DecodeOptions(6, False, window, guard))
    ko, lo, pos_o = np.array(ks), 0, 0
    worst = 0.0
    for k, f in zip(ks, fillers):
        ref, _, _ = oracle.decode_cb(k, f, llr[lo:lo + 3 * (k + 4)], 6, False, window=window,
                                     guard=guard)
        err, hard = llr_close(post[pos_o:pos_o + k], ref)
        worst = max(worst, err)
        assert hard == 0, (k, window, guard)
        lo += 3 * (k + 4)
        pos_o += k
    assert worst <= RTOL, worst


def test_config1_parity_and_ber(tc, decoder, oracle):
    """Config 1: 1000 blocks, K=1024, 0.5 dB, 8 iterations, no early stop: every posterior
    against the reference decoder (oracle, bitwise equal to the reference) and BER/BLER."""
    n, k = 1000, 1024
    llr, bits = awgn_blocks(tc, [k] * n, 0.5, seed=1)
    post, _, _ = decoder.decode([k] * n, llr)
    lo = np.arange(n, dtype=np.int64) * 3 * (k + 4)
    oo = np.arange(n, dtype=np.int64) * k
    ref, _, _ = oracle.decode_batch(np.full(n, k, np.int32), np.zeros(n, np.int32), llr, lo, oo, 8)
    err, hard = llr_close(post, ref)
    assert err <= RTOL and hard == 0, (err, hard)
    truth = np.concatenate(bits)
    ge = ((post >= 0) != truth).reshape(n, k)
    ce = ((ref >= 0) != truth).reshape(n, k)
    lo_b, hi_b = wilson(int(ce.any(1).sum()), n)
    assert lo_b <= ge.any(1).mean() <= hi_b
    lo_e, hi_e = wilson(int(ce.sum()), n * k)
    assert lo_e <= ge.mean() <= hi_e


def test_early_stop_matches_oracle(tc, decoder, oracle):
    """CRC24B early stop per block (lte_turbo.cpp:792-804): same stopping iteration, flag and
    posterior as the reference; blocks with filler included."""
    ks = [1024, 6144, 40 * 3, 2048, 512, 6144, 3008, 104]
    fillers = [0, 8, 0, 24, 0, 0, 16, 8]
    for eb in (0.4, 1.0, 2.5):
        llr, _ = awgn_blocks(tc, ks, eb, seed=int(eb * 10), fillers=fillers, crc24b=True)
        post, ok, used = decoder.decode(ks, llr, fillers, tc.DecodeOptions(8, True))
        lo = po = 0
        for j, (k, f) in enumerate(zip(ks, fillers)):
            ref, rok, rused = oracle.decode_cb(k, f, llr[lo:lo + 3 * (k + 4)], 8, True)
            assert (bool(ok[j]), int(used[j])) == (rok, rused), (eb, k)
            err, hard = llr_close(post[po:po + k], ref)
            assert err <= RTOL and hard == 0, (eb, k, err)
            lo += 3 * (k + 4)
            po += k


def test_reference_roundtrip_cases(tc):
    """The reference's own roundtrip tests (test_main.cpp:58-344) through
    decode_transport_block on every GPU backend."""
    for tbs, a, c in [(40, 7, 3), (512, 11, 5), (6112, 19, 11), (12000, 17, 9)]:
        bits = ((np.arange(tbs) * a + c) & 1).astype(np.uint8)
        seg = tc.segment_transport_block(tc.append_crc24a(bits))
        g = sum(3 * (b.size + 4) for b in seg.code_blocks)
        p = tc.LteTurboCodecParams(transport_block_bits=tbs, g_total=g, max_iterations=6)
        enc = tc.encode_transport_block(p, bits)
        for be in (tc.DecoderBackend.GpuStage1Exact, tc.DecoderBackend.GpuStage2Windowed,
                   tc.DecoderBackend.GpuB200Plain):
            dec = tc.decode_transport_block(p, enc, be)
            assert np.array_equal(dec.tb_bits, bits) and dec.transport_block_crc_ok, (tbs, be)
            assert all(dec.code_block_crc_ok) and np.all(np.isfinite(dec.posterior_llr))


def test_device_memory_mode_matches_host_mode(tc, decoder):
    import torch

    ks = [6144, 40, 1056, 2112]
    llr, _ = awgn_blocks(tc, ks, 0.7, seed=4)
    host_post, host_ok, host_it = decoder.decode(ks, llr)
    cbs, llr_len, post_len = tc.Decoder.layout(ks)
    x = torch.from_numpy(llr).cuda()
    out = torch.zeros(post_len, dtype=torch.float32, device="cuda")
    it = torch.zeros(len(ks), dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream()
    decoder.decode_device(cbs, len(ks), x.data_ptr(), llr_len, out.data_ptr(), post_len,
                          0, it.data_ptr(), stream=s.cuda_stream)
    s.synchronize()
    assert np.array_equal(out.cpu().numpy(), host_post)
    assert np.array_equal(it.cpu().numpy().astype(np.uint32), host_it)


def test_edge_cases_and_errors(tc, decoder):
    post, ok, it = decoder.decode([], np.zeros(0, np.float32))
    assert post.size == 0
    llr, _ = awgn_blocks(tc, [40], 3.0, seed=2)
    p1, _, _ = decoder.decode([40], llr, options=tc.DecodeOptions(1))
    assert p1.shape == (40,) and np.all(np.isfinite(p1))
    p0, _, it0 = decoder.decode([40], llr, options=tc.DecodeOptions(0))
    assert np.all(p0 == 0) and it0[0] == 0
    with pytest.raises(tc.OutOfRange):
        decoder.decode([44], np.zeros(3 * 48, np.float32))
    with pytest.raises(tc.InvalidArgument):
        decoder.decode([40], llr, options=tc.DecodeOptions(8, False, 64, 12))  # guard % 8
    with pytest.raises(tc.InvalidArgument):
        decoder.decode([40], llr[:-1])
    with pytest.raises(tc.InvalidArgument):
        decoder.decode([40], llr, [40])  # filler >= K


def test_scales_of_one_are_the_plain_decoder(tc, decoder):
    ks = [1024, 6144]
    llr, _ = awgn_blocks(tc, ks, 0.6, seed=8)
    a = decoder.decode(ks, llr)[0]
    b = decoder.decode(ks, llr, options=tc.DecodeOptions(8, scales=[1.0] * 16))[0]
    assert np.array_equal(a, b)


def test_config2_full_size_properties(tc, decoder, oracle):
    """Config 2 shape (4096 blocks of K=6144 per call, 8 iterations) at 1.2 dB: every block the
    GPU gets wrong, and a fixed sample of the rest, decodes to the same hard decisions and
    posteriors (1e-3) in the oracle, so the residual block errors are the reference decoder's
    own; the block error rate stays small."""
    n, k = 4096, 6144
    llr, bits = awgn_blocks(tc, [k] * n, 1.2, seed=12)
    post, _, _ = decoder.decode([k] * n, llr)
    truth = np.concatenate(bits)
    assert np.all(np.isfinite(post))
    bad = np.flatnonzero(((post >= 0) != truth).reshape(n, k).any(1))
    assert bad.size <= 0.02 * n, bad.size
    for i in list(bad[:32]) + [0, 1, 2047, 4095]:
        ref, _, _ = oracle.decode_cb(k, 0, llr[i * 3 * (k + 4):(i + 1) * 3 * (k + 4)], 8)
        err, hard = llr_close(post[i * k:(i + 1) * k], ref)
        assert err <= RTOL and hard == 0, (i, err, hard)


def test_concurrent_calls_on_one_decoder(tc, decoder):
    """Calls on one decoder from several host threads (the reference fans Stage 2 decodes out
    with std::async, lte_turbo.cpp:941-951) give the results of the same calls made one by one."""
    from concurrent.futures import ThreadPoolExecutor

    jobs = []
    for i in range(8):
        ks = [6144, 1024, 40 + 8 * i, 2048]
        llr, _ = awgn_blocks(tc, ks, 0.4 + 0.1 * i, seed=300 + i)
        jobs.append((ks, llr, tc.DecodeOptions(6, i % 2 == 1, 0, -1,
                                               tc.SCHEDULE_PERSISTENT if i % 3 == 0 else tc.SCHEDULE_PLAIN)))
    serial = [decoder.decode(ks, llr, options=o) for ks, llr, o in jobs]
    with ThreadPoolExecutor(4) as pool:
        threaded = list(pool.map(lambda j: decoder.decode(j[0], j[1], options=j[2]), jobs))
    for a, b in zip(serial, threaded):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


def test_decoders_can_be_created_and_destroyed_repeatedly(tc):
    llr, _ = awgn_blocks(tc, [1024], 1.0, seed=5)
    ref = None
    for _ in range(12):
        d = tc.Decoder(0)
        post, _, _ = d.decode([1024], llr)
        ref = post if ref is None else ref
        assert np.array_equal(post, ref)
        d.close()
