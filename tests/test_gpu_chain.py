"""The device transport-block chain (config 3): LLR de-rate matching on the GPU, batched
decoding, CRC24B/CRC24A and reassembly, against the host de-rate matcher (bit for bit) and the
reference CPU chain (oracle restatement of derate + turbo_decode_code_block_cpu +
decode_transport_block)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_device_derate_is_bit_exact(tc, decoder):
    import torch

    rng = np.random.default_rng(17)
    table = [e.k for e in tc.qpp_interleaver_table()]
    blocks = []
    for _ in range(60):
        k = table[int(rng.integers(0, 188))]
        f = int(rng.integers(0, 3)) * 8 if k > 64 else 0
        e = int(rng.integers(1, 4 * k))
        blocks.append((k, f, e, int(rng.integers(0, 4))))
    blocks += [(6144, 0, 30000, 3), (40, 0, 1, 0), (40, 16, 500, 2), (6144, 32, 18444, 0)]
    arr, e_len, llr_len = tc.Decoder.rm_blocks(blocks)
    x = rng.normal(0, 4, e_len).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    out = torch.full((llr_len,), float("nan"), device="cuda")
    decoder.derate_device(blocks, xd.data_ptr(), e_len, out.data_ptr(), llr_len)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    e_pos = l_pos = 0
    for k, f, e, rv in blocks:
        ref = tc.derate_match_llr(k, f, x[e_pos:e_pos + e], rv)
        assert np.array_equal(got[l_pos:l_pos + 3 * (k + 4)].view(np.uint32), ref.view(np.uint32)), (k, f, e, rv)
        e_pos += e
        l_pos += 3 * (k + 4)


def test_device_derate_covers_every_block_size(tc, decoder):
    """Every one of the 188 block sizes, each redundancy version, fillers 0-56 and E on both
    sides of the valid circular-buffer length (punctured and repeated): the device de-rate
    matcher, whose circular-buffer ranks are computed in closed form per interleaver column,
    equals the host matcher (a position walk) bit for bit."""
    import torch

    rng = np.random.default_rng(23)
    blocks = []
    for i, k in enumerate(e.k for e in tc.qpp_interleaver_table()):
        for rv in range(4):
            f = ((i + rv) % 8) * 8 if k > 64 else 0
            e = int(rng.integers(k // 2, 3 * (k + 4))) if rv % 2 == 0 else int(rng.integers(3 * (k + 4), 7 * k))
            blocks.append((k, f, e, rv))
    arr, e_len, llr_len = tc.Decoder.rm_blocks(blocks)
    x = rng.normal(0, 4, e_len).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    out = torch.full((llr_len,), float("nan"), device="cuda")
    decoder.derate_device(blocks, xd.data_ptr(), e_len, out.data_ptr(), llr_len)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    e_pos = l_pos = 0
    for k, f, e, rv in blocks:
        ref = tc.derate_match_llr(k, f, x[e_pos:e_pos + e], rv)
        assert np.array_equal(got[l_pos:l_pos + 3 * (k + 4)].view(np.uint32), ref.view(np.uint32)), (k, f, e, rv)
        e_pos += e
        l_pos += 3 * (k + 4)


def test_transport_block_chain_matches_reference(tc, decoder, oracle):
    """Config-3 transport blocks (uneven TBS, K+/K-, filler, CRC24B, rate 0.3-0.9): the device
    chain gives the reference chain's posteriors (1e-3), decoded bits and CRC flags -- bits may
    differ only at ties, where the reference posterior is within 1e-4 of zero -- and the same
    stopping iterations."""
    from conftest import llr_close
    from turbo_cpp_b200.workloads import config3_transport_blocks

    tbs, blocks, e_llr, truth, ebs = config3_transport_blocks(10, seed=3)
    for es in (False, True):
        bits, tb_ok, cb_ok, iters, post = decoder.decode_tbs(
            tbs, blocks, e_llr, tc.DecodeOptions(8, es), want_posterior=True)
        e_pos = cb = p_pos = 0
        for t, (size, ncb) in enumerate(tbs):
            hard_all, tie_all = [], []
            for r in range(ncb):
                k, f, e, rv = blocks[cb + r]
                d012 = oracle.derate_llr(k, f, e_llr[e_pos:e_pos + e], rv)
                e_pos += e
                ref, ok, used = oracle.decode_cb(k, f, d012, 8, es)
                err, hard_bad = llr_close(post[p_pos:p_pos + k], ref)
                p_pos += k
                assert err <= 1e-3 and hard_bad == 0, (t, r, err, hard_bad)
                assert int(iters[cb + r]) == used, (t, r)
                hard = (ref >= 0).astype(np.uint8)[f:]
                tie = (np.abs(ref) < 1e-4)[f:]
                if ncb > 1:
                    if not tie.any():
                        assert bool(cb_ok[cb + r]) == oracle.crc_check(1, hard)
                    hard, tie = hard[:-24], tie[:-24]
                hard_all.append(hard)
                tie_all.append(tie)
            stream, ties = np.concatenate(hard_all), np.concatenate(tie_all)
            diff = bits[t] != stream[:-24]
            assert not np.any(diff & ~ties[:-24]), t
            if not ties.any():
                assert bool(tb_ok[t]) == oracle.crc_check(0, stream), t
            cb += ncb
    # high Eb/N0 transport blocks decode to the transmitted bits
    good = [t for t in range(len(tbs)) if ebs[t] > 2.0]
    assert good and all(np.array_equal(bits[t], truth[t]) and tb_ok[t] for t in good)


def test_harq_combining_matches_host_derate_sums(tc, decoder):
    """tc_derate_combine_llr_device: 1-4 transmissions per code block (rv cycling 0, 2, 3, 1,
    punctured and repeated E, fillers) give exactly the sum, in transmission order, of the host
    de-rate matcher's output per transmission."""
    import torch

    rng = np.random.default_rng(41)
    table = np.array([e.k for e in tc.qpp_interleaver_table()])
    tx, host, e_parts = [], [], []
    e_off = llr_off = 0
    for b in range(24):
        k = int(rng.choice(table))
        f = int(rng.integers(0, 4)) * 8 if b % 3 == 0 else 0
        f = min(f, k - 8)
        acc = None
        for t in range(int(rng.integers(1, 5))):
            rv = (0, 2, 3, 1)[t]
            e = int(rng.integers(k // 3, 3 * (k + 4) + 2 * k))
            x = (rng.standard_normal(e) * 4).astype(np.float32)
            d = tc.derate_match_llr(k, f, x, rv)
            acc = d if acc is None else acc + d
            tx.append((k, f, e, rv, e_off, llr_off))
            e_parts.append(x)
            e_off += e
        host.append(acc)
        llr_off += 3 * (k + 4)
    e_llr = torch.from_numpy(np.concatenate(e_parts)).cuda()
    out = torch.full((llr_off,), 9.0, device="cuda")
    decoder.derate_combine_device(tx, e_llr.data_ptr(), e_llr.numel(), out.data_ptr(), llr_off)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), np.concatenate(host))
    with pytest.raises(tc.InvalidArgument):  # filler disagrees inside one code block's group
        k0, f0 = tx[0][0], tx[0][1]
        bad = [tx[0], (k0, (f0 + 8) % k0) + tx[0][2:]]
        decoder.derate_combine_device(bad, e_llr.data_ptr(), e_llr.numel(), out.data_ptr(), llr_off)


@pytest.mark.parametrize("schedule", ["plain", "persistent"])
def test_transport_blocks_async_host_calls(tc, schedule):
    """TC_MEM_HOST_ASYNC transport-block calls (enqueued on the worker workspaces, several in
    flight) give the synchronous call's bits, CRC flags and iterations once synchronised."""
    import torch
    from turbo_cpp_b200.workloads import config3_transport_blocks

    dec = tc.Decoder(0)
    sched = tc.SCHEDULE_PLAIN if schedule == "plain" else tc.SCHEDULE_PERSISTENT
    o = tc.DecodeOptions(8, True, 0, -1, sched)
    calls = []
    for i in range(4):
        tbs, blocks, e_llr, truth, _ = config3_transport_blocks(12, seed=60 + i)
        tba, nbits = tc.Decoder.tb_descriptors(tbs)
        arr, e_len, _ = tc.Decoder.rm_blocks(blocks)
        x = torch.from_numpy(np.ascontiguousarray(e_llr, np.float32)).pin_memory()
        bits = torch.zeros(nbits, dtype=torch.uint8).pin_memory()
        tb_ok = torch.zeros(len(tbs), dtype=torch.uint8).pin_memory()
        cb_ok = torch.zeros(len(blocks), dtype=torch.uint8).pin_memory()
        it = torch.zeros(len(blocks), dtype=torch.int32).pin_memory()
        dec.decode_tbs_async(tba, len(tbs), arr, len(blocks), e_len, x.data_ptr(), nbits,
                             bits.data_ptr(), tb_ok.data_ptr(), cb_ok.data_ptr(), it.data_ptr(),
                             options=o)
        calls.append((tbs, blocks, e_llr, tba, arr, x, bits, tb_ok, cb_ok, it))
    dec.sync()
    for tbs, blocks, e_llr, tba, arr, x, bits, tb_ok, cb_ok, it in calls:
        ref_bits, ref_tb, ref_cb, ref_it = dec.decode_tbs(tbs, blocks, e_llr, o)
        assert np.array_equal(bits.numpy(), np.concatenate(ref_bits))
        assert np.array_equal(tb_ok.numpy().astype(bool), np.asarray(ref_tb, bool))
        assert np.array_equal(cb_ok.numpy().astype(bool), np.asarray(ref_cb, bool))
        assert np.array_equal(it.numpy().astype(np.uint32), np.asarray(ref_it, np.uint32))


def test_transport_block_graph_with_autotuned_schedule(tc, decoder):
    """Config-3 style transport blocks on device buffers with SCHEDULE_AUTO (after tc_autotune
    on the same code blocks) and graph replay: the first call captures de-rate matching,
    decoding and the finish kernel, later calls replay them; every call equals the eager
    (uncaptured) decode of the same inputs, including after new LLRs are written into the same
    input buffer."""
    import torch
    from turbo_cpp_b200.workloads import config3_transport_blocks

    tbs, blocks, e_llr, _, _ = config3_transport_blocks(24, seed=5)
    tbs2, blocks2, e_llr2, _, _ = config3_transport_blocks(24, seed=5, llr_seed=77)
    assert tbs2 == tbs and blocks2 == blocks and not np.array_equal(e_llr, e_llr2)
    arr, e_len, llr_len = tc.Decoder.rm_blocks(blocks)
    tba, nbits = tc.Decoder.tb_descriptors(tbs)
    n_tb, n_cb = len(tbs), len(blocks)
    stream = torch.cuda.Stream()
    x = torch.from_numpy(np.ascontiguousarray(e_llr, np.float32)).cuda()

    def run(opts):
        bits = torch.zeros(nbits, dtype=torch.uint8, device="cuda")
        tb_ok = torch.zeros(n_tb, dtype=torch.uint8, device="cuda")
        cb_ok = torch.zeros(n_cb, dtype=torch.uint8, device="cuda")
        it = torch.zeros(n_cb, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        decoder.decode_tbs_device(tba, n_tb, arr, n_cb, e_len, x.data_ptr(), nbits,
                                  bits.data_ptr(), tb_ok.data_ptr(), cb_ok.data_ptr(),
                                  it.data_ptr(), options=opts, stream=stream.cuda_stream)
        stream.synchronize()
        return [t.cpu().numpy() for t in (bits, tb_ok, cb_ok, it)]

    # the decode request the chain makes: its de-rate-matched blocks, tuned once
    d012 = torch.zeros(llr_len, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    decoder.derate_device(blocks, x.data_ptr(), e_len, d012.data_ptr(), llr_len,
                          stream=stream.cuda_stream)
    cbs, _, post_len = tc.Decoder.layout([b[0] for b in blocks], [b[1] for b in blocks])
    post = torch.empty(post_len, dtype=torch.float32, device="cuda")
    tuned = decoder.autotune(cbs, n_cb, d012.data_ptr(), llr_len, post.data_ptr(), post_len,
                             tc.DecodeOptions(8, True), stream.cuda_stream)
    stream.synchronize()
    sched = tc.SCHEDULE_PERSISTENT if tuned["schedule"] == 1 else tc.SCHEDULE_PLAIN
    eager = run(tc.DecodeOptions(8, True, tuned["window"], -1, sched))
    auto_graph = tc.DecodeOptions(8, True, 0, -1, tc.SCHEDULE_AUTO, graph=True)
    for _ in range(3):  # capture, then replays
        got = run(auto_graph)
        for a, b in zip(got, eager):
            assert np.array_equal(a, b)
    # new LLRs in the same buffer: the replayed graph decodes them
    x.copy_(torch.from_numpy(np.ascontiguousarray(e_llr2, np.float32)))
    eager2 = run(tc.DecodeOptions(8, True, tuned["window"], -1, sched))
    got2 = run(auto_graph)
    for a, b in zip(got2, eager2):
        assert np.array_equal(a, b)
    assert not np.array_equal(eager2[3], eager[3]) or not np.array_equal(eager2[0], eager[0])
