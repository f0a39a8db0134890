"""The TS 36.212 code on the GPU (DecodeOptions.convention = CONVENTION_3GPP; off by default).

The decoder's other trellis, tail mapping and CRC24B are checked against the oracle's
restatement of 36.212 running the same windows (flags and iterations equal, posteriors within
1e-3), on both schedules; then the convention is shown to select the code (graph cache kept
apart, LLRs of one code fail the other's CRC), and transport blocks of the 36.212 code make
the round trip through the device chain with the 36.212 CRC24A/CRC24B.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import llr_close, schedule_window

pytestmark = pytest.mark.gpu

KS = [40, 48, 512, 1056, 2048, 4096, 6144, 6144, 1024, 3200]
FILLERS = [0, 0, 0, 0, 0, 0, 0, 32, 16, 0]


def std_code_blocks(tc, ks, ebn0_db, seed, fillers=None):
    """BPSK/AWGN LLRs of 36.212 code blocks (K - 24 - F random bits + 36.212 CRC24B after F
    filler zeros; filler LLRs zeroed).  Returns (LLRs back to back, code-block bits)."""
    llrs, cbs = [], []
    for i, k in enumerate(ks):
        f = 0 if fillers is None else int(fillers[i])
        data = tc.random_bits(seed * 1009 + i, k - 24 - f)
        cb = np.concatenate([np.zeros(f, np.uint8), tc.append_crc24b(data, tc.CONVENTION_3GPP)])
        desc = tc.CodeBlockDescriptor(0, k, k + 4, 0, f, tc.qpp_index(k))
        e = tc.turbo_encode_code_block(desc, cb, tc.CONVENTION_3GPP)
        d = np.concatenate([e.systematic, e.parity0, e.parity1])
        sigma2 = 1.0 / (2.0 * (k / (3.0 * (k + 4))) * 10 ** (ebn0_db / 10.0))
        x = tc.awgn_llr(seed * 7919 + i, d, sigma2)
        x[:f] = 0.0
        x[k + 4:k + 4 + f] = 0.0
        llrs.append(x)
        cbs.append(cb)
    return np.concatenate(llrs), cbs


@pytest.mark.parametrize("persistent", [False, True])
def test_std_decode_matches_oracle(tc, decoder, oracle, persistent):
    llr, _ = std_code_blocks(tc, KS, 0.7, seed=3)
    sched = tc.SCHEDULE_PERSISTENT if persistent else tc.SCHEDULE_PLAIN
    post, ok, used = decoder.decode(KS, llr, FILLERS, tc.DecodeOptions(
        8, True, 0, -1, sched, convention=tc.CONVENTION_3GPP))
    lo = po = 0
    flags = []
    for i, k in enumerate(KS):
        ref, rok, rused = oracle.std_decode_cb(k, FILLERS[i], llr[lo:lo + 3 * (k + 4)], 8, True,
                                               window=schedule_window(k, persistent), guard=96)
        assert (bool(ok[i]), int(used[i])) == (rok, rused), (i, k)
        err, hard = llr_close(post[po:po + k], ref)
        assert err <= 1e-3 and hard == 0, (i, k, err)
        flags.append(rok)
        lo += 3 * (k + 4)
        po += k
    assert any(flags) and not all(flags), flags  # both branches of the early stop ran


def test_std_full_trellis_matches_oracle(tc, decoder, oracle):
    llr, _ = std_code_blocks(tc, [40, 1056, 6144], 1.0, seed=4)
    post, ok, used = decoder.decode([40, 1056, 6144], llr, None, tc.DecodeOptions(
        6, False, 6144, -1, convention=tc.CONVENTION_3GPP))
    lo = po = 0
    for k in (40, 1056, 6144):
        ref, _, _ = oracle.std_decode_cb(k, 0, llr[lo:lo + 3 * (k + 4)], 6)
        err, hard = llr_close(post[po:po + k], ref)
        assert err <= 1e-3 and hard == 0, (k, err)
        lo += 3 * (k + 4)
        po += k


def test_convention_selects_the_code(tc, decoder):
    """At 3 dB every 36.212 block decodes under its own convention and (nearly) none under the
    reference's; the same holds for the reference's blocks the other way round."""
    ks = [1056] * 24 + [6144] * 8
    std_llr, std_cb = std_code_blocks(tc, ks, 3.0, seed=5)
    bits, ref_llr = tc.awgn_code_blocks(6, ks, 3.0, None, True)
    for llr, conv, other in ((std_llr, tc.CONVENTION_3GPP, tc.CONVENTION_REFERENCE),
                             (ref_llr, tc.CONVENTION_REFERENCE, tc.CONVENTION_3GPP)):
        _, ok, _ = decoder.decode(ks, llr, None, tc.DecodeOptions(8, True, convention=conv))
        assert ok.all()
        _, ok_other, it = decoder.decode(ks, llr, None,
                                         tc.DecodeOptions(8, True, convention=other))
        assert ok_other.sum() <= 1 and (it[~ok_other] == 8).all()
    post, ok, _ = decoder.decode(ks, std_llr, None, tc.DecodeOptions(
        8, True, schedule=tc.SCHEDULE_PERSISTENT, convention=tc.CONVENTION_3GPP))
    assert ok.all() and np.array_equal((post >= 0).astype(np.uint8), np.concatenate(std_cb))


def test_graphs_keep_the_conventions_apart(tc, decoder):
    import torch

    ks = [512, 6144, 2048]
    llr, _ = std_code_blocks(tc, ks, 0.5, seed=7)
    cbs, llr_len, post_len = tc.Decoder.layout(ks)
    x = torch.from_numpy(llr).cuda()
    s = torch.cuda.Stream()
    p = torch.zeros(post_len, device="cuda")
    out = {}
    for conv in (tc.CONVENTION_3GPP, tc.CONVENTION_REFERENCE, tc.CONVENTION_3GPP):
        for graph in (False, True, True):
            p.zero_()
            torch.cuda.synchronize()
            decoder.decode_device(cbs, len(ks), x.data_ptr(), llr_len, p.data_ptr(), post_len,
                                  options=tc.DecodeOptions(6, False, graph=graph,
                                                           convention=conv),
                                  stream=s.cuda_stream)
            s.synchronize()
            out.setdefault(conv, []).append(p.cpu().numpy())
    for conv, runs in out.items():
        for r in runs[1:]:
            assert np.array_equal(r, runs[0]), conv
    assert not np.array_equal(out[tc.CONVENTION_3GPP][0], out[tc.CONVENTION_REFERENCE][0])


@pytest.mark.parametrize("persistent", [False, True])
def test_std_transport_blocks_through_the_device_chain(tc, decoder, persistent):
    tbs, blocks, llrs, truth = [], [], [], []
    for t, (size, rate) in enumerate([(1000, 0.5), (20000, 0.6), (6104, 0.4), (60000, 0.6)]):
        g = int(np.ceil(size / rate / 2.0)) * 2
        p = tc.LteTurboCodecParams(transport_block_bits=size, g_total=g,
                                   convention=tc.CONVENTION_3GPP)
        bits = tc.random_bits(100 + t, size)
        enc = tc.encode_transport_block(p, bits)
        rm = np.concatenate([b.rate_matched_bits for b in enc.code_blocks])
        sigma2 = 1.0 / (2.0 * (size / g) * 10 ** (3.0 / 10.0))
        llrs.append(tc.awgn_llr(200 + t, rm, sigma2))
        blocks += [(b.descriptor.k_r, b.descriptor.filler_count, b.descriptor.e_r, 0)
                   for b in enc.code_blocks]
        tbs.append((size, len(enc.code_blocks)))
        truth.append(bits)
    e_llr = np.concatenate(llrs)
    sched = tc.SCHEDULE_PERSISTENT if persistent else tc.SCHEDULE_PLAIN
    got, tb_ok, cb_ok, it = decoder.decode_tbs(tbs, blocks, e_llr, tc.DecodeOptions(
        8, True, schedule=sched, convention=tc.CONVENTION_3GPP))
    assert tb_ok.all() and cb_ok.all() and (it >= 1).all()
    for g_bits, t_bits in zip(got, truth):
        assert np.array_equal(g_bits, t_bits)
    # the same LLRs under the reference's code: no transport block passes its CRC24A
    _, tb_bad, _, _ = decoder.decode_tbs(tbs, blocks, e_llr,
                                         tc.DecodeOptions(8, True, schedule=sched))
    assert not tb_bad.any()


def test_std_reference_api_round_trip(tc):
    """encode_transport_block / decode_transport_block with LteTurboCodecParams.convention."""
    for size in (40, 5000, 14112):
        g = 3 * (size + 100)
        p = tc.LteTurboCodecParams(transport_block_bits=size, g_total=g, max_iterations=6,
                                   convention=tc.CONVENTION_3GPP)
        bits = tc.random_bits(size, size)
        enc = tc.encode_transport_block(p, bits)
        for be in (tc.DecoderBackend.GpuStage1Exact, tc.DecoderBackend.GpuB200Persistent):
            dec = tc.decode_transport_block(p, enc, be)
            assert dec.transport_block_crc_ok and all(dec.code_block_crc_ok)
            assert np.array_equal(dec.tb_bits, bits)


def test_graph_on_the_legacy_stream_is_refused(tc, decoder):
    """The legacy default stream cannot be captured: refused before any capture starts, and the
    decoder (and the same request on a created stream) works afterwards."""
    import torch

    ks = [1056, 40]
    llr, _ = std_code_blocks(tc, ks, 1.0, seed=8)
    cbs, llr_len, post_len = tc.Decoder.layout(ks)
    x = torch.from_numpy(llr).cuda()
    p = torch.zeros(post_len, device="cuda")
    opts = tc.DecodeOptions(4, graph=True, convention=tc.CONVENTION_3GPP)
    with pytest.raises(tc.InvalidArgument):
        decoder.decode_device(cbs, len(ks), x.data_ptr(), llr_len, p.data_ptr(), post_len,
                              options=opts)
    ref = decoder.decode(ks, llr, None, tc.DecodeOptions(4, convention=tc.CONVENTION_3GPP))[0]
    s = torch.cuda.Stream()
    decoder.decode_device(cbs, len(ks), x.data_ptr(), llr_len, p.data_ptr(), post_len,
                          options=opts, stream=s.cuda_stream)
    s.synchronize()
    assert np.array_equal(p.cpu().numpy(), ref)


def test_std_async_host_calls_and_autotuned_schedule(tc):
    """TC_MEM_HOST_ASYNC and the autotuner carry the convention: asynchronous calls equal the
    synchronous ones, and SCHEDULE_AUTO after tuning a 36.212 request decodes the 36.212 code."""
    import torch

    dec = tc.Decoder(0)
    ks = [6144] * 64 + [1056] * 32 + [40] * 8
    cbs, llr_len, post_len = tc.Decoder.layout(ks)
    conv = tc.CONVENTION_3GPP
    o = tc.DecodeOptions(8, True, schedule=tc.SCHEDULE_PERSISTENT, convention=conv)
    calls = []
    for i in range(3):
        llr, _ = std_code_blocks(tc, ks, 0.6 + 0.3 * i, seed=40 + i)
        x = torch.from_numpy(llr).pin_memory()
        p = torch.zeros(post_len).pin_memory()
        c = torch.zeros(len(ks), dtype=torch.uint8).pin_memory()
        it = torch.zeros(len(ks), dtype=torch.int32).pin_memory()
        dec.decode_async(cbs, len(ks), x.data_ptr(), llr_len, p.data_ptr(), post_len,
                         c.data_ptr(), it.data_ptr(), options=o)
        calls.append((llr, p, c, it))
    dec.sync()
    for llr, p, c, it in calls:
        post, ok, used = dec.decode(ks, llr, options=o)
        assert np.array_equal(p.numpy(), post)
        assert np.array_equal(c.numpy().astype(bool), ok)
        assert np.array_equal(it.numpy().astype(np.uint32), used)

    llr, cb_bits = std_code_blocks(tc, ks, 3.0, seed=45)
    x = torch.from_numpy(llr).cuda()
    out = torch.zeros(post_len, device="cuda")
    s = torch.cuda.Stream()
    best = dec.autotune(cbs, len(ks), x.data_ptr(), llr_len, out.data_ptr(), post_len,
                        options=tc.DecodeOptions(8, convention=conv), stream=s.cuda_stream)
    assert best["schedule"] in (0, 1) and best["ms"] > 0
    dec.decode_device(cbs, len(ks), x.data_ptr(), llr_len, out.data_ptr(), post_len,
                      options=tc.DecodeOptions(8, schedule=tc.SCHEDULE_AUTO, convention=conv),
                      stream=s.cuda_stream)
    s.synchronize()
    assert np.array_equal((out.cpu().numpy() >= 0).astype(np.uint8), np.concatenate(cb_bits))


# ---- the differentiable decoder on the 36.212 code (bars as tests/test_gpu_adjoint.py) ----
H_FD = 1e-4
RTOL_ADJ = 1e-4


def _std_gpu_vjp(tc, decoder, ks, llr, bits, scales, window=0, guard=-1):
    """GPU forward + backward on the 36.212 code: (posterior, d loss/d posterior, grad_llr,
    grad_scales), loss = mean BCE against the code-block bits."""
    import torch

    adj = tc.AdjointDecoder(decoder)
    iters = len(scales) // 2
    cbs, llr_len, post_len = tc.Decoder.layout(ks)
    s = torch.cuda.current_stream().cuda_stream
    x = torch.from_numpy(np.ascontiguousarray(llr, np.float32)).cuda()
    post = torch.zeros(post_len, device="cuda")
    tape = adj.forward(cbs, len(ks), x.data_ptr(), llr_len, post.data_ptr(), post_len, iters,
                       scales, window, guard, stream=s, convention=tc.CONVENTION_3GPP)
    b = torch.from_numpy(np.concatenate(bits).astype(np.float32)).cuda()
    gp = (torch.sigmoid(post) - b) / post.numel()
    gl = torch.zeros(llr_len, device="cuda")
    gs = torch.zeros(2 * iters, device="cuda")
    adj.backward(tape, gp.data_ptr(), gl.data_ptr(), gs.data_ptr(), stream=s)
    torch.cuda.synchronize()
    return post.cpu().numpy(), gp.cpu().numpy(), gl.cpu().numpy(), gs.cpu().numpy()


def _rel(got, ref):
    return float(np.abs(got - ref).max() / np.abs(ref).max())


def test_std_adjoint_gradient_check_k40(tc, decoder, oracle):
    """8 blocks of K=40 at 0.6 dB, 6 iterations, 12 scales: GPU gradients on the 36.212 code vs
    FP64 central differences of the oracle's 36.212 loss and vs its FP64 adjoint."""
    n, k, iters = 8, 40, 6
    llr, bits = std_code_blocks(tc, [k] * n, 0.6, seed=50)
    scales = np.random.default_rng(2).uniform(0.6, 1.2, 2 * iters)
    post, gp, g_llr, g_s = _std_gpu_vjp(tc, decoder, [k] * n, llr, bits,
                                        scales.astype(np.float32))
    l64 = llr.astype(np.float64).reshape(n, 3 * (k + 4))
    b64 = [b.astype(np.float64) for b in bits]

    def block_loss(i, l, s):
        p = oracle.adj_vjp(k, l, s, std=True)[0]
        return float(np.sum(np.logaddexp(0.0, p) - b64[i] * p)) / (n * k)

    fd_s = np.array([sum(block_loss(i, l64[i], scales + H_FD * e)
                         - block_loss(i, l64[i], scales - H_FD * e) for i in range(n)) / (2 * H_FD)
                     for e in np.eye(2 * iters)])
    fd_l = np.array([[(block_loss(i, l64[i] + H_FD * e, scales)
                       - block_loss(i, l64[i] - H_FD * e, scales)) / (2 * H_FD)
                      for e in np.eye(l64.shape[1])] for i in range(n)]).ravel()
    a_l, a_s = [], np.zeros(2 * iters)
    for i in range(n):
        p = oracle.adj_vjp(k, l64[i], scales, std=True)[0]
        _, _, g, s_ = oracle.adj_vjp(k, l64[i], scales,
                                     grad_post=(1 / (1 + np.exp(-p)) - b64[i]) / (n * k), std=True)
        a_l.append(g)
        a_s += s_
    a_l = np.concatenate(a_l)
    err = dict(fp64_scales_fd=_rel(a_s, fd_s), fp64_llr_fd=_rel(a_l, fd_l),
               scales_fd=_rel(g_s, fd_s), llr_fd=_rel(g_llr, fd_l), scales_adj=_rel(g_s, a_s),
               llr_adj=_rel(g_llr, a_l))
    print("36.212 K=40 gradient check (max rel):", err)
    assert err["fp64_scales_fd"] < 1e-5 and err["fp64_llr_fd"] < 1e-5, err
    assert max(err[key] for key in ("scales_fd", "llr_fd", "scales_adj", "llr_adj")) < RTOL_ADJ, err


def test_std_adjoint_windowed_vjp_and_autograd(tc, decoder, oracle):
    """K=1024, window 64, guard 32, 6 iterations on the 36.212 code: the GPU posterior and
    vector-Jacobian product against the FP64 36.212 adjoint fed the same d loss / d posterior;
    the torch autograd wrapper gives the same gradients."""
    import torch
    from turbo_cpp_b200.autograd import DifferentiableDecoder

    k, n, iters = 1024, 4, 6
    llr, bits = std_code_blocks(tc, [k] * n, 0.6, seed=51)
    scales = np.random.default_rng(5).uniform(0.7, 1.1, 2 * iters).astype(np.float32)
    post, gp, g_llr, g_s = _std_gpu_vjp(tc, decoder, [k] * n, llr, bits, scales, 64, 32)
    p64, a_l, a_s = [], [], np.zeros(2 * iters)
    for i in range(n):
        seg = llr[i * 3 * (k + 4):(i + 1) * 3 * (k + 4)].astype(np.float64)
        p, _, g, s_ = oracle.adj_vjp(k, seg, scales.astype(np.float64), 64, 32,
                                     grad_post=gp[i * k:(i + 1) * k].astype(np.float64), std=True)
        p64.append(p)
        a_l.append(g)
        a_s += s_
    err = dict(post=_rel(post, np.concatenate(p64)), scales=_rel(g_s, a_s),
               llr=_rel(g_llr, np.concatenate(a_l)))
    print("36.212 K=1024 windowed (max rel):", err)
    assert err["post"] < 1e-4 and err["scales"] < RTOL_ADJ and err["llr"] < RTOL_ADJ, err

    dd = DifferentiableDecoder([k] * n, window=64, guard=32, decoder=decoder,
                               convention=tc.CONVENTION_3GPP)
    x = torch.from_numpy(np.ascontiguousarray(llr, np.float32)).cuda().requires_grad_(True)
    sc = torch.from_numpy(scales).cuda().requires_grad_(True)
    out = dd(x, sc)
    b = torch.from_numpy(np.concatenate(bits).astype(np.float32)).cuda()
    torch.nn.functional.binary_cross_entropy_with_logits(out, b).backward()
    assert np.array_equal(out.detach().cpu().numpy(), post)
    assert np.allclose(x.grad.cpu().numpy(), g_llr, rtol=0, atol=1e-5 * np.abs(g_llr).max())
    assert np.allclose(sc.grad.cpu().numpy(), g_s, rtol=1e-4, atol=0)
