"""Configurations 3, 4 and 5 at their full sizes, checked through properties that do not depend
on size (the oracle checks sampled blocks; it is too slow for all of them):

* config 3 (512 transport blocks, 4444 code blocks): device de-rate matching is bit-exact for
  every block; on both schedules every transport block whose CRC24A passes decodes to the
  transmitted bits, and the two schedules' CRC pass rates agree;
* config 5 (20000 code blocks of mixed K, CRC24B early stop), both schedules: every block whose
  CRC24B passes equals the transmitted bits, blocks that never pass ran all 8 iterations, and a
  fixed sample matches the oracle running the same windows (flags, iterations, posteriors within
  1e-3);
* config 4 (1024 blocks of K=6144, 6 iterations, 12 scales): the batch gradient is additive
  over sub-batches (scales within float summation error, LLR gradients bit for bit), so every
  block's gradient is the one the K=40 and K=6144 checks validate.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import llr_close, schedule_window

pytestmark = pytest.mark.gpu


def test_config3_full_size(tc, decoder):
    import torch
    from turbo_cpp_b200.workloads import config3_transport_blocks

    tbs, blocks, e_llr, truth, _ = config3_transport_blocks(512, seed=33)
    assert len(blocks) > 4000
    # de-rate matching of every block on the device equals the host matcher
    x = torch.from_numpy(np.ascontiguousarray(e_llr, np.float32)).cuda()
    _, e_len, llr_len = tc.Decoder.rm_blocks(blocks)
    out = torch.zeros(llr_len, device="cuda")
    decoder.derate_device(blocks, x.data_ptr(), e_len, out.data_ptr(), llr_len)
    host, pos = [], 0
    for k, f, e, rv in blocks:
        host.append(tc.derate_match_llr(k, f, e_llr[pos:pos + e], rv))
        pos += e
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), np.concatenate(host))
    rates = []
    for sched in (tc.SCHEDULE_PLAIN, tc.SCHEDULE_PERSISTENT):
        bits_s, tb_ok, cb_ok, it = decoder.decode_tbs(tbs, blocks, e_llr,
                                                      tc.DecodeOptions(8, True, 0, -1, sched))
        for j in np.flatnonzero(tb_ok):
            assert np.array_equal(bits_s[j], truth[j]), (sched, j)
        assert np.all((it >= 1) & (it <= 8))
        rates.append(tb_ok.mean())
    assert 0.2 < rates[0] < 1.0 and abs(rates[0] - rates[1]) <= 0.02, rates


def test_config5_full_size(tc, decoder, oracle):
    import torch
    from turbo_cpp_b200.workloads import config5_code_blocks

    ks, llr, bits, eb = config5_code_blocks(20000, seed=55)
    cbs, llr_len, post_len = tc.Decoder.layout(ks)
    x = torch.from_numpy(llr).cuda()
    starts = np.concatenate([[0], np.cumsum(ks)[:-1]])
    llr_off = np.concatenate([[0], np.cumsum(3 * (ks.astype(np.int64) + 4))])
    pass_rate = []
    for sched in (tc.SCHEDULE_PLAIN, tc.SCHEDULE_PERSISTENT):
        p = torch.zeros(post_len, device="cuda")
        c = torch.zeros(ks.size, dtype=torch.uint8, device="cuda")
        it = torch.zeros(ks.size, dtype=torch.int32, device="cuda")
        decoder.decode_device(cbs, ks.size, x.data_ptr(), llr_len, p.data_ptr(), post_len,
                              c.data_ptr(), it.data_ptr(), options=tc.DecodeOptions(8, True, 0, -1, sched))
        torch.cuda.synchronize()
        post, ok, used = p.cpu().numpy(), c.cpu().numpy(), it.cpu().numpy()
        wrong = np.logical_or.reduceat((post >= 0) != bits, starts)
        assert not np.any(wrong & (ok == 1))  # a passing CRC24B means a correct block
        assert np.all((used >= 1) & (used <= 8)) and np.all(used[ok == 0] == 8)
        pass_rate.append(ok.mean())
        sample = list(np.flatnonzero(ok == 0)[:5]) + list(np.flatnonzero(ok == 1)[:5]) + [0, 19999]
        for i in sample:
            k = int(ks[i])
            win = schedule_window(k, sched == tc.SCHEDULE_PERSISTENT)
            ref, rok, rused = oracle.decode_cb(k, 0, llr[llr_off[i]:llr_off[i + 1]], 8, True,
                                               window=win, guard=96)
            assert (bool(ok[i]), int(used[i])) == (rok, rused), (sched, i)
            err, hard = llr_close(post[starts[i]:starts[i] + k], ref)
            assert err <= 1e-3 and hard == 0, (sched, i, err)
    assert abs(pass_rate[0] - pass_rate[1]) <= 0.01, pass_rate


def test_config4_gradient_is_additive_over_sub_batches(tc, decoder):
    import torch

    n, k, iters = 1024, 6144, 6
    bits, x = decoder.awgn_code_blocks_device(4321, [k] * n, 0.6)
    scales = np.linspace(0.9, 1.05, 2 * iters).astype(np.float32)
    adj = tc.AdjointDecoder(decoder)
    total = n * k

    def grads(first, count):
        cbs, llr_len, post_len = tc.Decoder.layout([k] * count)
        xs = x[first * 3 * (k + 4):(first + count) * 3 * (k + 4)].contiguous()
        post = torch.zeros(post_len, device="cuda")
        tape = adj.forward(cbs, count, xs.data_ptr(), llr_len, post.data_ptr(), post_len, iters,
                           scales)
        b = bits[first * k:(first + count) * k].float()
        gp = (torch.sigmoid(post) - b) / total  # the full batch's mean-BCE normalisation
        gl = torch.zeros(llr_len, device="cuda")
        gs = torch.zeros(2 * iters, device="cuda")
        adj.backward(tape, gp.data_ptr(), gl.data_ptr(), gs.data_ptr())
        torch.cuda.synchronize()
        return gl.cpu().numpy(), gs.cpu().numpy().astype(np.float64)

    gl_all, gs_all = grads(0, n)
    parts = [grads(j * 256, 256) for j in range(4)]
    assert np.array_equal(gl_all, np.concatenate([p[0] for p in parts]))
    gs_sum = sum(p[1] for p in parts)
    assert np.abs(gs_sum - gs_all).max() <= 1e-5 * np.abs(gs_all).max()
