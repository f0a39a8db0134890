"""CUDA-graph replay, autotuning and the persistent schedule's failure path (B200).

The failure test makes a device-side wait run out on purpose through the documented testing hook
(a progress count that nothing ever sets): the wait is bounded (one second of the GPU timer),
the kernel finishes, the host gets TC_ERR_TIMEOUT and the decoder keeps working afterwards.
No GPU fault, trap or hang is involved."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import awgn_blocks, llr_close

pytestmark = pytest.mark.gpu


def _dev(tc, ks, llr, fillers=None):
    import torch

    cbs, llr_len, post_len = tc.Decoder.layout(ks, fillers)
    x = torch.from_numpy(llr).cuda()
    out = torch.zeros(post_len, dtype=torch.float32, device="cuda")
    return cbs, llr_len, post_len, x, out


@pytest.mark.parametrize("schedule", [0, 1])
def test_graph_capture_and_replay(tc, decoder, schedule):
    import torch

    ks = [6144, 1024, 40, 2112, 512]
    llr_a, _ = awgn_blocks(tc, ks, 0.7, seed=41)
    llr_b, _ = awgn_blocks(tc, ks, 0.9, seed=42)
    ref_a = decoder.decode(ks, llr_a, options=tc.DecodeOptions(8, schedule=schedule))[0]
    ref_b = decoder.decode(ks, llr_b, options=tc.DecodeOptions(8, schedule=schedule))[0]
    cbs, ll, pl, x, out = _dev(tc, ks, llr_a)
    s = torch.cuda.Stream()
    opts = tc.DecodeOptions(8, schedule=schedule, graph=True)
    for _ in range(2):  # capture, then replay
        decoder.decode_device(cbs, len(ks), x.data_ptr(), ll, out.data_ptr(), pl, options=opts,
                              stream=s.cuda_stream)
        s.synchronize()
        assert np.array_equal(out.cpu().numpy(), ref_a)
    x.copy_(torch.from_numpy(llr_b))  # new data in the same buffer: the replay decodes it
    out.zero_()
    decoder.decode_device(cbs, len(ks), x.data_ptr(), ll, out.data_ptr(), pl, options=opts,
                          stream=s.cuda_stream)
    s.synchronize()
    assert np.array_equal(out.cpu().numpy(), ref_b)


def test_autotune_and_auto_schedule(tc, tmp_path):
    import torch

    dec = tc.Decoder(0)
    ks = [6144] * 256 + [1024] * 64
    llr, _ = awgn_blocks(tc, ks, 0.8, seed=43)
    cbs, ll, pl, x, out = _dev(tc, ks, llr)
    s = torch.cuda.Stream()
    best = dec.autotune(cbs, len(ks), x.data_ptr(), ll, out.data_ptr(), pl, stream=s.cuda_stream)
    assert best["schedule"] in (0, 1) and best["window"] % 8 == 0 and best["ms"] > 0
    ref = dec.decode(ks, llr)[0]
    dec.decode_device(cbs, len(ks), x.data_ptr(), ll, out.data_ptr(), pl,
                      options=tc.DecodeOptions(8, schedule=tc.SCHEDULE_AUTO),
                      stream=s.cuda_stream)
    s.synchronize()
    err, hard = llr_close(out.cpu().numpy(), ref, rtol=2e-3)  # both within 1e-3 of the trellis
    assert err <= 2e-3 and hard <= 2
    path = str(tmp_path / "tuning.txt")
    dec.save_tuning(path)
    dec2 = tc.Decoder(0)
    dec2.load_tuning(path)
    with open(path) as f:
        assert any(line.startswith("es=0,it=8") for line in f)
    bad = tmp_path / "bad.txt"
    bad.write_text("es=0 sideways 12 1.0\n")
    with pytest.raises(tc.InvalidArgument):
        dec2.load_tuning(str(bad))


def test_persistent_wait_limit_reports_timeout(tc):
    dec = tc.Decoder(0)
    ks = [6144] * 8
    llr, _ = awgn_blocks(tc, ks, 1.0, seed=44)
    opts = tc.DecodeOptions(2, schedule=tc.SCHEDULE_PERSISTENT)
    dec.inject_stall(3)
    with pytest.raises(tc.DeviceTimeout):
        dec.decode(ks, llr, options=opts)
    dec.inject_stall(-1)
    post, _, _ = dec.decode(ks, llr, options=opts)  # the context and the decoder still work
    ref, _, _ = dec.decode(ks, llr, options=tc.DecodeOptions(2))
    assert np.all(np.isfinite(post)) and llr_close(post, ref, rtol=2e-3)[0] <= 2e-3


@pytest.mark.parametrize("schedule", ["plain", "persistent"])
def test_async_host_calls_match_synchronous_ones(tc, decoder, schedule):
    """TC_MEM_HOST_ASYNC: five calls in a row on different inputs (pinned host buffers), then
    one sync: every call's posterior, CRC flags and iteration counts equal a synchronous
    host-memory call on the same input."""
    import torch

    sched = tc.SCHEDULE_PLAIN if schedule == "plain" else tc.SCHEDULE_PERSISTENT
    rng = np.random.default_rng(23)
    table = np.array([e.k for e in tc.qpp_interleaver_table()])
    ks = rng.choice(table, 300)
    cbs, llr_len, post_len = tc.Decoder.layout(ks)
    o = tc.DecodeOptions(8, True, 0, -1, sched)
    calls = []
    for i in range(5):
        llr, _ = awgn_blocks(tc, ks, 0.6 + 0.2 * i, seed=30 + i, crc24b=True)
        x = torch.from_numpy(llr).pin_memory()
        p = torch.full((post_len,), 7.0).pin_memory()
        c = torch.zeros(len(ks), dtype=torch.uint8).pin_memory()
        it = torch.zeros(len(ks), dtype=torch.int32).pin_memory()
        decoder.decode_async(cbs, len(ks), x.data_ptr(), llr_len, p.data_ptr(), post_len,
                             c.data_ptr(), it.data_ptr(), options=o)
        calls.append((llr, x, p, c, it))
    decoder.sync()
    for llr, x, p, c, it in calls:
        post, ok, used = decoder.decode(ks, llr, options=o)
        assert np.array_equal(p.numpy(), post)
        assert np.array_equal(c.numpy().astype(bool), np.asarray(ok, bool))
        assert np.array_equal(it.numpy().astype(np.uint32), np.asarray(used, np.uint32))
