"""Persistent batched schedule (one launch for all iterations, warp tasks from a device queue,
per-block CRC24B early stop) against the reference decoder, on the same inputs as the plain
schedule's tests.  Tolerance as in test_gpu_decoder.py."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import awgn_blocks, llr_close, wilson

pytestmark = pytest.mark.gpu
RTOL = 1e-3


def persistent(tc, iters=8, early=False, window=0, guard=-1, scales=None):
    return tc.DecodeOptions(iters, early, window, guard, tc.SCHEDULE_PERSISTENT, scales)


def test_golden_vectors_persistent(tc, decoder, golden):
    from test_gpu_decoder import _golden_cases

    cases = _golden_cases(golden)
    groups = {}
    for c in cases:
        groups.setdefault((c["it"], c["es"]), []).append(c)
    for (it, es), cs in groups.items():
        post, ok, used = decoder.decode([c["k"] for c in cs], np.concatenate([c["llr"] for c in cs]),
                                        [c["f"] for c in cs], persistent(tc, it, es))
        pos = 0
        for j, c in enumerate(cs):
            err, hard = llr_close(post[pos:pos + c["k"]], c["post"])
            pos += c["k"]
            assert err <= RTOL and hard == 0, (c["k"], it, es, err, hard)
            assert bool(ok[j]) == c["ok"] and int(used[j]) == c["used"]


def test_config1_persistent(tc, decoder, oracle):
    n, k = 1000, 1024
    llr, bits = awgn_blocks(tc, [k] * n, 0.5, seed=1)
    post, _, _ = decoder.decode([k] * n, llr, options=persistent(tc))
    lo = np.arange(n, dtype=np.int64) * 3 * (k + 4)
    oo = np.arange(n, dtype=np.int64) * k
    ref, _, _ = oracle.decode_batch(np.full(n, k, np.int32), np.zeros(n, np.int32), llr, lo, oo, 8)
    err, hard = llr_close(post, ref)
    assert err <= RTOL and hard == 0, (err, hard)


def test_mixed_k_early_stop_persistent(tc, decoder, oracle):
    """Blocks of uneven K (40..6144, P ~ K, as config 5), CRC24B payloads, per-block Eb/N0,
    early stop: stopping iteration, flag and posterior of every block equal the reference's."""
    rng = np.random.default_rng(5)
    table = np.array([e.k for e in tc.qpp_interleaver_table()])
    ks = rng.choice(table, size=96, p=table / table.sum())
    ks[:3] = [40, 6144, 104]
    eb = rng.uniform(0.0, 2.0, ks.size).astype(np.float32)
    fillers = [0] * ks.size
    bits, llr = tc.awgn_code_blocks(9, ks, eb, fillers, True)
    post, ok, used = decoder.decode(ks, llr, fillers, persistent(tc, 8, True))
    lo = po = 0
    stopped = 0
    for j, k in enumerate(ks):
        k = int(k)
        ref, rok, rused = oracle.decode_cb(k, 0, llr[lo:lo + 3 * (k + 4)], 8, True)
        assert (bool(ok[j]), int(used[j])) == (rok, rused), (j, k)
        err, hard = llr_close(post[po:po + k], ref)
        assert err <= RTOL and hard == 0, (j, k, err)
        stopped += rok
        lo += 3 * (k + 4)
        po += k
    assert 0 < stopped < ks.size  # the mix exercises both stopped and full-length blocks


def test_persistent_equals_plain_schedule_quality(tc, decoder):
    """Config-2-like batch at 0.6 dB: both schedules reach the same BLER (95 % interval)."""
    n, k = 512, 6144
    llr, bits = awgn_blocks(tc, [k] * n, 0.6, seed=21)
    a, _, _ = decoder.decode([k] * n, llr)
    b, _, _ = decoder.decode([k] * n, llr, options=persistent(tc))
    truth = np.concatenate(bits)
    ea = ((a >= 0) != truth).reshape(n, k).any(1)
    eb = ((b >= 0) != truth).reshape(n, k).any(1)
    lo, hi = wilson(int(ea.sum()), n)
    assert lo <= eb.mean() <= hi
    err, hard = llr_close(b, a, rtol=2e-3)  # both within 1e-3 of the full trellis
    assert err <= 2e-3
