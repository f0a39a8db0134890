"""Extreme inputs against the reference decoder (the oracle restatement of
turbo_decode_code_block_cpu): very large and saturated LLR magnitudes, where the exact max*
correction underflows and the state metrics span thousands; totally erased blocks (all LLRs
zero), where every metric ties; and blocks with 30 % or 50 % of their LLRs erased.  Both
schedules against the oracle running the same windows, with the usual bar |gpu - ref| <=
1e-3 max(|ref|, 1) (widened for the scaled inputs, see there), hard decisions identical except
where |ref| is within the bar, CRC flags and iteration counts equal.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import schedule_window

pytestmark = pytest.mark.gpu

KS = [40, 512, 1056, 6144, 2048, 6144]


def _check(tc, decoder, oracle, llr, early_stop, iters=8, spread=0.0):
    """Both schedules against the oracle running the same windows (guard 96); returns the
    oracle's full-trellis posterior of the batch.  spread > 0 widens the bar of each block to
    spread x its largest |posterior| where that is larger (float32 metrics in the thousands)."""
    full = []
    for persistent in (False, True):
        sched = tc.SCHEDULE_PERSISTENT if persistent else tc.SCHEDULE_PLAIN
        post, ok, used = decoder.decode(KS, llr, None,
                                        tc.DecodeOptions(iters, early_stop, 0, -1, sched))
        assert np.all(np.isfinite(post)), sched
        lo = po = 0
        for i, k in enumerate(KS):
            seg = llr[lo:lo + 3 * (k + 4)]
            ref, rok, rused = oracle.decode_cb(k, 0, seg, iters, early_stop,
                                               window=schedule_window(k, persistent), guard=96)
            assert (bool(ok[i]), int(used[i])) == (rok, rused), (sched, i)
            got = post[po:po + k].astype(np.float64)
            tol = np.maximum(1e-3 * np.maximum(np.abs(ref), 1.0), spread * np.abs(ref).max())
            over = float((np.abs(got - ref) / tol).max())
            hard = int((((got >= 0) != (ref >= 0)) & (np.abs(ref) > tol)).sum())
            assert over <= 1.0 and hard == 0, (sched, i, over, hard)
            if not persistent:
                full.append(oracle.decode_cb(k, 0, seg, iters, early_stop)[0])
            lo += 3 * (k + 4)
            po += k
    return np.concatenate(full)


@pytest.mark.parametrize("scale", [40.0, 1000.0])
def test_large_llr_magnitudes(tc, decoder, oracle, scale):
    """A 0.6 dB batch scaled by 40 (metric differences of hundreds: every max* correction
    underflows to zero) and by 1000 (saturated LLRs in the tens of thousands).  With metrics in
    the thousands one float32 rounding is 1e-4 to 4e-3, so a small posterior formed from them
    agrees between two float32 implementations only to a fraction of the block's dynamic range:
    the bar is the usual one or 1e-4 of the block's largest |posterior|, whichever is larger
    (flags, iteration counts and hard decisions exact)."""
    _, llr = tc.awgn_code_blocks(71, KS, 0.6, None, True)
    ref = _check(tc, decoder, oracle, (llr * scale).astype(np.float32), True, spread=1e-4)
    assert np.abs(ref).max() > 10 * scale


def test_totally_erased_blocks(tc, decoder, oracle):
    """All LLRs zero: every metric ties, the posterior is zero everywhere, hard decisions are
    all ones, CRC24B never passes and every block runs all iterations."""
    llr = np.zeros(int(3 * (np.asarray(KS) + 4).sum()), np.float32)
    ref = _check(tc, decoder, oracle, llr, True, iters=4)
    assert np.all(ref == 0)
    post, ok, used = decoder.decode(KS, llr, None, tc.DecodeOptions(4, True))
    assert np.all(post == 0) and not np.any(ok) and np.all(used == 4)


@pytest.mark.parametrize("fraction", [0.3, 0.5])
def test_partly_erased_blocks(tc, decoder, oracle, fraction):
    """30 % / 50 % of each block's LLRs zeroed at random (heavy puncturing) at 3 dB: with 30 %
    every block stops early after 2-6 iterations, with 50 % none does."""
    _, llr = tc.awgn_code_blocks(72, KS, 3.0, None, True)
    rng = np.random.default_rng(72)
    llr = np.where(rng.random(llr.size) < fraction, 0.0, llr).astype(np.float32)
    _check(tc, decoder, oracle, llr, True)
