"""The FP64 differentiable decoder and its hand-written adjoint (oracle/turbo_oracle.c,
or_adj_vjp), the checker of the GPU adjoint.  CPU only.

* Forward: with unit scales it is the reference decoder (golden posteriors of the reference's
  turbo_decode_code_block_cpu, full trellis) and the oracle's float windowed schedule.
* Backward: central finite differences in FP64 (h = 1e-4) of the mean binary cross-entropy of
  the posterior against the true bits, with respect to every input LLR and all scales; on the
  windowed schedule the next-iteration seeds are held at the values the unperturbed run used
  (they are constants of the differentiated function).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import llr_close

H = 1e-4


def _bce(post, bits):
    """mean BCE with logits and its gradient w.r.t. the logits (LLR > 0 <=> bit 1)"""
    return (float(np.mean(np.logaddexp(0.0, post) - bits * post)),
            (1.0 / (1.0 + np.exp(-post)) - bits) / post.size)


def _case(tc, k, ebn0, seed, iters):
    bits, llr = tc.awgn_code_blocks(seed, [k], ebn0)
    rng = np.random.default_rng(seed)
    return llr.astype(np.float64), bits.astype(np.float64), rng.uniform(0.6, 1.2, 2 * iters)


def _fd_check(oracle, k, llr, bits, scales, window, guard, positions):
    post, seeds, _, _ = oracle.adj_vjp(k, llr, scales, window, guard)
    _, gp = _bce(post, bits)
    _, _, g_llr, g_s = oracle.adj_vjp(k, llr, scales, window, guard, grad_post=gp,
                                      frozen_seeds=seeds)

    def loss(l, s):
        return _bce(oracle.adj_vjp(k, l, s, window, guard, frozen_seeds=seeds)[0], bits)[0]

    fd_s = np.array([(loss(llr, scales + H * e) - loss(llr, scales - H * e)) / (2 * H)
                     for e in np.eye(scales.size)])
    fd_l = np.empty(len(positions))
    for j, i in enumerate(positions):
        e = np.zeros_like(llr)
        e[i] = H
        fd_l[j] = (loss(llr + e, scales) - loss(llr - e, scales)) / (2 * H)
    err_s = np.abs(fd_s - g_s).max() / np.abs(fd_s).max()
    err_l = np.abs(fd_l - g_llr[positions]).max() / np.abs(fd_l).max()
    return err_s, err_l


def test_forward_with_unit_scales_is_the_reference_decoder(oracle, golden):
    """Golden posteriors of the reference (full trellis, no early stop cases)."""
    pos_l = pos_p = 0
    n = 0
    for k, f, it, es, ok, used, eb in golden["dec_meta"]:
        k = int(k)
        llr = golden["dec_llr"][pos_l:pos_l + 3 * (k + 4)]
        ref = golden["dec_post"][pos_p:pos_p + k]
        pos_l += 3 * (k + 4)
        pos_p += k
        if es or f:
            continue
        post, _, _, _ = oracle.adj_vjp(k, llr, np.ones(2 * int(it)))
        err, hard = llr_close(post.astype(np.float32), ref)
        assert err <= 1e-4 and hard == 0, (k, err)
        n += 1
    assert n >= 3


@pytest.mark.parametrize("window,guard", [(64, 32), (128, 96), (32, 0)])
def test_windowed_forward_matches_float_schedule(oracle, tc, window, guard):
    k = 1024
    llr, _, _ = _case(tc, k, 0.6, 5, 4)
    post, _, _, _ = oracle.adj_vjp(k, llr, np.ones(8), window, guard)
    ref, _, _ = oracle.decode_cb(k, 0, llr.astype(np.float32), 4, False, window=window,
                                 guard=guard)
    err, hard = llr_close(post.astype(np.float32), ref)
    assert err <= 1e-4 and hard == 0, err


def test_gradient_k40_full_trellis_vs_finite_differences(oracle, tc):
    """K=40, 6 iterations, 12 scales, every one of the 132 input LLRs."""
    k = 40
    llr, bits, scales = _case(tc, k, 0.6, 11, 6)
    err_s, err_l = _fd_check(oracle, k, llr, bits, scales, 0, 0, np.arange(llr.size))
    assert err_s < 1e-6 and err_l < 1e-6, (err_s, err_l)


@pytest.mark.parametrize("k,window,guard", [(40, 16, 8), (256, 64, 32), (512, 64, 64)])
def test_gradient_windowed_vs_finite_differences(oracle, tc, k, window, guard):
    """Windowed schedule with frozen seeds; a fixed sample of 64 input LLRs (tails included)."""
    llr, bits, scales = _case(tc, k, 0.4, k + window, 3)
    rng = np.random.default_rng(k)
    tails = [k, k + 1, k + 2, k + 3, 2 * k + 7, 3 * k + 11]
    pos = np.unique(np.concatenate([rng.choice(3 * (k + 4), 58, replace=False), tails]))
    err_s, err_l = _fd_check(oracle, k, llr, bits, scales, window, guard, pos)
    assert err_s < 1e-6 and err_l < 1e-6, (err_s, err_l)


def test_scale_gradient_is_the_extrinsic_correlation(oracle, tc):
    """d loss / d scale of the last lower SISO = sum over positions of d loss / d e2 * x; with
    e2 entering the posterior directly, a zero scale there gives d/ds = sum gp * x where x is
    the unscaled extrinsic (x = posterior(s=1) - posterior(s=0))."""
    k = 104
    llr, bits, _ = _case(tc, k, 1.0, 21, 2)
    s1 = np.ones(4)
    s0 = s1.copy()
    s0[3] = 0.0
    p1, _, _, _ = oracle.adj_vjp(k, llr, s1)
    p0, _, _, _ = oracle.adj_vjp(k, llr, s0)
    _, gp = _bce(p0, bits)
    _, _, _, g_s = oracle.adj_vjp(k, llr, s0, grad_post=gp)
    assert abs(g_s[3] - float(np.dot(gp, p1 - p0))) <= 1e-9 * max(1.0, abs(g_s[3]))


@pytest.mark.parametrize("k,window,guard,iters,bound", [(1024, 64, 32, 6, 2e-3),
                                                        (1024, 128, 96, 6, 1e-6)])
def test_frozen_seed_gradient_vs_true_gradient(oracle, tc, k, window, guard, iters, bound):
    """The differentiated function treats the next-iteration seeds as constants.  Here the true
    gradient of the windowed decoder -- seeds recomputed by every perturbed run, i.e. not frozen
    -- is taken by FP64 central differences and compared with the frozen-seed adjoint.  Measured
    worst relative error over the 12 scales and 64 sampled LLRs: 5.6e-4 with window 64 and guard
    32 (the training schedule), 1.5e-8 with window 128 and guard 96, where the seeds barely move
    the posteriors; the directions agree to cosine similarity 1 - 1e-9 or better."""
    llr, bits, scales = _case(tc, k, 0.6, k + window, iters)
    post, seeds, _, _ = oracle.adj_vjp(k, llr, scales, window, guard)
    _, gp = _bce(post, bits)
    _, _, g_llr, g_s = oracle.adj_vjp(k, llr, scales, window, guard, grad_post=gp,
                                      frozen_seeds=seeds)

    def loss(l, s):  # seeds follow the perturbed run
        return _bce(oracle.adj_vjp(k, l, s, window, guard)[0], bits)[0]

    fd_s = np.array([(loss(llr, scales + H * e) - loss(llr, scales - H * e)) / (2 * H)
                     for e in np.eye(scales.size)])
    pos = np.random.default_rng(k).choice(3 * (k + 4), 64, replace=False)
    fd_l = np.empty(pos.size)
    for j, i in enumerate(pos):
        e = np.zeros_like(llr)
        e[i] = H
        fd_l[j] = (loss(llr + e, scales) - loss(llr - e, scales)) / (2 * H)
    err_s = np.abs(fd_s - g_s).max() / np.abs(fd_s).max()
    err_l = np.abs(fd_l - g_llr[pos]).max() / np.abs(fd_l).max()
    cos_s = np.dot(fd_s, g_s) / np.linalg.norm(fd_s) / np.linalg.norm(g_s)
    assert err_s < bound and err_l < bound, (err_s, err_l)
    assert cos_s > 1.0 - 1e-6
