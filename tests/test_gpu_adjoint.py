"""The GPU adjoint (tc_adjoint_forward / tc_adjoint_backward) against the FP64 oracle.

Loss: mean binary cross-entropy of the posterior LLRs against the true bits over all blocks of
a call (LLR > 0 <=> bit 1).  Bars, written here once:
* gradient check on K=40 blocks (full trellis), 6 iterations, 12 scales: the GPU gradients
  (every input LLR, every scale) match FP64 central finite differences (h = 1e-4) and the FP64
  CPU adjoint to 1e-4 relative (max |difference| / max |reference|, per gradient);
* windowed schedule (K = 1024 and 6144, window 64, guard 32): the GPU vector-Jacobian product
  matches the FP64 adjoint of the same schedule, fed the same d loss / d posterior, to 1e-4;
* the forward posterior is the plain decoder's with the same scales, bit for bit.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import awgn_blocks

pytestmark = pytest.mark.gpu
H = 1e-4
RTOL = 1e-4


def _gpu(tc, decoder, ks, llr, bits, scales, window=0, guard=-1, adj=None, grad_post=None):
    """GPU forward + backward; returns (posterior, d loss/d posterior, grad_llr, grad_scales)."""
    import torch

    adj = adj or tc.AdjointDecoder(decoder)
    iters = len(scales) // 2
    cbs, llr_len, post_len = tc.Decoder.layout(ks)
    s = torch.cuda.current_stream().cuda_stream
    x = torch.from_numpy(np.ascontiguousarray(llr, np.float32)).cuda()
    post = torch.zeros(post_len, device="cuda")
    tape = adj.forward(cbs, len(ks), x.data_ptr(), llr_len, post.data_ptr(), post_len, iters,
                       scales, window, guard, stream=s)
    if grad_post is None:
        b = torch.from_numpy(np.concatenate(bits).astype(np.float32)).cuda()
        gp = (torch.sigmoid(post) - b) / post.numel()
    else:
        gp = torch.from_numpy(np.ascontiguousarray(grad_post, np.float32)).cuda()
    gl = torch.zeros(llr_len, device="cuda")
    gs = torch.zeros(2 * iters, device="cuda")
    adj.backward(tape, gp.data_ptr(), gl.data_ptr(), gs.data_ptr(), stream=s)
    torch.cuda.synchronize()
    return post.cpu().numpy(), gp.cpu().numpy(), gl.cpu().numpy(), gs.cpu().numpy()


def _oracle_vjp(oracle, ks, llr, scales, window, guard, grad_post):
    """FP64 adjoint per block with the given d loss / d posterior; block results concatenated."""
    gl, gs, lo, po = [], np.zeros(len(scales)), 0, 0
    for k in ks:
        n = 3 * (k + 4)
        _, _, g, s = oracle.adj_vjp(k, llr[lo:lo + n], scales, window, guard,
                                    grad_post=grad_post[po:po + k])
        gl.append(g)
        gs += s
        lo += n
        po += k
    return np.concatenate(gl), gs


def _rel(got, ref):
    return float(np.abs(got - ref).max() / np.abs(ref).max())


def test_gradient_check_k40(tc, decoder, oracle):
    """16 blocks of K=40 at 0.6 dB, 6 iterations, 12 scales (random in [0.6, 1.2]): GPU vs
    FP64 central finite differences of the FP64 loss, and vs the FP64 adjoint."""
    n, k, iters = 16, 40, 6
    llr, bits = awgn_blocks(tc, [k] * n, 0.6, seed=40)
    scales = np.random.default_rng(1).uniform(0.6, 1.2, 2 * iters)
    post, gp, g_llr, g_s = _gpu(tc, decoder, [k] * n, llr, bits, scales.astype(np.float32))
    l64 = llr.astype(np.float64).reshape(n, 3 * (k + 4))
    b64 = [b.astype(np.float64) for b in bits]

    def block_loss(i, l, s):  # block i's share of the batch mean
        p = oracle.adj_vjp(k, l, s)[0]
        return float(np.sum(np.logaddexp(0.0, p) - b64[i] * p)) / (n * k)

    def batch_loss(s):
        return sum(block_loss(i, l64[i], s) for i in range(n))

    fd_s = np.array([(batch_loss(scales + H * e) - batch_loss(scales - H * e)) / (2 * H)
                     for e in np.eye(2 * iters)])
    fd_l = np.empty_like(l64)
    for i in range(n):
        for j in range(l64.shape[1]):
            e = np.zeros(l64.shape[1])
            e[j] = H
            fd_l[i, j] = (block_loss(i, l64[i] + e, scales) - block_loss(i, l64[i] - e, scales)) / (2 * H)
    fd_l = fd_l.ravel()
    # FP64 adjoint with FP64's own d loss / d posterior
    gp64 = np.concatenate([(1 / (1 + np.exp(-oracle.adj_vjp(k, l64[i], scales)[0])) - b64[i]) / (n * k)
                           for i in range(n)])
    a_l, a_s = _oracle_vjp(oracle, [k] * n, l64.ravel(), scales, 0, 0, gp64)
    err = dict(fp64_scales_fd=_rel(a_s, fd_s), fp64_llr_fd=_rel(a_l, fd_l),
               scales_fd=_rel(g_s, fd_s), llr_fd=_rel(g_llr, fd_l), scales_adj=_rel(g_s, a_s),
               llr_adj=_rel(g_llr, a_l))
    print("K=40 gradient check (max rel):", err)
    # the FP64 adjoint itself (the finite differences' own truncation error is ~1e-6 here)
    assert err["fp64_scales_fd"] < 1e-5 and err["fp64_llr_fd"] < 1e-5, err
    assert max(err[key] for key in ("scales_fd", "llr_fd", "scales_adj", "llr_adj")) < RTOL, err


@pytest.mark.parametrize("k,n", [(1024, 8), (6144, 4)])
def test_windowed_vjp_matches_fp64(tc, decoder, oracle, k, n):
    """Window 64, guard 32, 6 iterations: the GPU vector-Jacobian product against the FP64
    adjoint of the same schedule, both fed the GPU's d loss / d posterior."""
    iters = 6
    llr, bits = awgn_blocks(tc, [k] * n, 0.6, seed=k + n)
    scales = np.random.default_rng(k).uniform(0.7, 1.1, 2 * iters).astype(np.float32)
    post, gp, g_llr, g_s = _gpu(tc, decoder, [k] * n, llr, bits, scales, 64, 32)
    a_l, a_s = _oracle_vjp(oracle, [k] * n, llr.astype(np.float64), scales.astype(np.float64),
                           64, 32, gp.astype(np.float64))
    # the FP64 forward of the same schedule gives the same posterior
    p64 = np.concatenate([oracle.adj_vjp(k, llr[i * 3 * (k + 4):(i + 1) * 3 * (k + 4)],
                                         scales.astype(np.float64), 64, 32)[0] for i in range(n)])
    err = dict(post=_rel(post, p64), scales=_rel(g_s, a_s), llr=_rel(g_llr, a_l))
    print(f"K={k} windowed (max rel):", err)
    assert err["post"] < 1e-4 and err["scales"] < RTOL and err["llr"] < RTOL, err


def test_forward_is_the_scaled_plain_decoder(tc, decoder):
    ks = [6144, 40, 1056, 512]
    llr, bits = awgn_blocks(tc, ks, 0.8, seed=3)
    scales = np.linspace(0.7, 1.0, 12).astype(np.float32)
    post, _, _, _ = _gpu(tc, decoder, ks, llr, bits, scales, 64, 32)
    ref, _, _ = decoder.decode(ks, llr, options=tc.DecodeOptions(6, False, 64, 32, scales=list(scales)))
    assert np.array_equal(post, ref)


def test_backward_is_deterministic_and_tapes_are_checked(tc, decoder):
    import torch

    ks = [1024, 6144, 40]
    llr, bits = awgn_blocks(tc, ks, 0.6, seed=9)
    adj = tc.AdjointDecoder(decoder)
    sc = np.ones(12, np.float32)
    r1 = _gpu(tc, decoder, ks, llr, bits, sc, adj=adj)
    r2 = _gpu(tc, decoder, ks, llr, bits, sc, adj=adj)
    for a, b in zip(r1, r2):
        assert np.array_equal(a, b)
    # a backward pass of a replaced tape is refused
    cbs, llr_len, post_len = tc.Decoder.layout(ks)
    x = torch.from_numpy(llr).cuda()
    post = torch.zeros(post_len, device="cuda")
    t1 = adj.forward(cbs, len(ks), x.data_ptr(), llr_len, post.data_ptr(), post_len, 6)
    t2 = adj.forward(cbs, len(ks), x.data_ptr(), llr_len, post.data_ptr(), post_len, 6)
    assert t2 != t1
    g = torch.zeros(llr_len, device="cuda")
    gs = torch.zeros(12, device="cuda")
    with pytest.raises(tc.InvalidArgument):
        adj.backward(t1, post.data_ptr(), g.data_ptr(), gs.data_ptr())
    # grad_llr must be 16-byte aligned (the buffer is 4 floats longer, so a misaligned view
    # would still lie inside it); the refusal comes before any launch
    g_pad = torch.zeros(llr_len + 4, device="cuda")
    with pytest.raises(tc.InvalidArgument):
        adj.backward(t2, post.data_ptr(), g_pad.data_ptr() + 4, gs.data_ptr())
    adj.backward(t2, post.data_ptr(), g.data_ptr(), gs.data_ptr())
    torch.cuda.synchronize()
    with pytest.raises(tc.InvalidArgument):
        adj.forward(cbs, len(ks), x.data_ptr(), llr_len, post.data_ptr(), post_len, 6, window=60)
