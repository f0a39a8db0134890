"""tc_decode_noalloc: the decode entry point that allocates no device memory.

It exists for callers that may not call cudaMalloc/cudaFree (a real-time receiver thread that
cannot take their synchronisation and latency, a program whose device memory belongs to another
allocator, a plug-in handed only its buffers); all of its scratch comes from a fixed array in the
library.  These tests call it through the C ABI and compare it with tc_decode, the entry point
that allocates, at the tolerance the other decoder tests use, on two calls in a row (the second
with other inputs and options, so leftovers of the first call in the shared array would show),
and check that an oversized request is refused.  This file is collected last on purpose.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import awgn_blocks, llr_close

pytestmark = pytest.mark.gpu
RTOL = 1e-3
SCRATCH_LIMIT = 32 << 20


def _noalloc(tc, ks, fillers, llr_host, options, stream):
    import torch

    lib = tc.load_library()
    cbs, llr_len, post_len = tc.Decoder.layout(ks, fillers)
    x = torch.from_numpy(llr_host).cuda()
    post = torch.full((post_len,), float("nan"), dtype=torch.float32, device="cuda")
    ok = torch.zeros(len(ks), dtype=torch.uint8, device="cuda")
    it = torch.zeros(len(ks), dtype=torch.int32, device="cuda")
    opt, _keep = tc.Decoder._opts(options, tc.MEM_DEVICE, stream.cuda_stream)
    need = C.c_size_t()
    rc = lib.tc_decode_noalloc(len(ks), C.addressof(cbs), llr_len, x.data_ptr(), post_len,
                               post.data_ptr(), ok.data_ptr(), it.data_ptr(), C.addressof(opt),
                               C.addressof(need))
    assert rc == 0, lib.tc_last_error()
    stream.synchronize()
    return post.cpu().numpy(), ok.cpu().numpy().astype(bool), it.cpu().numpy(), need.value


def test_noalloc_matches_allocating_decoder_twice(tc, decoder):
    import torch

    stream = torch.cuda.Stream()
    cases = [
        # mixed sizes with filler, 8 iterations, no early stop
        ([6144, 40, 1024, 2112, 512, 6144], [0, 0, 8, 0, 16, 24], 0.6, tc.DecodeOptions(8), False),
        # other sizes, CRC24B blocks with early stop, another window
        ([1056, 6144, 3008, 104], [0, 8, 0, 0], 1.1,
         tc.DecodeOptions(8, True, 168, 96), True),
    ]
    for seed, (ks, fillers, eb, opts, crc) in enumerate(cases):
        llr, _ = awgn_blocks(tc, ks, eb, seed=300 + seed, fillers=fillers, crc24b=crc)
        ref_post, ref_ok, ref_it = decoder.decode(ks, llr, fillers, opts)
        post, ok, it, need = _noalloc(tc, ks, fillers, llr, opts, stream)
        assert 0 < need <= SCRATCH_LIMIT
        err, hard = llr_close(post, ref_post)
        assert err <= RTOL and hard == 0, (seed, err, hard)
        assert np.array_equal(ok, ref_ok) and np.array_equal(it.astype(np.uint32), ref_it)


def test_noalloc_refuses_oversized_requests(tc):
    import torch

    lib = tc.load_library()
    ks = [6144] * 400
    cbs, llr_len, post_len = tc.Decoder.layout(ks)
    x = torch.zeros(llr_len, dtype=torch.float32, device="cuda")
    post = torch.zeros(post_len, dtype=torch.float32, device="cuda")
    opt, _ = tc.Decoder._opts(tc.DecodeOptions(8), tc.MEM_DEVICE, 0)
    need = C.c_size_t()
    rc = lib.tc_decode_noalloc(len(ks), C.addressof(cbs), llr_len, x.data_ptr(), post_len,
                               post.data_ptr(), None, None, C.addressof(opt), C.addressof(need))
    assert rc == 7  # TC_ERR_CAPACITY
    assert need.value > SCRATCH_LIMIT and b"scratch" in lib.tc_last_error()
    torch.cuda.synchronize()
    assert torch.count_nonzero(post).item() == 0  # nothing was launched
