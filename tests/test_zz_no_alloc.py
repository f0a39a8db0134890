"""tc_decode_noalloc: the decode entry point that allocates no device memory.

It exists for callers that may not call cudaMalloc/cudaFree (a real-time receiver thread that
cannot take their synchronisation and latency, a program whose device memory belongs to another
allocator, a plug-in handed only its buffers); all of its scratch comes from a fixed array in the
library.  These tests call it through the C ABI and compare it with tc_decode, the entry point
that allocates, at the tolerance the other decoder tests use, on two calls in a row (the second
with other inputs and options, so leftovers of the first call in the shared array would show),
check that an oversized request is refused, that a call leaves the device's free memory
unchanged, and that a call made while its stream is capturing is refused.  This file is
collected last on purpose.
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


def test_noalloc_allocates_no_device_memory(tc):
    """After a first call (which sets the device up and, with the same options, loads every
    kernel the second call runs), a larger call changes the device's free memory by nothing: all
    of its scratch is the library's own array."""
    import torch

    stream = torch.cuda.Stream()
    small = [1024, 40]
    llr, _ = awgn_blocks(tc, small, 0.8, seed=320)
    _noalloc(tc, small, [0, 0], llr, tc.DecodeOptions(8, True), stream)
    ks = [6144] * 48 + [2048, 40]
    llr, _ = awgn_blocks(tc, ks, 0.8, seed=321)
    lib = tc.load_library()
    cbs, llr_len, post_len = tc.Decoder.layout(ks)
    x = torch.from_numpy(llr).cuda()
    post = torch.empty(post_len, dtype=torch.float32, device="cuda")
    ok = torch.zeros(len(ks), dtype=torch.uint8, device="cuda")
    it = torch.zeros(len(ks), dtype=torch.int32, device="cuda")
    opt, _keep = tc.Decoder._opts(tc.DecodeOptions(8, True), tc.MEM_DEVICE, stream.cuda_stream)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    rc = lib.tc_decode_noalloc(len(ks), C.addressof(cbs), llr_len, x.data_ptr(), post_len,
                               post.data_ptr(), ok.data_ptr(), it.data_ptr(), C.addressof(opt),
                               None)
    assert rc == 0, lib.tc_last_error()
    stream.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert np.all(np.isfinite(post.cpu().numpy()))


def test_noalloc_refuses_a_capturing_stream(tc):
    """The descriptors are copied from call-local host memory, so a call on a stream that is
    being captured is refused before anything is enqueued (the capture stays valid)."""
    import torch

    lib = tc.load_library()
    ks = [1024]
    cbs, llr_len, post_len = tc.Decoder.layout(ks)
    x = torch.zeros(llr_len, dtype=torch.float32, device="cuda")
    post = torch.zeros(post_len, dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    opt, _ = tc.Decoder._opts(tc.DecodeOptions(8), tc.MEM_DEVICE, stream.cuda_stream)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        rc = lib.tc_decode_noalloc(len(ks), C.addressof(cbs), llr_len, x.data_ptr(), post_len,
                                   post.data_ptr(), None, None, C.addressof(opt), None)
    assert rc == 1  # TC_ERR_INVALID_ARGUMENT
    assert b"captured" in lib.tc_last_error()
    del graph
