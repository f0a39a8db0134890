"""Torch-facing differentiable decoder: posterior LLRs as a function of the channel LLRs and
the per-half-iteration extrinsic scales, with gradients from the library's hand-written adjoint
(tc_adjoint_forward / tc_adjoint_backward) through the thin libtorch autograd Function in
csrc/torch_adjoint.cpp.  Used by the scale-training harness (turbo_cpp_b200.train)."""
from __future__ import annotations

import importlib.util
from typing import Optional, Sequence

from . import AdjointDecoder, Decoder, load_library
from .build import TORCH_EXT_NAME, torch_ext_path

_ext = None


def extension():
    """The compiled torch extension (built in-tree by turbo_cpp_b200/build.py); raises if it is
    missing -- there is no fallback."""
    global _ext
    if _ext is None:
        import torch  # noqa: F401  (loads libtorch / libc10, which the extension links)

        load_library()  # the ctypes mirror's copy of libturbo_b200.so: the extension links it
        spec = importlib.util.spec_from_file_location(TORCH_EXT_NAME, torch_ext_path())
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        _ext = mod
    return _ext


class DifferentiableDecoder:
    """posterior = dd(llr, scales) for blocks of sizes ``ks`` stored back to back
    ([d0|d1|d2] per block, K posteriors per block), ``len(scales) // 2`` unrolled iterations
    without early stop, on the windowed schedule (window, guard; 0 / -1 = 64 / 32), for the
    code ``convention`` names (CONVENTION_REFERENCE or CONVENTION_3GPP)."""

    def __init__(self, ks: Sequence[int], fillers: Optional[Sequence[int]] = None,
                 window: int = 0, guard: int = -1, device: int = 0,
                 decoder: Optional[Decoder] = None, convention: int = 0):
        import torch

        self.decoder = decoder or Decoder(device)
        self.adjoint = AdjointDecoder(self.decoder)
        cbs, self.llr_len, self.post_len = Decoder.layout(ks, fillers)
        self.code_blocks = torch.tensor(
            [[cbs[i].k, cbs[i].filler, cbs[i].llr_offset, cbs[i].out_offset] for i in range(len(ks))],
            dtype=torch.int64)
        self.window, self.guard = int(window), int(guard)
        self.convention = int(convention)
        self._ext = extension()

    def __call__(self, llr, scales):
        if llr.numel() != self.llr_len:
            raise ValueError("llr: wrong length for these blocks")
        return self._ext.decode(llr, scales, self.adjoint._h.value, self.code_blocks,
                                self.post_len, self.window, self.guard, self.convention)
