"""turbo_cpp_b200 -- LTE turbo codec with an exact Log-MAP decoder for NVIDIA B200 (sm_100a).

Python mirror of the Wiseung/Turbo_CPP public API (include/turbo_cpp/lte_turbo.h) over the C ABI
of ``libturbo_b200.so`` (include/turbo_b200.h).  The codec chain (CRC, segmentation, encoding,
rate matching, de-rate matching) runs on the host in C++; decoding runs only on the GPU.  There is
no CPU decoder here: without a CUDA device ``Decoder`` raises.
"""
from __future__ import annotations

import ctypes as C
import enum
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

__all__ = [
    "LIB_PATH", "TurboError", "InvalidArgument", "OutOfRange", "CudaError", "NoDevice",
    "DeviceTimeout", "CapacityExceeded", "load_library", "qpp_interleaver_table",
    "qpp_entry_for_k", "qpp_permutation", "qpp_inverse_permutation", "append_crc24a",
    "append_crc24b", "append_crc16", "append_crc8", "check_crc24a", "check_crc24b",
    "check_crc16", "check_crc8", "segment_transport_block", "SegmentationResult",
    "CodeBlockDescriptor", "EncodedCodeBlock", "EncodedTransportBlock", "DecodedTransportBlock",
    "LteTurboCodecParams", "LteChannelType", "DecoderBackend", "turbo_encode_code_block",
    "encode_transport_block", "compute_e", "rate_match", "derate_match_code_block",
    "derate_match_llr", "random_bits", "awgn_llr", "awgn_code_blocks", "Decoder", "DecodeOptions",
    "turbo_decode_code_block_gpu", "decode_transport_block", "MEM_HOST", "MEM_DEVICE",
    "SCHEDULE_PLAIN", "SCHEDULE_PERSISTENT", "SCHEDULE_AUTO",
]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libturbo_b200.so")

MEM_HOST, MEM_DEVICE, MEM_HOST_ASYNC = 0, 1, 2
SCHEDULE_PLAIN, SCHEDULE_PERSISTENT, SCHEDULE_AUTO = 0, 1, 2
CONVENTION_REFERENCE, CONVENTION_3GPP = 0, 1  # the reference's code; TS 36.212 (new)


# ------------------------------------------------------------------------------------------
# errors: the reference throws std::invalid_argument / std::out_of_range / std::runtime_error
# ------------------------------------------------------------------------------------------
class TurboError(RuntimeError):
    status = 3


class InvalidArgument(TurboError, ValueError):
    status = 1


class OutOfRange(TurboError, IndexError):
    status = 2


class CudaError(TurboError):
    status = 4


class NoDevice(TurboError):
    status = 5


class DeviceTimeout(TurboError):
    status = 6


class CapacityExceeded(TurboError):
    status = 7


_ERRORS = {c.status: c for c in (TurboError, InvalidArgument, OutOfRange, CudaError, NoDevice,
                                 DeviceTimeout, CapacityExceeded)}


class _CodeBlock(C.Structure):
    _fields_ = [("k", C.c_int32), ("filler", C.c_int32), ("llr_offset", C.c_int64),
                ("out_offset", C.c_int64)]


class _Options(C.Structure):
    _fields_ = [("max_iterations", C.c_uint32), ("early_stop", C.c_uint32), ("window", C.c_int32),
                ("guard", C.c_int32), ("memory", C.c_uint32), ("schedule", C.c_uint32),
                ("scales", C.c_void_p), ("graph", C.c_uint32), ("stream", C.c_void_p),
                ("convention", C.c_uint32)]


class _RmBlock(C.Structure):
    _fields_ = [("k", C.c_int32), ("filler", C.c_int32), ("e", C.c_int32), ("rv", C.c_uint32),
                ("e_offset", C.c_int64), ("llr_offset", C.c_int64)]


# numpy views of the descriptor structs (same field order, sizes and alignment)
_CODE_BLOCK_DTYPE = np.dtype([("k", np.int32), ("filler", np.int32), ("llr_offset", np.int64),
                              ("out_offset", np.int64)])
_RM_BLOCK_DTYPE = np.dtype([("k", np.int32), ("filler", np.int32), ("e", np.int32),
                            ("rv", np.uint32), ("e_offset", np.int64), ("llr_offset", np.int64)])
assert _CODE_BLOCK_DTYPE.itemsize == C.sizeof(_CodeBlock)
assert _RM_BLOCK_DTYPE.itemsize == C.sizeof(_RmBlock)


class _TransportBlock(C.Structure):
    _fields_ = [("tbs", C.c_int64), ("first_cb", C.c_int32), ("n_cb", C.c_int32),
                ("bits_offset", C.c_int64)]


class _TuneResult(C.Structure):
    _fields_ = [("schedule", C.c_int32), ("window", C.c_int32), ("ms", C.c_double)]


class _Seg(C.Structure):
    _fields_ = [(n, C.c_size_t) for n in ("c", "c_plus", "c_minus", "k_plus", "k_minus",
                                          "filler_bits", "l")]


_lib: Optional[C.CDLL] = None
_VP, _SZ, _I32, _U32, _U64 = C.c_void_p, C.c_size_t, C.c_int32, C.c_uint32, C.c_uint64

# (name, argtypes); every function returns int status except the two string getters
_SIGNATURES = {
    "tc_version": [],
    "tc_qpp_table_size": [],
    "tc_qpp_entry": [C.c_int, _VP, _VP, _VP],
    "tc_qpp_index": [_I32, _VP],
    "tc_qpp_permutation": [_I32, _VP],
    "tc_qpp_inverse_permutation": [_I32, _VP],
    "tc_crc_append": [C.c_int, _VP, _SZ, _VP],
    "tc_crc_check": [C.c_int, _VP, _SZ, _VP],
    "tc_segment_transport_block": [_VP, _SZ, _VP, _VP, _SZ],
    "tc_turbo_encode": [_I32, _I32, _VP, _VP],
    "tc_crc_append_conv": [C.c_int, C.c_int, _VP, _SZ, _VP],
    "tc_crc_check_conv": [C.c_int, C.c_int, _VP, _SZ, _VP],
    "tc_segment_transport_block_conv": [C.c_int, _VP, _SZ, _VP, _VP, _SZ],
    "tc_turbo_encode_conv": [C.c_int, _I32, _I32, _VP, _VP],
    "tc_compute_e": [_SZ, _SZ, _SZ, _U32, _U32, _VP],
    "tc_rate_match": [_I32, _I32, _VP, _SZ, _U32, _VP],
    "tc_derate_match_bits": [_I32, _I32, _VP, _SZ, _U32, _VP],
    "tc_derate_match_llr": [_I32, _I32, _VP, _SZ, _U32, _VP],
    "tc_random_bits": [_U64, _U64, _SZ, _VP],
    "tc_awgn_llr": [_U64, _U64, _VP, _SZ, C.c_double, _VP],
    "tc_awgn_code_blocks": [_U64, _SZ, _VP, _VP, _VP, C.c_int, _VP, _VP, C.c_int],
    "tc_decoder_create": [C.c_int, _VP],
    "tc_decoder_destroy": [_VP],
    "tc_decode_options_init": [_VP],
    "tc_decode": [_VP, _SZ, _VP, _SZ, _VP, _SZ, _VP, _VP, _VP, _VP],
    "tc_decode_noalloc": [_SZ, _VP, _SZ, _VP, _SZ, _VP, _VP, _VP, _VP, _VP],
    "tc_decoder_sync": [_VP],
    "tc_derate_match_llr_device": [_VP, _SZ, _VP, _SZ, _VP, _SZ, _VP, _VP],
    "tc_decode_transport_blocks": [_VP, _SZ, _VP, _SZ, _VP, _SZ, _VP, _SZ, _VP, _VP, _VP, _VP,
                                   _VP, _VP],
    "tc_decoder_inject_stall": [_VP, C.c_int],
    "tc_autotune": [_VP, _SZ, _VP, _SZ, _VP, _SZ, _VP, _VP, _VP],
    "tc_autotune_save": [_VP, C.c_char_p],
    "tc_autotune_load": [_VP, C.c_char_p],
    "tc_decoder_set_timing": [_VP, C.c_int],
    "tc_decoder_timing": [_VP, _VP, C.c_int],
    "tc_derate_combine_llr_device": [_VP, _SZ, _VP, _SZ, _VP, _SZ, _VP, _VP],
    "tc_awgn_code_blocks_device": [_VP, _U64, _SZ, _VP, _VP, _VP, C.c_int, _VP, _VP, _VP],
    "tc_turbo_encode_device": [_VP, _SZ, _VP, _VP, _VP, _VP, _VP],
    "tc_rate_match_device": [_VP, _SZ, _VP, _SZ, _VP, _SZ, _VP, _VP],
    "tc_adjoint_create": [_VP, _VP],
    "tc_adjoint_destroy": [_VP],
    "tc_adjoint_forward": [_VP, _SZ, _VP, _SZ, _VP, _SZ, _VP, C.c_uint32, _VP, C.c_int32,
                           C.c_int32, _VP, _VP],
    "tc_adjoint_forward_conv": [C.c_int, _VP, _SZ, _VP, _SZ, _VP, _SZ, _VP, C.c_uint32, _VP,
                                C.c_int32, C.c_int32, _VP, _VP],
    "tc_adjoint_backward": [_VP, C.c_uint64, _VP, _VP, _VP, _VP],
    "tc_adjoint_launches": [_VP, _VP],
}


class _Timing(C.Structure):
    _fields_ = [("launches", C.c_uint64), ("siso_launches", C.c_uint64), ("siso_ms", C.c_double),
                ("trellis_steps", C.c_uint64)]


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Loads libturbo_b200.so (built by ``turbo_cpp_b200/build.py``); raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python turbo_cpp_b200/build.py`")
    lib = C.CDLL(path)
    for name, args in _SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    for name in ("tc_status_name", "tc_last_error"):
        getattr(lib, name).restype = C.c_char_p
    lib.tc_status_name.argtypes = [C.c_int]
    lib.tc_last_error.argtypes = []
    _lib = lib
    return lib


def _call(name: str, *args) -> None:
    lib = load_library()
    rc = getattr(lib, name)(*args)
    if rc != 0:
        msg = lib.tc_last_error().decode(errors="replace")
        raise _ERRORS.get(rc, TurboError)(f"{name}: {lib.tc_status_name(rc).decode()}: {msg}")


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _u8(bits) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(bits, dtype=np.uint8) & 1)


# ------------------------------------------------------------------------------------------
# QPP (lte_turbo.h:77-81, 94-95, 108-109)
# ------------------------------------------------------------------------------------------
@dataclass(frozen=True)
class QppEntry:
    k: int
    f1: int
    f2: int


def qpp_interleaver_table() -> list[QppEntry]:
    lib = load_library()
    out = []
    for i in range(lib.tc_qpp_table_size()):
        k, f1, f2 = C.c_int32(), C.c_int32(), C.c_int32()
        _call("tc_qpp_entry", i, C.addressof(k), C.addressof(f1), C.addressof(f2))
        out.append(QppEntry(k.value, f1.value, f2.value))
    return out


def qpp_entry_for_k(k: int) -> QppEntry:
    idx = C.c_int32()
    _call("tc_qpp_index", int(k), C.addressof(idx))
    return qpp_interleaver_table()[idx.value]


def qpp_index(k: int) -> int:
    idx = C.c_int32()
    _call("tc_qpp_index", int(k), C.addressof(idx))
    return idx.value


def qpp_permutation(k: int) -> np.ndarray:
    p = np.empty(int(k), np.int32)
    _call("tc_qpp_permutation", int(k), _ptr(p))
    return p


def qpp_inverse_permutation(k: int) -> np.ndarray:
    p = np.empty(int(k), np.int32)
    _call("tc_qpp_inverse_permutation", int(k), _ptr(p))
    return p


# ------------------------------------------------------------------------------------------
# CRC (lte_turbo.h:97-104)
# ------------------------------------------------------------------------------------------
_CRC_LEN = (24, 24, 16, 8)


def _crc_append(kind: int, bits, convention: int = CONVENTION_REFERENCE) -> np.ndarray:
    b = _u8(bits)
    out = np.empty(b.size + _CRC_LEN[kind], np.uint8)
    _call("tc_crc_append_conv", int(convention), kind, _ptr(b), b.size, _ptr(out))
    return out


def _crc_check(kind: int, bits, convention: int = CONVENTION_REFERENCE) -> bool:
    b = _u8(bits)
    ok = C.c_int()
    _call("tc_crc_check_conv", int(convention), kind, _ptr(b), b.size, C.addressof(ok))
    return bool(ok.value)


# convention: CONVENTION_REFERENCE (the reference's generator arrays) or CONVENTION_3GPP
def append_crc24a(bits, convention=CONVENTION_REFERENCE): return _crc_append(0, bits, convention)
def append_crc24b(bits, convention=CONVENTION_REFERENCE): return _crc_append(1, bits, convention)
def append_crc16(bits, convention=CONVENTION_REFERENCE): return _crc_append(2, bits, convention)
def append_crc8(bits, convention=CONVENTION_REFERENCE): return _crc_append(3, bits, convention)
def check_crc24a(bits, convention=CONVENTION_REFERENCE): return _crc_check(0, bits, convention)
def check_crc24b(bits, convention=CONVENTION_REFERENCE): return _crc_check(1, bits, convention)
def check_crc16(bits, convention=CONVENTION_REFERENCE): return _crc_check(2, bits, convention)
def check_crc8(bits, convention=CONVENTION_REFERENCE): return _crc_check(3, bits, convention)


# ------------------------------------------------------------------------------------------
# segmentation (lte_turbo.h:83-92, 106)
# ------------------------------------------------------------------------------------------
@dataclass
class SegmentationResult:
    c: int
    c_plus: int
    c_minus: int
    k_plus: int
    k_minus: int
    filler_bits: int
    l: int
    code_blocks: list


def segment_transport_block(bits_with_crc, convention: int = CONVENTION_REFERENCE
                            ) -> SegmentationResult:
    b = _u8(bits_with_crc)
    s = _Seg()
    conv = int(convention)
    _call("tc_segment_transport_block_conv", conv, _ptr(b), b.size, C.addressof(s), None, 0)
    total = s.c_plus * s.k_plus + s.c_minus * s.k_minus
    cbs = np.empty(total, np.uint8)
    _call("tc_segment_transport_block_conv", conv, _ptr(b), b.size, C.addressof(s), _ptr(cbs),
          cbs.size)
    blocks, pos = [], 0
    for r in range(s.c):
        kr = s.k_minus if r < s.c_minus else s.k_plus
        blocks.append(cbs[pos:pos + kr].copy())
        pos += kr
    return SegmentationResult(s.c, s.c_plus, s.c_minus, s.k_plus, s.k_minus, s.filler_bits, s.l,
                              blocks)


# ------------------------------------------------------------------------------------------
# encoder / rate matching (lte_turbo.h:13-65, 111-118)
# ------------------------------------------------------------------------------------------
class LteChannelType(enum.Enum):
    UL_SCH = 0
    DL_SCH = 1
    PCH = 2
    MCH = 3


class DecoderBackend(enum.Enum):
    """Reference backends (lte_turbo.h:20-24) plus the B200 schedules.

    CpuReference is not provided by this library (decoding is GPU only) and raises; the
    reference's GPU backends map onto the B200 decoder: GpuStage1Exact decodes the full trellis
    (window >= K), GpuStage2Windowed uses the windowed schedule."""
    CpuReference = 0
    GpuStage1Exact = 1
    GpuStage2Windowed = 2
    GpuB200Plain = 3
    GpuB200Persistent = 4


@dataclass
class LteTurboCodecParams:
    channel_type: LteChannelType = LteChannelType.DL_SCH
    transport_block_bits: int = 0
    g_total: int = 0
    rv: int = 0
    num_layers: int = 1
    mod_order: int = 2
    n_soft: int = 0
    max_iterations: int = 8
    enable_early_stop: bool = False
    convention: int = 0  # CONVENTION_REFERENCE; CONVENTION_3GPP: the TS 36.212 code (new)


@dataclass
class CodeBlockDescriptor:
    block_index: int = 0
    k_r: int = 0
    d_r: int = 0
    e_r: int = 0
    filler_count: int = 0
    qpp_index: int = 0


@dataclass
class EncodedCodeBlock:
    descriptor: CodeBlockDescriptor
    cb_bits: np.ndarray
    systematic: np.ndarray
    parity0: np.ndarray
    parity1: np.ndarray
    rate_matched_bits: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint8))


@dataclass
class EncodedTransportBlock:
    params: LteTurboCodecParams
    tb_bits_with_crc: np.ndarray
    code_blocks: list
    transport_bits: np.ndarray


@dataclass
class DecodedTransportBlock:
    tb_bits: np.ndarray
    code_block_crc_ok: list
    transport_block_crc_ok: bool
    iterations_used: int
    posterior_llr: Optional[np.ndarray]


def turbo_encode_code_block(descriptor: CodeBlockDescriptor, cb_bits,
                            convention: int = CONVENTION_REFERENCE) -> EncodedCodeBlock:
    b = _u8(cb_bits)
    k = int(descriptor.k_r)
    if b.size != k:
        raise InvalidArgument("code block length mismatch")
    d = np.empty(3 * (k + 4), np.uint8)
    _call("tc_turbo_encode_conv", int(convention), k, int(descriptor.filler_count), _ptr(b),
          _ptr(d))
    desc = CodeBlockDescriptor(descriptor.block_index, k, k + 4, descriptor.e_r,
                               descriptor.filler_count, qpp_index(k))
    return EncodedCodeBlock(desc, b.copy(), d[:k + 4].copy(), d[k + 4:2 * k + 8].copy(),
                            d[2 * k + 8:].copy())


def compute_e(r: int, g_total: int, c: int, num_layers: int, mod_order: int) -> int:
    e = C.c_size_t()
    _call("tc_compute_e", r, g_total, c, num_layers, mod_order, C.addressof(e))
    return e.value


def rate_match(k: int, filler: int, d012, e: int, rv: int) -> np.ndarray:
    d = _u8(d012)
    out = np.empty(int(e), np.uint8)
    _call("tc_rate_match", int(k), int(filler), _ptr(d), int(e), int(rv), _ptr(out))
    return out


def encode_transport_block(params: LteTurboCodecParams, transport_bits) -> EncodedTransportBlock:
    """CRC24A, segmentation, per-block encoding and rate matching (lte_turbo.cpp:690-720)."""
    bits = _u8(transport_bits)
    if params.transport_block_bits != bits.size:
        raise InvalidArgument("transport block size does not match params")
    conv = int(params.convention)
    with_crc = append_crc24a(bits, conv)
    seg = segment_transport_block(with_crc, conv)
    blocks = []
    for r, cb in enumerate(seg.code_blocks):
        k = cb.size
        desc = CodeBlockDescriptor(r, k, k + 4,
                                   compute_e(r, params.g_total, seg.c, params.num_layers,
                                             params.mod_order),
                                   seg.filler_bits if r == 0 else 0, qpp_index(k))
        enc = turbo_encode_code_block(desc, cb, conv)
        d012 = np.concatenate([enc.systematic, enc.parity0, enc.parity1])
        enc.rate_matched_bits = rate_match(k, desc.filler_count, d012, desc.e_r, params.rv)
        blocks.append(enc)
    return EncodedTransportBlock(params, with_crc, blocks, bits.copy())


def derate_match_code_block(params: LteTurboCodecParams, descriptor: CodeBlockDescriptor,
                            rate_matched_bits) -> np.ndarray:
    """Hard bits -> [d0|d1|d2] LLRs of +-8 per bit (lte_turbo.cpp:722-734)."""
    b = _u8(rate_matched_bits)
    k = int(descriptor.k_r)
    out = np.empty(3 * (k + 4), np.float32)
    _call("tc_derate_match_bits", k, int(descriptor.filler_count), _ptr(b), b.size,
          int(params.rv), _ptr(out))
    return out


def derate_match_llr(k: int, filler: int, e_llr, rv: int) -> np.ndarray:
    """LLR-domain de-rate matching: soft values summed where the reference adds +-8."""
    x = np.ascontiguousarray(e_llr, np.float32)
    out = np.empty(3 * (int(k) + 4), np.float32)
    _call("tc_derate_match_llr", int(k), int(filler), _ptr(x), x.size, int(rv), _ptr(out))
    return out


def random_bits(seed: int, n: int, first: int = 0) -> np.ndarray:
    out = np.empty(int(n), np.uint8)
    _call("tc_random_bits", int(seed), int(first), int(n), _ptr(out))
    return out


def awgn_llr(seed: int, bits, sigma2: float, first: int = 0) -> np.ndarray:
    b = _u8(bits)
    out = np.empty(b.size, np.float32)
    _call("tc_awgn_llr", int(seed), int(first), _ptr(b), b.size, float(sigma2), _ptr(out))
    return out


def awgn_code_blocks(seed: int, ks, ebn0_db, fillers=None, crc24b: bool = False,
                     threads: int = 0):
    """Seeded BPSK/AWGN code blocks (C++, multi-threaded).  Returns (info bits per block as one
    array, LLRs [d0|d1|d2] per block back to back)."""
    ks = np.ascontiguousarray(ks, np.int32)
    n = ks.size
    f = np.zeros(n, np.int32) if fillers is None else np.ascontiguousarray(fillers, np.int32)
    eb = np.ascontiguousarray(np.broadcast_to(np.asarray(ebn0_db, np.float32), (n,)))
    bits = np.empty(int(ks.sum()), np.uint8)
    llr = np.empty(int(3 * (ks.astype(np.int64) + 4).sum()), np.float32)
    _call("tc_awgn_code_blocks", int(seed), n, _ptr(ks), _ptr(f), _ptr(eb), int(bool(crc24b)),
          _ptr(bits), _ptr(llr), int(threads))
    return bits, llr


# ------------------------------------------------------------------------------------------
# GPU decoder
# ------------------------------------------------------------------------------------------
@dataclass
class DecodeOptions:
    max_iterations: int = 8
    early_stop: bool = False
    window: int = 0          # 0: default (128); >= K: full trellis
    guard: int = -1          # <0: default (96)
    schedule: int = SCHEDULE_PLAIN
    scales: Optional[Sequence[float]] = None  # 2 per iteration; None = 1.0
    graph: bool = False      # device memory: capture once, replay the CUDA graph
    convention: int = 0      # CONVENTION_REFERENCE; CONVENTION_3GPP: LLRs of the TS 36.212 code


class Decoder:
    """Owns a tc_decoder (device buffers, QPP tables, stream) on one GPU."""

    def __init__(self, device: int = 0):
        lib = load_library()
        self._lib = lib
        h = C.c_void_p()
        _call("tc_decoder_create", int(device), C.addressof(h))
        self._h = h
        self.device = int(device)

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.tc_decoder_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _opts(o: DecodeOptions, memory: int, stream: int = 0):
        opt = _Options()
        opt.max_iterations = int(o.max_iterations)
        opt.early_stop = int(bool(o.early_stop))
        opt.window = int(o.window)
        opt.guard = int(o.guard)
        opt.memory = memory
        opt.schedule = int(o.schedule)
        keep = None
        if o.scales is not None:
            keep = np.ascontiguousarray(o.scales, np.float32)
            if keep.size < 2 * o.max_iterations:
                raise InvalidArgument("scales needs 2 entries per iteration")
            opt.scales = keep.ctypes.data
        opt.graph = int(bool(o.graph))
        opt.stream = stream or None
        opt.convention = int(o.convention)
        return opt, keep

    def inject_stall(self, task: int) -> None:
        """Testing hook: persistent decodes time out waiting on `task` (-1 turns it off)."""
        _call("tc_decoder_inject_stall", self._h, int(task))

    def sync(self) -> None:
        """Waits for enqueued work; raises DeviceTimeout if a device-side wait gave up."""
        _call("tc_decoder_sync", self._h)

    def decode_async(self, cbs, n_cb: int, llr_ptr: int, llr_len: int, post_ptr: int,
                     post_len: int, crc_ptr: int = 0, iters_ptr: int = 0,
                     options: Optional[DecodeOptions] = None) -> None:
        """TC_MEM_HOST_ASYNC: host pointers (pinned for overlap, e.g. torch pin_memory()
        tensors); enqueues copy-in, decode and copy-out and returns.  Results are valid after
        sync(); consecutive calls overlap one call's copies with earlier calls' decoding."""
        o = options or DecodeOptions()
        opt, _keep = self._opts(o, MEM_HOST_ASYNC)
        _call("tc_decode", self._h, int(n_cb), C.addressof(cbs), int(llr_len), llr_ptr,
              int(post_len), post_ptr, crc_ptr or None, iters_ptr or None, C.addressof(opt))

    def autotune(self, cbs, n_cb: int, llr_ptr: int, llr_len: int, post_ptr: int, post_len: int,
                 options: Optional[DecodeOptions] = None, stream: int = 0) -> dict:
        """Times the candidate schedules/windows on this device-memory request and remembers the
        fastest for SCHEDULE_AUTO; returns {schedule, window, ms}."""
        o = options or DecodeOptions()
        opt, _keep = self._opts(o, MEM_DEVICE, stream)
        r = _TuneResult()
        _call("tc_autotune", self._h, int(n_cb), C.addressof(cbs), int(llr_len), llr_ptr,
              int(post_len), post_ptr, C.addressof(opt), C.addressof(r))
        return {"schedule": r.schedule, "window": r.window, "ms": r.ms}

    @staticmethod
    def rm_blocks(blocks):
        """tc_rm_block array from (k, filler, e, rv) tuples; E LLRs back to back, outputs
        [d0|d1|d2] back to back."""
        b = np.asarray(blocks, np.int64).reshape(-1, 4)
        n = b.shape[0]
        e_off = np.concatenate([[0], np.cumsum(b[:, 2])])
        llr_off = np.concatenate([[0], np.cumsum(3 * (b[:, 0] + 4))])
        rec = np.zeros(max(n, 1), dtype=_RM_BLOCK_DTYPE)
        rec["k"][:n], rec["filler"][:n], rec["e"][:n], rec["rv"][:n] = b[:, 0], b[:, 1], b[:, 2], b[:, 3]
        rec["e_offset"][:n], rec["llr_offset"][:n] = e_off[:-1], llr_off[:-1]
        arr = (_RmBlock * max(n, 1)).from_buffer(rec)  # shares (and keeps) rec's memory
        return arr, int(e_off[-1]), int(llr_off[-1])

    def derate_device(self, blocks, e_ptr: int, e_len: int, out_ptr: int, llr_len: int,
                      stream: int = 0) -> None:
        """LLR-domain de-rate matching on the GPU (device pointers)."""
        arr, _, _ = self.rm_blocks(blocks)
        _call("tc_derate_match_llr_device", self._h, len(blocks), C.addressof(arr), int(e_len),
              e_ptr, int(llr_len), out_ptr, stream or None)

    # -- test-vector generation on the device (torch CUDA tensors out) --
    def awgn_code_blocks_device(self, seed: int, ks, ebn0_db, fillers=None, crc24b: bool = False,
                                stream: int = 0):
        """The device version of awgn_code_blocks: returns (bits uint8, LLRs float32) as CUDA
        tensors in the same layout, bits identical to the host generator's."""
        import torch

        ks = np.ascontiguousarray(ks, np.int32)
        n = ks.size
        f = np.zeros(n, np.int32) if fillers is None else np.ascontiguousarray(fillers, np.int32)
        eb = np.ascontiguousarray(np.broadcast_to(np.asarray(ebn0_db, np.float32), (n,)))
        dev = torch.device("cuda", self.device)
        bits = torch.empty(int(ks.sum()), dtype=torch.uint8, device=dev)
        llr = torch.empty(int(3 * (ks.astype(np.int64) + 4).sum()), dtype=torch.float32, device=dev)
        _call("tc_awgn_code_blocks_device", self._h, int(seed), n, _ptr(ks), _ptr(f), _ptr(eb),
              int(bool(crc24b)), bits.data_ptr(), llr.data_ptr(), stream or None)
        return bits, llr

    def turbo_encode_device(self, ks, bits, fillers=None, stream: int = 0):
        """Encodes blocks stored back to back in the CUDA uint8 tensor `bits`; returns their
        [d0|d1|d2] bits back to back (CUDA uint8 tensor)."""
        import torch

        ks = np.ascontiguousarray(ks, np.int32)
        f = np.zeros(ks.size, np.int32) if fillers is None else np.ascontiguousarray(fillers, np.int32)
        d = torch.empty(int(3 * (ks.astype(np.int64) + 4).sum()), dtype=torch.uint8,
                        device=bits.device)
        _call("tc_turbo_encode_device", self._h, ks.size, _ptr(ks), _ptr(f), bits.data_ptr(),
              d.data_ptr(), stream or None)
        return d

    def rate_match_device(self, blocks, d012, stream: int = 0):
        """blocks = (k, filler, e, rv) per block, encoded bits back to back in the CUDA uint8
        tensor d012; returns the E rate-matched bits per block back to back."""
        import torch

        arr, e_len, d_len = self.rm_blocks(blocks)
        out = torch.empty(max(e_len, 1), dtype=torch.uint8, device=d012.device)
        _call("tc_rate_match_device", self._h, len(blocks), C.addressof(arr), int(d012.numel()),
              d012.data_ptr(), int(e_len), out.data_ptr(), stream or None)
        return out[:e_len]

    def derate_combine_device(self, transmissions, e_ptr: int, e_len: int, out_ptr: int,
                              llr_len: int, stream: int = 0) -> None:
        """HARQ soft combining on the GPU: transmissions = (k, filler, e, rv, e_offset,
        llr_offset) tuples, those of one code block consecutive with the same llr_offset; each
        code block's [d0|d1|d2] becomes the sum of its transmissions' de-rate-matched LLRs."""
        arr = (_RmBlock * max(len(transmissions), 1))()
        for i, (k, f, e, rv, eo, lo) in enumerate(transmissions):
            arr[i].k, arr[i].filler, arr[i].e, arr[i].rv = int(k), int(f), int(e), int(rv)
            arr[i].e_offset, arr[i].llr_offset = int(eo), int(lo)
        _call("tc_derate_combine_llr_device", self._h, len(transmissions), C.addressof(arr),
              int(e_len), e_ptr, int(llr_len), out_ptr, stream or None)

    @staticmethod
    def tb_descriptors(tbs):
        """tc_transport_block array for tbs = list of (TBS, n_cb) in order, bits back to back.
        Returns (array, total decoded bits)."""
        tba = (_TransportBlock * max(len(tbs), 1))()
        first = bits = 0
        for i, (size, ncb) in enumerate(tbs):
            tba[i].tbs, tba[i].first_cb, tba[i].n_cb, tba[i].bits_offset = (
                int(size), first, int(ncb), bits)
            first += int(ncb)
            bits += int(size)
        return tba, bits

    def decode_tbs_async(self, tba, n_tb: int, arr, n_cb: int, e_len: int, e_llr_ptr: int,
                         bits_len: int, bits_ptr: int, tb_ok_ptr: int = 0, cb_ok_ptr: int = 0,
                         iters_ptr: int = 0, options: Optional[DecodeOptions] = None) -> None:
        """tc_decode_transport_blocks with TC_MEM_HOST_ASYNC: host pointers (pinned for
        overlap), descriptors from tb_descriptors() and rm_blocks(); returns once enqueued.
        Results are valid after sync()."""
        o = options or DecodeOptions()
        opt, _keep = self._opts(o, MEM_HOST_ASYNC)
        _call("tc_decode_transport_blocks", self._h, int(n_tb), C.addressof(tba), int(n_cb),
              C.addressof(arr), int(e_len), e_llr_ptr, int(bits_len), bits_ptr,
              tb_ok_ptr or None, cb_ok_ptr or None, iters_ptr or None, None, C.addressof(opt))

    def decode_tbs_device(self, tba, n_tb: int, arr, n_cb: int, e_len: int, e_llr_ptr: int,
                          bits_len: int, bits_ptr: int, tb_ok_ptr: int = 0, cb_ok_ptr: int = 0,
                          iters_ptr: int = 0, options: Optional[DecodeOptions] = None,
                          stream: int = 0) -> None:
        """tc_decode_transport_blocks with TC_MEM_DEVICE: device pointers, descriptors from
        tb_descriptors() and rm_blocks(), ordered on `stream`; returns once enqueued.  With
        options.graph the chain is captured once per request key and replayed (needs a created
        stream); SCHEDULE_AUTO applies the autotuning table."""
        o = options or DecodeOptions()
        opt, _keep = self._opts(o, MEM_DEVICE, stream)
        _call("tc_decode_transport_blocks", self._h, int(n_tb), C.addressof(tba), int(n_cb),
              C.addressof(arr), int(e_len), e_llr_ptr, int(bits_len), bits_ptr,
              tb_ok_ptr or None, cb_ok_ptr or None, iters_ptr or None, None, C.addressof(opt))

    def decode_tbs(self, tbs, blocks, e_llr, options: Optional[DecodeOptions] = None,
                   want_posterior: bool = False):
        """Many transport blocks through the device chain (host arrays): tbs = list of
        (TBS, n_cb); blocks = (k, filler, e, rv) per code block in transport-block order;
        e_llr = their rate-matched LLRs back to back.  Returns (bits per TB, tb_crc_ok,
        cb_crc_ok, iterations per code block[, posterior])."""
        o = options or DecodeOptions()
        arr, e_len, _ = self.rm_blocks(blocks)
        x = np.ascontiguousarray(e_llr, np.float32)
        if x.size != e_len:
            raise InvalidArgument(f"expected {e_len} rate-matched LLRs, got {x.size}")
        tba, bits = self.tb_descriptors(tbs)
        out = np.zeros(bits, np.uint8)
        tb_ok = np.zeros(len(tbs), np.uint8)
        cb_ok = np.zeros(len(blocks), np.uint8)
        it = np.zeros(len(blocks), np.uint32)
        post = np.zeros(sum(int(b[0]) for b in blocks), np.float32) if want_posterior else None
        opt, _keep = self._opts(o, MEM_HOST)
        _call("tc_decode_transport_blocks", self._h, len(tbs), C.addressof(tba), len(blocks),
              C.addressof(arr), e_len, _ptr(x), bits, _ptr(out), _ptr(tb_ok), _ptr(cb_ok),
              _ptr(it), _ptr(post) if post is not None else None, C.addressof(opt))
        per_tb, pos = [], 0
        for size, _ in tbs:
            per_tb.append(out[pos:pos + int(size)])
            pos += int(size)
        res = (per_tb, tb_ok.astype(bool), cb_ok.astype(bool), it)
        return res + (post,) if want_posterior else res

    def save_tuning(self, path: str) -> None:
        _call("tc_autotune_save", self._h, os.fsencode(path))

    def load_tuning(self, path: str) -> None:
        _call("tc_autotune_load", self._h, os.fsencode(path))

    def set_timing(self, on: bool) -> None:
        _call("tc_decoder_set_timing", self._h, int(bool(on)))

    def timing(self, reset: bool = False) -> dict:
        t = _Timing()
        _call("tc_decoder_timing", self._h, C.addressof(t), int(bool(reset)))
        return dict(launches=t.launches, siso_launches=t.siso_launches, siso_ms=t.siso_ms,
                    trellis_steps=t.trellis_steps)

    @staticmethod
    def layout(ks: Sequence[int], fillers: Optional[Sequence[int]] = None):
        """Descriptor array for blocks stored back to back: [d0|d1|d2] per block, K posteriors."""
        ks = np.asarray(ks, np.int64)
        n = ks.size
        fillers = np.zeros(n, np.int64) if fillers is None else np.asarray(fillers, np.int64)
        llr_off = np.concatenate([[0], np.cumsum(3 * (ks + 4))])
        out_off = np.concatenate([[0], np.cumsum(ks)])
        rec = np.zeros(max(n, 1), dtype=_CODE_BLOCK_DTYPE)
        rec["k"][:n], rec["filler"][:n] = ks, fillers
        rec["llr_offset"][:n], rec["out_offset"][:n] = llr_off[:-1], out_off[:-1]
        cbs = (_CodeBlock * max(n, 1)).from_buffer(rec)  # shares (and keeps) rec's memory
        return cbs, int(llr_off[-1]), int(out_off[-1])

    def decode(self, ks, llr, fillers=None, options: Optional[DecodeOptions] = None):
        """Host arrays in, host arrays out (synchronous).  Returns (posterior, crc_ok, iters)."""
        o = options or DecodeOptions()
        ks = np.asarray(ks, np.int64)
        cbs, llr_len, post_len = self.layout(ks, fillers)
        x = np.ascontiguousarray(llr, np.float32)
        if x.size != llr_len:
            raise InvalidArgument(f"expected {llr_len} LLRs, got {x.size}")
        post = np.zeros(post_len, np.float32)
        ok = np.zeros(ks.size, np.uint8)
        it = np.zeros(ks.size, np.uint32)
        opt, _keep = self._opts(o, MEM_HOST)
        _call("tc_decode", self._h, ks.size, C.addressof(cbs), llr_len, _ptr(x), post_len,
              _ptr(post), _ptr(ok), _ptr(it), C.addressof(opt))
        return post, ok.astype(bool), it

    def decode_device(self, cbs, n_cb: int, llr_ptr: int, llr_len: int, post_ptr: int,
                      post_len: int, crc_ptr: int = 0, iters_ptr: int = 0,
                      options: Optional[DecodeOptions] = None, stream: int = 0) -> None:
        """Device pointers (e.g. torch tensors' data_ptr()); ordered on ``stream`` (a
        cudaStream_t as an int; 0 = the legacy default stream)."""
        o = options or DecodeOptions()
        opt, _keep = self._opts(o, MEM_DEVICE, stream)
        _call("tc_decode", self._h, int(n_cb), C.addressof(cbs), int(llr_len), llr_ptr,
              int(post_len), post_ptr, crc_ptr or None, iters_ptr or None, C.addressof(opt))


class AdjointDecoder:
    """The differentiable decoder (tc_adjoint_*): a taped forward pass over ``iterations``
    unrolled iterations with an extrinsic scale per half-iteration, and the hand-written
    backward pass (d loss / d LLRs and d loss / d scales from d loss / d posterior).  Device
    buffers only (e.g. torch tensors' data_ptr()), ordered on ``stream``."""

    def __init__(self, decoder: Decoder):
        self._dec = decoder  # the tables live in the decoder: keep it alive
        self._lib = decoder._lib
        h = C.c_void_p()
        _call("tc_adjoint_create", decoder._h, C.addressof(h))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.tc_adjoint_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, cbs, n_cb: int, llr_ptr: int, llr_len: int, post_ptr: int, post_len: int,
                iterations: int, scales=None, window: int = 0, guard: int = -1,
                stream: int = 0, convention: int = CONVENTION_REFERENCE) -> int:
        """Decodes and records the tape; returns the tape id for backward().  convention: the
        code of the LLRs (CONVENTION_REFERENCE or CONVENTION_3GPP)."""
        sc = None
        if scales is not None:
            sc = np.ascontiguousarray(scales, np.float32)
            if sc.size != 2 * iterations:
                raise InvalidArgument("scales: two per iteration")
        tape = C.c_uint64()
        _call("tc_adjoint_forward_conv", int(convention), self._h, int(n_cb), C.addressof(cbs),
              int(llr_len), llr_ptr, int(post_len), post_ptr, int(iterations),
              None if sc is None else _ptr(sc), int(window), int(guard), stream or None,
              C.addressof(tape))
        return tape.value

    def backward(self, tape: int, grad_post_ptr: int, grad_llr_ptr: int, grad_scales_ptr: int,
                 stream: int = 0) -> None:
        _call("tc_adjoint_backward", self._h, int(tape), grad_post_ptr, grad_llr_ptr,
              grad_scales_ptr, stream or None)

    def launches(self) -> int:
        n = C.c_uint64()
        _call("tc_adjoint_launches", self._h, C.addressof(n))
        return n.value


_default_decoders: dict = {}


def _decoder(device: int = 0) -> Decoder:
    d = _default_decoders.get(device)
    if d is None:
        d = _default_decoders[device] = Decoder(device)
    return d


def turbo_decode_code_block_gpu(descriptor: CodeBlockDescriptor, d0_llr, d1_llr, d2_llr,
                                max_iterations: int = 8, enable_early_stop: bool = False,
                                window: int = 0, guard: int = -1):
    """One code block, as turbo_decode_code_block_gpu_stage2 (lte_turbo.h:138-145).

    Returns (posterior[K], crc_ok, iterations_used)."""
    k = int(descriptor.k_r)
    parts = [np.asarray(x, np.float32) for x in (d0_llr, d1_llr, d2_llr)]
    if any(p.size != k + 4 for p in parts):
        raise InvalidArgument("invalid LLR sizes for turbo decode")
    post, ok, it = _decoder().decode(
        [k], np.concatenate(parts), [descriptor.filler_count],
        DecodeOptions(max_iterations, enable_early_stop, window, guard))
    return post, bool(ok[0]), int(it[0])


def decode_transport_block(params: LteTurboCodecParams, encoded: EncodedTransportBlock,
                           backend: DecoderBackend = DecoderBackend.GpuB200Plain
                           ) -> DecodedTransportBlock:
    """De-rate matching, GPU decoding of all code blocks in one call, then hard decisions,
    filler strip, CRC24B per block (C > 1) and CRC24A (lte_turbo.cpp:891-980)."""
    if backend == DecoderBackend.CpuReference:
        raise InvalidArgument("CPU decoding is not part of turbo_cpp_b200; use a GPU backend")
    blocks = encoded.code_blocks
    ks = [b.descriptor.k_r for b in blocks]
    fillers = [b.descriptor.filler_count for b in blocks]
    llr = np.concatenate([derate_match_code_block(params, b.descriptor, b.rate_matched_bits)
                          for b in blocks])
    window = 6144 if backend == DecoderBackend.GpuStage1Exact else 0
    schedule = SCHEDULE_PERSISTENT if backend == DecoderBackend.GpuB200Persistent else SCHEDULE_PLAIN
    conv = int(params.convention)
    post, ok, it = _decoder().decode(ks, llr, fillers, DecodeOptions(
        params.max_iterations, params.enable_early_stop, window, -1, schedule,
        convention=conv))
    tb, cb_ok, pos = [], [], 0
    for b in blocks:
        k = b.descriptor.k_r
        hard = (post[pos:pos + k] >= 0).astype(np.uint8)[b.descriptor.filler_count:]
        pos += k
        good = True
        if len(blocks) > 1:
            good = check_crc24b(hard, conv)
            hard = hard[:-24]
        tb.append(hard)
        cb_ok.append(good)
    tb_bits = np.concatenate(tb) if tb else np.zeros(0, np.uint8)
    return DecodedTransportBlock(tb_bits[:-24].copy(), cb_ok, check_crc24a(tb_bits, conv),
                                 int(it.max()) if len(it) else 0, post)
