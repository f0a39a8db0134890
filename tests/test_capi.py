"""The C-ABI library loads, exports every symbol include/*.h declares, and reports errors as
status codes.  CPU only: no decoding without a GPU."""
from __future__ import annotations

import ctypes as C
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        names |= set(re.findall(r"TC_API\s+[\w\s\*]+?\b(tc_\w+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("tc_decoder_create", "tc_decode", "tc_derate_match_llr", "tc_crc_check",
                 "tc_segment_transport_block", "tc_turbo_encode", "tc_rate_match"):
        assert must in names


def test_library_exports_every_declared_symbol(tc):
    lib = tc.load_library()
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", tc.LIB_PATH], capture_output=True,
                         text=True).stdout
    exported = set(re.findall(r"\bT\s+(tc_\w+)", out))
    assert set(declared_symbols()) <= exported
    assert all(n.startswith("tc_") for n in exported)  # nothing else leaks at the boundary


def test_status_codes(tc):
    lib = tc.load_library()
    idx = C.c_int32()
    assert lib.tc_qpp_index(41, C.addressof(idx)) == 2  # TC_ERR_OUT_OF_RANGE
    assert b"unsupported" in lib.tc_last_error()
    assert lib.tc_qpp_index(6144, C.addressof(idx)) == 0 and idx.value == 187
    assert lib.tc_last_error() == b""
    assert lib.tc_crc_append(9, None, 0, None) == 1  # TC_ERR_INVALID_ARGUMENT
    assert lib.tc_status_name(4) == b"TC_ERR_CUDA"
    bits = np.zeros(40, np.uint8)
    out = np.zeros(3 * 44, np.uint8)
    assert lib.tc_turbo_encode(40, 40, bits.ctypes.data, out.ctypes.data) == 1  # filler >= K
    assert lib.tc_turbo_encode(44, 0, bits.ctypes.data, out.ctypes.data) == 2
    assert lib.tc_rate_match(40, 0, out.ctypes.data, 10, 4, out.ctypes.data) == 1  # rv > 3
    assert lib.tc_decode(None, 0, None, 0, None, 0, None, None, None, None) == 1
    e = C.c_size_t()
    assert lib.tc_compute_e(0, 101, 1, 1, 2, C.addressof(e)) == 1  # G not a multiple of NL*Qm


def test_python_errors_map_to_reference_exception_kinds(tc):
    with pytest.raises(ValueError):          # std::invalid_argument
        tc.turbo_encode_code_block(tc.CodeBlockDescriptor(k_r=40), np.zeros(39, np.uint8))
    with pytest.raises(IndexError):          # std::out_of_range
        tc.qpp_permutation(7)


def test_decoder_without_device_fails_loudly(tc):
    """Without a GPU there is no fallback: creating a decoder reports TC_ERR_NO_DEVICE."""
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(tc.NoDevice):
        tc.Decoder(0)
    with pytest.raises(tc.InvalidArgument):
        tc.decode_transport_block(tc.LteTurboCodecParams(), None, tc.DecoderBackend.CpuReference)


def test_header_is_plain_c(tc, tmp_path):
    """include/turbo_b200.h compiles as C99 with -pedantic -Werror, and a C program linked to
    libturbo_b200.so calls the CPU-side entry points (36.212 CRC check value, option defaults,
    segmentation sizes, QPP, encoder, error status); its view of tc_decode_options has the
    size the Python binding uses."""
    import shutil

    if shutil.which("gcc") is None:
        pytest.skip("gcc is not available")
    lib_dir = os.path.join(ROOT, "turbo_cpp_b200", "lib")
    exe = str(tmp_path / "c_api_check")
    r = subprocess.run(["gcc", "-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror",
                        "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "cpp", "c_api_check.c"), "-o", exe,
                        "-L", lib_dir, "-lturbo_b200", f"-Wl,-rpath,{lib_dir}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.split() == ["c", "api", "ok", str(C.sizeof(tc._Options))]
