"""TEST INFRASTRUCTURE ONLY: ctypes loaders for the oracle libraries.

``liboracle.so`` is the C restatement of the Wiseung/Turbo_CPP CPU codec chain
(``turbo_oracle.c``); ``_ref/libturbo_ref.so`` is the reference's own ``src/lte_turbo.cpp``
built CPU-only with a C shim (``ref_shim.cpp``).  Only ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may use this package; the
product library (``turbo_cpp_b200``) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libturbo_ref.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")

CRC24A, CRC24B, CRC16, CRC8 = 0, 1, 2, 3
CRC_LEN = {CRC24A: 24, CRC24B: 24, CRC16: 16, CRC8: 8}


def build(ref_root: str | None = None) -> None:
    """Compile liboracle.so and, when the reference sources are given (`ref_root`, else the
    TURBO_CPP_REF environment variable) and exist, _ref/libturbo_ref.so.  Without them the
    reference library is skipped with a notice (a prebuilt one is kept)."""
    ref_root = ref_root or os.environ.get("TURBO_CPP_REF", "")
    subprocess.run(["make", "-s", "-C", HERE, "all", f"REF={ref_root}"], check=True)


def _sig(lib, name, res, args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args
    return f


class _Lib:
    """Common wrappers; ``prefix`` is ``or_`` for the restatement, ``ref_`` for the reference."""

    def __init__(self, path: str, prefix: str):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.path = path
        self.lib = C.CDLL(path)
        self.prefix = prefix


class Oracle(_Lib):
    def __init__(self, path: str = ORACLE_SO):
        super().__init__(path, "or_")
        L = self.lib
        _sig(L, "or_qpp_count", C.c_int, [])
        _sig(L, "or_qpp_entry", None, [C.c_int] + [C.POINTER(C.c_int32)] * 3)
        _sig(L, "or_qpp_index", C.c_int, [C.c_int32])
        _sig(L, "or_qpp_perm", None, [C.c_int32, _i32p])
        _sig(L, "or_crc_append", None, [C.c_int, _u8p, C.c_size_t, _u8p])
        _sig(L, "or_crc_check", C.c_int, [C.c_int, _u8p, C.c_size_t])
        _sig(L, "or_segment", C.c_int, [_u8p, C.c_size_t, C.POINTER(SegInfo), C.c_void_p])
        _sig(L, "or_turbo_encode", None, [C.c_int32, C.c_int32, _u8p, _u8p, _u8p, _u8p])
        _sig(L, "or_compute_e", C.c_int64, [C.c_size_t] * 5)
        _sig(L, "or_rate_match", None,
             [C.c_int32, C.c_int32, _u8p, _u8p, _u8p, C.c_size_t, C.c_int32, _u8p])
        _sig(L, "or_derate_bits", None,
             [C.c_int32, C.c_int32, _u8p, C.c_size_t, C.c_int32, _f32p])
        _sig(L, "or_derate_llr", None,
             [C.c_int32, C.c_int32, _f32p, C.c_size_t, C.c_int32, _f32p])
        _sig(L, "or_decode_cb", None,
             [C.c_int32, C.c_int32, _f32p, C.c_int32, C.c_int32, _f32p,
              C.POINTER(C.c_int32), C.POINTER(C.c_int32)])
        _sig(L, "or_decode_cb_windowed", None,
             [C.c_int32, C.c_int32, _f32p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _f32p,
              C.POINTER(C.c_int32), C.POINTER(C.c_int32)])
        batch_args = [C.c_int32, _i32p, _i32p, _i64p, _f32p, _i64p, _f32p, C.c_int32,
                      C.c_int32]
        _sig(L, "or_decode_batch", None, batch_args + [_i32p, _i32p, C.c_int32])
        _sig(L, "or_decode_batch_windowed", None,
             batch_args + [C.c_int32, C.c_int32, _i32p, _i32p, C.c_int32])
        _sig(L, "or_std_crc_append", None, [C.c_int, _u8p, C.c_size_t, _u8p])
        _sig(L, "or_std_crc_check", C.c_int, [C.c_int, _u8p, C.c_size_t])
        _sig(L, "or_std_turbo_encode", None, [C.c_int32, C.c_int32, _u8p, _u8p, _u8p, _u8p])
        _sig(L, "or_std_decode_cb_windowed", None,
             [C.c_int32, C.c_int32, _f32p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _f32p,
              C.POINTER(C.c_int32), C.POINTER(C.c_int32)])
        _f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        _f64n = C.POINTER(C.c_double)
        _sig(L, "or_adj_seed_count", C.c_int64, [C.c_int32, C.c_int32, C.c_int32])
        _sig(L, "or_adj_vjp", None,
             [C.c_int32, _f64p, C.c_int32, _f64p, C.c_int32, C.c_int32] + [_f64n] * 6)
        _sig(L, "or_std_adj_vjp", None,
             [C.c_int32, _f64p, C.c_int32, _f64p, C.c_int32, C.c_int32] + [_f64n] * 6)

    # -- QPP --
    def qpp_table(self):
        out = []
        for i in range(self.lib.or_qpp_count()):
            k, f1, f2 = C.c_int32(), C.c_int32(), C.c_int32()
            self.lib.or_qpp_entry(i, C.byref(k), C.byref(f1), C.byref(f2))
            out.append((k.value, f1.value, f2.value))
        return out

    def qpp_perm(self, k: int) -> np.ndarray:
        p = np.empty(k, np.int32)
        self.lib.or_qpp_perm(k, p)
        return p

    # -- CRC --
    def crc_append(self, kind: int, bits) -> np.ndarray:
        b = np.ascontiguousarray(bits, np.uint8)
        out = np.empty(b.size + CRC_LEN[kind], np.uint8)
        self.lib.or_crc_append(kind, b, b.size, out)
        return out

    def crc_check(self, kind: int, bits) -> bool:
        b = np.ascontiguousarray(bits, np.uint8)
        return bool(self.lib.or_crc_check(kind, b, b.size))

    # -- segmentation --
    def segment(self, bits):
        b = np.ascontiguousarray(bits, np.uint8)
        info = SegInfo()
        rc = self.lib.or_segment(b, b.size, C.byref(info), None)
        if rc != 0:
            raise ValueError(f"segmentation failed ({rc})")
        total = info.c_plus * info.k_plus + info.c_minus * info.k_minus
        cbs = np.empty(total, np.uint8)
        self.lib.or_segment(b, b.size, C.byref(info), cbs.ctypes.data_as(C.c_void_p))
        return info.as_dict(), cbs

    # -- encoder / rate matching --
    def turbo_encode(self, k: int, filler: int, cb) -> np.ndarray:
        cbb = np.ascontiguousarray(cb, np.uint8)
        d = [np.empty(k + 4, np.uint8) for _ in range(3)]
        self.lib.or_turbo_encode(k, filler, cbb, *d)
        return np.concatenate(d)

    def compute_e(self, r, g_total, c, nl, qm) -> int:
        return int(self.lib.or_compute_e(r, g_total, c, nl, qm))

    def rate_match(self, k: int, filler: int, d012, e: int, rv: int) -> np.ndarray:
        d = k + 4
        a = np.ascontiguousarray(d012, np.uint8)
        out = np.empty(e, np.uint8)
        self.lib.or_rate_match(d, filler, np.ascontiguousarray(a[:d]),
                               np.ascontiguousarray(a[d:2 * d]),
                               np.ascontiguousarray(a[2 * d:]), e, rv, out)
        return out

    def derate_bits(self, k: int, filler: int, e_bits, rv: int) -> np.ndarray:
        b = np.ascontiguousarray(e_bits, np.uint8)
        out = np.empty(3 * (k + 4), np.float32)
        self.lib.or_derate_bits(k + 4, filler, b, b.size, rv, out)
        return out

    def derate_llr(self, k: int, filler: int, e_llr, rv: int) -> np.ndarray:
        b = np.ascontiguousarray(e_llr, np.float32)
        out = np.empty(3 * (k + 4), np.float32)
        self.lib.or_derate_llr(k + 4, filler, b, b.size, rv, out)
        return out

    # -- decoder --
    def decode_cb(self, k, filler, llr, iters=8, early_stop=False, window=0, guard=0):
        """window=0: the reference's full-trellis decoder; window>0: the windowed schedule."""
        llr = np.ascontiguousarray(llr, np.float32)
        post = np.empty(k, np.float32)
        ok, used = C.c_int32(), C.c_int32()
        if window:
            self.lib.or_decode_cb_windowed(k, filler, llr, iters, int(early_stop), window, guard,
                                           post, C.byref(ok), C.byref(used))
        else:
            self.lib.or_decode_cb(k, filler, llr, iters, int(early_stop), post, C.byref(ok),
                                  C.byref(used))
        return post, bool(ok.value), used.value

    # -- the TS 36.212 code (no reference counterpart) --
    def std_crc_append(self, kind: int, bits) -> np.ndarray:
        b = np.ascontiguousarray(bits, np.uint8)
        out = np.empty(b.size + CRC_LEN[kind], np.uint8)
        self.lib.or_std_crc_append(kind, b, b.size, out)
        return out

    def std_crc_check(self, kind: int, bits) -> bool:
        b = np.ascontiguousarray(bits, np.uint8)
        return bool(self.lib.or_std_crc_check(kind, b, b.size))

    def std_turbo_encode(self, k: int, filler: int, cb) -> np.ndarray:
        cbb = np.ascontiguousarray(cb, np.uint8)
        d = [np.empty(k + 4, np.uint8) for _ in range(3)]
        self.lib.or_std_turbo_encode(k, filler, cbb, *d)
        return np.concatenate(d)

    def std_decode_cb(self, k, filler, llr, iters=8, early_stop=False, window=0, guard=0):
        """The windowed schedule (window 0: full trellis) on the TS 36.212 code."""
        llr = np.ascontiguousarray(llr, np.float32)
        post = np.empty(k, np.float32)
        ok, used = C.c_int32(), C.c_int32()
        self.lib.or_std_decode_cb_windowed(k, filler, llr, iters, int(early_stop), window, guard,
                                           post, C.byref(ok), C.byref(used))
        return post, bool(ok.value), used.value

    # -- FP64 differentiable decoder (scaled extrinsics, windowed schedule) and its adjoint --
    def adj_vjp(self, k, llr, scales, window=0, guard=0, grad_post=None, frozen_seeds=None,
                std=False):
        """Returns (posterior, seeds used, grad_llr, grad_scales); the gradients are the
        vector-Jacobian product with grad_post (None: forward only, gradients None).
        len(scales) // 2 iterations.  std: the TS 36.212 code."""
        def ptr(a):
            return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))
        scales = np.ascontiguousarray(scales, np.float64)
        iters = scales.size // 2
        llr = np.ascontiguousarray(llr, np.float64)
        post = np.empty(k, np.float64)
        seeds = np.empty(self.lib.or_adj_seed_count(k, iters, window), np.float64)
        fz = None if frozen_seeds is None else np.ascontiguousarray(frozen_seeds, np.float64)
        gp = None if grad_post is None else np.ascontiguousarray(grad_post, np.float64)
        g_llr = np.empty(3 * (k + 4), np.float64) if gp is not None else None
        g_s = np.empty(scales.size, np.float64) if gp is not None else None
        f = self.lib.or_std_adj_vjp if std else self.lib.or_adj_vjp
        f(k, llr, iters, scales, window, guard, ptr(fz), ptr(gp), ptr(post), ptr(g_llr), ptr(g_s),
          ptr(seeds))
        return post, seeds, g_llr, g_s

    def decode_batch(self, ks, fillers, llr, llr_off, out_off, iters=8, early_stop=False,
                     window=0, guard=0, threads=0):
        ks = np.ascontiguousarray(ks, np.int32)
        fillers = np.ascontiguousarray(fillers, np.int32)
        llr_off = np.ascontiguousarray(llr_off, np.int64)
        out_off = np.ascontiguousarray(out_off, np.int64)
        n = ks.size
        post = np.zeros(int(out_off[-1] + ks[-1]) if n else 0, np.float32)
        ok = np.zeros(n, np.int32)
        used = np.zeros(n, np.int32)
        llr = np.ascontiguousarray(llr, np.float32)
        if window:
            self.lib.or_decode_batch_windowed(n, ks, fillers, llr_off, llr, out_off, post, iters,
                                              int(early_stop), window, guard, ok, used, threads)
        else:
            self.lib.or_decode_batch(n, ks, fillers, llr_off, llr, out_off, post, iters,
                                     int(early_stop), ok, used, threads)
        return post, ok.astype(bool), used


class Reference(_Lib):
    """The reference's own CPU code (oracle/_ref/libturbo_ref.so)."""

    def __init__(self, path: str = REF_SO):
        super().__init__(path, "ref_")
        L = self.lib
        _sig(L, "ref_qpp_count", C.c_int, [])
        _sig(L, "ref_qpp_entry", None, [C.c_int] + [C.POINTER(C.c_int32)] * 3)
        _sig(L, "ref_qpp_perm", C.c_int, [C.c_int32, _i32p])
        _sig(L, "ref_crc_append", None, [C.c_int, _u8p, C.c_size_t, _u8p])
        _sig(L, "ref_crc_check", C.c_int, [C.c_int, _u8p, C.c_size_t])
        _sig(L, "ref_segment", C.c_int, [_u8p, C.c_size_t, _i64p, C.c_void_p])
        _sig(L, "ref_turbo_encode", C.c_int, [C.c_int32, C.c_int32, _u8p, _u8p, _u8p, _u8p])
        _sig(L, "ref_encode_tb", C.c_int,
             [C.c_size_t, C.c_size_t, C.c_uint32, C.c_uint32, C.c_uint32, _u8p, _i32p, _i32p,
              _i32p, _i64p, C.c_int32, _u8p, C.c_size_t])
        _sig(L, "ref_derate_bits", C.c_int,
             [C.c_int32, C.c_int32, C.c_uint32, _u8p, C.c_size_t, _f32p])
        _sig(L, "ref_decode_cb", C.c_int,
             [C.c_int32, C.c_int32, _f32p, C.c_int32, C.c_int, _f32p, C.POINTER(C.c_int),
              C.POINTER(C.c_int32)])
        _sig(L, "ref_decode_batch", C.c_int,
             [C.c_int32, _i32p, _i32p, _i64p, _f32p, _i64p, _f32p, C.c_int32, C.c_int, _i32p,
              _i32p, C.c_int])
        _sig(L, "ref_roundtrip_tb", C.c_int,
             [C.c_size_t, C.c_size_t, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int,
              _u8p, _u8p, C.POINTER(C.c_int), C.POINTER(C.c_int32), C.c_void_p, C.c_size_t])

    def qpp_table(self):
        out = []
        for i in range(self.lib.ref_qpp_count()):
            k, f1, f2 = C.c_int32(), C.c_int32(), C.c_int32()
            self.lib.ref_qpp_entry(i, C.byref(k), C.byref(f1), C.byref(f2))
            out.append((k.value, f1.value, f2.value))
        return out

    def qpp_perm(self, k: int) -> np.ndarray:
        p = np.empty(k, np.int32)
        if self.lib.ref_qpp_perm(k, p) != 0:
            raise ValueError("unsupported K")
        return p

    def crc_append(self, kind, bits):
        b = np.ascontiguousarray(bits, np.uint8)
        out = np.empty(b.size + CRC_LEN[kind], np.uint8)
        self.lib.ref_crc_append(kind, b, b.size, out)
        return out

    def crc_check(self, kind, bits) -> bool:
        b = np.ascontiguousarray(bits, np.uint8)
        return bool(self.lib.ref_crc_check(kind, b, b.size))

    def segment(self, bits):
        b = np.ascontiguousarray(bits, np.uint8)
        info = np.zeros(7, np.int64)
        if self.lib.ref_segment(b, b.size, info, None) != 0:
            raise ValueError("segmentation failed")
        c, cp, cm, kp, km, f, l = (int(x) for x in info)
        cbs = np.empty(cp * kp + cm * km, np.uint8)
        self.lib.ref_segment(b, b.size, info, cbs.ctypes.data_as(C.c_void_p))
        return dict(c=c, c_plus=cp, c_minus=cm, k_plus=kp, k_minus=km, filler=f, l=l), cbs

    def turbo_encode(self, k, filler, cb):
        cbb = np.ascontiguousarray(cb, np.uint8)
        d = [np.empty(k + 4, np.uint8) for _ in range(3)]
        if self.lib.ref_turbo_encode(k, filler, cbb, *d) != 0:
            raise ValueError("encode failed")
        return np.concatenate(d)

    def encode_tb(self, bits, g_total, rv=0, nl=1, qm=2):
        b = np.ascontiguousarray(bits, np.uint8)
        cap = 64
        n = np.zeros(1, np.int32)
        ks = np.zeros(cap, np.int32)
        fs = np.zeros(cap, np.int32)
        es = np.zeros(cap, np.int64)
        rm = np.zeros(g_total + 64, np.uint8)
        rc = self.lib.ref_encode_tb(b.size, g_total, rv, nl, qm, b, n, ks, fs, es, cap, rm, rm.size)
        if rc != 0:
            raise ValueError(f"encode_tb failed ({rc})")
        c = int(n[0])
        return ks[:c].copy(), fs[:c].copy(), es[:c].copy(), rm[: int(es[:c].sum())].copy()

    def derate_bits(self, k, filler, e_bits, rv):
        b = np.ascontiguousarray(e_bits, np.uint8)
        out = np.empty(3 * (k + 4), np.float32)
        if self.lib.ref_derate_bits(k, filler, rv, b, b.size, out) != 0:
            raise ValueError("derate failed")
        return out

    def decode_cb(self, k, filler, llr, iters=8, early_stop=False):
        llr = np.ascontiguousarray(llr, np.float32)
        post = np.empty(k, np.float32)
        ok, used = C.c_int(), C.c_int32()
        if self.lib.ref_decode_cb(k, filler, llr, iters, int(early_stop), post, C.byref(ok),
                                  C.byref(used)) != 0:
            raise ValueError("decode failed")
        return post, bool(ok.value), used.value

    def decode_batch(self, ks, fillers, llr, llr_off, out_off, iters=8, early_stop=False,
                     threads=0):
        ks = np.ascontiguousarray(ks, np.int32)
        fillers = np.ascontiguousarray(fillers, np.int32)
        llr_off = np.ascontiguousarray(llr_off, np.int64)
        out_off = np.ascontiguousarray(out_off, np.int64)
        n = ks.size
        post = np.zeros(int(out_off[-1] + ks[-1]) if n else 0, np.float32)
        ok = np.zeros(n, np.int32)
        used = np.zeros(n, np.int32)
        if self.lib.ref_decode_batch(n, ks, fillers, llr_off,
                                     np.ascontiguousarray(llr, np.float32), out_off, post, iters,
                                     int(early_stop), ok, used, threads) != 0:
            raise ValueError("decode batch failed")
        return post, ok.astype(bool), used

    def roundtrip_tb(self, bits, g_total, iters=6, early_stop=False, rv=0, nl=1, qm=2):
        b = np.ascontiguousarray(bits, np.uint8)
        tb = np.zeros(b.size, np.uint8)
        ok, used = C.c_int(), C.c_int32()
        post = np.zeros(b.size + 24 * 20 + 6144, np.float32)
        rc = self.lib.ref_roundtrip_tb(b.size, g_total, rv, nl, qm, iters, int(early_stop), b, tb,
                                       C.byref(ok), C.byref(used),
                                       post.ctypes.data_as(C.c_void_p), post.size)
        if rc != 0:
            raise ValueError(f"roundtrip failed ({rc})")
        return tb, bool(ok.value), used.value


class SegInfo(C.Structure):
    _fields_ = [(n, C.c_size_t) for n in ("c", "c_plus", "c_minus", "k_plus", "k_minus",
                                          "filler", "l")]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


def reference_available() -> bool:
    return os.path.exists(REF_SO)
