"""Generates tests/golden/reference_vectors.npz from the reference itself.

Runs the Wiseung/Turbo_CPP CPU code (oracle/_ref/libturbo_ref.so, built by oracle/Makefile from
the reference sources) on seeded inputs and stores inputs and outputs.  The fixture pins the
oracle restatement and the product's host codec without needing the reference at test time.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import CRC_LEN, Reference  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_vectors.npz")


def load(path: str = OUT) -> dict:
    """Reads the fixture back, unpacking the bit arrays."""
    z = np.load(path)
    out = {}
    for name in z.files:
        if name.endswith("__n"):
            continue
        v = z[name]
        if name + "__n" in z.files:
            v = np.unpackbits(v)[: int(z[name + "__n"][0])]
        out[name] = v
    return out


def awgn(rng, d012, k, ebn0_db):
    r = k / (3 * (k + 4))
    s2 = 1.0 / (2 * r * 10 ** (ebn0_db / 10))
    y = (2.0 * d012 - 1.0) + rng.normal(0.0, np.sqrt(s2), d012.size)
    return (2.0 * y / s2).astype(np.float32)


def main() -> None:
    ref = Reference()
    rng = np.random.default_rng(20261203)
    g: dict[str, np.ndarray] = {}

    g["qpp_table"] = np.array(ref.qpp_table(), np.int32)
    for k in (40, 1024, 6144):
        g[f"qpp_perm_{k}"] = ref.qpp_perm(k)

    # CRC: append for every kind over assorted lengths (0 .. 300 and 2 long strings)
    lens = list(range(0, 64)) + [100, 255, 256, 300, 6120, 6144]
    crc_bits, crc_off = [], [0]
    for n in lens:
        crc_bits.append(rng.integers(0, 2, n).astype(np.uint8))
        crc_off.append(crc_off[-1] + n)
    g["crc_in"] = np.concatenate(crc_bits)
    g["crc_off"] = np.array(crc_off, np.int64)
    for kind in range(4):
        g[f"crc_out_{kind}"] = np.concatenate([ref.crc_append(kind, b)[b.size:] for b in crc_bits])

    # segmentation: sizes around every boundary plus the config-3 range
    bs = [1, 40, 41, 63, 6143, 6144, 6145, 6168, 12000, 12024, 18432, 40000, 97896 + 24,
          75000, 6120 * 16 + 1]
    bs += [int(x) for x in rng.integers(1000, 97920, 12)]
    seg_info, seg_bits, seg_in = [], [], []
    for b in bs:
        bits = rng.integers(0, 2, b).astype(np.uint8)
        info, cbs = ref.segment(bits)
        seg_in.append(bits)
        seg_info.append([b, info["c"], info["c_plus"], info["c_minus"], info["k_plus"],
                         info["k_minus"], info["filler"], info["l"], cbs.size])
        seg_bits.append(cbs)
    g["seg_info"] = np.array(seg_info, np.int64)
    g["seg_in"] = np.concatenate(seg_in)
    g["seg_out"] = np.concatenate(seg_bits)

    # encoder: assorted K with and without filler
    enc_cases = [(40, 0), (40, 16), (64, 0), (512, 8), (1024, 0), (2048, 24), (6144, 0),
                 (6144, 32), (528, 0), (1056, 0), (4032, 4)]
    enc_in, enc_out = [], []
    for k, f in enc_cases:
        cb = rng.integers(0, 2, k).astype(np.uint8)
        cb[:f] = 0
        enc_in.append(cb)
        enc_out.append(ref.turbo_encode(k, f, cb))
    g["enc_cases"] = np.array(enc_cases, np.int32)
    g["enc_in"] = np.concatenate(enc_in)
    g["enc_out"] = np.concatenate(enc_out)

    # transport-block encode (CRC24A + segmentation + encode + rate matching) and +-8 de-rate
    tb_cases = [(40, 3 * 68, 0), (512, 3 * 540, 0), (512, 1000, 1), (1000, 3000, 2),
                (1000, 1800, 3), (6112, 3 * 6148, 0), (12000, 36000, 0), (12000, 20000, 2),
                (30000, 48000, 1), (97896, 97896 * 2 + 16, 0), (4000, 16000, 3)]
    tb_in, tb_cb, tb_rm, tb_der = [], [], [], []
    for tbs, gt, rv in tb_cases:
        bits = rng.integers(0, 2, tbs).astype(np.uint8)
        ks, fs, es, rm = ref.encode_tb(bits, gt, rv=rv)
        tb_in.append(bits)
        pos = 0
        for k, f, e in zip(ks, fs, es):
            tb_cb.append([tbs, gt, rv, k, f, e])
            chunk = rm[pos:pos + e]
            pos += e
            tb_der.append(ref.derate_bits(int(k), int(f), chunk, rv))
        tb_rm.append(rm)
    g["tb_cases"] = np.array(tb_cases, np.int64)
    g["tb_in"] = np.concatenate(tb_in)
    g["tb_cb"] = np.array(tb_cb, np.int64)
    g["tb_rm"] = np.concatenate(tb_rm)
    g["tb_derate"] = np.concatenate(tb_der)

    # decoder: seeded BPSK/AWGN blocks, (K, filler, Eb/N0, iterations, early_stop)
    dec_cases = [(40, 0, 0.5, 8, 0), (64, 0, 1.0, 6, 0), (104, 16, 1.5, 8, 1), (512, 0, 0.5, 8, 0),
                 (1024, 0, 0.5, 8, 0), (1024, 0, 1.5, 8, 1), (1024, 0, 0.0, 8, 0),
                 (2048, 40, 1.0, 4, 0), (6144, 0, 0.6, 8, 0), (6144, 8, 1.2, 8, 1),
                 (3008, 0, 3.0, 8, 0), (40, 0, 6.0, 1, 0)]
    dec_llr, dec_post, dec_meta = [], [], []
    for k, f, eb, it, es in dec_cases:
        cb = rng.integers(0, 2, k).astype(np.uint8)
        cb[:f] = 0
        if es:  # a block that carries CRC24B (payload + CRC), as segmented blocks do
            from oracle import Oracle
            body = cb[f:k - 24]
            cb[f:] = Oracle().crc_append(1, body)
        d012 = ref.turbo_encode(k, f, cb)
        llr = awgn(rng, d012, k, eb)
        llr[:f] = 0.0                      # filler is an erasure in d0 and d1
        llr[k + 4:k + 4 + f] = 0.0
        post, ok, used = ref.decode_cb(k, f, llr, it, bool(es))
        dec_llr.append(llr)
        dec_post.append(post)
        dec_meta.append([k, f, it, es, int(ok), used, int(round(eb * 10))])
    g["dec_meta"] = np.array(dec_meta, np.int64)
    g["dec_llr"] = np.concatenate(dec_llr)
    g["dec_post"] = np.concatenate(dec_post)
    g["dec_bits_note"] = np.array([0], np.int8)

    # transport-block roundtrips of the reference's own tests (test_main.cpp:58-344):
    # alternating bit patterns, noise-free +-8 LLRs
    rt = [(40, 3 * 68, 6, 7, 3), (512, 3 * 540, 6, 11, 5), (6112, 3 * 6148, 6, 19, 11),
          (12000, 3 * (6016 + 4) + 3 * (6080 + 4), 6, 17, 9)]
    rt_out = []
    for tbs, gt, it, a, c in rt:
        bits = ((np.arange(tbs) * a + c) & 1).astype(np.uint8)
        tb, ok, used = ref.roundtrip_tb(bits, gt, iters=it)
        rt_out.append([tbs, gt, it, a, c, int(ok), used, int(np.array_equal(tb, bits))])
    g["roundtrip"] = np.array(rt_out, np.int64)

    # bit arrays are stored packed (np.packbits) with their length under "<name>__n"
    for name in [n for n, v in g.items() if v.dtype == np.uint8]:
        g[name + "__n"] = np.array([g[name].size], np.int64)
        g[name] = np.packbits(g[name])
    np.savez_compressed(OUT, **g)
    print(f"wrote {OUT} ({os.path.getsize(OUT) / 1024:.0f} KiB)")


if __name__ == "__main__":
    main()
