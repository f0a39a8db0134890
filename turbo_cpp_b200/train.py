"""Scale-training harness: learns the 2 per-iteration extrinsic scale factors of the unrolled
Log-MAP turbo decoder by Adam on the mean binary cross-entropy of the posterior LLRs against the
true information bits, with gradients from the hand-written adjoint.  Every step decodes a
freshly seeded batch (seed + step): BPSK over AWGN at a fixed Eb/N0, rate 1/3 with tails,
generated on the GPU (the same bits and LLRs as the host generator for the same seed).

    python -m turbo_cpp_b200.train --steps 200 --blocks 1024 --k 6144 --ebn0 0.6 \\
        --iterations 6 --out scales.json
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from typing import Callable, Optional

import numpy as np


def train_scales(steps: int = 200, n_blocks: int = 1024, k: int = 6144, ebn0_db: float = 0.6,
                 iterations: int = 6, lr: float = 0.01, seed: int = 4000, window: int = 0,
                 guard: int = -1, device: int = 0,
                 callback: Optional[Callable[[dict], None]] = None):
    """Returns (trained scales as a float32 array of 2*iterations, per-step history, held-out
    record).  The learning rate decays from lr to lr/10 over the run (cosine, one scheduler
    step per Adam step).  The held-out record is the loss / BER / BLER of one fixed batch
    (seed + 1000000) with the initial scales (all 1) and with the trained ones: the training
    batches are too noisy to show progress."""
    import torch
    import torch.nn.functional as F

    from .autograd import DifferentiableDecoder

    dev = torch.device("cuda", device)
    ks = [k] * n_blocks
    dd = DifferentiableDecoder(ks, window=window, guard=guard, device=device)
    scales = torch.nn.Parameter(torch.ones(2 * iterations, device=dev))
    opt = torch.optim.Adam([scales], lr=lr)
    # cosine decay to lr/10: the batch-to-batch noise of the loss otherwise keeps the scales
    # moving by about lr around their optimum
    sched = torch.optim.lr_scheduler.LambdaLR(
        opt, lambda i: 0.1 + 0.45 * (1.0 + np.cos(np.pi * min(i, steps) / max(steps, 1))))
    history = []
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    gen = dd.decoder.awgn_code_blocks_device
    vbits, vx = gen(seed + 1000000, ks, ebn0_db)
    vb = vbits.to(torch.float32)

    def held_out(sc):
        with torch.no_grad():
            post = dd(vx, sc)
            errs = ((post >= 0).float() != vb).float().view(n_blocks, k)
            return dict(loss=float(F.binary_cross_entropy_with_logits(post, vb)),
                        ber=float(errs.mean()), bler=float(errs.amax(1).mean()))

    held = {"initial": held_out(scales.detach())}
    for step in range(steps):
        bits, x = gen(seed + step, ks, ebn0_db)
        b = bits.to(torch.float32)
        ev[0].record()
        post = dd(x, scales)
        loss = F.binary_cross_entropy_with_logits(post, b)
        opt.zero_grad(set_to_none=True)
        loss.backward()
        ev[1].record()
        opt.step()
        sched.step()
        with torch.no_grad():
            errs = ((post >= 0).float() != b).float().view(n_blocks, k)
        rec = dict(step=step, lr=float(opt.param_groups[0]["lr"]), loss=float(loss.detach()),
                   ber=float(errs.mean()),
                   bler=float(errs.amax(1).mean()), ms=ev[0].elapsed_time(ev[1]),
                   scales=[float(v) for v in scales.detach().cpu()])
        history.append(rec)
        if callback:
            callback(rec)
    held["trained"] = held_out(scales.detach())
    return scales.detach().cpu().numpy().astype(np.float32), history, held


def wilson(k: int, n: int, z: float = 1.96):
    """95% Wilson score interval of a binomial proportion k/n."""
    if n == 0:
        return (0.0, 1.0)
    p = k / n
    d = 1 + z * z / n
    c = (p + z * z / (2 * n)) / d
    h = z * np.sqrt(p * (1 - p) / n + z * z / (4 * n * n)) / d
    return (float(c - h), float(c + h))


def sign_test_p(a: int, b: int) -> float:
    """Two-sided exact binomial (sign) test of a vs b discordant pairs under p = 1/2."""
    from math import comb

    n = a + b
    if n == 0:
        return 1.0
    tail = sum(comb(n, i) for i in range(0, min(a, b) + 1)) / 2.0 ** n
    return float(min(1.0, 2.0 * tail))


def evaluate_bler(scale_sets, n_blocks: int = 8192, k: int = 6144, ebn0_db: float = 0.6,
                  iterations: int = 8, seed: int = 9000000, batch: int = 1024, device: int = 0):
    """Held-out block error rates of the production decoder (tc_decode, plain schedule, default
    windows, no early stop) with each scale set (None = the unscaled decoder) on the same
    n_blocks fresh blocks.  Returns one record per set: BER, BLER with its 95% Wilson interval,
    and the per-block error flags (for paired comparisons)."""
    import torch

    from . import SCHEDULE_PLAIN, DecodeOptions, Decoder

    dec = Decoder(device)
    ks = [k] * batch
    cbs, llr_len, post_len = Decoder.layout(ks)
    post = torch.empty(post_len, dtype=torch.float32, device=f"cuda:{device}")
    stream = torch.cuda.current_stream(device)
    flags = [[] for _ in scale_sets]
    bit_err = [0] * len(scale_sets)
    for j in range(0, n_blocks, batch):
        bits, x = dec.awgn_code_blocks_device(seed + j, ks, ebn0_db)
        for i, sc in enumerate(scale_sets):
            o = DecodeOptions(iterations, False, 0, -1, SCHEDULE_PLAIN,
                              scales=None if sc is None else [float(v) for v in sc])
            dec.decode_device(cbs, batch, x.data_ptr(), llr_len, post.data_ptr(), post_len,
                              options=o, stream=stream.cuda_stream)
            err = ((post >= 0).to(torch.uint8) != bits).view(batch, k)
            bit_err[i] += int(err.sum())
            flags[i].append(err.any(1).cpu().numpy())
    dec.close()
    out = []
    for i in range(len(scale_sets)):
        f = np.concatenate(flags[i])[:n_blocks]
        kerr = int(f.sum())
        out.append(dict(blocks=int(f.size), block_errors=kerr, bler=kerr / f.size,
                        bler_ci95=wilson(kerr, f.size), ber=bit_err[i] / (f.size * k),
                        flags=f))
    return out


def sweep(lrs, steps: int, n_blocks: int = 1024, k: int = 6144, ebn0_db: float = 0.6,
          iterations: int = 8, window: int = 128, guard: int = 96, eval_blocks: int = 8192,
          seed: int = 4000, device: int = 0, log=print):
    """Trains the scales once per learning rate and evaluates every result, and the unscaled
    decoder, on the same held-out blocks.  Returns a JSON-ready record."""
    runs = []
    for lr in lrs:
        t0 = time.time()
        sc, hist, held = train_scales(steps, n_blocks, k, ebn0_db, iterations, lr, seed, window,
                                      guard, device)
        runs.append(dict(lr=lr, steps=steps, scales=[float(v) for v in sc], held_out=held,
                         wall_s=time.time() - t0,
                         final_loss=float(np.mean([h["loss"] for h in hist[-20:]]))))
        log(f"lr {lr}: scales " + " ".join(f"{v:.3f}" for v in sc) + f" held-out {held}")
    ev = evaluate_bler([None] + [r["scales"] for r in runs], eval_blocks, k, ebn0_db, iterations,
                       device=device)
    base = ev[0]
    for r, e in zip(runs, ev[1:]):
        fixed = int(np.sum(base["flags"] & ~e["flags"]))  # unscaled fails, scaled decodes
        broke = int(np.sum(~base["flags"] & e["flags"]))
        r["eval"] = {key: e[key] for key in ("blocks", "block_errors", "bler", "bler_ci95", "ber")}
        r["paired"] = dict(fixed=fixed, broken=broke, sign_test_p=sign_test_p(fixed, broke))
    best = min(runs, key=lambda r: r["held_out"]["trained"]["loss"])
    gain = (best["eval"]["bler_ci95"][1] < base["bler_ci95"][0]
            and best["paired"]["sign_test_p"] < 0.05)
    return dict(
        k=k, ebn0_db=ebn0_db, iterations=iterations, window=window, guard=guard,
        blocks_per_step=n_blocks, steps=steps, lrs=list(lrs),
        unscaled_eval={key: base[key] for key in ("blocks", "block_errors", "bler", "bler_ci95",
                                                  "ber")},
        runs=runs, chosen_lr=best["lr"], scales=best["scales"],
        selection="the run with the lowest held-out BCE loss (training-side validation batch)",
        result=("BLER gain outside the 95% interval" if gain else
                "no gain: the trained decoder's BLER is inside the unscaled decoder's 95% "
                "interval (or the paired sign test is not significant)"))


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--blocks", type=int, default=1024)
    ap.add_argument("--k", type=int, default=6144)
    ap.add_argument("--ebn0", type=float, default=0.6)
    ap.add_argument("--iterations", type=int, default=6)
    ap.add_argument("--lr", type=float, default=0.01)
    ap.add_argument("--seed", type=int, default=4000)
    ap.add_argument("--window", type=int, default=0)
    ap.add_argument("--guard", type=int, default=-1)
    ap.add_argument("--out", default="")
    ap.add_argument("--every", type=int, default=10)
    ap.add_argument("--sweep", default="", help="comma-separated learning rates: train once per "
                    "rate, evaluate all on --eval-blocks held-out blocks, write the record")
    ap.add_argument("--eval-blocks", type=int, default=8192)
    a = ap.parse_args(argv)
    t0 = time.time()
    if a.sweep:
        rec = sweep([float(v) for v in a.sweep.split(",")], a.steps, a.blocks, a.k, a.ebn0,
                    a.iterations, a.window or 128, a.guard if a.guard >= 0 else 96,
                    a.eval_blocks, a.seed)
        rec["command"] = "python -m turbo_cpp_b200.train " + " ".join(argv or sys.argv[1:])
        rec["wall_s"] = time.time() - t0
        if a.out:
            with open(a.out, "w") as f:
                json.dump(rec, f, indent=1)
        print(json.dumps({key: rec[key] for key in ("scales", "chosen_lr", "unscaled_eval",
                                                    "result")}))
        for r in rec["runs"]:
            print(json.dumps({key: r[key] for key in ("lr", "eval", "paired")}))
        return

    def show(r):
        if r["step"] % a.every == 0 or r["step"] == a.steps - 1:
            print(f"step {r['step']:4d} loss {r['loss']:.6f} ber {r['ber']:.3e} "
                  f"bler {r['bler']:.3f} step_ms {r['ms']:.2f} scales "
                  + " ".join(f"{v:.3f}" for v in r["scales"]), flush=True)

    sc, hist, held = train_scales(a.steps, a.blocks, a.k, a.ebn0, a.iterations, a.lr, a.seed, a.window,
                            a.guard, callback=show)
    out = dict(scales=[float(v) for v in sc], steps=a.steps, blocks=a.blocks, k=a.k,
               ebn0_db=a.ebn0, iterations=a.iterations, lr=a.lr, seed=a.seed,
               wall_s=time.time() - t0, held_out=held, history=hist)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(out, f)
    print(json.dumps({key: out[key] for key in ("scales", "wall_s", "held_out")}))


if __name__ == "__main__":
    main()
