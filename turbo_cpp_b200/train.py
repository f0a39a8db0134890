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
    a = ap.parse_args(argv)
    t0 = time.time()

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
