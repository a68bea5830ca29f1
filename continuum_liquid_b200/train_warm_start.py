"""Train the learned pressure warm start on the GPU and write its weights.

    python -m continuum_liquid_b200.train_warm_start [--iterations 2500] [--out PATH]

Training data are the solver's own solves: for the 128^3 collider pool (seeds 0..9) and the 256^3
block (seeds 0..2), every step after the first two contributes (right-hand side, operator, solid
mask, previous-step pressure, pressure converged to 1e-6). The network is trained with Adam
(lr 1e-3, batch 8) on random 64^3 crops, each crop's squared error weighted by the relative residual
its previous-step pressure starts from (``iterations`` x 8 crops; 2500 iterations are the 20k
crops). It is then evaluated on held-out seeds 100..104 of both scenes: flexible-CG cycles to 1e-6
from the previous-step pressure and from the solver's choice between it and the network's guess.
The weights, the loss history and the evaluation go to one .npz file (default: the package's
weights/warm_start_unet.npz, which the solver and bench.py load).
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import learned, scenes
from .backend import Backend


def capture(kernels, factory, seeds, steps):
    frames = []
    for s in seeds:
        frames += learned.capture_frames(kernels, factory(s), steps=steps, skip=2)
        torch.cuda.empty_cache()
    return frames


def summarise(rows):
    prev = sum(r["previous"]["cycles"] for r in rows)
    lrn = sum(r["learned"]["cycles"] for r in rows)
    used = sum(1 for r in rows if r["learned"]["guess"] == "learned")
    return {"frames": len(rows), "cycles_previous": prev, "cycles_learned": lrn, "learned_guess_used": used,
            "initial_rel_previous_mean": float(np.mean([r["previous"]["initial_rel"] for r in rows])),
            "learned_rel_mean": float(np.mean([r["learned"]["learned_rel"] or np.nan for r in rows]))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--iterations", type=int, default=2500)
    ap.add_argument("--out", default=str(learned.default_weights_path()))
    ap.add_argument("--pool-seeds", type=int, default=10)
    ap.add_argument("--block-seeds", type=int, default=3)
    ap.add_argument("--steps", type=int, default=24, help="steps captured per 128^3 run (256^3 runs: a third)")
    ap.add_argument("--eval-seeds", type=int, default=5)
    args = ap.parse_args()
    k = Backend(0)
    t0 = time.perf_counter()
    pool = lambda s: scenes.collider_pool(128, seed=s)  # noqa: E731
    block = lambda s: scenes.block(256, seed=s)  # noqa: E731
    train_frames = capture(k, pool, range(args.pool_seeds), args.steps)
    train_frames += capture(k, block, range(args.block_seeds), max(4, args.steps // 3))
    capture_s = time.perf_counter() - t0
    net = learned.UNet(k, seed=0)
    t0 = time.perf_counter()
    history = learned.train(net, train_frames, iterations=args.iterations, batch=8, crop=64, lr=1e-3, seed=0,
                            log_every=100, weighted=True)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    evaluation = {}
    for name, factory, steps in (("collider_pool_128", pool, 12), ("block_256", block, 8)):
        frames = capture(k, factory, range(100, 100 + args.eval_seeds), steps)
        evaluation[name] = summarise(learned.evaluate(k, net, frames))
        del frames
        torch.cuda.empty_cache()
    meta = {"iterations": args.iterations, "batch": 8, "crop": 64, "lr": 1e-3, "train_frames": len(train_frames),
            "capture_s": capture_s, "train_s": train_s, "loss_every_100": history, "evaluation": evaluation}
    net.save(args.out, meta)
    print(json.dumps(meta), flush=True)


if __name__ == "__main__":
    main()
