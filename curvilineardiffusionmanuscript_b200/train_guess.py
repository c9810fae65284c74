"""Trainer of the guess network's checkpoint for the 1024² multi-Gaussian problem.

    python -m curvilineardiffusionmanuscript_b200.train_guess [--n 1024] [--seeds 250]
        [--steps-per-seed 8] [--train-steps 3000] [--out PATH]

Generates APT trajectories of the seeded multi-Gaussian problem with the
library's own FP64 solver (seeds 1000.., disjoint from the benchmark's timed
seed 12345), trains the network on 16 random 128² crops per Adam step in the
library's kernels, and writes the FP32 parameter vector with
GuessNet.save (an .npz holding `params`).  bench.py loads the checkpoint
written to weights/guess_multigauss1024.npz beside this file.
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

from . import learned, problems

DEFAULT_CHECKPOINT = Path(__file__).resolve().parent / "weights" / "guess_multigauss1024.npz"


def train_multigauss(n: int = 1024, nseeds: int = 250, steps_per_seed: int = 8, train_steps: int = 3000,
                     seed0: int = 1000, net_seed: int = 1):
    """(net, info): a GuessNet trained on trajectories of multi_gaussian_2d(n, seed)."""
    import torch
    make = lambda seed: problems.multi_gaussian_2d(n, seed=seed, device="cuda")
    t0 = time.time()
    skipped = []
    trajs = learned.generate_trajectories(make, seeds=list(range(seed0, seed0 + nseeds)), nsteps=steps_per_seed,
                                          skipped=skipped)
    t1 = time.time()
    net = learned.GuessNet(seed=net_seed)
    pr0 = make(seed0)
    losses = learned.train(net, trajs, pr0.mesh, pr0.kappa.k0, pr0.kappa.n, steps=train_steps, batch=16, crop=128,
                           lr=2e-3)
    torch.cuda.synchronize()
    info = {"n": n, "apt_steps": len(trajs) * steps_per_seed, "seeds": [seed0, seed0 + nseeds - 1],
            "seeds_diverged": len(skipped), "data_s": round(t1 - t0, 1), "train_s": round(time.time() - t1, 1),
            "train_steps": train_steps, "loss_first": float(sum(losses[:10]) / 10),
            "loss_last": float(sum(losses[-50:]) / 50)}
    del trajs
    torch.cuda.empty_cache()
    return net, info


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--seeds", type=int, default=250)
    ap.add_argument("--steps-per-seed", type=int, default=8)
    ap.add_argument("--train-steps", type=int, default=3000)
    ap.add_argument("--out", default=str(DEFAULT_CHECKPOINT))
    a = ap.parse_args()
    net, info = train_multigauss(a.n, a.seeds, a.steps_per_seed, a.train_steps)
    out = Path(a.out)
    out.parent.mkdir(parents=True, exist_ok=True)
    net.save(out)
    net.close()
    print(json.dumps({"checkpoint": str(out), "training": info}), flush=True)


if __name__ == "__main__":
    main()
