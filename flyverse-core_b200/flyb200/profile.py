"""A short, eager run of the whole-fly step for profilers (every kernel launched separately).

    python -m flyb200.profile [--batch 64] [--steps 5] [--warmup 2] [--part whole|lif|optic]

Builds flyb200.synthetic.whole_fly_config5 (167,106 neurons, 25.6 M edges), warms up, then runs
`--steps` steps of the chosen part. Used for the launch list and the per-kernel captures whose
summaries live in profiles/.
"""
from __future__ import annotations

import argparse

import torch

from . import synthetic
from .whole import WholeFly


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--part", default="whole", choices=["whole", "lif", "optic"])
    args = ap.parse_args()
    cfg = synthetic.whole_fly_config5(seed=0)
    eng = WholeFly(cfg, args.batch, device="cuda", seed=1, launch="step")
    eng.optic.pr_in.normal_(0.0, 0.2)
    eng.step(args.warmup)
    torch.cuda.synchronize()
    for _ in range(args.steps):
        if args.part == "whole":
            eng.step(1)
        elif args.part == "lif":
            eng.lif.step(1)
        else:
            eng.optic.substeps(1)
    torch.cuda.synchronize()
    eng.lif.check()
    print(f"profiled {args.steps} {args.part} steps at batch {args.batch}: {eng.n_neurons:,} neurons")


if __name__ == "__main__":
    main()
