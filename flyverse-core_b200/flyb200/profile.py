"""A short, eager run of the whole-fly step for profilers (every kernel launched separately).

    python -m flyb200.profile [--batch 64] [--steps 5] [--warmup 2] [--part whole|lif|optic|tracer|pull]
                              [--lif-block 256] [--lif-ipt 0|1|2|4] [--lif-staged] [--lif-defer] [--lif-grid 0]
                              [--lif-pull] [--density 0.024]
                              [--optic-launch step|persistent] [--optic-variant 0] [--optic-grid 0] [--optic-long-row 0]
                              [--no-overlap]
    python -m flyb200.profile --breakdown [--batch 64] [--steps 50]
    (--per-call K: K whole-fly steps per call, `--steps` calls; --settle S: S steps first, from CUDA graphs)

Builds flyb200.synthetic.whole_fly_config5 (167,106 neurons, 25.6 M edges), warms up, then runs
`--steps` steps of the chosen part. Used for the launch list and the per-kernel captures whose
summaries live in profiles/. `--part pull` fills the LIF pull buffer with random spikes at
`--density` (per neuron, fly and step; 0.024 is the whole fly's steady firing at 64 flies) and
runs the pull delivery of one group of steps (Brain.pull_group: 4 at 64 flies) `--steps` times. `--breakdown` instead times each stage of the step on its own with
CUDA events (stream-ordered, warm L2) and prints one JSON line of microseconds per stage.
"""
from __future__ import annotations

import argparse
import json

import torch

from . import synthetic
from .optic import spmm
from .whole import WholeFly


def _time_us(fn, reps: int) -> float:
    fn()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        fn()
    e.record()
    e.synchronize()
    return 1000.0 * s.elapsed_time(e) / reps


def _graph_us(fn, reps: int = 20) -> float:
    """Device microseconds of one fn() call, from a CUDA graph of `reps` calls (no host gaps)."""
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            for _ in range(reps):
                fn()
    torch.cuda.current_stream().wait_stream(s)
    us = _time_us(g.replay, 5) / reps
    del g
    return us


def breakdown(eng: WholeFly, reps: int) -> dict:
    """Microseconds per stage of one whole-fly step, each stage repeated alone inside a CUDA graph
    (so small kernels are not measured through host launch gaps)."""
    o = eng.cfg.optic
    rate, drive = eng.lif._st["rate"], eng.lif._st["drive"]
    stages = {
        "spk_in = W_rs rate": lambda: spmm(eng.W_rs, rate, eng.optic.spk_in, x_div=100.0, x_lo=0.0, x_hi=3.0,
                                           alpha=o.gain_fb, y_index=eng.rs_rows),
        "optic substep": lambda: eng.optic.substeps(1, carry=True),
        "drive = W_sr dr": lambda: spmm(eng.W_sr, eng.optic.dr_out, drive, y_index=eng.sr_rows, alpha=o.gain_out_mv,
                                        y_lo=-o.drive_clip_mv, y_hi=o.drive_clip_mv),
        "lif step": lambda: eng.lif.step(1),
        "whole step (eager)": lambda: eng.step(1),
    }
    for wpr in (1, 2, 4, 8):
        stages[f"W_rs, {wpr} warps/row"] = (lambda w=wpr: spmm(eng.W_rs, rate, eng.optic.spk_in, x_div=100.0, x_lo=0.0,
                                                              x_hi=3.0, alpha=o.gain_fb, y_index=eng.rs_rows,
                                                              warps_per_row=w))
        stages[f"W_sr, {wpr} warps/row"] = (lambda w=wpr: spmm(eng.W_sr, eng.optic.dr_out, drive, y_index=eng.sr_rows,
                                                              alpha=o.gain_out_mv, y_lo=-o.drive_clip_mv,
                                                              y_hi=o.drive_clip_mv, warps_per_row=w))
    out = {k: (_time_us(f, reps) if "eager" in k else _graph_us(f)) for k, f in stages.items()}
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            eng.step(10)
    torch.cuda.current_stream().wait_stream(s)
    out["whole step (graph of 10)"] = _time_us(g.replay, max(1, reps // 10)) / 10
    del g
    return out


def trace_eyes(args) -> None:
    """`--batch` flies' eyes (1,634 columns x 7 rays) traced in their own rooms, `--steps` times."""
    from . import world as W
    from .batch_world import BatchWorld
    _, dirs, w = synthetic.eye_grid()
    bw = BatchWorld([W.make_room(i)[0] for i in range(args.batch)], "cuda")
    bw.set_eye(dirs, w)
    bw.set_pose(*synthetic.fly_poses(args.batch, seed=0))
    for _ in range(args.warmup + args.steps):
        out = bw.trace_eye()
    torch.cuda.synchronize()
    print(f"traced {args.steps} frames of {args.batch} eyes: {out.shape[1]} columns, mean radiance "
          f"{float(out.mean()):.4f}")


def pull_steps(eng, steps: int, density: float) -> None:
    """Pull delivery of whole groups of LIF steps (Brain.pull_group), `steps` groups, from spike
    words filled at `density` per (neuron, fly, step)."""
    import ctypes as ct
    from . import _abi
    b = eng.lif
    if not b._pull_active():
        raise ValueError("pull delivery needs 32, 64, 128 or 256 flies and the count ring")
    a = b._args
    a.flags, a.nsteps, a.n_first, a.n_count = b._flags(False), 1, 0, 0
    b._set_pull(a)
    g = torch.Generator(device=b.device).manual_seed(1)
    bits = (torch.rand(b._pull_bits.numel(), 32, device=b.device, generator=g) < density).to(torch.int64)
    words = (bits << torch.arange(32, device=b.device)).sum(-1)
    b._pull_bits.copy_(torch.where(words >= 2**31, words - 2**32, words).to(torch.int32))
    del bits, words
    L = b.pull_group
    a.pull_steps = L
    b._pull_state.zero_()
    stream = torch.cuda.current_stream(b.device).cuda_stream
    for _ in range(steps):
        rc = _abi.lib().flyb_lif_pull(ct.byref(a), stream)
        if rc:
            raise RuntimeError(f"flyb_lif_pull: error {rc}")
    torch.cuda.synchronize()
    b._pull_state[:2].copy_(b._clock[:2])
    print(f"pulled {steps} groups of {L} steps at batch {b.B}, density {density}: "
          f"{int(b._pull_t[1].numel()) // 32:,} chunks")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--part", default="whole", choices=["whole", "lif", "optic", "tracer", "pull"])
    ap.add_argument("--lif-pull", action="store_true", help="LIF spikes delivered by the pull kernel")
    ap.add_argument("--density", type=float, default=0.024, help="spike density for --part pull")
    ap.add_argument("--breakdown", action="store_true")
    ap.add_argument("--settle", type=int, default=0, help="steps replayed from CUDA graphs of 20 before the "
                                                           "profiled ones (3,000: the steady firing the bench times)")
    ap.add_argument("--per-call", type=int, default=1, help="whole-fly steps per WholeFly.step call (the pull "
                                                             "delivers whole groups of steps within a call)")
    ap.add_argument("--lif-block", type=int, default=256)
    ap.add_argument("--lif-ipt", type=int, default=0, help="LIF items per thread (0: automatic)")
    ap.add_argument("--lif-staged", action="store_true", help="LIF step through the bulk-copy kernel")
    ap.add_argument("--no-overlap", action="store_true", help="run the LIF step after the optic chain")
    ap.add_argument("--lif-grid", type=int, default=0, help="staged LIF block cap (0: every resident block)")
    ap.add_argument("--lif-defer", action="store_true", help="LIF spikes delivered by a second kernel")
    ap.add_argument("--optic-launch", default="step", choices=["step", "persistent"])
    ap.add_argument("--optic-variant", type=int, default=0)
    ap.add_argument("--optic-long-row", type=int, default=0, help="rows longer than this are split across a "
                    "block (0: the library default)")
    ap.add_argument("--optic-grid", type=int, default=0, help="persistent optic block cap")
    args = ap.parse_args()
    if args.part == "tracer":
        trace_eyes(args)
        return
    cfg = synthetic.whole_fly_config5(seed=0)
    eng = WholeFly(cfg, args.batch, device="cuda", seed=1, launch="step", overlap=not args.no_overlap)
    eng.lif.block, eng.lif.items_per_thread, eng.lif.staged = args.lif_block, args.lif_ipt, args.lif_staged
    eng.lif.grid, eng.lif.defer = args.lif_grid, args.lif_defer
    eng.lif.pull = args.lif_pull or args.part == "pull"
    eng.optic.launch, eng.optic.variant, eng.optic.grid = args.optic_launch, args.optic_variant, args.optic_grid
    if args.optic_long_row:
        eng.optic.set_long_rows(args.optic_long_row)
    eng.lif._make_args()
    eng.optic.pr_in.normal_(0.0, 0.2)
    eng.step(args.warmup)
    if args.settle > 0:
        stream = torch.cuda.Stream()
        stream.wait_stream(torch.cuda.current_stream())
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.stream(stream):
            with torch.cuda.graph(graph, stream=stream):
                eng.step(20)
        torch.cuda.current_stream().wait_stream(stream)
        for _ in range(args.settle // 20):
            graph.replay()
        del graph
    torch.cuda.synchronize()
    if args.breakdown:
        res = breakdown(eng, max(10, args.steps))
        eng.lif.check()
        print(json.dumps({"batch": args.batch, "us": res}))
        return
    if args.part == "pull":
        pull_steps(eng, args.steps, args.density)
        return
    for _ in range(args.steps):
        if args.part == "whole":
            eng.step(args.per_call)
        elif args.part == "lif":
            eng.lif.step(1)
        else:
            eng.optic.substeps(1, carry=True)
    torch.cuda.synchronize()
    eng.lif.check()
    print(f"profiled {args.steps} {args.part} steps at batch {args.batch}: {eng.n_neurons:,} neurons")


if __name__ == "__main__":
    main()
