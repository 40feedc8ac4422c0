"""Launch-parameter autotuner for the native steps, cached per (graph, batch, activity bucket).

The best launch shape depends on the graph, the batch and how many cells spike per step: at B = 1
the step is latency-bound and a persistent cooperative launch (one launch for many steps, a grid
barrier per step) wins; at B = 64 the state streams from HBM and one launch per step, with the
state staged through shared memory by bulk copies, keeps more bytes in flight. `tune_lif` times
each candidate (launch mode x block size x items per thread x spike delivery) for a few steps on a
copy of the live state, restores the state, installs the fastest and caches it under the key;
`tune_optic` does the same for the optic substep's launch mode and kernel shape.
"""
from __future__ import annotations

import hashlib
import math

import numpy as np
import torch

CACHE: dict = {}
OPTIC_VARIANTS = 6          # flyb_optic_args.variant values; a batch width has a subset of them
# (launch, block, items per thread, delivery): "fused" delivers spikes inside the update kernel,
# "staged" runs per-step launches through the bulk-copy kernel, "defer" lists the spikers and
# delivers them from a second, load-balanced kernel, "staged-defer" does both
LIF_CANDIDATES = (("step", 256, 4, "fused"), ("step", 256, 2, "fused"), ("step", 256, 1, "fused"),
                  ("step", 256, 2, "staged"), ("step", 512, 2, "staged"), ("step", 256, 4, "staged"),
                  ("step", 256, 2, "defer"), ("step", 256, 1, "defer"), ("step", 128, 2, "defer"),
                  ("step", 256, 4, "defer"), ("step", 256, 2, "staged-defer"), ("step", 512, 2, "staged-defer"),
                  ("step", 256, 4, "staged-defer"), ("persistent", 256, 4, "fused"), ("persistent", 512, 2, "fused"),
                  ("step", 256, 2, "pull"), ("step", 256, 1, "pull"), ("step", 256, 2, "staged-pull"),
                  ("step", 512, 2, "staged-pull"), ("step", 128, 2, "staged"), ("step", 128, 2, "staged-defer"),
                  ("step", 128, 2, "staged-pull"))


def graph_key(brain) -> str:
    h = hashlib.sha1()
    h.update(brain._out_ptr.cpu().numpy().tobytes())
    h.update(str((brain.n, brain.nnz, brain.ring_mode)).encode())
    return h.hexdigest()[:16]


def activity_bucket(brain, steps: int = 20) -> int:
    """log2 bucket of the fraction of (neuron, fly) pairs spiking per step, measured on a copy."""
    saved = brain.state_dict()
    before = float(brain.spike_counts.sum())
    rec = brain.record_activity
    brain.record_activity = True
    brain.step(steps)
    rate = (float(brain.spike_counts.sum()) - before) / (steps * brain.n * brain.B)
    brain.record_activity = rec
    brain.load_state_dict(saved)
    return int(math.floor(math.log2(max(rate, 1e-7))))


def _time(fn, reps: int) -> float:
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        fn()
    e.record()
    e.synchronize()
    return s.elapsed_time(e) / reps


def tune_lif(brain, steps: int = 10, candidates=LIF_CANDIDATES) -> dict:
    """Install and return the fastest LIF launch choice for this brain; state is left unchanged.
    A brain with per-neuron clocks or the slow receptor tone has one launch shape (the extended
    kernel): nothing to tune."""
    if getattr(brain, "_kvec", None) is not None or getattr(brain, "slow", None) is not None:
        return {"launch": "step", "block": 256, "items_per_thread": 1, "delivery": "extended", "ms_per_step": None}
    key = ("lif", graph_key(brain), brain.B, activity_bucket(brain))
    if key in CACHE:
        _apply(brain, CACHE[key])
        return CACHE[key]
    saved = brain.state_dict()
    results = {}
    if not brain.can_pull():             # pull delivery: count ring and 32-fly groups only
        candidates = [c for c in candidates if "pull" not in c[3]]
    for launch, block, ipt, delivery in candidates:
        _apply(brain, {"launch": launch, "block": block, "items_per_thread": ipt, "delivery": delivery})
        brain.step(2)
        results[(launch, block, ipt, delivery)] = _time(lambda: brain.step(steps), 1) / steps
        brain.load_state_dict(saved)
    best = min(results, key=results.get)
    choice = {"launch": best[0], "block": best[1], "items_per_thread": best[2], "delivery": best[3],
              "ms_per_step": results[best],
              "all": {f"{k[0]}-{k[3]}/{k[1]}/{k[2]}": v for k, v in results.items()}}
    CACHE[key] = choice
    _apply(brain, choice)
    return choice


def _apply(brain, choice: dict) -> None:
    brain.launch, brain.block = choice["launch"], choice["block"]
    brain.items_per_thread = choice.get("items_per_thread", 0)
    delivery = choice.get("delivery", "fused")
    brain.staged = delivery in ("staged", "staged-defer", "staged-pull")
    brain.defer = delivery in ("defer", "staged-defer")
    brain.pull = delivery in ("pull", "staged-pull")
    brain._make_args()


# Row lengths above which a row is shared by a whole block (OpticCore.set_long_rows): the split
# pays at many flies per row gather; at one fly a row of a few hundred entries is better left to
# its warp slot.
OPTIC_LONG_ROWS = (192, 384, 512, 768, 1024, 2048)


def tune_optic(core, steps: int = 10) -> dict:
    """Pick the optic substep's launch mode, kernel shape (fly lanes x flies per lane x lanes per
    row, flyb_optic_args.variant) and long-row threshold by timing each on a copy of the state."""
    key = ("optic", core.m, core.W.nnz, core.B)
    if key in CACHE:
        core.launch, core.variant = CACHE[key]["launch"], CACHE[key]["variant"]
        core.set_long_rows(CACHE[key]["long_row"])
        return CACHE[key]
    v, a = core.v_s.clone(), core.adapt_s.clone()
    results = {}
    for long_row in OPTIC_LONG_ROWS:
        core.set_long_rows(long_row)
        for launch in ("step", "persistent"):
            for variant in range(OPTIC_VARIANTS):
                core.launch, core.variant = launch, variant
                try:
                    core.substeps(2)
                except RuntimeError:                 # no such shape for this batch width
                    continue
                results[(launch, variant, long_row)] = _time(lambda: core.substeps(steps, carry=True), 1) / steps
                core.v_s.copy_(v)
                core.adapt_s.copy_(a)
    best = min(results, key=results.get)
    CACHE[key] = {"launch": best[0], "variant": best[1], "long_row": best[2], "ms_per_step": results[best],
                  "all": {f"{k[0]}/{k[1]}/{k[2]}": t for k, t in results.items()}}
    core.launch, core.variant = best[0], best[1]
    core.set_long_rows(best[2])
    return CACHE[key]


def summary() -> list:
    return [{"key": list(map(str, k)), **{kk: vv for kk, vv in v.items() if kk != "all"}} for k, v in CACHE.items()]
