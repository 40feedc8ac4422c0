#!/usr/bin/env python
"""Headline benchmark: neuron-steps/s of the whole-fly brain step at 167,106 neurons.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl flyb200|reference]

Workload (synthetic, seeded; the MaleCNS data is not available): flyb200.synthetic.whole_fly_config5,
167,106 neurons = 89,390 graded optic units + 71,618 LIF + 6,098 Poisson-driven sensory cells,
25.6 M edges (~124 M synapses), dt 0.1 ms, optic <-> LIF coupling every step, a drifting grating on
5,895 photoreceptors. One step advances all 167,106 neurons of every fly once (flyb200.whole).

  value          neuron-steps/s of B=64 flies per GPU (whole job over N GPUs, weak scaling),
                 steps replayed from a CUDA graph at steady firing; state > L2, so no flush is needed
  e2e            the same B=64 step through the public API with, every step, the radiance copied in
                 from pinned host memory and the motor readout copied out, 20 steps per CUDA graph
                 and the host synchronising on each graph's readouts (the eager launch-by-launch
                 figure is reported beside it)
  roofline       the dominant kernel (LIF step or optic substep): algorithmic bytes / CUDA-event time
                 against the measured HBM copy rate, with ncu's DRAM bytes per launch
  cpu_baseline   the C oracle port (oracle/) on this host's cores from this run's settled state
  batch1         the plain single-instance kernels (B=1) at the same steady firing, tuned there
                 like the batched engine, graph-replayed (the "vs plain" ratio uses it) and eager
                 with L2 flushed between steps
  adjoint        optic-lobe adjoint over 200 substeps (89,390 units, 6 M nnz, checkpoint 20) over
                 the forward pass time
  fp64_max_err   max |FP32 - FP64| of the optic state after 200 substeps (config 3, whole-fly lobe)
  batch256       the whole fly at 256 flies (config 5's width)
  uneven_*       uneven rollouts: config 5 at 256 flies (episodes of 200-2,000 steps) and config 4
                 (config 2's graph + config 3's lobe) at 64 flies (500-4,000 steps, 20-200 Hz)
  reference_gpu  the reference's own CUDA path (baseline/_ref, its neural.cu kernels) beside ours on
                 config 2's LIF and config 3's optic substep at 1 and 64 flies, on this GPU
  reference_own_cpu  the reference's own CPU code (Brain.step, OpticLobe._substep) on host cores
  tracer         the eye's ray tracer at 64 flies x 1,634 columns x 7 rays, beside the reference's
                 torch tracer on this GPU and the C oracle on host cores
`--impl reference` times the CPU port alone on this host's cores (the reference's own CPU
implementation of the path, restated in oracle/), from one fly settled the same number of steps
and widened to the same 64 flies, and prints the same line with impl "reference".
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
for _p in (ROOT, ROOT / "flyverse-core_b200"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

import numpy as np  # noqa: E402
import torch  # noqa: E402

METRIC = "neuron-steps/s at 167k neurons (batch 1 & 64, vs plain); adjoint/forward cost"
BATCH = 64
L2_BYTES = 126 * 2**20


def load_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


# ------------------------------------------------------------------ clocks during the timed region
class Clocks:
    """SM clock and clock-event reasons sampled during the timed region, two ways: nvidia-smi's
    clocks line every 200 ms, and NVML every 2 ms (a timed region can be shorter than 200 ms).
    Read-only: no clock or other GPU setting is changed."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    REASONS = (("sw_power_cap", 0x4), ("hw_slowdown", 0x8), ("sw_thermal_slowdown", 0x20),
               ("hw_thermal_slowdown", 0x40), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, index: int):
        self.index, self.proc = index, None
        self.path = Path(tempfile.mkstemp(prefix="flyb_clocks_", suffix=".csv")[1])
        self.nvml, self.stop, self.thread, self.handle, self.max_mhz = [], threading.Event(), None, None, None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        p = torch.cuda.get_device_properties(self.index)
        try:
            bus = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _sample(self):
        nv, h = self.handle
        while not self.stop.is_set():
            try:
                self.nvml.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM),
                                  nv.nvmlDeviceGetCurrentClocksEventReasons(h)))
            except Exception:
                return
            time.sleep(0.002)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        try:
            self.handle = self._nvml_handle()
            self.max_mhz = self.handle[0].nvmlDeviceGetMaxClockInfo(self.handle[1], self.handle[0].NVML_CLOCK_SM)
            self.thread = threading.Thread(target=self._sample, daemon=True)
            self.thread.start()
        except Exception:
            self.thread = None
        return self

    def __exit__(self, *exc):
        self.stop.set()
        if self.thread is not None:
            self.thread.join(timeout=5)
        if self.proc is not None:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self) -> dict:
        rows = [r.split(",") for r in self.path.read_text().splitlines() if r.strip()] if self.path.exists() else []
        self.path.unlink(missing_ok=True)
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if rows:
            names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
            out = {"sm_mhz": float(np.median([float(r[1]) for r in rows])), "sm_max_mhz": float(rows[0][2]),
                   "reasons": sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.strip().lower() == "active"}),
                   "samples": len(rows)}
        if self.nvml:
            sm = [c for c, _ in self.nvml]
            reasons = sorted({n for _, m in self.nvml for n, bit in self.REASONS if m & bit})
            out["nvml"] = {"sm_mhz": float(np.median(sm)), "sm_min_mhz": float(min(sm)), "samples": len(sm),
                           "reasons": reasons, "period_ms": 2}
            if out["sm_mhz"] is None:
                out["sm_mhz"], out["sm_max_mhz"] = float(np.median(sm)), float(self.max_mhz)
            out["reasons"] = sorted(set(out["reasons"]) | set(reasons))
        if not rows and not self.nvml:
            out["reasons"] = ["unsampled"]
        return out


# ------------------------------------------------------------------ helpers
def flush_l2(buf: torch.Tensor) -> None:
    buf.add_(1.0)


def events_time(fn, reps: int, flush=None) -> float:
    """Mean device ms of fn() over reps, each bracketed by CUDA events on the current stream."""
    total = 0.0
    for _ in range(reps):
        if flush is not None:
            flush()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        fn()
        e.record()
        e.synchronize()
        total += s.elapsed_time(e)
    return total / reps


def build_engine(cfg, batch, device, launch, fly0=0):
    from flyb200.whole import WholeFly
    eng = WholeFly(cfg, batch, device=device, seed=1, launch=launch)
    eng.lif.fly0 = fly0              # this rank's flies draw their own Poisson streams
    eng.lif._make_args()
    o = cfg.optic
    rad = torch.from_numpy(o.grating(0.0, batch, seed=fly0)).to(device)
    a_pr = photoreceptor_contrast(cfg, rad)
    eng.set_photoreceptors(a_pr)
    return eng


def photoreceptor_contrast(cfg, rad: torch.Tensor, tables=None) -> torch.Tensor:
    """Held photoreceptor activity [n_pr][B] of a radiance frame (B, n_col, 4): channel-weighted
    intensity, contrast against the frame mean (the stage's steady state). `tables` = the device
    copies of (sensitivity, photoreceptor column) when the call is captured in a graph."""
    o = cfg.optic
    if tables is None:
        tables = (torch.from_numpy(o.sens).to(rad.device), torch.from_numpy(o.pr_column.astype(np.int64)).to(rad.device))
    sens, col = tables
    ip = (rad[:, col, :] * sens[None]).sum(-1)                            # (B, n_pr)
    con = ((ip - ip.mean(1, keepdim=True)) / (ip.mean(1, keepdim=True) + 0.02)).clamp(-1.0, 2.0)
    return con.t().contiguous()


def graph_chunk(steps: int, most: int = 26) -> int:
    """Steps per captured graph: a divisor of `steps` (so exactly `steps` are timed), a multiple of
    4 when possible (whole groups of the pull delivery at 64 flies, so every replay pulls at group
    ends), else even (an odd count ends each replay with a copy of the optic dr back to its start)."""
    divs = [d for d in range(min(most, steps), 0, -1) if steps % d == 0]
    by4 = [d for d in divs if d % 4 == 0]
    even = [d for d in divs if d % 2 == 0]
    return (by4 or even or divs)[0]


def to_group_end(eng, at_least: int = 2) -> int:
    """Steps (at least `at_least`) that bring the engine's step count to a multiple of 4, so that a
    graph of a multiple of 4 steps captured next pulls at the ends of whole delivery groups."""
    k = at_least
    while (eng.lif.step_count + k) % 4:
        k += 1
    return k


def capture(eng, steps: int):
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            eng.step(steps)
    torch.cuda.current_stream().wait_stream(s)
    return g


# ------------------------------------------------------------------ measurements
# Steps run before timing: the synthetic whole-fly network starts at rest and its firing climbs to
# a steady level (~220 Hz mean, ~29 M synaptic events per step at 64 flies) within ~2,000 steps of
# 0.1 ms; timed steps start from that steady state, the onset (the first steps from rest) is
# reported beside them.
SETTLE_STEPS = 3000


def measure_batched(cfg, device, steps, warmup, fly0, batch=BATCH, settle=SETTLE_STEPS):
    """Engine, captured graph of `chunk` steps, replays to time, and the onset figures: the
    network is tuned and timed from rest, run `settle` steps, then tuned again (the launch choice
    depends on the spike density) and recaptured for the timed steady-state steps."""
    from flyb200 import autotune
    eng = build_engine(cfg, batch, device, "step", fly0)
    eng.step(max(3, warmup))
    eng.tuned = {"lif": autotune.tune_lif(eng.lif, steps=10), "optic": autotune.tune_optic(eng.optic, steps=10)}
    eng.step(to_group_end(eng))    # the tuners restored the state: a step re-derives the carried dr
    chunk = graph_chunk(steps)
    g = capture(eng, chunk)
    reps = steps // chunk
    g.replay()
    torch.cuda.synchronize()
    ev0 = eng.lif.synaptic_events
    onset_ms = time_graph(g, reps) / (chunk * reps)
    onset = {"ms_per_step": onset_ms, "synaptic_events_per_step": (eng.lif.synaptic_events - ev0) / (chunk * reps),
             "lif": {k: v for k, v in eng.tuned["lif"].items() if k != "all"},
             "note": f"the first {max(3, warmup) + 3 + chunk * (reps + 1)} steps from rest"}
    for _ in range(max(0, settle) // chunk):
        g.replay()
    torch.cuda.synchronize()
    del g
    eng.tuned["lif"] = autotune.tune_lif(eng.lif, steps=10)
    eng.step(to_group_end(eng))
    g = capture(eng, chunk)
    g.replay()
    torch.cuda.synchronize()
    onset["value"] = eng.n_neurons * batch / (onset_ms / 1000.0)
    return eng, g, chunk, reps, onset


def time_graph(g, reps) -> float:
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    s.record()
    for _ in range(reps):
        g.replay()
    e.record()
    e.synchronize()
    return s.elapsed_time(e)


def kernel_roofline(eng, reps=20) -> dict:
    """The LIF step and the optic substep timed alone with CUDA events (B=64), after one untimed
    call of each (the first whole-range LIF step sizes its spike list). The LIF is timed over calls
    of one delivery group (Brain.pull_group steps: the updates and one pull) started at a group
    boundary, per step."""
    L = eng.lif.pull_group if eng.lif._pull_active() else 1
    eng.lif.step(to_group_end(eng, 1))
    eng.optic.substeps(1, carry=True)
    torch.cuda.synchronize()
    lif_ms = events_time(lambda: eng.lif.step(L), reps) / L
    opt_ms = events_time(lambda: eng.optic.substeps(1, carry=True), reps)
    lif_b, opt_b = eng.lif_bytes_per_step(group=L), eng.optic_bytes_per_step()
    return {"lif_ms": lif_ms, "optic_ms": opt_ms, "lif_bytes": lif_b, "optic_bytes": opt_b, "lif_group": L}


def measure_l2_gather(device, rows: int = 89_390, n_idx: int = 6_000_000) -> dict:
    """L2 -> SM gather ceiling on this GPU: flyb_gather_probe reads n_idx random 256-byte rows of a
    [rows][64] float array (the optic substep's dr gathers at 64 flies, L2-resident), best of 8 and
    16 blocks per SM; TB/s of row bytes + index bytes."""
    import ctypes as ct
    from flyb200 import _abi
    lib = _abi.lib()
    g = torch.Generator(device="cpu").manual_seed(7)
    idx = torch.randint(0, rows, (n_idx,), generator=g, dtype=torch.int32).to(device)
    x = torch.zeros(rows, 64, device=device)
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    out = torch.empty(sms * 16 * 256, device=device)
    stream = torch.cuda.current_stream(device).cuda_stream
    best = 0.0
    for bps in (8, 16):
        call = lambda: lib.flyb_gather_probe(ct.c_void_p(x.data_ptr()), rows, ct.c_void_p(idx.data_ptr()), n_idx,
                                             ct.c_void_p(out.data_ptr()), bps, ct.c_void_p(stream))
        for _ in range(3):
            if call():
                raise RuntimeError("flyb_gather_probe failed")
        ms = events_time(call, 10)
        best = max(best, (n_idx * 256 + n_idx * 4) / (ms / 1000.0) / 1e12)
    return {"tbs": best, "rows": rows, "gathers": n_idx, "row_bytes": 256}


def read_traffic() -> dict:
    """Per-launch DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of the ncu captures
    summarised in profiles/traffic.txt: one `<kernel> <bytes>` pair per line."""
    tp = ROOT / "profiles" / "traffic.txt"
    out = {}
    if tp.exists():
        for line in tp.read_text().splitlines():
            parts = line.split()
            if len(parts) >= 2 and not line.startswith("#"):
                try:
                    out[parts[0]] = float(parts[1])
                except ValueError:
                    pass
    return out


def measure_plain(cfg, device, steps, warmup, settle=SETTLE_STEPS) -> dict:
    """The plain single-instance kernels (one fly), settled to the same steady firing as the batched
    engine and tuned there as it is (LIF launch and delivery, optic shape and long-row threshold),
    timed two ways: replayed from a CUDA graph of 20 steps with the L2 left warm (like the batched
    figure), and launched eagerly step by step with the L2 flushed between timed steps."""
    from flyb200 import autotune
    eng = build_engine(cfg, 1, device, "step")
    eng.step(max(3, warmup))
    g = capture(eng, 20)              # settle to the steady firing the batched figures are timed at
    for _ in range(max(0, settle) // 20):
        g.replay()
    torch.cuda.synchronize()
    del g
    tuned = {"lif": autotune.tune_lif(eng.lif, steps=10), "optic": autotune.tune_optic(eng.optic, steps=10)}
    eng.step(to_group_end(eng))       # the tuners restored the state: a step re-derives the carried dr
    g = capture(eng, 20)
    g.replay()
    torch.cuda.synchronize()
    graph_ms = time_graph(g, 10) / 200
    del g
    eng.step(1)
    buf = torch.zeros(int(2 * L2_BYTES // 4), device=device)
    n = min(steps, 50)
    eager_ms = events_time(lambda: eng.step(1), n, flush=lambda: flush_l2(buf))
    del buf, eng
    torch.cuda.empty_cache()
    N = cfg.n_rate + cfg.n_spiking
    return {"graph": {"value": N / (graph_ms / 1000.0), "ms_per_step": graph_ms,
                      "how": "CUDA graph of 20 steps replayed back to back, L2 warm"},
            "eager_flushed": {"value": N / (eager_ms / 1000.0), "ms_per_step": eager_ms,
                              "how": "one call per step, L2 flushed between timed steps"},
            "tuned": {part: {k: v for k, v in t.items() if k in ("launch", "delivery", "variant", "long_row")}
                      for part, t in tuned.items()}}


def measure_adjoint(device) -> dict:
    from flyb200 import synthetic
    from flyb200.adjoint import OpticAdjoint
    cfg = synthetic.optic_config3(seed=3)
    rng = np.random.default_rng(0)
    m, T = cfg.m, 200
    pr = torch.from_numpy((rng.standard_normal((m, 1)) * 0.2).astype(np.float32)).to(device)
    spk = torch.zeros(m, 1, device=device)
    eng = OpticAdjoint(cfg.W0, cfg.pair_id, len(cfg.gain0), cfg.type_of, cfg.n_types, cfg.b, pr, spk,
                       dt_ms=cfg.dt_ms, batch=1, checkpoint=20, device=device)
    eng.set_params(torch.from_numpy(cfg.gain0), torch.from_numpy(cfg.tau_of_type))
    v0 = torch.from_numpy((rng.standard_normal((m, 1)) * 0.2).astype(np.float32)).to(device)
    a0 = torch.zeros(m, 1, device=device)
    w = torch.zeros(m, 1, device=device)
    w[:50], w[50:100] = 1 / 50, -1 / 50
    eng.forward(v0, a0, T)
    eng.backward(w)
    fwd = events_time(lambda: eng.forward(v0, a0, T), 3)
    bwd = events_time(lambda: eng.backward(w), 3)
    eng.check()
    return {"forward_ms": fwd, "backward_ms": bwd, "ratio": bwd / fwd, "units": m, "nnz": int(cfg.W0.nnz), "steps": T,
            "checkpoint": 20}


def measure_e2e(cfg, eng, device, steps, chunk: int = 20) -> dict:
    """Public-API loop: every step copies its own radiance frame in from pinned host memory, forms
    the photoreceptor activity, steps the whole fly and copies its motor readout out to pinned host
    memory. The copies run on two copy streams, so a step's input arrives while the previous step
    computes and its readout leaves while the next one does; `chunk` steps are captured as one CUDA
    graph and the host synchronises on every chunk's readouts (it reads `chunk` results at once).
    The launch-by-launch loop with a synchronisation per step is reported beside it."""
    from flyb200 import cuda as fcuda
    o, B = cfg.optic, eng.B
    frames = np.stack([o.grating(0.5 * i, B, seed=0) for i in range(chunk)])
    rad_host = torch.from_numpy(frames).pin_memory()                # (chunk, B, columns, 4)
    rad_dev = torch.empty_like(rad_host, device=device)
    groups = np.array_split(eng.lif_position[np.asarray(cfg.vpn_idx[:900])], 90)   # stored LIF order
    ptr = torch.tensor(np.r_[0, np.cumsum([len(g) for g in groups])], dtype=torch.int32, device=device)
    idx = torch.tensor(np.concatenate(groups), dtype=torch.int32, device=device)
    out_host = torch.empty(chunk, B, 90, dtype=torch.float64).pin_memory()
    out_dev = torch.empty(chunk, B, 90, dtype=torch.float64, device=device)
    rate_nb = eng.lif._st["rate"]                     # [N][B]: the readout reads the native layout
    n = max(chunk, min(steps, 100) // chunk * chunk)
    copy_in, copy_out = torch.cuda.Stream(device), torch.cuda.Stream(device)

    frame_ms = eng.dt_ms             # one radiance frame per step

    def one(i: int) -> None:
        rad_dev[i].copy_(rad_host[i], non_blocking=True)
        eng.set_radiance(rad_dev[i], frame_ms)
        eng.step(1)
        out_host[i].copy_(fcuda.group_means_native(ptr, idx, rate_nb, out_dev[i]), non_blocking=True)

    a_pr = torch.empty(chunk, cfg.optic.n_pr, B, device=device)

    def pipelined() -> None:
        # inputs: each frame's copy and its photoreceptor stage on the input stream (they do not
        # depend on the brain; the stage's state advances frame by frame there); steps, per-step
        # input installation and readouts on the main stream; readout copies on the output stream
        main = torch.cuda.current_stream(device)
        copy_in.wait_stream(main)
        arrived = []
        with torch.cuda.stream(copy_in):
            for i in range(chunk):
                rad_dev[i].copy_(rad_host[i], non_blocking=True)
                eng.set_radiance(rad_dev[i], frame_ms, a_pr=a_pr[i])
                arrived.append(torch.cuda.Event())
                arrived[-1].record(copy_in)

        def before(i):
            main.wait_event(arrived[i])
            eng.set_photoreceptors(a_pr[i])

        def after(i):
            fcuda.group_means_native(ptr, idx, rate_nb, out_dev[i])
            done = torch.cuda.Event()
            done.record(main)
            copy_out.wait_event(done)
            with torch.cuda.stream(copy_out):
                out_host[i].copy_(out_dev[i], non_blocking=True)

        eng.step(chunk, before=before, after=after)
        main.wait_stream(copy_out)

    for _ in range(3):
        one(0)
        torch.cuda.current_stream().synchronize()
    t0 = time.perf_counter()
    for k in range(n):
        one(k % chunk)
        torch.cuda.current_stream().synchronize()           # the host reads this step's readout
    dt_eager = time.perf_counter() - t0
    eng.step(to_group_end(eng, 0))                          # the graph below starts at a group boundary
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            pipelined()
    torch.cuda.current_stream().wait_stream(s)
    for _ in range(2):
        g.replay()
        torch.cuda.current_stream().synchronize()
    ev0 = eng.lif.synaptic_events
    t0 = time.perf_counter()
    for _ in range(n // chunk):
        g.replay()
        torch.cuda.current_stream().synchronize()           # the host reads `chunk` readouts
    dt = time.perf_counter() - t0
    events = (eng.lif.synaptic_events - ev0) / n
    del g
    return {"value": eng.n_neurons * B * n / dt, "unit": "neuron-steps/s",
            "h2d_bytes_per_step": int(rad_host[0].numel() * 4), "d2h_bytes_per_step": int(out_host[0].numel() * 8),
            "steps": n, "synaptic_events_per_step": events,
            "path": f"per step: radiance H2D (pinned) + photoreceptor stage on an input stream, whole-fly step, "
                    f"motor readout D2H on an output stream; {chunk} steps per CUDA graph, host sync per graph",
            "eager": {"value": eng.n_neurons * B * n / dt_eager, "note": "launched one by one, host sync every step"}}


class OraclePort:
    """The whole-fly step restated in C (oracle/), run on host cores in the engine's order: spike
    input, optic substep, VPN drive, LIF step. The LIF population is in the engine's stored order
    (WholeFly.lif_order), so a settled engine's state can be copied in as it is."""

    def __init__(self, cfg, batch: int, threads: int):
        import oracle
        from flyb200 import _abi
        from flyb200.brain import LIFParams, lif_coefficients, out_edges
        from flyb200.weights import lif_weights
        self.oracle, self.cfg, self.B, self.threads = oracle, cfg, batch, threads
        o = cfg.optic
        n = cfg.n_spiking
        driven = np.unique(o.W_sr.tocoo().row)
        order = np.concatenate([np.setdiff1d(np.arange(n), driven), driven])      # WholeFly.lif_order
        pos = np.empty(n, np.int64)
        pos[order] = np.arange(n)
        self.p = LIFParams(**{**cfg.lif.params, "dt": 0.1})
        W, _ = lif_weights(cfg.lif.c.subset(order), self.p)
        self.ptr, self.edges, mode = out_edges(W, self.p.w_syn)
        self.st = oracle.LifState(n, batch, 19, mode, self.p.v_rest)
        self.st.poisson_p[pos[np.asarray(cfg.sensory_idx)], :] = np.float32(cfg.lif.poisson_hz) * np.float32(self.p.dt / 1000.0)
        self.Wr = o.W_rr()
        self.a = np.exp(-0.1 / o.tau_of_type[o.type_of].astype(np.float32)).astype(np.float32)
        self.aad = float(np.exp(-0.1 / o.adapt_tau_ms))
        self.v = np.zeros((o.m, batch), np.float32)
        self.ad = np.zeros((o.m, batch), np.float32)
        rad = o.grating(0.0, batch, seed=0)
        ip = (rad[:, o.pr_column, :] * o.sens[None]).sum(-1)
        mean = ip.mean(1, keepdims=True)
        a_pr = np.clip((ip - mean) / (mean + 0.02), -1.0, 2.0).T.astype(np.float32)
        M = o.W_rp.tocsr()
        self.pr = oracle.spmm(M.indptr, M.indices, M.data, a_pr, batch, rows=o.m, alpha=o.gain_in)
        self.Wrs = o.W_rs.tocsc()[:, order].tocsr()
        self.Wsr = o.W_sr.tocsr()[order]
        self.P = lif_coefficients(self.p, False)
        self.flags = _abi.LIF_POISSON | _abi.LIF_COUNTS
        self.events = 0

    @classmethod
    def from_engine(cls, eng, threads: int, flies: int | None = None):
        """The engine's state (its first `flies` flies) copied into a port."""
        B = eng.B if flies is None else flies
        port = cls(eng.cfg, B, threads)
        lif = eng.lif
        for name, oname in (("v", "v"), ("g", "g"), ("refrac", "refrac"), ("rate", "rate"), ("spike_counts", "counts"),
                            ("spikes", "spikes"), ("adapt", "adapt"), ("res", "res"), ("drive", "drive"),
                            ("poisson_p", "poisson_p")):
            getattr(port.st, oname)[...] = lif._st[name][:, :B].cpu().numpy()
        port.st.ring[...] = lif.ring[:, :, :B].cpu().numpy()
        clock = lif._clock.cpu().numpy()
        port.st.step, port.st.ring_pos = int(clock[0]), int(clock[1]) % lif.R
        port.v[...] = eng.optic.v_s[:, :B].cpu().numpy()
        port.ad[...] = eng.optic.adapt_s[:, :B].cpu().numpy()
        port.pr[...] = eng.optic.pr_in[:, :B].cpu().numpy()
        return port

    def widen(self, batch: int):
        """A port of `batch` flies, each starting from fly 0's state (their Poisson streams differ)."""
        wide = OraclePort.__new__(OraclePort)
        wide.__dict__ = dict(self.__dict__)
        st = self.st.copy()
        for name in self.oracle.LifState.NAMES:
            setattr(st, name, np.ascontiguousarray(np.repeat(getattr(self.st, name)[:, :1], batch, axis=1)))
        st.ring = np.ascontiguousarray(np.repeat(self.st.ring[:, :, :1], batch, axis=2))
        st.batch = batch
        wide.st, wide.B = st, batch
        wide.v = np.ascontiguousarray(np.repeat(self.v[:, :1], batch, axis=1))
        wide.ad = np.ascontiguousarray(np.repeat(self.ad[:, :1], batch, axis=1))
        wide.pr = np.ascontiguousarray(np.repeat(self.pr[:, :1], batch, axis=1))
        return wide

    def step(self) -> None:
        o, st, ora, B = self.cfg.optic, self.st, self.oracle, self.B
        spk = ora.spmm(self.Wrs.indptr, self.Wrs.indices, self.Wrs.data, st.rate, B, rows=o.m, x_div=100.0, x_lo=0.0,
                       x_hi=3.0, alpha=o.gain_fb)
        ora.optic_run(self.v, self.ad, self.Wr.indptr, self.Wr.indices, self.Wr.data, self.pr, spk, self.a, o.b,
                      o.gain_rr, o.adapt_gain, self.aad, 1, threads=self.threads)
        dr = (np.clip(self.v + o.b[:, None], 0, 1) - o.b[:, None]).astype(np.float32)
        ora.spmm(self.Wsr.indptr, self.Wsr.indices, self.Wsr.data, dr, B, rows=self.cfg.n_spiking, y=st.drive,
                 alpha=o.gain_out_mv, y_lo=-o.drive_clip_mv, y_hi=o.drive_clip_mv)
        self.events += ora.lif_run(st, self.ptr, self.edges, self.P, n_delay=18, flags=self.flags, nsteps=1, seed=1,
                                   threads=self.threads)[1]

    def rate(self, steps: int) -> dict:
        """neuron-steps/s over `steps` timed steps (after one untimed step)."""
        self.step()
        ev0 = self.events
        t0 = time.perf_counter()
        for _ in range(steps):
            self.step()
        dt = time.perf_counter() - t0
        n = self.cfg.n_rate + self.cfg.n_spiking
        return {"value": n * self.B * steps / dt, "unit": "neuron-steps/s", "cores": self.threads, "kind": "port",
                "ms_per_step": dt / steps * 1000.0, "synaptic_events_per_step": (self.events - ev0) / steps,
                "mean_rate_hz": float(self.st.rate.mean())}


def measure_tracer(device, batch: int = BATCH, reps: int = 50, cpu: bool = True) -> dict:
    """The eye's ray tracer: 1,634 columns x 7 rays per fly in its own make_room scene, fused
    column sums, at `batch` flies. Device time of the one launch; the frame-level path (poses from
    the host, column radiance on the device) beside the reference's own torch tracer run on this
    GPU from baseline/_ref when it is installed; the C oracle on host cores."""
    from flyb200 import synthetic
    from flyb200 import world as W
    from flyb200.batch_world import BatchWorld
    _, dirs, w = synthetic.eye_grid()
    n_col, k = dirs.shape[:2]
    scenes = [W.make_room(i)[0] for i in range(batch)]
    bw = BatchWorld(scenes, device)
    bw.set_eye(dirs, w)
    pose = synthetic.fly_poses(batch, seed=0)
    bw.set_pose(*pose)
    out = torch.empty(batch, n_col, 4, device=device)
    for _ in range(3):
        bw.trace_eye(out)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(reps):                 # back to back: device time per launch, no host gaps
        bw.trace_eye(out)
    t1.record()
    t1.synchronize()
    ms = t0.elapsed_time(t1) / reps
    rays = batch * n_col * k

    def frame():
        bw.column_radiance(*pose, out=out)
        torch.cuda.current_stream().synchronize()

    for _ in range(3):
        frame()
    t0 = time.perf_counter()
    for _ in range(reps):
        frame()
    frame_ms = (time.perf_counter() - t0) / reps * 1000.0
    res = {"workload": f"{batch} flies x {n_col} columns x {k} rays, make_room scenes (20 spheres, 8 boxes, "
                       "6 planes), shadows and value-noise detail, column sums fused",
           "rays_per_frame": rays, "ms": ms, "rays_per_s": rays / (ms / 1000.0),
           "frame_ms": frame_ms, "frame_note": "poses from host numpy -> column radiance on the device, synchronised"}
    ref = reference_tracer(device, scenes, dirs, w, pose, out, reps=max(3, reps // 10))
    if ref is not None:
        res["reference_gpu"] = ref
        res["frame_speedup_vs_reference"] = ref["frame_ms"] / frame_ms
    if cpu:
        import oracle
        sample = 8
        blob = np.stack([W.pack_scene(sc) for sc in scenes[:sample]])
        args = dict(origins=pose[0][:sample], eye_dirs=dirs.reshape(-1, 3),
                    pose=np.concatenate([v[:sample] for v in pose[1:]], 1), weights=w, shared_origin=True, batch=sample)
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        cols = oracle.trace(blob, bw._scene_shape, bw.detail, threads=threads, **args)
        dt = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": sample * n_col * k / dt, "unit": "rays/s", "cores": threads, "kind": "port",
                               "sample": f"{sample} of the {batch} flies on the C oracle"}
        res["oracle_bit_exact"] = bool(np.array_equal(cols, out[:sample].cpu().numpy()))
    return res


def reference_tracer(device, scenes, dirs, w, pose, ours, reps: int):
    """The reference's stock tracer (flyverse.world / batch_world from baseline/_ref) on this GPU
    for the same scenes and poses, as BatchSim.column_radiance calls it (host numpy turn, captured
    trace, weighted sum); None when it is not installed."""
    ref_dir = ROOT / "baseline" / "_ref"
    if not (ref_dir / "flyverse" / "world.py").exists():
        return None
    sys.path.insert(0, str(ref_dir))
    try:
        from flyverse import batch_world as rbw
        from flyverse import world as rw
    except Exception as e:               # noqa: BLE001 - report, do not fail the bench
        return {"unavailable": f"import failed: {e}"}
    finally:
        sys.path.remove(str(ref_dir))
    worlds = []
    for i in range(len(scenes)):
        wr = rw.make_room(i)[0]
        wr.device = device
        worlds.append(wr)
    bw = rbw.BatchWorld(worlds, device)
    wts = torch.as_tensor(w, dtype=torch.float32, device=device)
    eye, f, left, up = pose

    def frame():
        rotation = np.stack([f, left, up], axis=2)
        directions = dirs.reshape(1, -1, 3) @ rotation.transpose(0, 2, 1)
        origins = np.broadcast_to(eye[:, None], directions.shape)
        rad = bw.trace(torch.from_numpy(np.ascontiguousarray(origins, dtype=np.float32)),
                       torch.from_numpy(np.ascontiguousarray(directions, dtype=np.float32)), cuda_graphs=True)
        col = (rad.reshape(len(worlds), *dirs.shape[:2], 4) * wts[None, None, :, None]).sum(2)
        torch.cuda.current_stream().synchronize()
        return col

    col = frame()
    for _ in range(2):
        frame()
    t0 = time.perf_counter()
    for _ in range(reps):
        frame()
    frame_ms = (time.perf_counter() - t0) / reps * 1000.0
    diff = (col - ours).abs()
    res = {"frame_ms": frame_ms, "reps": reps, "max_abs_diff": float(diff.max()),
           "columns_differing_over_1e-4": int((diff > 1e-4).any(-1).sum()),
           "note": "the reference's torch tracer on this GPU (CUDA-graph captured), same scenes and poses"}
    del bw, worlds
    torch.cuda.empty_cache()
    return res


# ------------------------------------------------------------------ the reference's own code
REF_DIR = ROOT / "baseline" / "_ref"


def reference_modules():
    """flyverse (the unmodified reference, installed under baseline/_ref): {name: module}, or
    {"unavailable": why}."""
    if not (REF_DIR / "flyverse" / "brain.py").exists():
        return {"unavailable": "the reference is not installed under baseline/_ref"}
    import importlib
    os.environ.setdefault("FLYVERSE_CUDA_CACHE", tempfile.mkdtemp(prefix="flyverse_cuda_"))
    sys.path.insert(0, str(REF_DIR))
    try:
        return {k: importlib.import_module(f"flyverse.{k}") for k in ("brain", "connectome", "cuda", "optic")}
    except Exception as e:                # noqa: BLE001 - report, do not fail the bench
        return {"unavailable": f"import failed: {e}"}
    finally:
        sys.path.remove(str(REF_DIR))


def reference_brain(ref, cfg2, device, batch):
    """The reference's Brain on config 2's graph, event-driven, with the benchmark's model constants."""
    import pandas as pd
    c = cfg2.c
    rc = ref["connectome"].Connectome(c.neurons[["bodyId", "type", "superclass", "nt"]].copy(), c.W.copy(),
                                      pd.Series(np.arange(c.n), index=c.neurons.bodyId.to_numpy()))
    cuda = torch.device(device).type == "cuda"
    b = ref["brain"].Brain(rc, ref["brain"].LIFParams(**cfg2.params, event_driven=True), device=device, seed=0,
                           batch=batch, cuda_kernels=True if cuda else None)
    b.set_poisson(cfg2.poisson_idx, cfg2.poisson_hz)
    b.record_activity = True
    return b


def graph_ms_per_step(step, steps: int, reps: int, generator=None) -> float:
    """Device ms per step of `step(steps)` captured once as a CUDA graph and replayed `reps` times."""
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    if generator is not None:
        g.register_generator_state(generator)
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            step(steps)
    torch.cuda.current_stream().wait_stream(s)
    g.replay()
    ms = time_graph(g, reps) / (steps * reps)
    del g
    return ms


def reference_lif_gpu(ref, cfg2, device, batch) -> dict:
    """The reference's CUDA LIF step (flyverse/cuda.py + kernels/neural.cu, compiled by its own nvcc
    call for this GPU: g decay, event scatter, torch.rand, fused update) on config 2's graph, eager
    and captured in a CUDA graph of n_delay steps (its FlyBrain replays such graphs), after 500
    steps from rest."""
    b = reference_brain(ref, cfg2, device, batch)
    b.step(500)
    torch.cuda.synchronize()
    eager = events_time(lambda: b.step(1), 50)
    graph = graph_ms_per_step(b.step, b.n_delay, 10, b.gen)
    return {"eager_ms": eager, "graph_ms": graph, "path": "native neural.cu (launch_events, launch_lif), cuda_sparse=torch"}


def ours_lif(cfg2, device, batch) -> float:
    """This library's Brain on the same graph and constants: device ms per step, graph-replayed
    chunks of 20 steps after 500 steps from rest, the launch shape autotuned."""
    from flyb200 import autotune
    from flyb200.brain import Brain, LIFParams
    b = Brain(cfg2.c, LIFParams(**cfg2.params), device=device, seed=0, batch=batch, launch="step")
    b.set_poisson(cfg2.poisson_idx, cfg2.poisson_hz)
    b.record_activity = True
    b.step(500)
    autotune.tune_lif(b, steps=10)
    b.step(4 - b.step_count % 4)
    return graph_ms_per_step(b.step, 20, 10)


def reference_optic_gpu(ref, cfg3, device, batch) -> dict:
    """The reference's CUDA optic substep on config 3's lobe (optic.py:585-589: the recurrent
    product through its `_mv` with torch's sparse CSR (cuSPARSE, its default cuda_sparse) or its
    warp CSR kernel, then launch_optic), under a held random input."""
    from types import SimpleNamespace
    optic, cuda = ref["optic"], ref["cuda"]
    W = cfg3.W_rr()
    rng = np.random.default_rng(0)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32), device=device)  # noqa: E731
    out = {}
    for sparse in ("torch", "warp"):
        M = optic._csr(W, device, cuda_sparse=sparse)
        lobe = SimpleNamespace(v=t(np.zeros((batch, cfg3.m))), adapt=t(np.zeros((batch, cfg3.m))), B=batch,
                               n_rate=cfg3.m, p=optic.OpticParams(adapt_tau_ms=cfg3.adapt_tau_ms, dt_ms=cfg3.dt_ms),
                               _a=t(cfg3.a), b_vec=t(cfg3.b), _a_ad=cfg3.aad, _cuda_dr=t(np.zeros((batch, cfg3.m))))
        pr, spk = t(rng.standard_normal((batch, cfg3.m)) * 0.2), t(np.zeros((batch, cfg3.m)))
        cuda.optic_dr(lobe.v, lobe.b_vec, lobe._cuda_dr)

        def substeps(n):
            for _ in range(n):
                cuda.optic_update(lobe, optic._mv(M, lobe._cuda_dr), pr, spk)

        substeps(5)
        torch.cuda.synchronize()
        out[sparse] = {"eager_ms": events_time(lambda: substeps(1), 20), "graph_ms": graph_ms_per_step(substeps, 10, 5)}
    return out


def ours_optic(cfg3, device, batch) -> tuple:
    """This library's fused substep on the same lobe: device ms per substep (autotuned shape) and
    the tuner's choice (launch, kernel shape, long-row threshold)."""
    from flyb200 import autotune
    from flyb200.optic import OpticCore
    core = OpticCore(cfg3.W_rr(), cfg3.a, cfg3.b, batch=batch, device=device, gain_rr=cfg3.gain_rr,
                     adapt_gain=cfg3.adapt_gain, aad=cfg3.aad, launch="step")
    rng = np.random.default_rng(0)
    core.pr_in.copy_(torch.from_numpy((rng.standard_normal((cfg3.m, batch)) * 0.2).astype(np.float32)))
    pick = autotune.tune_optic(core, steps=10)
    core.substeps(2)
    tuned = {k: pick[k] for k in ("launch", "variant", "long_row")}
    return graph_ms_per_step(lambda n: core.substeps(n, carry=True), 10, 5), tuned


def measure_reference_gpu(device, cfg2, cfg3) -> dict:
    """The reference's own GPU kernels (its stock cuda_kernels=True path from baseline/_ref) beside
    this library's kernels on the same configurations and this GPU: config 2's LIF at 1 and 64
    flies, config 3's optic substep at 1 and 64 flies."""
    ref = reference_modules()
    if "unavailable" in ref:
        return ref
    res = {"lif_c2": {}, "optic_c3": {}}
    for B in (1, 64):
        try:
            r = reference_lif_gpu(ref, cfg2, device, B)
            r["ours_ms"] = ours_lif(cfg2, device, B)
            r["speedup_vs_graph"] = r["graph_ms"] / r["ours_ms"]
        except Exception as e:            # noqa: BLE001 - report, do not fail the bench
            r = {"unavailable": f"{type(e).__name__}: {e}"}
        res["lif_c2"][f"B{B}"] = r
        torch.cuda.empty_cache()
        try:
            r = reference_optic_gpu(ref, cfg3, device, B)
            r["ours_ms"], r["ours_tuned"] = ours_optic(cfg3, device, B)
            r["speedup_vs_best_graph"] = min(v["graph_ms"] for v in r.values()
                                             if isinstance(v, dict) and "graph_ms" in v) / r["ours_ms"]
        except Exception as e:            # noqa: BLE001
            r = {"unavailable": f"{type(e).__name__}: {e}"}
        res["optic_c3"][f"B{B}"] = r
        torch.cuda.empty_cache()
    return res


def reference_own_cpu(cfg2, cfg3, threads: int) -> dict:
    """The reference's own CPU code on this host (torch CPU, `threads` threads): Brain.step of
    config 2 at one fly (event-driven, after 100 steps from rest; median of 5 runs of 20 steps) and
    OpticLobe._substep of config 3 at one fly (median of 5 runs of 5 substeps)."""
    ref = reference_modules()
    if "unavailable" in ref:
        return ref
    torch.set_num_threads(threads)
    b = reference_brain(ref, cfg2, "cpu", 1)
    b.step(100)
    runs = []
    for _ in range(5):
        t0 = time.perf_counter()
        b.step(20)
        runs.append((time.perf_counter() - t0) / 20)
    lif_s = float(np.median(runs))
    optic = ref["optic"]
    W = cfg3.W_rr()
    lobe = object.__new__(optic.OpticLobe)
    lobe.p = optic.OpticParams(adapt_tau_ms=cfg3.adapt_tau_ms, dt_ms=cfg3.dt_ms)
    lobe.slow, lobe._hooks = None, False
    lobe.W_rr = torch.sparse_csr_tensor(torch.from_numpy(W.indptr.astype(np.int64)),
                                        torch.from_numpy(W.indices.astype(np.int64)), torch.from_numpy(W.data),
                                        size=W.shape)
    lobe._a, lobe.b_vec, lobe._a_ad = torch.from_numpy(cfg3.a), torch.from_numpy(cfg3.b), cfg3.aad
    lobe.v, lobe.adapt = torch.zeros(1, cfg3.m), torch.zeros(1, cfg3.m)
    rng = np.random.default_rng(0)
    pr = torch.from_numpy((rng.standard_normal((1, cfg3.m)) * 0.2).astype(np.float32))
    spk = torch.zeros(1, cfg3.m)
    optic.OpticLobe._substep(lobe, pr, spk)
    runs = []
    for _ in range(5):
        t0 = time.perf_counter()
        for _ in range(5):
            optic.OpticLobe._substep(lobe, pr, spk)
        runs.append((time.perf_counter() - t0) / 5)
    opt_s = float(np.median(runs))
    return {"lif_c2_b1": {"ms_per_step": lif_s * 1000, "neuron_steps_per_s": cfg2.c.n / lif_s},
            "optic_c3_b1": {"ms_per_substep": opt_s * 1000, "unit_steps_per_s": cfg3.m / opt_s},
            "cores": threads, "code": "flyverse.brain.Brain.step (event_driven) / flyverse.optic.OpticLobe._substep, "
                                      "torch CPU, from baseline/_ref"}


# ------------------------------------------------------------------ uneven rollouts
def measure_uneven(cfg, device, batch: int, lengths: tuple, steps: int, warm: int, chunk: int = 20,
                   seed: int = 0) -> dict:
    """Uneven rollouts: every fly runs episodes back to back, lengths uniform on `lengths` steps,
    each with its own Poisson rate (uniform 20-200 Hz on the sensory cells); a fly whose episode
    ends inside a replay of `chunk` steps is reset after that replay (WholeFly.reset: state, pending
    input and spike history to rest; BatchSim's per-row resets, batch_sim.py:282-304) and starts
    the next episode with a new rate while the others run on. `steps` steps are timed on the device
    (replays and resets) after `warm` steps; the autotuners pick the launch shapes after the warm-up."""
    from flyb200 import autotune
    from flyb200.whole import WholeFly
    rng = np.random.default_rng(seed)
    eng = WholeFly(cfg, batch, device=device, seed=seed + 1, launch="step")
    eng.set_poisson_rates(rng.uniform(20.0, 200.0, batch))
    eng.set_radiance(torch.from_numpy(cfg.optic.grating(0.0, batch, seed=seed)).to(device), 0.1)
    left = rng.integers(lengths[0], lengths[1] + 1, batch)
    eng.step(chunk)
    left -= chunk
    g = capture(eng, chunk)

    def run(n_replays: int) -> int:
        nonlocal left
        resets = 0
        for _ in range(n_replays):
            g.replay()
            left -= chunk
            done = np.flatnonzero(left <= 0)
            if done.size:
                eng.reset(done, rng.uniform(20.0, 200.0, done.size))
                left[done] = rng.integers(lengths[0], lengths[1] + 1, done.size)
                resets += int(done.size)
        return resets

    run(warm // chunk)
    torch.cuda.synchronize()
    del g
    eng.tuned = {"lif": autotune.tune_lif(eng.lif, steps=10), "optic": autotune.tune_optic(eng.optic, steps=10)}
    eng.step(chunk)                              # keeps the step count a multiple of the chunk
    left -= chunk
    g = capture(eng, chunk)
    torch.cuda.synchronize()
    ev0 = eng.lif.synaptic_events
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record()
    resets = run(steps // chunk)
    t1.record()
    t1.synchronize()
    ms = t0.elapsed_time(t1)
    n_steps = steps // chunk * chunk
    eng.lif.check()
    out = {"value": eng.n_neurons * batch * n_steps / (ms / 1000.0), "unit": "neuron-steps/s",
           "ms_per_step": ms / n_steps, "flies": batch, "episode_steps": list(lengths), "timed_steps": n_steps,
           "episodes_ended": resets, "synaptic_events_per_step": (eng.lif.synaptic_events - ev0) / n_steps,
           "lif": {k: v for k, v in eng.tuned["lif"].items() if k != "all"},
           "note": f"episode ends take effect at the end of the {chunk}-step replay they fall in"}
    del g, eng
    torch.cuda.empty_cache()
    return out


# ------------------------------------------------------------------ FP32 against FP64
def fp64_error(device, cfg3, eng) -> dict:
    """max |FP32 - FP64| of the optic state after 200 substeps: config 3's lobe at one fly from rest
    under a held random input, and the whole fly's lobe continued from the settled engine (its first
    8 flies, their held inputs), each against the FP64 oracle from the same start."""
    import oracle
    from flyb200.optic import OpticCore
    out = {}
    W = cfg3.W_rr()
    rng = np.random.default_rng(0)
    pr = (rng.standard_normal((cfg3.m, 1)) * 0.2).astype(np.float32)
    core = OpticCore(W, cfg3.a, cfg3.b, batch=1, device=device, gain_rr=cfg3.gain_rr, adapt_gain=cfg3.adapt_gain,
                     aad=cfg3.aad, launch="step")
    core.pr_in.copy_(torch.from_numpy(pr))
    core.substeps(200)
    v64, a64 = np.zeros((cfg3.m, 1)), np.zeros((cfg3.m, 1))
    oracle.optic_run_f64(v64, a64, W.indptr, W.indices, W.data, pr, np.zeros_like(pr), cfg3.a, cfg3.b, cfg3.gain_rr,
                         cfg3.adapt_gain, cfg3.aad, 200)
    out["C3_b1_200_substeps"] = _err(core.v_s.cpu().numpy(), v64, cfg3.b)
    o, B = eng.cfg.optic, 8
    W = o.W_rr()
    a = np.exp(-0.1 / o.tau_of_type[o.type_of].astype(np.float32)).astype(np.float32)
    aad = float(np.exp(-0.1 / o.adapt_tau_ms))
    v0 = eng.optic.v_s[:, :B].cpu().numpy()
    ad0 = eng.optic.adapt_s[:, :B].cpu().numpy()
    pr = eng.optic.pr_in[:, :B].cpu().numpy()
    spk = eng.optic.spk_in[:, :B].cpu().numpy()
    core = OpticCore(W, a, o.b, batch=B, device=device, gain_rr=o.gain_rr, adapt_gain=o.adapt_gain, aad=aad,
                     launch="step")
    for dst, src in ((core.v_s, v0), (core.adapt_s, ad0), (core.pr_in, pr), (core.spk_in, spk)):
        dst.copy_(torch.from_numpy(src))
    core.substeps(200)
    v64, a64 = v0.astype(np.float64), ad0.astype(np.float64)
    oracle.optic_run_f64(v64, a64, W.indptr, W.indices, W.data, pr, spk, a, o.b, o.gain_rr, o.adapt_gain, aad, 200)
    out["C5_lobe_8_flies_200_substeps"] = _err(core.v_s.cpu().numpy(), v64, o.b)
    return out


def _err(v32: np.ndarray, v64: np.ndarray, b: np.ndarray) -> dict:
    r32 = np.clip(v32 + b[:, None], 0, 1)
    r64 = np.clip(v64 + b[:, None], 0, 1)
    return {"v_abs": float(np.abs(v32 - v64).max()), "rate_abs": float(np.abs(r32 - r64).max()),
            "v_scale": float(np.abs(v64).max())}


# ------------------------------------------------------------------ arms
def arm_config(world: int) -> dict:
    """The workload both arms report (the reference arm times a bounded sample of it)."""
    return {"workload": "whole fly 167,106 neurons (89,390 optic + 71,618 LIF + 6,098 sensory), 25.6M edges, "
                        "dt 0.1 ms, optic<->LIF coupling every step", "batch_per_gpu": BATCH,
            "flies_total": BATCH * world, "l2": "state of 64 flies > 126 MB L2; no flush needed",
            "parallelism": f"fly shards x{world}, no per-step collective",
            "state": f"steady firing after {SETTLE_STEPS} settling steps"}


def reference_arm(args) -> None:
    """The CPU port of the path (the C oracle; the reference itself is Python/torch and has no C
    implementation of the step to build) on every host thread, same metric, config and state: one
    fly settled for the same number of steps from rest, its state given to all 64 flies (their
    Poisson streams differ), then whole 64-fly steps timed."""
    from flyb200 import synthetic
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg = synthetic.whole_fly_config5(seed=0)
    threads = os.cpu_count() or 1
    one = OraclePort(cfg, 1, threads)
    t0 = time.perf_counter()
    for _ in range(SETTLE_STEPS):
        one.step()
    settle_s = time.perf_counter() - t0
    port = one.widen(BATCH)
    steps = max(2, min(args.steps, 6))
    r = port.rate(steps)
    r["sample"] = (f"{steps} whole-fly steps x {BATCH} flies ({cfg.n_rate + cfg.n_spiking:,} neurons) on the C oracle, "
                   f"from a fly settled {SETTLE_STEPS} steps ({settle_s:.0f} s, untimed; {r.pop('mean_rate_hz'):.0f} Hz "
                   f"mean)")
    line = {"metric": METRIC, "value": r["value"], "unit": "neuron-steps/s", "n_gpus": args.gpus, "steps": steps,
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded whole_fly_config5)",
            "config": arm_config(args.gpus), "impl": "reference", "cpu_baseline": r,
            "e2e": {"value": r["value"], "unit": "neuron-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="flyb200", choices=["flyb200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="the headline, roofline and e2e only")
    args = ap.parse_args()
    if args.impl == "reference":
        reference_arm(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=device)
    from flyb200 import synthetic
    from flyb200 import build as fbuild
    fbuild.build()
    cfg = synthetic.whole_fly_config5(seed=0)
    N = cfg.n_rate + cfg.n_spiking
    eng, g, chunk, reps, onset = measure_batched(cfg, device, args.steps, args.warmup, fly0=rank * BATCH)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = eng.lif.synaptic_events
    with Clocks(local) as clk:
        ms = time_graph(g, reps)
    clocks = clk.summary()
    timed_steps = chunk * reps
    events_per_step = (eng.lif.synaptic_events - ev0) / timed_steps
    if world > 1:
        t = torch.tensor([ms], device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        del g                      # no collective is captured; release the graph before the group
        dist.destroy_process_group()
    value = N * BATCH * world * timed_steps / (ms / 1000.0)
    launches = eng.launches(chunk) * reps
    eng.lif.check()
    if rank != 0:
        return
    roof = kernel_roofline(eng)
    peaks = load_peaks()
    lif_gbs = roof["lif_bytes"] / (roof["lif_ms"] / 1000.0) / 1e9
    opt_gbs = roof["optic_bytes"] / (roof["optic_ms"] / 1000.0) / 1e9
    dom = "lif" if roof["lif_ms"] >= roof["optic_ms"] else "optic"
    achieved = lif_gbs if dom == "lif" else opt_gbs
    threads = os.cpu_count() or 1
    cpu = None
    if not args.no_cpu_baseline:             # the same settled state, copied into the C oracle
        cpu = OraclePort.from_engine(eng, threads).rate(3)
        cpu["sample"] = (f"3 whole-fly steps x {BATCH} flies ({N:,} neurons) on the C oracle, from this run's settled "
                         f"state ({cpu.pop('mean_rate_hz'):.0f} Hz mean)")
    e2e = measure_e2e(cfg, eng, device, args.steps)
    traffic = read_traffic().get(dom)
    l2 = measure_l2_gather(device)
    optic_l2_bytes = int(cfg.optic.W0.nnz) * BATCH * 4 + roof["optic_bytes"]     # dr gathers + the streamed bytes
    extras = {}
    if not args.no_extras:
        cfg3 = synthetic.optic_config3(seed=3)
        extras["fp64_max_err"] = fp64_error(device, cfg3, eng)
        del g
        autotune_summary = {k: {kk: vv for kk, vv in v.items() if kk != "all"} for k, v in eng.tuned.items()}
        state = f"steady firing after {SETTLE_STEPS} settling steps (mean rate {float(eng.lif.rate.mean()):.0f} Hz)"
        del eng
        torch.cuda.empty_cache()
        # the whole fly at 256 flies (config 5's width), even lengths from the steady state
        n256 = min(args.steps, 40)
        eng256, g256, c256, r256, onset256 = measure_batched(cfg, device, n256, args.warmup, fly0=0, batch=256)
        ev256 = eng256.lif.synaptic_events
        ms256 = time_graph(g256, r256) / (c256 * r256)
        extras["batch256"] = {"value": N * 256 / (ms256 / 1000.0), "ms_per_step": ms256, "steps": c256 * r256,
                              "synaptic_events_per_step": (eng256.lif.synaptic_events - ev256) / (c256 * r256),
                              "onset": {k: onset256[k] for k in ("value", "ms_per_step", "synaptic_events_per_step")},
                              "autotune": {k: {kk: vv for kk, vv in v.items() if kk != "all"}
                                           for k, v in eng256.tuned.items()}}
        del g256, eng256
        torch.cuda.empty_cache()
        extras["uneven_c5_b256"] = measure_uneven(cfg, device, 256, (200, 2000), 2000, 600)
        cfg4 = synthetic.batched_config4(seed=0)
        extras["uneven_c4_b64"] = measure_uneven(cfg4, device, BATCH, (500, 4000), 2000, 1000)
        plain = measure_plain(cfg, device, args.steps, args.warmup)
        extras["reference_gpu"] = measure_reference_gpu(device, cfg4.lif, cfg3)
        if not args.no_cpu_baseline:
            extras["reference_own_cpu"] = reference_own_cpu(cfg4.lif, cfg3, threads)
        del cfg4
        adj = measure_adjoint(device)
        extras["tracer"] = measure_tracer(device, cpu=not args.no_cpu_baseline)
        extras["onset"] = onset
        extras["autotune"] = autotune_summary
        extras["state"] = state
    line = {
        "metric": METRIC, "value": value, "unit": "neuron-steps/s", "n_gpus": world, "steps": timed_steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms / timed_steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded whole_fly_config5)",
        "config": arm_config(world),
        **{k: v for k, v in extras.items() if k != "fp64_max_err"},
        "synaptic_events_per_s": events_per_step * world * timed_steps / (ms / 1000.0),
        "synaptic_events_per_step": events_per_step,
        "roofline": {"bound": "hbm", "kernel": f"{dom} step (B=64)", "achieved": achieved, "peak": peaks["hbm_gbs"],
                     "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                     "peak_source": peaks["source"], "lif_gbs": lif_gbs, "optic_gbs": opt_gbs,
                     "lif_ms": roof["lif_ms"], "optic_ms": roof["optic_ms"], "lif_bytes": roof["lif_bytes"],
                     "optic_bytes": roof["optic_bytes"], "lif_group": roof["lif_group"],
                     "l2_gather": {"kernel": "optic step (B=64)", "bytes": optic_l2_bytes,
                                   "achieved_tbs": optic_l2_bytes / (roof["optic_ms"] / 1000.0) / 1e12,
                                   "peak_tbs": l2["tbs"],
                                   "frac": optic_l2_bytes / (roof["optic_ms"] / 1000.0) / 1e12 / l2["tbs"],
                                   "peak_source": "flyb_gather_probe, measured in this run",
                                   "note": "the optic substep gathers nnz x 64 x 4 B of L2-resident dr"}},
        "cpu_baseline": cpu,
        "e2e": e2e,
    }
    if not args.no_extras:
        line["batch1"] = plain
        line["batched_over_plain"] = value / world / plain["graph"]["value"]
        line["adjoint"] = adj
        line["fp64_max_err"] = extras["fp64_max_err"]
    line["gpu_launches"] = launches
    line["clocks"] = clocks
    print(json.dumps(line))


if __name__ == "__main__":
    main()
