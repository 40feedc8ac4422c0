#!/usr/bin/env python
"""Headline benchmark: neuron-steps/s of the whole-fly brain step at 167,106 neurons.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl flyb200|reference]

Workload (synthetic, seeded; the MaleCNS data is not available): flyb200.synthetic.whole_fly_config5,
167,106 neurons = 89,390 graded optic units + 71,618 LIF + 6,098 Poisson-driven sensory cells,
25.6 M edges (~124 M synapses), dt 0.1 ms, optic <-> LIF coupling every step, a drifting grating on
5,895 photoreceptors. One step advances all 167,106 neurons of every fly once (flyb200.whole).

  value          neuron-steps/s of B=64 flies per GPU (whole job over N GPUs, weak scaling),
                 steps replayed from a CUDA graph; state > L2, so no flush is needed
  batch1         the plain single-instance kernels (B=1, one launch per kernel per step), L2 flushed
                 between timed steps, for the "vs plain" ratio
  adjoint        optic-lobe adjoint over 200 substeps (89,390 units, 6 M nnz, checkpoint 20) over
                 the forward pass time
  e2e            the same B=64 step through the public API with, every step, the radiance copied in
                 from pinned host memory and the motor readout copied out, the calls captured once
                 as a CUDA graph and the host synchronising on every step's readout (the eager
                 launch-by-launch figure is reported beside it)
  roofline       the LIF step kernel: algorithmic bytes / CUDA-event time against measured HBM copy
  tracer         the eye's ray tracer at 64 flies x 1,634 columns x 7 rays: device time, the frame
                 path beside the reference's own torch tracer on the same GPU (baseline/_ref), and
                 the C oracle on host cores
  cpu_baseline   the C oracle port (oracle/) on this host's cores, a bounded sample of the workload
`--impl reference` times that CPU port alone on the same config and prints the same line.
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
    """Steps per captured graph: a divisor of `steps` (so exactly `steps` are timed), even when
    possible (an odd count ends each replay with a copy of the optic dr back to its start buffer)."""
    divs = [d for d in range(min(most, steps), 0, -1) if steps % d == 0]
    even = [d for d in divs if d % 2 == 0]
    return (even or divs)[0]


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
    eng.step(2)                    # the tuners restored the state: one step re-derives the carried dr
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
    eng.step(2)
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
    call of each (the first whole-range LIF step sizes its spike list)."""
    eng.lif.step(1)
    eng.optic.substeps(1, carry=True)
    torch.cuda.synchronize()
    lif_ms = events_time(lambda: eng.lif.step(1), reps)
    opt_ms = events_time(lambda: eng.optic.substeps(1, carry=True), reps)
    lif_b, opt_b = eng.lif_bytes_per_step(), eng.optic_bytes_per_step()
    return {"lif_ms": lif_ms, "optic_ms": opt_ms, "lif_bytes": lif_b, "optic_bytes": opt_b}


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


def measure_plain(cfg, device, steps, warmup, settle=SETTLE_STEPS):
    eng = build_engine(cfg, 1, device, "step")
    eng.step(max(3, warmup))
    g = capture(eng, 10)              # settle to the steady firing the batched figures are timed at
    for _ in range(max(0, settle) // 10):
        g.replay()
    torch.cuda.synchronize()
    del g
    eng.step(1)
    buf = torch.zeros(int(2 * L2_BYTES // 4), device=device)
    n = min(steps, 50)
    ms = events_time(lambda: eng.step(1), n, flush=lambda: flush_l2(buf))
    del buf
    return eng, ms


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


def measure_e2e(cfg, eng, device, steps, chunk: int = 10) -> dict:
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
            "path": f"per step: its radiance frame H2D from pinned memory and the photoreceptor stage "
                    f"(flyb_photoreceptor, input stream), the photoreceptor input installed and the whole fly "
                    f"stepped, motor readout D2H to pinned memory (output stream); {chunk} steps per CUDA graph "
                    f"(WholeFly.step with per-step before/after calls), the host synchronising on each graph's "
                    f"readouts",
            "eager": {"value": eng.n_neurons * B * n / dt_eager,
                      "note": "the same calls launched one by one, the host synchronising every step"}}


def cpu_port_rate(cfg, batch: int, steps: int, threads: int) -> dict:
    """The oracle whole-fly step on host cores: neuron-steps/s over a bounded sample."""
    import oracle
    from flyb200 import _abi
    from flyb200.brain import LIFParams, lif_coefficients, out_edges
    from flyb200.weights import lif_weights
    p = LIFParams(**cfg.lif.params)
    W, _ = lif_weights(cfg.lif.c, p)
    ptr, edges, mode = out_edges(W, p.w_syn)
    n = cfg.n_spiking
    st = oracle.LifState(n, batch, 19, mode, p.v_rest)
    st.poisson_p[cfg.sensory_idx, :] = np.float32(cfg.lif.poisson_hz) * np.float32(p.dt / 1000.0)
    o = cfg.optic
    Wr = o.W_rr()
    tau = o.tau_of_type[o.type_of].astype(np.float32)
    a = np.exp(-0.1 / tau).astype(np.float32)
    aad = float(np.exp(-0.1 / o.adapt_tau_ms))
    m = o.m
    v = np.zeros((m, batch), np.float32)
    ad = np.zeros((m, batch), np.float32)
    rng = np.random.default_rng(0)
    pr = (rng.standard_normal((m, batch)) * 0.1).astype(np.float32)
    Wrs, Wsr = o.W_rs.tocsr(), o.W_sr.tocsr()
    P = lif_coefficients(p, False)
    flags = _abi.LIF_POISSON | _abi.LIF_COUNTS

    def step():
        spk = oracle.spmm(Wrs.indptr, Wrs.indices, Wrs.data, st.rate, batch, rows=m, x_div=100.0, x_lo=0.0, x_hi=3.0,
                          alpha=o.gain_fb)
        oracle.optic_run(v, ad, Wr.indptr, Wr.indices, Wr.data, pr, spk, a, o.b, o.gain_rr, o.adapt_gain, aad, 1,
                         threads=threads)
        dr = (np.clip(v + o.b[:, None], 0, 1) - o.b[:, None]).astype(np.float32)
        oracle.spmm(Wsr.indptr, Wsr.indices, Wsr.data, dr, batch, rows=n, y=st.drive, alpha=o.gain_out_mv,
                    y_lo=-o.drive_clip_mv, y_hi=o.drive_clip_mv)
        oracle.lif_run(st, ptr, edges, P, n_delay=18, flags=flags, nsteps=1, seed=1, threads=threads)

    step()
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    dt = time.perf_counter() - t0
    return {"value": (m + n) * batch * steps / dt, "unit": "neuron-steps/s", "cores": threads,
            "kind": "port", "sample": f"{steps} whole-fly steps x {batch} flies ({m + n:,} neurons) on the C oracle"}


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


# ------------------------------------------------------------------ arms
def arm_config(world: int) -> dict:
    """The workload both arms report (the reference arm times a bounded sample of it)."""
    return {"workload": "whole fly 167,106 neurons (89,390 optic + 71,618 LIF + 6,098 sensory), 25.6M edges, "
                        "dt 0.1 ms, optic<->LIF coupling every step", "batch_per_gpu": BATCH,
            "flies_total": BATCH * world, "l2": "state of 64 flies > 126 MB L2; no flush needed",
            "parallelism": f"fly shards x{world}, no per-step collective",
            "state": f"our arm: steady firing after {SETTLE_STEPS} settling steps (onset from rest reported "
                     f"under 'onset'); reference arm: a sample of the first steps from rest"}


def reference_arm(args) -> None:
    """The CPU port of the path (the C oracle; the reference itself is Python/torch and is not
    installed on the GPU machines), timed on every host thread, same metric and config."""
    from flyb200 import synthetic
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg = synthetic.whole_fly_config5(seed=0)
    threads = os.cpu_count() or 1
    batch = 8
    r = cpu_port_rate(cfg, batch, max(1, min(args.steps, 6)), threads)
    n = cfg.n_rate + cfg.n_spiking
    line = {"metric": METRIC, "value": r["value"], "unit": "neuron-steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": n * BATCH / r["value"] * 1000.0, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded whole_fly_config5)",
            "config": {**arm_config(args.gpus), "sample": f"{batch} flies per timed step; ms_per_step is a "
                                                         f"{BATCH}-fly step at the sampled rate"},
            "impl": "reference", "cpu_baseline": r,
            "e2e": {"value": r["value"], "unit": "neuron-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="flyb200", choices=["flyb200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
    eng.lif.check()
    if rank != 0:
        return
    roof = kernel_roofline(eng)
    peaks = load_peaks()
    lif_gbs = roof["lif_bytes"] / (roof["lif_ms"] / 1000.0) / 1e9
    opt_gbs = roof["optic_bytes"] / (roof["optic_ms"] / 1000.0) / 1e9
    dom = "lif" if roof["lif_ms"] >= roof["optic_ms"] else "optic"
    achieved = lif_gbs if dom == "lif" else opt_gbs
    # the whole-fly configuration at 256 flies (its uneven-rollout variant runs through BatchSim)
    n256 = min(args.steps, 40)
    eng256, g256, c256, r256, onset256 = measure_batched(cfg, device, n256, args.warmup, fly0=0, batch=256)
    ev256 = eng256.lif.synaptic_events
    ms256 = time_graph(g256, r256) / (c256 * r256)
    batch256 = {"value": N * 256 / (ms256 / 1000.0), "ms_per_step": ms256, "steps": c256 * r256,
                "synaptic_events_per_step": (eng256.lif.synaptic_events - ev256) / (c256 * r256),
                "onset": {k: onset256[k] for k in ("value", "ms_per_step", "synaptic_events_per_step")},
                "autotune": {k: {kk: vv for kk, vv in v.items() if kk != "all"} for k, v in eng256.tuned.items()}}
    del g256, eng256
    torch.cuda.empty_cache()
    plain_eng, plain_ms = measure_plain(cfg, device, args.steps, args.warmup)
    batch1 = N / (plain_ms / 1000.0)
    adj = measure_adjoint(device)
    tracer = measure_tracer(device, cpu=not args.no_cpu_baseline)
    e2e = measure_e2e(cfg, eng, device, args.steps)
    traffic = read_traffic().get(dom)
    l2 = measure_l2_gather(device)
    o = cfg.optic
    optic_l2_bytes = int(o.W0.nnz) * BATCH * 4 + roof["optic_bytes"]     # dr gathers + the streamed bytes
    cpu = None
    if not args.no_cpu_baseline:
        cpu = cpu_port_rate(cfg, 8, 3, os.cpu_count() or 1)
    line = {
        "metric": METRIC, "value": value, "unit": "neuron-steps/s", "n_gpus": world, "steps": timed_steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms / timed_steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded whole_fly_config5)",
        "config": arm_config(world),
        "batch1": {"value": batch1, "ms_per_step": plain_ms, "l2": "flushed between timed steps",
                   "launches": "one launch per kernel per step"},
        "batched_over_plain": value / world / batch1,
        "batch256": batch256,
        "adjoint": adj,
        "tracer": tracer,
        "synaptic_events_per_s": events_per_step * world * timed_steps / (ms / 1000.0),
        "synaptic_events_per_step": events_per_step,
        "state": f"steady firing after {SETTLE_STEPS} settling steps (mean rate {float(eng.lif.rate.mean()):.0f} Hz)",
        "onset": onset,
        "roofline": {"bound": "hbm", "kernel": f"{dom} step (B=64)", "achieved": achieved, "peak": peaks["hbm_gbs"],
                     "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                     "peak_source": peaks["source"], "lif_gbs": lif_gbs, "optic_gbs": opt_gbs,
                     "lif_ms": roof["lif_ms"], "optic_ms": roof["optic_ms"], "lif_bytes": roof["lif_bytes"],
                     "optic_bytes": roof["optic_bytes"],
                     "l2_gather": {"kernel": "optic step (B=64)", "bytes": optic_l2_bytes,
                                   "achieved_tbs": optic_l2_bytes / (roof["optic_ms"] / 1000.0) / 1e12,
                                   "peak_tbs": l2["tbs"],
                                   "frac": optic_l2_bytes / (roof["optic_ms"] / 1000.0) / 1e12 / l2["tbs"],
                                   "peak_source": "flyb_gather_probe, measured in this run",
                                   "note": "the optic substep gathers nnz x 64 x 4 B of L2-resident dr"}},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "autotune": {k: {kk: vv for kk, vv in v.items()} for k, v in eng.tuned.items()},
        "gpu_launches": eng.launches(chunk) * reps,
        "clocks": clocks,
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
