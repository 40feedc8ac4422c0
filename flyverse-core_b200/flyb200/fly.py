"""The frame loop around the brain step: the drop-in for the brain-step part of flyverse/fly.py.

`FlyBrain` holds a batched `Brain` and, when the connectome has an eye, an `OpticLobe`, and
advances them frame by frame exactly as flyverse/fly.py:448-610 does: fractional milliseconds carry
over, the optic frame runs once per frame on the held radiance and writes the LIF drive, pulses
from `stimulate` end on a LIF step boundary, and with `cuda_graphs=True` each distinct frame shape
(steps, ring position, Poisson on, radiance present, optic remainder) is captured once and replayed.
Captured frames advance the device step clock themselves, so replays draw fresh Poisson numbers.
Senses, motor programs and the body of the reference are outside the brain step; inputs arrive as
Poisson rates (`set_input`, `stimulate`) and radiance (`vision`), outputs as group means (`motor`).
Groups registered with `set_motor` are reduced at the end of every frame, inside the captured
graph, straight from the fly-minor rate state, and copied asynchronously into pinned host memory;
`motor()` then only waits for that copy.
"""
from __future__ import annotations

import math
from dataclasses import asdict

import numpy as np
import torch

from . import cuda as fcuda
from .brain import Brain, LIFParams
from .connectome import PHOTORECEPTOR_TYPES
from .optic import OpticLobe, OpticParams
from .retina import build_retina
from .weights import receptor_gain


class PoissonSchedule:
    """The Poisson forcing of a FlyBrain (fly.py:312-396): held inputs, set by name and kept until
    replaced, and timed pulses. The forcing a step sees is, per (fly, neuron), the larger of the
    held probability and that of every pulse still running; a pulse of `ms` runs for whole LIF steps
    (ceil(ms / dt) of them) and ends when the clock reaches its end time (1e-9 ms tolerance).
    Probabilities per step are float32 rate x (dt / 1000), as the brain's `set_poisson`."""

    EPS_MS = 1e-9

    def __init__(self, brain: Brain):
        self.brain = brain
        self.held = torch.zeros_like(brain.poisson_p)       # (B, N)
        self.held_on: dict[str, bool] = {}                  # input name -> any positive rate
        self.pulses: list = []                              # [rows (k,), rates (B, k) Hz float32, end ms]

    def per_step(self, hz) -> torch.Tensor:
        return torch.as_tensor(hz, dtype=torch.float32, device=self.brain.device) * (self.brain.p.dt / 1000)

    def hold(self, name: str, idx, hz) -> None:
        cols = self.brain._idx(idx)
        prob = self.per_step(np.asarray(hz, dtype=np.float32))
        self.held[:, cols] = prob
        self.held_on[name] = bool(np.any(np.asarray(hz) > 0))
        if self.pulses:
            self.apply()
            return
        self.brain.poisson_p[:, cols] = prob          # no pulse can sit above the held rates
        self.brain._poisson_on = any(self.held_on.values())

    def add_pulse(self, rows: np.ndarray, hz: np.ndarray, end_ms: float) -> None:
        self.pulses.append((rows.copy(), hz, end_ms))
        self.apply()

    def next_end(self) -> float | None:
        return min(end for _, _, end in self.pulses) if self.pulses else None

    def ends_before(self, t_ms: float) -> bool:
        return any(end < t_ms - self.EPS_MS for _, _, end in self.pulses)

    def apply(self) -> None:
        """Write held and running pulses into the brain's forcing at the brain's current time."""
        now = self.brain.t
        self.pulses = [pl for pl in self.pulses if pl[2] > now + self.EPS_MS]
        forcing = self.brain.poisson_p
        forcing.copy_(self.held)
        for rows, hz, _ in self.pulses:
            cols = self.brain._idx(rows)
            forcing[:, cols] = torch.maximum(forcing[:, cols], self.per_step(hz))
        self.brain._poisson_on = any(self.held_on.values()) or any(bool((hz > 0).any()) for _, hz, _ in self.pulses)

    def clear(self, rows=None) -> None:
        """Forget the held inputs and pulses of fly rows `rows` (all flies, and the input names,
        when None); the forcing itself is rewritten by the next `apply`."""
        if rows is None:
            self.held.zero_()
            self.held_on.clear()
            self.pulses.clear()
            return
        self.held[self.brain._idx(rows)] = 0
        for _, hz, _ in self.pulses:
            hz[rows] = 0


class FlyBrain:
    BRAIN_TENSORS = ("v", "g", "refrac", "drive", "poisson_p", "rate", "spikes", "spike_counts", "adapt", "res")
    OPTIC_TENSORS = ("v", "adapt", "I_lp", "I_mean", "contrast", "delta_rate", "g_slow", "g_slow_cls", "_slow_in_s",
                     "stream_adapt_state")

    # reference constructor arguments for parts outside the brain step: accepted at these defaults
    OUTSIDE_THE_BRAIN = {"modules": None, "eye_geometry": None, "nt_source": None, "dataset": None, "optic": "auto",
                         "preset": "raw", "instruments": None}

    def __init__(self, c, *, batch: int = 1, device=None, seed: int = 0, lif_params: LIFParams | None = None,
                 optic_params: OpticParams | None = None, cuda_graphs: bool = False, retina=None,
                 launch: str = "persistent", receptor=None, cuda_kernels=None, cuda_sparse: str = "torch",
                 cuda_compact: bool = True, **outside):
        """The reference's constructor (fly.py:41-44): `cuda_kernels`, `cuda_sparse` and
        `cuda_compact` reach the Brain with the reference's meaning; modules, instruments, presets,
        NT sources and eye geometry are parts outside the brain step, accepted at their defaults."""
        for name, value in outside.items():
            if name not in self.OUTSIDE_THE_BRAIN:
                raise TypeError(f"FlyBrain got an unexpected keyword argument {name!r}")
            if value is not self.OUTSIDE_THE_BRAIN[name] and value != self.OUTSIDE_THE_BRAIN[name]:
                raise ValueError(f"FlyBrain argument {name}={value!r} is outside the brain step flyb200 provides "
                                 f"(only {self.OUTSIDE_THE_BRAIN[name]!r} is accepted)")
        if c is None:
            raise ValueError("FlyBrain needs the connectome `c` (connectome.load(cache_dir)); the dataset is not bundled")
        if c.n == 0:
            raise ValueError("FlyBrain needs at least one neuron")
        self.c = c
        lp = lif_params or LIFParams()
        self.brain = Brain(c, lp, device=device, seed=seed, batch=batch, launch=launch, receptor=receptor,
                           cuda_kernels=cuda_kernels, cuda_sparse=cuda_sparse, cuda_compact=cuda_compact)
        self.B, self.device = self.brain.B, self.brain.device
        self.brain.record_activity = True
        self.cuda_graphs = bool(cuda_graphs)
        self._graphs = {}
        self.retina = self.optic = None
        has_eye = "hex1" in c.neurons and bool(c.neurons.type.isin(PHOTORECEPTOR_TYPES).any()) and \
            bool((c.neurons.superclass == "ol_intrinsic").any())
        if retina is not None or has_eye:
            self.retina = retina if retina is not None else build_retina(c)
            if self.retina.n_columns:
                self.optic = OpticLobe(c, self.retina, optic_params, device=self.device, batch=self.B,
                                       receptor=receptor, receptor_gain=receptor_gain(lp), slow=self.brain.slow,
                                       launch=launch)
                self.optic.relax()
                self.brain.freeze(self.optic.rate_idx)
                if lp.prune_frozen:
                    self.brain.prune(self.optic.rate_idx)
        if lp.dt_by_module:             # per-module clocks (fly.py:98-107)
            from .regions import clock_periods
            self.brain.set_clocks(clock_periods(c, lp.dt, lp.dt_by_module))
        self._radiance = None
        self._pending_ms = 0.0
        self.poisson = PoissonSchedule(self.brain)
        self._activity_ms = np.zeros(self.B)
        self._motor = None                # (names, ptr, idx, device means, pinned means, event)
        self._motor_fresh = False
        # parity runs: uniform_source(n) -> (n, B, N) Poisson uniforms for the next n LIF steps (the
        # reference generator's draws, in the order it made them); frames then run eagerly
        self.uniform_source = None

    @property
    def t(self) -> float:
        return self.brain.t

    # ------------------------------------------------------------------ inputs
    def vision(self, radiance) -> None:
        """Hold a radiance frame [UV, B, G, R] until the next call: (columns, 4), the same for every
        fly, or (B, columns, 4); values must be finite and nonnegative (fly.py:298-309)."""
        if self.optic is None:
            raise ValueError("this connectome subset has no eye: vision is unavailable")
        cols = self.retina.n_columns
        frame = torch.as_tensor(radiance, dtype=torch.float32, device=self.device)
        if tuple(frame.shape) == (cols, 4):
            frame = frame.expand(self.B, cols, 4)
        elif tuple(frame.shape) != (self.B, cols, 4):
            raise ValueError(f"radiance of shape {tuple(frame.shape)}: expected ({self.B}, {cols}, 4) or ({cols}, 4)")
        if bool((~torch.isfinite(frame) | (frame < 0)).any()):
            raise ValueError("radiance values must be finite and nonnegative")
        if self._radiance is None:
            self._radiance = frame.clone()
        else:
            self._radiance.copy_(frame)

    def look(self, world, eye, forward, left, up) -> None:
        """Trace every fly's eye in its own scene of `world` (a BatchWorld, one scene per fly) from
        eye positions (B, 3) and orientations forward/left/up (B, 3 each), and hold the column
        radiance as `vision` does; the radiance stays on the device (one trace launch)."""
        if self.optic is None:
            raise ValueError("vision is absent from this connectome subset")
        if getattr(world, "B", None) != self.B:
            raise ValueError("the world must hold one scene per fly")
        if world._eye is None or world._eye[2] != self.retina.n_columns:
            world.set_eye(*self.retina.ray_directions())
        if self._radiance is None:
            self._radiance = torch.zeros(self.B, self.retina.n_columns, 4, device=self.device)
        world.column_radiance(eye, forward, left, up, out=self._radiance)

    def set_input(self, name: str, idx, hz) -> None:
        """Hold a named sensory Poisson input: rates `hz` (Hz; scalar, per neuron or (B, k)) on
        neurons `idx` until the input is set again (the reference's `_input`, fly.py:312-324)."""
        self.poisson.hold(name, idx, hz)

    def stimulate(self, selection, hz, ms) -> None:
        """A Poisson pulse of `hz` on the selected neurons for `ms` (rounded up to whole LIF steps),
        combined with the held inputs by maximum (fly.py:375-385)."""
        if not (math.isfinite(ms) and ms > 0):
            raise ValueError(f"a pulse lasts a positive finite time, not {ms} ms")
        rows = self.c.indices(selection)
        rates = np.array(np.broadcast_to(np.asarray(hz, dtype=np.float32), (self.B, len(rows))))
        dt = self.brain.p.dt
        if not np.isfinite(rates).all() or rates.min(initial=0.0) < 0 or (rates * dt).max(initial=0.0) > 1000:
            raise ValueError(f"pulse rates must be finite, in [0, {1000 / dt:g}] Hz")
        self.poisson.add_pulse(rows, rates, self.t + math.ceil(ms / dt) * dt)

    def _refresh_poisson(self) -> None:
        self.poisson.apply()

    # ------------------------------------------------------------------ stepping (fly.py:398-610)
    def step(self, ms: float = 10.0) -> float:
        """Advance a frame; fractional LIF steps carry over. Returns the simulated ms."""
        if not math.isfinite(ms) or ms < 0:
            raise ValueError("ms must be finite and nonnegative")
        total = self._pending_ms + ms
        steps = int(math.floor((total + 1e-9) / self.brain.p.dt))
        elapsed = steps * self.brain.p.dt
        self._pending_ms = max(0.0, total - elapsed)
        if not steps:
            return 0.0
        if self.cuda_graphs and self.uniform_source is None and not self.poisson.ends_before(self.t + elapsed):
            self._graph_frame(steps)
            self._mark_readout()
            if self.poisson.pulses:
                self.poisson.apply()
            self._activity_ms += elapsed
            return elapsed
        self._vision_frame(elapsed)
        remaining = steps
        while remaining:
            count = remaining
            end = self.poisson.next_end()
            if end is not None:            # stop at the next pulse end (a LIF step boundary)
                count = min(count, max(1, int(round((end - self.t) / self.brain.p.dt))))
            self.brain.step(count, uniforms=self._uniforms(count))
            remaining -= count
            if self.poisson.pulses:
                self.poisson.apply()
        self._readout()
        self._mark_readout()
        self._activity_ms += elapsed
        return elapsed

    def _uniforms(self, n: int):
        if self.uniform_source is None:
            return None
        return self.uniform_source(n)

    def _vision_frame(self, elapsed: float) -> None:
        if self.optic is not None and self._radiance is not None:
            self.optic.step_frame(self._radiance, self.brain.rate, elapsed, out=self.brain._st["drive"])

    def _frame(self, steps: int) -> None:
        self._vision_frame(steps * self.brain.p.dt)
        self.brain.step(steps)
        self._readout()

    def _graph_frame(self, steps: int) -> None:
        b, o = self.brain, self.optic
        if getattr(self, "_graph_weights_version", None) != b._weights_version:
            self._graphs.clear()
            self._graph_weights_version = b._weights_version
        pending = o._pending_ms if o is not None else 0.0
        key = (steps, b.buf_pos, b._poisson_on, b.record_activity, self._radiance is not None, round(pending, 9))
        if key not in self._graphs:
            if len(self._graphs) >= 8:
                self._frame(steps)
                return
            stream = torch.cuda.Stream(device=self.device)
            stream.wait_stream(torch.cuda.current_stream(self.device))
            graph = torch.cuda.CUDAGraph()
            scalars = b.t, b.step_count, b.buf_pos
            with torch.cuda.stream(stream):
                with torch.cuda.graph(graph, stream=stream):
                    self._frame(steps)            # recorded, not run: the device clock is untouched
            torch.cuda.current_stream(self.device).wait_stream(stream)
            b.t, b.step_count, b.buf_pos = scalars
            if o is not None:
                o._pending_ms = pending
            self._graphs[key] = graph
        self._graphs[key].replay()
        b.t += steps * b.p.dt
        b.step_count += steps
        b.buf_pos = (b.buf_pos + steps) % b.R
        if o is not None and self._radiance is not None:
            total = pending + steps * b.p.dt
            o._pending_ms = max(0.0, total - int(math.floor((total + 1e-9) / o.p.dt_ms)) * o.p.dt_ms)

    # ------------------------------------------------------------------ outputs
    def _group_table(self, groups: dict):
        names = list(groups)
        idx = [np.asarray(groups[k], np.int64).ravel() for k in names]
        for i in idx:
            if len(i) and (i.min() < 0 or i.max() >= self.brain.n):
                raise IndexError("motor group index out of range")
        ptr = torch.tensor(np.r_[0, np.cumsum([len(i) for i in idx])], dtype=torch.int32, device=self.device)
        flat = torch.tensor(np.concatenate(idx) if idx else np.zeros(0, np.int64), dtype=torch.int32, device=self.device)
        return names, ptr, flat

    def _launch_means(self, ptr, flat, out) -> None:
        fcuda.group_means_native(ptr, flat, self.brain._st["rate"], out)

    def set_motor(self, groups: dict | None) -> None:
        """Register the motor groups that every frame reads out (None to stop): {name: neuron
        indices}. The group means are reduced on the device at the end of each frame, inside the
        captured graph, and copied without a synchronisation into pinned host memory."""
        self._graphs.clear()                    # captured frames hold the previous readout buffers
        self._motor, self._motor_fresh = None, False
        if not groups:
            return
        names, ptr, flat = self._group_table(groups)
        out = torch.zeros(self.B, len(names), dtype=torch.float64, device=self.device)
        host = torch.zeros(self.B, len(names), dtype=torch.float64, pin_memory=True)
        self._motor = (names, ptr, flat, out, host, torch.cuda.Event())
        self._motor_groups = {k: np.asarray(groups[k], np.int64).ravel().copy() for k in names}

    def _readout(self) -> None:
        """Queue the registered readout on the current stream (recorded when a frame is captured)."""
        if self._motor is not None:
            _, ptr, flat, out, host, _ = self._motor
            self._launch_means(ptr, flat, out)
            host.copy_(out, non_blocking=True)

    def _mark_readout(self) -> None:
        if self._motor is not None:
            self._motor[5].record(torch.cuda.current_stream(self.device))
            self._motor_fresh = True

    def _same_groups(self, groups: dict) -> bool:
        held = getattr(self, "_motor_groups", None)
        return held is not None and list(groups) == list(held) and \
            all(np.array_equal(np.asarray(groups[k], np.int64).ravel(), held[k]) for k in held)

    def motor(self, groups: dict | None = None) -> dict:
        """{name: (B,) mean rate in Hz} of named neuron groups (the native motor readout,
        flyverse/motor.py:232-270). With no argument, or the groups given to `set_motor`, the means
        of the last frame come from the frame's own readout; other groups cost one reduction and
        one synchronising copy."""
        if self._motor is not None and (groups is None or self._same_groups(groups)):
            if not self._motor_fresh:           # no frame since registration, reset or restore
                self._readout()
                self._mark_readout()
            names, _, _, _, host, event = self._motor
            event.synchronize()
            means = host.numpy().copy()
            return {k: means[:, n] for n, k in enumerate(names)}
        if groups is None:
            raise ValueError("no motor groups registered; pass groups or call set_motor")
        names, ptr, flat = self._group_table(groups)
        out = torch.zeros(self.B, len(names), dtype=torch.float64, device=self.device)
        self._launch_means(ptr, flat, out)
        means = out.cpu().numpy()
        return {k: means[:, n] for n, k in enumerate(names)}

    def reset(self, rows=None) -> None:
        """Return flies `rows` (every fly when None) to rest: brain, optic lobe, their held inputs and
        pulses, activity time (fly.py:682-707). A full reset also restarts the clock, drops the held
        radiance and the captured frames."""
        self._motor_fresh = False
        self.brain.reset(rows)
        if self.optic is not None:
            self.optic.reset(rows)
        if rows is None:
            self._restart()
        else:
            rows = np.asarray(rows)
            self.poisson.clear(rows)
            self._activity_ms[rows] = 0.0
        self.poisson.apply()

    def _restart(self) -> None:
        self.poisson.clear()
        self._pending_ms = 0.0
        self._activity_ms[:] = 0.0
        self._graphs.clear()
        self._radiance = None
        self.brain.restart_clock()

    def state_dict(self) -> dict:
        o = self.optic
        return {"version": 1, "body_ids": self.c.neurons.bodyId.to_numpy().copy(),
                "lif_params": asdict(self.brain.p), "optic_params": asdict(o.p) if o is not None else None,
                "brain": self.brain.state_dict(),
                "optic": {k: getattr(o, k).detach().cpu().clone() for k in self.OPTIC_TENSORS} if o is not None else None,
                "optic_fresh": o._fresh_u8.cpu().clone() if o is not None else None,
                "optic_pending_ms": o._pending_ms if o is not None else 0.0,
                "radiance": self._radiance.detach().cpu().clone() if self._radiance is not None else None,
                "base_poisson": self.poisson.held.cpu().clone(), "inputs_on": dict(self.poisson.held_on),
                "pulses": [(i.copy(), h.copy(), e) for i, h, e in self.poisson.pulses], "pending_ms": self._pending_ms,
                "activity_ms": self._activity_ms.copy()}

    def load_state_dict(self, state: dict) -> None:
        if state["version"] != 1 or not np.array_equal(state["body_ids"], self.c.neurons.bodyId.to_numpy()):
            raise ValueError("state version/connectome does not match")
        if state["lif_params"] != asdict(self.brain.p):
            raise ValueError("state simulation parameters do not match")
        self._graphs.clear()
        self._motor_fresh = False
        self.brain.load_state_dict(state["brain"])
        o = self.optic
        if o is not None:
            for k in self.OPTIC_TENSORS:
                if k in state["optic"]:          # the slow tone's state is absent from older checkpoints
                    getattr(o, k).copy_(state["optic"][k].to(self.device))
            o._fresh_u8.copy_(state["optic_fresh"].to(self.device))
            o._pending_ms = state["optic_pending_ms"]
            o.r0 = o.b_vec[None].clone()
        self._radiance = state["radiance"].to(self.device).clone() if state["radiance"] is not None else None
        self.poisson.held.copy_(state["base_poisson"].to(self.device))
        self.poisson.held_on = dict(state["inputs_on"])
        self.poisson.pulses = [(i.copy(), h.copy(), e) for i, h, e in state["pulses"]]
        self._pending_ms, self._activity_ms = state["pending_ms"], state["activity_ms"].copy()
