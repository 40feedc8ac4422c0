"""Batched rollouts of uneven length around one batched FlyBrain (the brain-step part of
flyverse/batch_sim.py:86-343).

Every row is an independent fly sharing the graph. `step()` runs one 10 ms frame for all rows:
the caller's stimulus (radiance and/or Poisson rates per row) goes in, or, with `world` (a
BatchWorld, one scene per fly) and `pose(frame, fb) -> (eye, forward, left, up)`, every eye is
ray traced on the device (batch_sim.py:192-201), then the frame runs through
FlyBrain (graph-captured when `cuda_graphs`), the motor groups' mean rates come out. Rows whose
episode length is used up are reset on their own (`FlyBrain.reset(rows)`, batch_sim.py:282-304)
and start a new episode of a freshly drawn length; the shared clock and Poisson streams go on.
The body and behaviour programs of the reference are not part of the brain step.
"""
from __future__ import annotations

from dataclasses import dataclass, replace

import numpy as np

from .brain import LIFParams
from .fly import FlyBrain
from .optic import OpticParams


@dataclass
class EpisodeStats:
    finished: int = 0
    frames: int = 0


# Keyword arguments of the reference's BatchSim (batch_sim.py:89-94) that configure the room, the
# body, the senses or the behaviour programs rather than the brain step: accepted at their
# reference defaults, refused by name otherwise (this package steps the brain only).
OUTSIDE_THE_BRAIN = {"seeds": None, "start": None, "sensory_cuda_graphs": None, "modules": None, "wind_speed": 0.3,
                     "wind_dir": 180.0, "fruit_set": "all", "fence": False, "program": "none", "escape_gating": False,
                     "proprioception": None, "preset": "raw", "instruments": None}


class BatchSim:
    FRAME_MS = 10.0

    def __init__(self, batch: int = 1, *, c=None, seed: int = 0, device=None, brain_dt: float = 0.5,
                 optic_dt: float = 1.0, cuda_graphs: bool = False, cuda_kernels=None, event_driven=None,
                 cuda_sparse: str = "torch", cuda_compact: bool = True, weight_dtype: str = "float32",
                 dt_by_module=None, prune_frozen: bool = True, lif_params: LIFParams | None = None,
                 optic_params: OpticParams | None = None, episode_frames=(50, 400), groups: dict | None = None,
                 stimulus=None, retina=None, world=None, pose=None, **outside):
        """The reference's brain-step arguments keep their names and meaning: `cuda_kernels`
        (only True/None: the native step is the only path), `event_driven`, `cuda_sparse`,
        `cuda_compact`, `weight_dtype`, `dt_by_module`, `prune_frozen` go into the LIF parameters
        and the Brain. Room, body, sense and program arguments are accepted at their defaults
        only (OUTSIDE_THE_BRAIN)."""
        for name, value in outside.items():
            if name not in OUTSIDE_THE_BRAIN:
                raise TypeError(f"BatchSim got an unexpected keyword argument {name!r}")
            if value != OUTSIDE_THE_BRAIN[name]:
                raise ValueError(f"BatchSim argument {name}={value!r} configures the room, body, senses or programs, "
                                 f"which flyb200 does not simulate (only its default {OUTSIDE_THE_BRAIN[name]!r} is "
                                 f"accepted)")
        if c is None:
            raise ValueError("BatchSim needs the connectome `c` (connectome.load(cache_dir)); the dataset is not "
                             "bundled")
        if cuda_kernels is False:
            raise ValueError("cuda_kernels=False asks for the torch path, which flyb200 does not have")
        if not isinstance(batch, (int, np.integer)) or batch < 1:
            raise ValueError("batch must be a positive integer")
        if not np.isfinite(brain_dt) or brain_dt <= 0 or not np.isclose(self.FRAME_MS / brain_dt,
                                                                         round(self.FRAME_MS / brain_dt), rtol=0, atol=1e-8):
            raise ValueError("brain_dt must divide the 10 ms frame")
        self.B = int(batch)
        lp = lif_params or LIFParams(dt=brain_dt)
        if lp.dt != brain_dt:
            raise ValueError("lif_params.dt must equal brain_dt")
        lp = replace(lp, event_driven=event_driven if event_driven is not None else lp.event_driven,
                     weight_dtype=weight_dtype, prune_frozen=prune_frozen,
                     dt_by_module=dt_by_module if dt_by_module is not None else lp.dt_by_module)
        op = optic_params or OpticParams(dt_ms=optic_dt)
        self.fb = FlyBrain(c, batch=self.B, device=device, seed=seed, lif_params=lp, optic_params=op,
                           cuda_graphs=cuda_graphs, retina=retina, cuda_sparse=cuda_sparse, cuda_compact=cuda_compact)
        self.rng = np.random.default_rng(seed)
        self.episode_frames = episode_frames
        self.frames_left = self._draw(self.B)
        self.groups = groups or {}
        self.fb.set_motor(self.groups or None)
        self.stimulus = stimulus
        if (world is None) != (pose is None):
            raise ValueError("a traced world needs a pose callback and vice versa")
        self.world, self.pose = world, pose
        self.stats = EpisodeStats()
        self.frame = 0

    def _draw(self, k: int) -> np.ndarray:
        lo, hi = self.episode_frames
        return self.rng.integers(lo, hi + 1, k)

    def step(self) -> dict:
        """One frame for every row; returns the motor readout and the rows that were reset."""
        if self.stimulus is not None:
            radiance, inputs = self.stimulus(self.frame, self.fb)
            if radiance is not None:
                self.fb.vision(radiance)
            for name, (idx, hz) in (inputs or {}).items():
                self.fb.set_input(name, idx, hz)
        if self.world is not None:
            self.fb.look(self.world, *self.pose(self.frame, self.fb))
        self.fb.step(self.FRAME_MS)
        out = self.fb.motor() if self.groups else {}
        self.frame += 1
        self.stats.frames += self.B
        self.frames_left -= 1
        done = np.flatnonzero(self.frames_left <= 0)
        if len(done):
            self.reset(done)
            self.stats.finished += len(done)
        out["reset_rows"] = done
        return out

    def reset(self, rows=None) -> None:
        """Reset rows (all if None) to rest with fresh episode lengths (batch_sim.py:282-304)."""
        if rows is None:
            self.fb.reset()
            self.frames_left = self._draw(self.B)
            return
        rows = np.asarray(rows)
        self.fb.reset(rows)
        self.frames_left[rows] = self._draw(len(rows))

    def save_state(self) -> dict:
        return {"fb": self.fb.state_dict(), "rng": self.rng.bit_generator.state, "frames_left": self.frames_left.copy(),
                "frame": self.frame}

    def load_state(self, state: dict) -> None:
        self.fb.load_state_dict(state["fb"])
        self.rng.bit_generator.state = state["rng"]
        self.frames_left = state["frames_left"].copy()
        self.frame = state["frame"]
