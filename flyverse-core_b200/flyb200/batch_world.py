"""Independent scenes traced together, one per fly (the scene side of flyverse/batch_world.py), and
the eye: every fly's ommatidial sample rays traced and averaged into column radiance in one launch.

All scenes of a batch have the same primitive counts; a ray of row b only sees scene b. The packed
scenes are one (B, floats) device tensor, so moving a sphere in some rows is an in-place copy and
captured frames keep reading the same buffer.
"""
from __future__ import annotations

import numpy as np
import torch

from .world import World, _device, launch_trace, pack_scene


class BatchWorld(World):
    def __init__(self, worlds, device=None):
        self.worlds = list(worlds)
        if not self.worlds:
            raise ValueError("BatchWorld needs at least one scene")
        self.B = len(self.worlds)
        self.device = _device(device if device is not None else self.worlds[0].device)
        self.detail = self.worlds[0].detail
        self._packed = False
        self._eye = None

    def _shape(self) -> tuple:
        shapes = [(len(w.spheres), len(w.boxes), len(w.planes)) for w in self.worlds]
        if any(s != shapes[0] for s in shapes):
            raise ValueError("batched scenes must have matching primitive counts")
        if any(w.detail != self.detail for w in self.worlds):
            raise ValueError("batched scenes must share the texture detail setting")
        return shapes[0]

    def _pack(self, device: torch.device) -> None:
        self._scene_shape = self._shape()
        self._scene = torch.from_numpy(np.stack([pack_scene(w) for w in self.worlds])).to(device)
        self._packed = True

    def move_sphere(self, idx, center, radii=None, *, rows=None):
        """Move/resize sphere `idx` in `rows` (all by default), in place (batch_world.py:62-75)."""
        rows = np.arange(self.B) if rows is None else np.asarray(rows, dtype=int)
        centers = np.broadcast_to(np.asarray(center, float), (len(rows), 3))
        sizes = None if radii is None else np.broadcast_to(np.asarray(radii, float), (len(rows), 3))
        if not 0 <= idx < len(self.worlds[0].spheres) or np.any((rows < 0) | (rows >= self.B)):
            raise IndexError("sphere/scene index out of range")
        for j, row in enumerate(rows):
            s = self.worlds[row].spheres[idx]
            s.center = tuple(float(v) for v in centers[j])
            if sizes is not None:
                s.radii = tuple(float(v) for v in sizes[j])
        if self._packed:
            self._scene[:, 6 * idx:6 * idx + 3].copy_(
                torch.tensor([w.spheres[idx].center for w in self.worlds], dtype=torch.float32))
            if sizes is not None:
                self._scene[:, 6 * idx + 3:6 * idx + 6].copy_(
                    torch.tensor([w.spheres[idx].radii for w in self.worlds], dtype=torch.float32))

    @torch.no_grad()
    def trace(self, origins, dirs, *, cuda_graphs: bool = False) -> torch.Tensor:
        """(B, M, 4) radiance of (B, M, 3) rays, row b in scene b (batch_world.py:77-92)."""
        if cuda_graphs and self.device.type != "cuda":
            raise ValueError("ray-tracing CUDA graphs require a CUDA device")
        o, d = torch.as_tensor(origins), torch.as_tensor(dirs)
        if o.shape != d.shape or o.ndim != 3 or o.shape[0] != self.B or o.shape[2] != 3:
            raise ValueError("batched rays must have shape (batch, rays, 3)")
        device = self._ready()
        o = o.to(device, torch.float32).contiguous()
        d = d.to(device, torch.float32).contiguous()
        out = torch.empty(self.B, o.shape[1], 4, dtype=torch.float32, device=device)
        launch_trace(self._scene, self._scene_shape, self.detail, out, origins=o, dirs=d, rays=o.shape[1],
                     batch=self.B)
        return out

    # ------------------------------------------------------------------ the eye
    def set_eye(self, directions, weights) -> None:
        """Body-frame sample rays of every column, (n_col, k, 3), and their (k,) weights
        (`Retina.ray_directions()`); kept on the device in double, as the reference turns them."""
        dirs = np.asarray(directions, dtype=np.float64)
        w = np.asarray(weights, dtype=np.float32).ravel()
        if dirs.ndim != 3 or dirs.shape[2] != 3 or dirs.shape[1] != len(w) or not 1 <= len(w) <= 256:
            raise ValueError("eye directions must be (columns, k, 3) with k weights, 1 <= k <= 256")
        device = self._ready()
        self._eye = (torch.from_numpy(np.ascontiguousarray(dirs.reshape(-1, 3))).to(device),
                     torch.from_numpy(w).to(device), dirs.shape[0])
        self._pose = torch.zeros(self.B, 9, dtype=torch.float64, device=device)
        self._eye_pos = torch.zeros(self.B, 3, dtype=torch.float32, device=device)

    def set_pose(self, eye, forward, left, up) -> None:
        """Eye positions (B, 3) and orientations forward/left/up (B, 3 each) for the next eye
        traces, copied into the device buffers that `trace_eye` (and a graph that captured it)
        reads."""
        if self._eye is None:
            raise ValueError("set_eye() first")
        pose = np.concatenate([np.asarray(v, dtype=np.float64).reshape(self.B, 3) for v in (forward, left, up)], 1)
        self._pose.copy_(torch.from_numpy(pose))
        self._eye_pos.copy_(torch.from_numpy(np.asarray(eye, dtype=np.float32).reshape(self.B, 3)))

    @torch.no_grad()
    def trace_eye(self, out: torch.Tensor | None = None) -> torch.Tensor:
        """(B, n_col, 4) radiance per column at the poses last given to `set_pose`: one launch,
        capturable in a CUDA graph."""
        if self._eye is None:
            raise ValueError("set_eye() first")
        device = self._ready()
        eye_dirs, w, n_col = self._eye
        if out is None:
            out = torch.empty(self.B, n_col, 4, dtype=torch.float32, device=device)
        elif out.shape != (self.B, n_col, 4) or out.dtype != torch.float32 or not out.is_contiguous():
            raise ValueError(f"out must be a contiguous float32 ({self.B}, {n_col}, 4) tensor")
        launch_trace(self._scene, self._scene_shape, self.detail, out, origins=self._eye_pos, eye_dirs=eye_dirs,
                     pose=self._pose, weights=w, shared_origin=True, rays=n_col * w.numel(), batch=self.B)
        return out

    def column_radiance(self, eye, forward, left, up, out: torch.Tensor | None = None) -> torch.Tensor:
        """(B, n_col, 4) radiance per column for flies at eye (B, 3) facing forward/left/up
        (B, 3 each): every sample ray d = x forward + y left + z up from the eye, traced in that
        fly's scene, weighted and summed over each column's samples in sample order
        (batch_sim.py:192-201). Writes into `out` when given (e.g. FlyBrain's held radiance)."""
        self.set_pose(eye, forward, left, up)
        return self.trace_eye(out)
