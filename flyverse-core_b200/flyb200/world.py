"""The fly's visual world: a spectral ray-traced room (the scene side of flyverse/world.py).

Light is carried in four channels [UV, B, G, R]. Geometry is spheres/ellipsoids, axis-aligned boxes
and planes, lit by one point light (hard shadows) and ambient light, with procedural patterns and
value-noise surface detail. Units are metres; world frame x forward, y left, z up.

`World` keeps the reference's scene description (dataclasses, `MATERIALS`, `make_room`) and its
calls (`trace`, `render_camera`, `move_sphere`, `invalidate`); tracing is one launch of the native
kernel `flyb_trace` over a packed scene that lives on the device. Packing happens on the host in
float32 exactly as the reference builds its scene tensors, so both trace the same numbers.
`flyb200.batch_world.BatchWorld` traces one scene per fly and the eye's columns in the same launch.
"""
from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _abi

INF = 1e9


@dataclass
class Material:
    name: str
    refl: tuple            # (UV, B, G, R) reflectance
    emit: tuple = (0, 0, 0, 0)
    pattern: int = 0       # 0 plain, 1 checks (refl2 the second colour), 2 wall stripes, 3 floor planks
    refl2: tuple = (0, 0, 0, 0)
    scale: float = 0.1     # pattern period (m)


# The room's materials (world.py:55-71): scene data, kept identical so that the same room gives the
# same radiance on both sides.
MATERIALS = {
    "wall": Material("wall", (0.45, 0.92, 0.95, 0.95), pattern=2, refl2=(0.20, 0.45, 0.50, 0.55), scale=0.5),
    "floor": Material("floor", (0.04, 0.10, 0.16, 0.24), pattern=3, refl2=(0.02, 0.05, 0.09, 0.14), scale=0.15),
    "ceiling": Material("ceiling", (0.40, 0.90, 0.90, 0.90)),
    "table": Material("table", (0.04, 0.10, 0.18, 0.30)),
    "cloth": Material("cloth", (0.50, 0.95, 0.95, 0.95), pattern=1, refl2=(0.05, 0.08, 0.15, 0.85), scale=0.03),
    "apple": Material("apple", (0.05, 0.08, 0.20, 0.85)),
    "banana": Material("banana", (0.10, 0.10, 0.85, 0.90)),
    "orange": Material("orange", (0.05, 0.05, 0.50, 0.95)),
    "grape": Material("grape", (0.30, 0.40, 0.15, 0.30)),
    "lime": Material("lime", (0.15, 0.20, 0.80, 0.30)),
    "blueberry": Material("blueberry", (0.55, 0.70, 0.20, 0.20)),
    "plate": Material("plate", (0.60, 0.95, 0.95, 0.95)),
    "lamp": Material("lamp", (0, 0, 0, 0), emit=(0.6, 1.0, 1.0, 1.0)),
    "black": Material("black", (0.01, 0.02, 0.02, 0.02)),
}


@dataclass
class Sphere:
    center: tuple
    radii: tuple          # (rx, ry, rz): an ellipsoid
    material: str


@dataclass
class Box:
    lo: tuple
    hi: tuple
    material: str


@dataclass
class Plane:
    point: tuple
    normal: tuple
    material: str


MAT_FLOATS, LIGHT_FLOATS = 16, 12


def scene_floats(n_sph: int, n_box: int, n_pln: int) -> int:
    n = _abi.lib().flyb_trace_scene_floats(n_sph, n_box, n_pln)
    if n < 0:
        raise ValueError("a scene holds at most 512 primitives")
    return n


def pack_scene(w) -> np.ndarray:
    """One scene as the kernel's float32 record (layout in include/flyb200.h, flyb_trace_args).
    Plane normals are normalised with torch on the CPU in float32, as the reference packs them
    (world.py:146-147), so both sides trace the same normal bits."""
    objs = list(w.spheres) + list(w.boxes) + list(w.planes)
    mats = [MATERIALS[o.material] for o in objs]
    for m in mats:
        if min(m.refl + m.refl2 + m.emit) < 0 or not m.scale > 0:
            raise ValueError(f"material {m.name}: reflectance and emission must be >= 0, the pattern period > 0")
    if min(tuple(w.light_color) + tuple(w.ambient)) < 0 or not w.detail >= 0:
        raise ValueError("light colour, ambient and detail must be >= 0")

    def f32(rows, width):
        return torch.tensor(rows, dtype=torch.float32).reshape(-1, width) if rows else torch.zeros(0, width)

    sph = torch.cat([f32([s.center for s in w.spheres], 3), f32([s.radii for s in w.spheres], 3)], 1)
    box = torch.cat([f32([b.lo for b in w.boxes], 3), f32([b.hi for b in w.boxes], 3)], 1)
    pn = f32([p.normal for p in w.planes], 3)
    pn = pn / pn.norm(dim=-1, keepdim=True).clamp_min(1e-9)
    pln = torch.cat([f32([p.point for p in w.planes], 3), pn], 1)
    mat = torch.zeros(len(objs) + 1, MAT_FLOATS)
    for i, m in enumerate(mats):
        mat[i, 0:4] = torch.tensor(m.refl, dtype=torch.float32)
        mat[i, 4:8] = torch.tensor(m.refl2, dtype=torch.float32)
        mat[i, 8:12] = torch.tensor(m.emit, dtype=torch.float32)
        mat[i, 12], mat[i, 13] = m.scale, float(m.pattern)
    mat[len(objs), 12] = 1.0
    light = torch.zeros(LIGHT_FLOATS)
    light[0:3] = torch.tensor(w.light_pos, dtype=torch.float32)
    light[3:7] = torch.tensor(w.light_color, dtype=torch.float32)
    light[7:11] = torch.tensor(w.ambient, dtype=torch.float32)
    out = torch.cat([sph.ravel(), box.ravel(), pln.ravel(), mat.ravel(), light]).numpy()
    assert out.size == scene_floats(len(w.spheres), len(w.boxes), len(w.planes))
    return out


def launch_trace(scene: torch.Tensor, shape: tuple, detail: float, out: torch.Tensor, *, origins: torch.Tensor,
                 dirs: torch.Tensor | None = None, eye_dirs: torch.Tensor | None = None,
                 pose: torch.Tensor | None = None, weights: torch.Tensor | None = None, shared_origin: bool = False,
                 rays: int, batch: int) -> None:
    """One flyb_trace launch on the current stream (arguments as in include/flyb200.h)."""
    if rays == 0:
        return
    tensors = [t for t in (scene, origins, dirs, eye_dirs, pose, weights, out) if t is not None]
    for t in tensors:
        if t.device != out.device or t.device.type != "cuda" or not t.is_contiguous():
            raise ValueError("the ray tracer takes contiguous tensors on one CUDA device")
    if out.data_ptr() % 16:
        raise ValueError("the radiance output must start on a 16-byte boundary")
    a = _abi.TraceArgs(batch=batch, rays=rays, n_sph=shape[0], n_box=shape[1], n_pln=shape[2],
                       shared_origin=int(shared_origin), samples=1 if weights is None else weights.numel(),
                       detail=float(detail), scene=_abi.ptr(scene), origins=_abi.ptr(origins), dirs=_abi.ptr(dirs),
                       eye_dirs=_abi.ptr(eye_dirs), pose=_abi.ptr(pose), weights=_abi.ptr(weights), out=_abi.ptr(out))
    with torch.cuda.device(out.device):
        rc = _abi.lib().flyb_trace(ct.byref(a), torch.cuda.current_stream(out.device).cuda_stream)
    if rc:
        raise RuntimeError(f"flyb_trace: error {rc}")


def _device(device) -> torch.device:
    d = torch.device(device if device is not None else "cuda")
    if d.type == "cuda" and d.index is None:
        d = torch.device("cuda", torch.cuda.current_device())
    return d


@dataclass
class World:
    spheres: list = field(default_factory=list)
    boxes: list = field(default_factory=list)
    planes: list = field(default_factory=list)
    light_pos: tuple = (0.0, 0.0, 2.3)
    light_color: tuple = (0.9, 1.8, 1.8, 1.8)     # UV, B, G, R power
    ambient: tuple = (0.12, 0.15, 0.15, 0.15)
    detail: float = 1.4                           # amplitude of the multi-scale surface noise (0: flat)
    device: object = "cuda"

    # ------------------------------------------------------------------ scene edits
    def move_sphere(self, idx: int, center, radii=None) -> None:
        """Move/resize sphere `idx` in place in the packed scene: no repack, and work already
        queued or captured keeps reading the same scene buffer."""
        s = self.spheres[idx]
        s.center = tuple(float(v) for v in center)
        if radii is not None:
            s.radii = tuple(float(v) for v in radii)
        if getattr(self, "_packed", False) and self._scene_shape == self._shape():
            self._scene[0, 6 * idx:6 * idx + 3].copy_(torch.tensor(s.center, dtype=torch.float32))
            if radii is not None:
                self._scene[0, 6 * idx + 3:6 * idx + 6].copy_(torch.tensor(s.radii, dtype=torch.float32))

    def invalidate(self) -> None:
        """Repack on the next trace after direct edits to geometry, materials or lighting."""
        self._packed = False

    def _shape(self) -> tuple:
        return len(self.spheres), len(self.boxes), len(self.planes)

    def _pack(self, device: torch.device) -> None:
        self._scene = torch.from_numpy(pack_scene(self))[None].to(device)
        self._scene_shape = self._shape()
        self._packed = True

    def _ready(self) -> torch.device:
        device = _device(self.device)
        if device.type != "cuda":
            raise ValueError("the ray tracer runs on a CUDA device")
        if not getattr(self, "_packed", False) or self._scene.device != device or self._scene_shape != self._shape():
            self._pack(device)
        return device

    # ------------------------------------------------------------------ tracing
    @torch.no_grad()
    def trace(self, origins, dirs, *, cuda_graphs: bool = False) -> torch.Tensor:
        """Radiance (M, 4) of rays from origins (M, 3) along unit dirs (M, 3) (world.py:214-262).
        The trace is a single launch, so there is nothing for `cuda_graphs` to capture; it is
        accepted for the reference's signature and, as there, needs a CUDA device. The result owns
        its storage."""
        if cuda_graphs and _device(self.device).type != "cuda":
            raise ValueError("ray-tracing CUDA graphs require a CUDA device")
        device = self._ready()
        o = torch.as_tensor(origins).to(device, torch.float32).contiguous()
        d = torch.as_tensor(dirs).to(device, torch.float32).contiguous()
        if o.shape != d.shape or o.ndim != 2 or o.shape[1] != 3:
            raise ValueError("rays must be (M, 3) origins and directions")
        out = torch.empty(o.shape[0], 4, dtype=torch.float32, device=device)
        launch_trace(self._scene, self._scene_shape, self.detail, out, origins=o, dirs=d, rays=o.shape[0], batch=1)
        return out

    @torch.no_grad()
    def render_camera(self, pos, forward, up, width=320, height=200, fov_deg=90.0) -> torch.Tensor:
        """Pinhole render -> (height, width, 4) radiance (world.py:302-318)."""
        device = self._ready()
        pos = torch.tensor(pos, dtype=torch.float32, device=device)
        f = torch.tensor(forward, dtype=torch.float32, device=device)
        f = f / f.norm()
        u = torch.tensor(up, dtype=torch.float32, device=device)
        r = torch.cross(f, u, dim=0)
        r = r / r.norm()
        u = torch.cross(r, f, dim=0)
        aspect = width / height
        tan = np.tan(np.deg2rad(fov_deg) / 2)
        xs = torch.linspace(-tan * aspect, tan * aspect, width, device=device)
        ys = torch.linspace(tan, -tan, height, device=device)
        gy, gx = torch.meshgrid(ys, xs, indexing="ij")
        d = f[None, None] + gx[..., None] * (-r)[None, None] + gy[..., None] * u[None, None]
        d = (d / d.norm(dim=-1, keepdim=True)).reshape(-1, 3)
        return self.trace(pos[None].expand_as(d), d).reshape(height, width, 4)


def make_room(seed: int = 0, fruit_set: str = "all") -> tuple[World, dict]:
    """A 4 x 4 x 2.6 m room with a table and fruit on it (world.py:321-362). Returns (world, info)."""
    w = World()
    w.planes += [Plane((0, 0, 0), (0, 0, 1), "floor"), Plane((0, 0, 2.6), (0, 0, -1), "ceiling"),
                 Plane((2, 0, 0), (-1, 0, 0), "wall"), Plane((-2, 0, 0), (1, 0, 0), "wall"),
                 Plane((0, 2, 0), (0, -1, 0), "wall"), Plane((0, -2, 0), (0, 1, 0), "wall")]
    # landmarks: a dark picture, a bright door, a black skirting strip
    w.boxes.append(Box((-0.6, 1.99, 1.0), (0.2, 2.0, 1.6), "black"))
    w.boxes.append(Box((1.99, -1.3, 0.0), (2.0, -0.5, 2.0), "plate"))
    w.boxes.append(Box((-2.0, -2.0, 0.0), (2.0, -1.99, 0.08), "black"))
    top = 0.75
    w.boxes.append(Box((-0.6, -0.4, top - 0.03), (0.6, 0.4, top), "cloth"))
    legs = [(sx, sy) for sx in (-0.55, 0.55) for sy in (-0.35, 0.35)]
    for sx, sy in legs:
        w.boxes.append(Box((sx - 0.025, sy - 0.025, 0), (sx + 0.025, sy + 0.025, top - 0.03), "table"))
    fruit = [Sphere((0.25, 0.15, top + 0.04), (0.04, 0.04, 0.04), "apple"),
             Sphere((-0.20, -0.10, top + 0.035), (0.035, 0.035, 0.035), "orange"),
             Sphere((0.05, -0.22, top + 0.02), (0.09, 0.02, 0.02), "banana"),
             Sphere((-0.30, 0.20, top + 0.025), (0.025, 0.025, 0.025), "lime")]
    rng = np.random.default_rng(seed)
    for k in range(9):                                   # a bunch of grapes
        fruit.append(Sphere((0.35 + 0.02 * rng.normal(), -0.05 + 0.015 * (k % 3) + 0.01 * rng.normal(),
                             top + 0.008 + 0.006 * (k // 3)), (0.008, 0.008, 0.008), "grape"))
    for _ in range(6):
        fruit.append(Sphere((-0.05 + 0.03 * rng.normal(), 0.28 + 0.03 * rng.normal(), top + 0.006),
                            (0.006, 0.006, 0.006), "blueberry"))
    if fruit_set == "apple":
        fruit = fruit[:1]
    elif fruit_set != "all":
        raise ValueError(f"unknown fruit set {fruit_set!r}")
    w.spheres += fruit
    w.spheres.append(Sphere(w.light_pos, (0.08, 0.08, 0.08), "lamp"))
    solids = [(-0.6, 0.6, -0.4, 0.4, top - 0.03, top)] + [(sx - 0.025, sx + 0.025, sy - 0.025, sy + 0.025, 0.0, top - 0.03)
                                                      for sx, sy in legs]
    info = {"table_top_z": top, "table_extent": (-0.6, 0.6, -0.4, 0.4), "room": (-2.0, 2.0, -2.0, 2.0, 0.0, 2.6),
            "solids": solids, "solid_labels": ["table"] + ["leg"] * 4,
            "fruit": [(s.material, s.center, max(s.radii)) for s in fruit]}
    return w, info
