"""The photoreceptor geometry the optic lobe consumes (flyverse/retina.py:49-162, the parts on the
brain-step path): each photoreceptor's connectome row, hex column and spectral sensitivity, and each
column's viewing direction with the sample rays of its acceptance cone, which the eye's ray tracer
casts."""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .connectome import PHOTORECEPTOR_TYPES

CHANNELS = ["UV", "B", "G", "R"]
# Relative spectral sensitivity per photoreceptor class over [UV, B, G, R] (retina.py:35-46): a data
# table of the model, kept identical so photoreceptor drive matches the reference.
SENSITIVITY = {
    "R1-R6": [0.50, 0.70, 1.00, 0.05], "R7p": [1.00, 0.05, 0.00, 0.00], "R7y": [1.00, 0.15, 0.00, 0.00],
    "R7d": [1.00, 0.05, 0.00, 0.00], "R7_unclear": [1.00, 0.10, 0.00, 0.00], "R8p": [0.20, 1.00, 0.10, 0.00],
    "R8y": [0.05, 0.30, 1.00, 0.10], "R8d": [1.00, 0.05, 0.00, 0.00], "R8_unclear": [0.12, 0.65, 0.55, 0.05],
    "R7R8_unclear": [0.60, 0.40, 0.30, 0.02],
}


@dataclass
class EyeGeometry:
    """Ommatidial layout (retina.py:49-56): spacing, where each eye's centre column looks, which
    hex diagonal points forward and up, the acceptance cone and rays cast per ommatidium."""
    interommatidial_deg: float = 4.6
    eye_center_azimuth_deg: float = 55.0
    anterior_sign: float = +1.0
    dorsal_sign: float = +1.0
    acceptance_deg: float = 4.5
    rays_per_ommatidium: int = 7


@dataclass
class Retina:
    pr_index: np.ndarray        # connectome row of each photoreceptor
    pr_column: np.ndarray       # column id 0..n_col-1
    pr_sens: np.ndarray         # (n_pr, 4)
    col_side: np.ndarray        # per column
    col_hex: np.ndarray         # (n_col, 2)
    col_dir: np.ndarray | None = None     # (n_col, 3) unit view direction, body frame (x fwd, y left, z up)
    col_az_el: np.ndarray | None = None   # (n_col, 2) azimuth (deg, + left), elevation (deg, + up)
    geometry: EyeGeometry = field(default_factory=EyeGeometry)

    @property
    def n_columns(self) -> int:
        return len(self.col_side)

    def ray_directions(self) -> tuple[np.ndarray, np.ndarray]:
        """(n_col, k, 3) body-frame sample directions and (k,) weights summing to 1 (retina.py:85-99):
        the column's axis plus k - 1 rays on a ring at half the acceptance angle, weighted by a
        Gaussian of the ring radius."""
        if self.col_az_el is None:
            raise ValueError("this retina has no viewing directions")
        g = self.geometry
        k = g.rays_per_ommatidium
        if k <= 1:
            return self.col_dir[:, None, :], np.ones(1)
        half = np.deg2rad(g.acceptance_deg / 2)
        ring = np.linspace(0, 2 * np.pi, k - 1, endpoint=False)
        offsets = np.concatenate([[[0.0, 0.0]], np.c_[half * np.cos(ring), half * np.sin(ring)]])
        weights = np.exp(-0.5 * (np.hypot(offsets[:, 0], offsets[:, 1]) / half) ** 2 * 2.0)
        weights /= weights.sum()
        az = np.deg2rad(self.col_az_el[:, 0])[:, None] + offsets[None, :, 0]
        el = np.deg2rad(self.col_az_el[:, 1])[:, None] + offsets[None, :, 1]
        return np.stack([np.cos(el) * np.cos(az), np.cos(el) * np.sin(az), np.sin(el)], axis=-1), weights


def column_directions(col_side: np.ndarray, col_hex: np.ndarray, g: EyeGeometry) -> tuple[np.ndarray, np.ndarray]:
    """Viewing direction of every column (retina.py:140-160): hex (h1, h2) to a plane with 120-degree
    axes, centred per eye, scaled by the interommatidial angle; the anterior-posterior coordinate
    sets azimuth (mirrored for the right eye) and the dorsal-ventral one sets elevation."""
    X = col_hex[:, 0] - 0.5 * col_hex[:, 1]
    Y = col_hex[:, 1] * np.sqrt(3) / 2
    e_dv = 0.5 * X + (np.sqrt(3) / 2) * Y
    e_ap = (np.sqrt(3) / 2) * X - 0.5 * Y
    az, el = np.zeros(len(col_side)), np.zeros(len(col_side))
    for side in ("L", "R"):
        s = col_side == side
        if not s.any():
            continue
        ap = (e_ap[s] - e_ap[s].mean()) * g.anterior_sign * g.interommatidial_deg
        dv = (e_dv[s] - e_dv[s].mean()) * g.dorsal_sign * g.interommatidial_deg
        lateral = g.eye_center_azimuth_deg - ap
        az[s] = lateral if side == "L" else -lateral
        el[s] = dv
    azr, elr = np.deg2rad(az), np.deg2rad(el)
    col_dir = np.stack([np.cos(elr) * np.cos(azr), np.cos(elr) * np.sin(azr), np.sin(elr)], axis=-1)
    return col_dir, np.c_[az, el]


def build_retina(c, geometry: EyeGeometry | None = None) -> Retina:
    """Columns = sorted distinct (side, hex1, hex2) of the photoreceptors (retina.py:108-162); the
    FAFB release lists its whole column grid, so columns without an R-cell axon are kept there. A
    subset keeps the viewing directions of the full eye it was cut from."""
    c.require("optic_columns")
    g = geometry or EyeGeometry()
    if c.reference is not c:
        full = build_retina(c.reference, g)
        body_ids = c.reference.neurons.bodyId.to_numpy()[full.pr_index]
        keep = np.isin(body_ids, c.neurons.bodyId.to_numpy())
        columns = np.unique(full.pr_column[keep])
        col_map = np.full(full.n_columns, -1, dtype=np.int64)
        col_map[columns] = np.arange(len(columns))
        return Retina(pr_index=c.index_of(body_ids[keep]), pr_column=col_map[full.pr_column[keep]],
                      pr_sens=full.pr_sens[keep], col_side=full.col_side[columns], col_hex=full.col_hex[columns],
                      col_dir=full.col_dir[columns], col_az_el=full.col_az_el[columns], geometry=g)
    nrn = c.neurons
    m = nrn.type.isin(PHOTORECEPTOR_TYPES) & nrn.hex1.notna()
    pr = nrn[m]
    keys = list(zip(pr.hex_side, pr.hex1.astype(int), pr.hex2.astype(int)))
    uniq = sorted(set(keys))
    if c.dataset == "fafb":
        grid = nrn[nrn.hex1.notna() & nrn.hex2.notna() & nrn.hex_side.notna()]
        uniq = sorted(set(uniq) | set(zip(grid.hex_side, grid.hex1.astype(int), grid.hex2.astype(int))))
    col_of = {k: i for i, k in enumerate(uniq)}
    col_side = np.array([k[0] for k in uniq])
    col_hex = np.array([[k[1], k[2]] for k in uniq], dtype=float).reshape(-1, 2)
    col_dir, az_el = column_directions(col_side, col_hex, g)
    return Retina(pr_index=np.flatnonzero(m.to_numpy()), pr_column=np.array([col_of[k] for k in keys], dtype=np.int64),
                  pr_sens=np.array([SENSITIVITY[t] for t in pr.type], dtype=np.float32).reshape(-1, 4),
                  col_side=col_side, col_hex=col_hex, col_dir=col_dir, col_az_el=az_el, geometry=g)
