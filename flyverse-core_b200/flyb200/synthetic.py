"""Seeded synthetic stand-ins for the MaleCNS graph at the benchmark sizes.

The connectome dataset is not shipped, so every workload runs on graphs drawn here with
`numpy.random.default_rng(seed)`. Each generator states its rule; the sizes are those the
reference's headline numbers are quoted on:

  lif_config1   2,000 LIF neurons, 20,000 uniform edges, counts 1+Geom0(0.3) (numpy geometric has
                support >= 1), presynaptic sign +1 w.p. 0.7, Poisson 150 Hz on 50 neurons.
  lif_config2   71,618 LIF neurons; out-degree round(lognormal(4.9, 1.2)) truncated to N, then
                scaled by largest-remainder rounding to exactly `edges` (15,000,000; the unscaled
                draw gives ~19.7 M); distinct uniform targets; counts geometric(0.2); sign +1 w.p.
                0.6 per presynaptic cell; Poisson 100 Hz on 2,000 designated neurons.
  optic_config3 89,390 rate units; in-degree round(lognormal(4.0, 1.0)) scaled to exactly `nnz`
                (6,000,000; unscaled ~8.0 M); distinct uniform presynaptic units; |w| from counts
                geometric(0.2), signed by the presynaptic type, normalised per row to sum |w| = 1;
                700 types round-robin; 5 % of units (35 types) rectifying T4/T5-like units
                (operating point 0) whose inhibitory inputs from 35 "delayed inhibition" types
                (tau 10 ms) carry a x5 pair gain; 5,895 photoreceptors on a hex eye driven by a
                drifting sinusoidal grating in 4 spectral channels.
  batched_config4  config 2's spiking graph coupled to config 3's lobe (the 64-fly uneven-rollout tier).
  eye_grid      the eye the ray tracer casts: two hexagonal column patches of radius 16 (817
                columns each, 1,634 in all, about the ommatidia of a fly's pair of eyes) through
                the retina's own geometry, 7 sample rays per column.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import pandas as pd
import scipy.sparse as sp

from .connectome import Connectome, from_arrays

# ------------------------------------------------------------------ sampling helpers


def scale_degrees(deg: np.ndarray, target: int, cap: int) -> np.ndarray:
    """Scale integer degrees to sum exactly `target` (largest-remainder rounding), each <= cap."""
    deg = np.minimum(deg.astype(np.int64), cap)
    x = deg * (target / max(int(deg.sum()), 1))
    base = np.minimum(np.floor(x).astype(np.int64), cap)
    rem = int(target - base.sum())
    frac = np.where(base < cap, x - base, -1.0)
    order = np.argsort(-frac, kind="stable")
    base[order[:rem]] += 1
    if base.sum() != target:
        raise ValueError("cannot place the requested number of edges under the degree cap")
    return base


def distinct_targets(rng: np.random.Generator, deg: np.ndarray, n: int) -> tuple[np.ndarray, np.ndarray]:
    """(row, col) pairs with deg[r] distinct uniform columns per row r (rejection of duplicates)."""
    rows = np.repeat(np.arange(len(deg), dtype=np.int64), deg)
    cols = rng.integers(0, n, rows.size, dtype=np.int64)
    big = np.flatnonzero(deg > n // 4)
    starts = np.concatenate([[0], np.cumsum(deg)])
    for r in big:                                  # dense rows: sample a permutation prefix directly
        cols[starts[r]:starts[r + 1]] = rng.choice(n, int(deg[r]), replace=False)
    for _ in range(64):
        key = rows * n + cols
        order = np.argsort(key, kind="stable")
        ks = key[order]
        dup = np.zeros(len(ks), bool)
        dup[1:] = ks[1:] == ks[:-1]
        if not dup.any():
            break
        idx = order[dup]
        cols[idx] = rng.integers(0, n, idx.size, dtype=np.int64)
    else:
        raise RuntimeError("duplicate rejection did not converge")
    return rows, cols


def neuron_table(n: int, *, type_names=None, superclass="cb_intrinsic", nt=None, body0: int = 1) -> pd.DataFrame:
    t = pd.DataFrame({"bodyId": np.arange(body0, body0 + n, dtype=np.int64)})
    t["type"] = type_names if type_names is not None else "LIF"
    t["superclass"] = superclass
    t["nt"] = nt if nt is not None else "acetylcholine"
    t["class"] = ""
    t["somaSide"] = ""
    return t


# ------------------------------------------------------------------ LIF configs
@dataclass
class LifConfig:
    name: str
    c: Connectome
    poisson_idx: np.ndarray
    poisson_hz: float | np.ndarray
    steps: int
    batch: int = 1
    dt: float = 0.1
    # LIFParams overrides that make the weights w_syn x signed integer counts (the model of the
    # benchmark configs: no cap, no fan-in scale, no gains, no adaptation, no depression).
    params: dict = field(default_factory=lambda: dict(conn_cap=0.0, input_norm_alpha=0.0, path_gain=[],
                                                      type_path_gain=[], same_type_gain=1.0, adapt_jump=0.0,
                                                      std_u=0.0, std_u_by_type={}, adapt_by_type={},
                                                      receptor_model=None, dt=0.1))


def _lif_graph(rng, n, pre, post, p_count, p_exc) -> sp.csr_matrix:
    count = rng.geometric(p_count, pre.size).astype(np.float32)
    sign = np.where(rng.random(n) < p_exc, 1.0, -1.0).astype(np.float32)
    W = sp.csr_matrix((count * sign[pre], (post, pre)), shape=(n, n), dtype=np.float32)
    W.sum_duplicates()
    W.sort_indices()
    return W


def lif_config1(seed: int = 0, n: int = 2000, edges: int = 20_000, n_poisson: int = 50,
                poisson_hz: float = 150.0, steps: int = 1000) -> LifConfig:
    rng = np.random.default_rng(seed)
    pre = rng.integers(0, n, edges)
    post = rng.integers(0, n, edges)
    W = _lif_graph(rng, n, pre, post, 0.3, 0.7)
    pidx = np.sort(rng.choice(n, n_poisson, replace=False))
    return LifConfig("plain LIF, 2,000 neurons / 20,000 edges", from_arrays(neuron_table(n), W), pidx, poisson_hz, steps)


def lif_config2(seed: int = 0, n: int = 71_618, edges: int | None = 15_000_000, n_poisson: int = 2000,
                poisson_hz: float = 100.0, steps: int = 10_000) -> LifConfig:
    rng = np.random.default_rng(seed)
    deg = np.minimum(np.round(rng.lognormal(4.9, 1.2, n)).astype(np.int64), n)
    if edges is not None:
        deg = scale_degrees(deg, edges, n)
    pre, post = distinct_targets(rng, deg, n)
    W = _lif_graph(rng, n, pre, post, 0.2, 0.6)
    pidx = np.sort(rng.choice(n, n_poisson, replace=False))
    return LifConfig(f"full-size spiking tier, {n:,} neurons / {W.nnz:,} edges", from_arrays(neuron_table(n), W),
                     pidx, poisson_hz, steps)


# ------------------------------------------------------------------ optic config
@dataclass
class OpticConfig:
    """Matrices and constants of a synthetic optic lobe (rows are postsynaptic units)."""
    m: int
    n_types: int
    type_of: np.ndarray          # (m,) int32
    tau_of_type: np.ndarray      # (n_types,) ms
    base_of_type: np.ndarray     # (n_types,) operating point
    W0: sp.csr_matrix            # unit-gain, row-normalised signed weights (m x m)
    pair_id: np.ndarray          # (nnz,) pair index of each W0 entry (CSR order)
    pairs: np.ndarray            # (n_pairs, 2) (pre type, post type)
    gain0: np.ndarray            # (n_pairs,) default pair gains
    W_rp: sp.csr_matrix          # m x n_pr
    W_rs: sp.csr_matrix          # m x n_spk
    W_sr: sp.csr_matrix          # n_spk x m
    n_pr: int
    n_col: int
    pr_column: np.ndarray
    pr_family: np.ndarray
    sens: np.ndarray             # (n_pr, 4)
    col_xy: np.ndarray           # (n_col, 2)
    dt_ms: float = 1.0
    gain_rr: float = 1.0
    gain_in: float = 3.0
    gain_fb: float = 0.5
    adapt_tau_ms: float = 400.0
    adapt_gain: float = 1.0
    gain_out_mv: float = 100.0
    drive_clip_mv: float = 35.0

    @property
    def a(self) -> np.ndarray:
        tau = self.tau_of_type[self.type_of].astype(np.float32)
        return np.exp(-self.dt_ms / tau).astype(np.float32)

    @property
    def b(self) -> np.ndarray:
        return self.base_of_type[self.type_of].astype(np.float32)

    @property
    def aad(self) -> float:
        return float(np.exp(-self.dt_ms / self.adapt_tau_ms))

    def W_rr(self, gains: np.ndarray | None = None) -> sp.csr_matrix:
        g = self.gain0 if gains is None else gains
        W = self.W0.copy()
        W.data = (W.data * g[self.pair_id]).astype(np.float32)
        return W

    def grating(self, t_ms: float, batch: int = 1, seed: int = 0) -> np.ndarray:
        """(batch, n_col, 4) radiance of a drifting sinusoidal grating (per-fly seeded direction)."""
        rng = np.random.default_rng(seed)
        theta = rng.uniform(0, 2 * np.pi, batch)
        phase = rng.uniform(0, 2 * np.pi, (batch, 4))
        k = 2 * np.pi / 8.0                       # 8 columns per cycle
        omega = 2 * np.pi * 2.0 / 1000.0          # 2 Hz
        proj = self.col_xy[None, :, 0] * np.cos(theta)[:, None] + self.col_xy[None, :, 1] * np.sin(theta)[:, None]
        arg = k * proj[:, :, None] - omega * t_ms + phase[:, None, :]
        return (0.5 + 0.4 * np.sin(arg)).astype(np.float32)


def optic_config3(seed: int = 0, m: int = 89_390, nnz: int | None = 6_000_000, n_pr: int = 5_895,
                  n_types: int = 700, n_spk: int = 71_618) -> OpticConfig:
    rng = np.random.default_rng(seed)
    type_of = (np.arange(m) % n_types).astype(np.int32)
    n_t45 = max(1, int(round(0.05 * n_types)))
    t45 = np.arange(n_t45)                                   # rectifying motion-detector types
    delayed = np.arange(n_t45, 2 * n_t45)                    # their delayed-inhibition input types
    inhibitory = np.zeros(n_types, bool)
    inhibitory[(np.arange(n_types) % 10) < 3] = True
    inhibitory[delayed] = True
    tau_cycle = np.array([6.0, 8.0, 10.0, 40.0, 150.0])
    tau_of_type = tau_cycle[np.arange(n_types) % len(tau_cycle)].astype(np.float32)
    tau_of_type[t45] = 10.0
    tau_of_type[delayed] = 10.0
    base_of_type = np.full(n_types, 0.5, np.float32)
    base_of_type[t45] = 0.0
    # recurrent block: in-degree per postsynaptic row
    deg = np.minimum(np.round(rng.lognormal(4.0, 1.0, m)).astype(np.int64), m)
    deg = np.maximum(deg, 1)
    if nnz is not None:
        deg = scale_degrees(deg, nnz, m)
    post, pre = distinct_targets(rng, deg, m)
    cnt = rng.geometric(0.2, post.size).astype(np.float32)
    sign = np.where(inhibitory[type_of[pre]], -1.0, 1.0).astype(np.float32)
    C = sp.csr_matrix((cnt * sign, (post, pre)), shape=(m, m), dtype=np.float32)
    C.sum_duplicates()
    C.sort_indices()
    rowsum = np.asarray(abs(C).sum(axis=1)).ravel()
    W0 = (sp.diags((1.0 / np.maximum(rowsum, 1.0)).astype(np.float32)) @ C).tocsr().astype(np.float32)
    W0.sort_indices()
    rows = np.repeat(np.arange(m), np.diff(W0.indptr))
    key = type_of[W0.indices].astype(np.int64) * n_types + type_of[rows]
    uniq, pair_id = np.unique(key, return_inverse=True)
    pairs = np.stack([uniq // n_types, uniq % n_types], axis=1).astype(np.int32)
    gain0 = np.ones(len(uniq), np.float32)
    gain0[np.isin(pairs[:, 0], delayed) & np.isin(pairs[:, 1], t45)] = 5.0      # delayed inhibition arm
    gain0[np.isin(pairs[:, 0], t45)] *= 2.0                                      # T4/T5 outputs
    # photoreceptors: 6 per column on a hex patch; the first 10 % of units (lamina) read their column
    n_col = int(np.ceil(n_pr / 6))
    pr_column = (np.arange(n_pr) % n_col).astype(np.int32)
    pr_family = np.array([0, 0, 0, 0, 1, 4], np.int32)[(np.arange(n_pr) // n_col) % 6]
    fam_sens = np.array([[0.45, 0.65, 0.95, 0.05], [0.95, 0.1, 0.0, 0.0], [0.9, 0.2, 0.0, 0.0],
                         [0.2, 0.95, 0.1, 0.0], [0.05, 0.35, 0.95, 0.1]], np.float32)
    sens = fam_sens[pr_family]
    width = int(np.ceil(np.sqrt(n_col)))
    h1, h2 = np.arange(n_col) % width, np.arange(n_col) // width
    col_xy = np.stack([h1 - 0.5 * h2, h2 * np.sqrt(3) / 2], axis=1).astype(np.float64)
    lam = np.arange(max(1, m // 10))
    members = [np.flatnonzero(pr_column == (i % n_col)) for i in range(n_col)]
    rp_rows = np.concatenate([np.full(len(members[i % n_col]), i) for i in lam])
    rp_cols = np.concatenate([members[i % n_col] for i in lam])
    rp_cnt = rng.geometric(0.2, rp_rows.size).astype(np.float32)
    W_rp = sp.csr_matrix((-rp_cnt, (rp_rows, rp_cols)), shape=(m, n_pr), dtype=np.float32)
    W_rp = (sp.diags((1.0 / np.maximum(np.asarray(abs(W_rp).sum(axis=1)).ravel(), 1.0)).astype(np.float32)) @ W_rp).tocsr()
    # spiking feedback (2 % of units, 20 inputs) and visual projection drive (5 % of LIF cells, 50 inputs)
    fb_rows = rng.choice(m, max(1, m // 50), replace=False)
    r, cidx = distinct_targets(rng, np.full(len(fb_rows), 20), n_spk)
    W_rs = sp.csr_matrix((rng.geometric(0.2, r.size).astype(np.float32) / 100.0, (fb_rows[r], cidx)),
                         shape=(m, n_spk), dtype=np.float32)
    vpn = rng.choice(n_spk, max(1, n_spk // 20), replace=False)
    r, cidx = distinct_targets(rng, np.full(len(vpn), 50), m)
    W_sr = sp.csr_matrix((rng.geometric(0.2, r.size).astype(np.float32) / 250.0, (vpn[r], cidx)),
                         shape=(n_spk, m), dtype=np.float32)
    for M in (W_rp, W_rs, W_sr):
        M.sum_duplicates()
        M.sort_indices()
    return OpticConfig(m=m, n_types=n_types, type_of=type_of, tau_of_type=tau_of_type, base_of_type=base_of_type,
                       W0=W0, pair_id=pair_id.astype(np.int32), pairs=pairs, gain0=gain0, W_rp=W_rp.astype(np.float32),
                       W_rs=W_rs, W_sr=W_sr, n_pr=n_pr, n_col=n_col, pr_column=pr_column, pr_family=pr_family,
                       sens=sens, col_xy=col_xy)


# ------------------------------------------------------------------ whole fly
@dataclass
class WholeFlyConfig:
    """167,106 neurons = n_rate graded optic units + n_lif spiking + n_sensory Poisson-driven spiking.

    Edge budget (total `edges`, default 25.6 M, counts geometric(0.2) so ~128 M synapses):
      rate <- rate  W_rr  `optic_nnz` (optic_config3's rule)
      spiking <- spiking  the rest after the three coupling blocks, lognormal(4.9, 1.2) out-degree
                          over all spiking cells (sensory included), scaled to the remainder
      spiking <- rate  W_sr  visual projection drive: 5 % of spiking cells, 50 rate inputs each ... scaled
      rate <- spiking  W_rs  feedback: 2 % of rate units, 20 spiking inputs each
      rate <- photoreceptor  W_rp  lamina (first 10 % of rate units), 6 photoreceptors of its column
    The photoreceptors are the optic lobe's input stage (driven by the grating), not counted in N.
    """
    lif: LifConfig
    optic: OpticConfig
    sensory_idx: np.ndarray        # spiking-population rows of the Poisson-driven sensory cells
    vpn_idx: np.ndarray            # spiking-population rows driven by the optic lobe (W_sr rows)
    n_rate: int
    n_spiking: int
    edges: int


def whole_fly_config5(seed: int = 0, n_rate: int = 89_390, n_lif: int = 71_618, n_sensory: int = 6_098,
                      edges: int = 25_600_000, optic_nnz: int = 6_000_000, n_pr: int = 5_895) -> WholeFlyConfig:
    rng = np.random.default_rng(seed)
    n_spk = n_lif + n_sensory
    optic = optic_config3(seed=seed + 1, m=n_rate, nnz=optic_nnz, n_pr=n_pr, n_spk=n_spk)
    coupling = optic.W_rp.nnz + optic.W_rs.nnz + optic.W_sr.nnz
    lif_edges = edges - optic_nnz - coupling
    deg = np.minimum(np.round(rng.lognormal(4.9, 1.2, n_spk)).astype(np.int64), n_spk)
    deg = scale_degrees(deg, lif_edges, n_spk)
    pre, post = distinct_targets(rng, deg, n_spk)
    W = _lif_graph(rng, n_spk, pre, post, 0.2, 0.6)
    sensory = np.arange(n_lif, n_spk)                          # the last block of the spiking population
    types = np.where(np.arange(n_spk) >= n_lif, "SENSORY", "LIF")
    table = neuron_table(n_spk, type_names=types)
    lif = LifConfig(f"whole fly, {n_rate + n_spk:,} neurons / {edges:,} edges", from_arrays(table, W), sensory,
                    100.0, 2000)
    vpn = np.unique(optic.W_sr.tocoo().row)
    return WholeFlyConfig(lif=lif, optic=optic, sensory_idx=sensory, vpn_idx=vpn, n_rate=n_rate, n_spiking=n_spk,
                          edges=int(W.nnz + optic.W0.nnz + coupling))


def batched_config4(seed: int = 0) -> WholeFlyConfig:
    """The batched-rollout tier: config 2's spiking graph (71,618 LIF neurons, 15 M edges, Poisson
    drive on its 2,000 designated cells) coupled to config 3's optic lobe (89,390 units, 6 M nnz)
    through the lobe's feedback (W_rs) and visual projection (W_sr) blocks. Per-fly Poisson rates
    and episode lengths are the caller's (the benchmark draws 20-200 Hz and 500-4,000 steps)."""
    lif = lif_config2(seed=seed)
    optic = optic_config3(seed=seed + 1, n_spk=lif.c.n)
    vpn = np.unique(optic.W_sr.tocoo().row)
    coupling = optic.W_rp.nnz + optic.W_rs.nnz + optic.W_sr.nnz
    return WholeFlyConfig(lif=lif, optic=optic, sensory_idx=np.asarray(lif.poisson_idx), vpn_idx=vpn,
                          n_rate=optic.m, n_spiking=lif.c.n, edges=int(lif.c.W.nnz + optic.W0.nnz + coupling))


def eye_grid(radius: int = 16):
    """(retina, ray directions (n_col, k, 3), weights (k,)) of two hexagonal column patches."""
    from .retina import EyeGeometry, Retina, column_directions
    cells = [(h1, h2) for h1 in range(-radius, radius + 1) for h2 in range(-radius, radius + 1) if abs(h1 - h2) <= radius]
    side = np.array(["L"] * len(cells) + ["R"] * len(cells))
    hexes = np.array(cells + cells, dtype=float)
    col_dir, az_el = column_directions(side, hexes, EyeGeometry())
    r = Retina(pr_index=np.zeros(0, np.int64), pr_column=np.zeros(0, np.int64), pr_sens=np.zeros((0, 4), np.float32),
               col_side=side, col_hex=hexes, col_dir=col_dir, col_az_el=az_el)
    return (r, *r.ray_directions())


def fly_poses(batch: int, seed: int = 0):
    """Eye positions and orientations (eye, forward, left, up) of flies walking and hovering over
    the table and floor of `world.make_room`, heading and pitch uniform."""
    rng = np.random.default_rng(seed)
    heading, pitch = rng.uniform(-np.pi, np.pi, batch), rng.uniform(-0.4, 0.4, batch)
    on_table = rng.random(batch) < 0.5
    eye = np.c_[rng.uniform(-1.5, 1.5, batch), rng.uniform(-1.5, 1.5, batch), rng.uniform(0.01, 1.5, batch)]
    eye[on_table] = np.c_[rng.uniform(-0.5, 0.5, on_table.sum()), rng.uniform(-0.3, 0.3, on_table.sum()),
                          0.751 + rng.uniform(0, 0.05, on_table.sum())]
    f = np.c_[np.cos(pitch) * np.cos(heading), np.cos(pitch) * np.sin(heading), np.sin(pitch)]
    left = np.c_[-np.sin(heading), np.cos(heading), np.zeros(batch)]
    return eye, f, left, np.cross(f, left)
