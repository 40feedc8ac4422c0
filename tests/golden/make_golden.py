"""Regenerate the golden fixtures of tests/golden/ from the reference's own CPU implementation.

    python tests/golden/make_golden.py --reference <flyverse checkout>   (or FLYVERSE_REFERENCE=<checkout>)

Runs in the build container only (the reference is not on the GPU machines): it imports
flyverse from the reference checkout and records what its CPU path produces on inputs both sides
can rebuild. Every random input is a torch CPU generator draw or a seeded numpy draw that the tests
regenerate; the fixtures store the reference's outputs and hashes of the inputs.

  lif_c1.npz      flyverse.brain.Brain (CPU, event-driven) on the 2,000-neuron benchmark graph,
                  three drive regimes x 1,000 steps: spike rasters (packed), final v / g / rate /
                  counts. Uniforms: torch.rand((1, N)) per step from Generator().manual_seed(regime).
  lif_19cell.npz  the same Brain with the default model constants (receptor_model=None) on the
                  19-cell graph of tests/test_bit_identity.py::graph(), batch 2, depression and
                  adaptation on: the shaped weights, rasters and final state.
  lif_19cell_adapt_by_type.npz  the same run with per-type adaptation jumps (ADAPT_BY_TYPE, the
                  reference's adapt_by_type): its per-neuron jump vector, rasters and final state.
  lif_19cell_clocks.npz  the same run with per-neuron clocks (Brain.set_clocks, periods 1/2/3 steps
                  by neuron index) on the reference's sparse-matmul path, which is where it runs them.
  lif_19cell_slow_{additive,gain,threshold}.npz  the 19-cell run with the slow receptor tone
                  (receptor_model="full", classical class at scale 0.5) in each slow_mode, with the
                  per-entry receptor arrays (connectome.receptor_signs) it was built from.
  lif_19cell_clocks_slow_{additive,gain,threshold}.npz  the same slow-tone runs with the clocks of
                  lif_19cell_clocks (the reference's clocked step, sparse-matmul path).
  lif_c1_clocks.npz  config 1 at 6.5 mV drive with per-neuron clocks of 1, 2 and 4 steps on the
                  reference's sparse-matmul path: rasters and final state.
  optic_hex.npz   flyverse.optic.OpticLobe (CPU) with default parameters on the 7-column hex patch
                  of tests/test_optic_hooks.py::hex_graph(), batch 2, three frames.
  optic_hex_slow_{additive,gain,threshold}.npz  the hex patch's OpticLobe with the receptor model's
                  slow tone (classical class at scale 2) in each slow_mode, three frames from a displaced start, with the
                  receptor record it was built from.
  optic_hex_hooks_{rectify,adapt,suppress,all}.npz  the hex patch's OpticLobe with the per-stream
                  hooks of HOOK_CASES (rectified, adapting and spatially suppressed Mi1 streams),
                  three frames.
  optic_synth.npz the reference's own `OpticLobe._substep` (optic.py:525-551), run on a
                  synthetic 3,000-unit lobe from flyb200.synthetic.optic_config3, 60 substeps.
  tracer.npz      flyverse.world / flyverse.batch_world (CPU): the reference tests' rays in
                  make_room(0), a 48 x 32 camera image, three batched rooms before and after a
                  per-row sphere move, and the eye: flyverse.retina.build_retina on a two-eye
                  hex grid (column directions, 7 sample rays per column) traced from four fly
                  poses and averaged into columns as BatchSim.column_radiance does.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys
from pathlib import Path

os.environ.setdefault("CUDA_VISIBLE_DEVICES", "-1")

import numpy as np
import pandas as pd
import scipy.sparse as sp
import torch

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "flyverse-core_b200"))

from flyb200 import synthetic  # noqa: E402

REGIMES = {"poisson": 0.0, "drive65": 6.5, "drive72": 7.2}


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def uniforms(seed: int, steps: int, shape) -> np.ndarray:
    gen = torch.Generator().manual_seed(seed)
    return np.stack([torch.rand(shape, generator=gen).numpy() for _ in range(steps)])


def lif_c1(ref) -> dict:
    cn, brain = ref["connectome"], ref["brain"]
    cfg = synthetic.lif_config1(seed=0)
    c = cfg.c
    out = {"W_sha": np.array(sha(c.W.data) + sha(c.W.indices) + sha(c.W.indptr))}
    for k, (name, drive) in enumerate(REGIMES.items()):
        rc = cn.Connectome(c.neurons[["bodyId", "type", "superclass", "nt"]].copy(), c.W.copy(),
                           pd.Series(np.arange(c.n), index=c.neurons.bodyId.to_numpy()))
        b = brain.Brain(rc, brain.LIFParams(**cfg.params, event_driven=True), device="cpu", seed=0)
        b.set_poisson(cfg.poisson_idx, cfg.poisson_hz)
        b.record_activity = True
        if drive:
            b.set_drive(np.arange(c.n), np.float32(drive))
        U = uniforms(k, cfg.steps, (1, c.n))
        b.gen.manual_seed(k)
        ras = np.zeros((cfg.steps, c.n), bool)
        for s in range(cfg.steps):
            b.step(1)
            ras[s] = b.spikes[0].numpy() > 0
        out[f"{name}_raster"] = np.packbits(ras, axis=1, bitorder="little")
        out[f"{name}_uniform_sha"] = np.array(sha(U))
        for key in ("v", "g", "rate", "spike_counts"):
            out[f"{name}_{key}"] = getattr(b, key)[0].numpy().copy()
        out[f"{name}_drive"] = np.float32(drive)
        out[f"{name}_seed"] = np.int64(k)
        print(f"lif_c1 {name}: {int(ras.sum())} spikes")
    return out


def lif_19cell_slow(ref, mode: str, clocks: bool = False) -> dict:
    """The 19-cell run with the receptor model's slow tone (receptor_model="full", classical class
    at scale 0.5) in one slow_mode: the per-entry receptor arrays the model read, the shaped fast
    and slow matrices, rasters, final state and tone. With `clocks`, periods 1, 2, 3 steps by
    neuron on the reference's sparse-matmul path (its clocked step carries the tone too)."""
    brain, cn = ref["brain"], ref["connectome"]
    tb = ref["test_bit_identity"]
    c = tb.graph()
    B, steps, seed = 2, 400, 7
    p = brain.LIFParams(receptor_model="full", event_driven=not clocks,
                        slow_gain_by_class={"metabotropic_classical": 0.5}, slow_mode=mode)
    rec = cn.receptor_signs(c, net_rule=p.receptor_net_rule, with_counts=True)
    b = brain.Brain(c, p, device="cpu", seed=seed, batch=B, receptor=rec)
    frozen = np.flatnonzero((c.neurons.superclass == "ol_intrinsic").to_numpy())
    b.freeze(frozen)
    b.prune(frozen)
    period = None
    if clocks:
        period = 1 + np.arange(c.n) % 3
        b.set_clocks(period)
    b.record_activity = True
    orn, jo, dnp = c.select(type="ORN_DM1"), c.select(type="~^JO-"), c.select(type="DNp01")
    b.set_poisson(orn, torch.tensor([[120.0], [40.0]]))
    b.set_poisson(jo, torch.tensor([[90.0, 10.0], [0.0, 150.0]]))
    b.set_drive(dnp, torch.tensor([[12.0], [0.0]]))
    gen = torch.Generator().manual_seed(seed)
    U = np.stack([torch.rand((B, c.n), generator=gen).numpy() for _ in range(steps)])
    ras = np.zeros((steps, B, c.n), bool)
    for s in range(steps):
        b.step(1)
        ras[s] = b.spikes.numpy() > 0
    W = b._W_cpu.tocsr()
    out = _table(c.neurons) | {"W_data": c.W.data, "W_indices": c.W.indices, "W_indptr": c.W.indptr,
                               "shaped_data": W.data, "shaped_indices": W.indices, "shaped_indptr": W.indptr,
                               "frozen": frozen, "orn": orn, "jo": jo, "dnp01": dnp, "raster": ras,
                               "uniform_sha": np.array(sha(U)), "seed": np.int64(seed), "steps": np.int64(steps),
                               "batch": np.int64(B), "slow_mode": np.array(mode), "slow_classes": np.array(b.slow_classes),
                               "rec_fast_sign": rec.fast_sign, "rec_slow_sign": rec.slow_sign,
                               "rec_fast_gain": rec.fast_gain, "rec_slow_gain": rec.slow_gain,
                               "rec_slow_class": rec.slow_class, "rec_count": rec.count}
    for k, S in b._W_slow_cpu.items():
        S = S.tocsr()
        out[f"slow_{k}_data"], out[f"slow_{k}_indices"], out[f"slow_{k}_indptr"] = S.data, S.indices, S.indptr
    for key in ("v", "g", "refrac", "adapt", "res", "rate", "spike_counts", "spikes", "g_slow"):
        out[f"final_{key}"] = getattr(b, key).numpy().copy()
    if period is not None:
        out["clock_period"] = period
    print(f"lif_19cell_slow ({mode}, clocks={clocks}): {int(ras.sum())} spikes, slow entries "
          f"{[(k, S.nnz) for k, S in b._W_slow_cpu.items()]}, max tone {float(b.g_slow.abs().max()):.3f} mV")
    return out


def lif_c1_clocks(ref) -> dict:
    """Config 1's drive regime 6.5 mV with per-neuron clocks of 1, 2 and 4 steps (by neuron index),
    on the reference's sparse-matmul path (where it runs clocks)."""
    cn, brain = ref["connectome"], ref["brain"]
    cfg = synthetic.lif_config1(seed=0)
    c = cfg.c
    rc = cn.Connectome(c.neurons[["bodyId", "type", "superclass", "nt"]].copy(), c.W.copy(),
                       pd.Series(np.arange(c.n), index=c.neurons.bodyId.to_numpy()))
    b = brain.Brain(rc, brain.LIFParams(**cfg.params, event_driven=False), device="cpu", seed=0)
    period = np.array([1, 2, 4])[np.arange(c.n) % 3]
    b.set_clocks(period)
    b.set_poisson(cfg.poisson_idx, cfg.poisson_hz)
    b.record_activity = True
    b.set_drive(np.arange(c.n), np.float32(6.5))
    seed = 1
    U = uniforms(seed, cfg.steps, (1, c.n))
    b.gen.manual_seed(seed)
    ras = np.zeros((cfg.steps, c.n), bool)
    for s in range(cfg.steps):
        b.step(1)
        ras[s] = b.spikes[0].numpy() > 0
    out = {"raster": np.packbits(ras, axis=1, bitorder="little"), "uniform_sha": np.array(sha(U)),
           "clock_period": period, "seed": np.int64(seed), "drive": np.float32(6.5)}
    for key in ("v", "g", "rate", "spike_counts"):
        out[key] = getattr(b, key)[0].numpy().copy()
    print(f"lif_c1_clocks: {int(ras.sum())} spikes")
    return out


def _table(n: pd.DataFrame) -> dict:
    return {f"nrn_{col}": n[col].fillna("").astype(str).to_numpy().astype("U") for col in ("type", "superclass", "nt", "class")} | \
        {"nrn_bodyId": n.bodyId.to_numpy().astype(np.int64)}


ADAPT_BY_TYPE = {"^ORN_": 3.0, "^JO-": 0.4, "^DNp": 2.5}


def lif_19cell(ref, adapt_by_type=None, clocks=False) -> dict:
    brain = ref["brain"]
    tb = ref["test_bit_identity"]
    c = tb.graph()
    B, steps, seed = 2, 400, 7
    # per-neuron clocks run on the reference's sparse-matmul path only (brain.py:624-625)
    p = brain.LIFParams(receptor_model=None, event_driven=not clocks, adapt_by_type=adapt_by_type)
    b = brain.Brain(c, p, device="cpu", seed=seed, batch=B)
    frozen = np.flatnonzero((c.neurons.superclass == "ol_intrinsic").to_numpy())
    b.freeze(frozen)
    b.prune(frozen)
    period = None
    if clocks:            # periods 1, 2, 3 steps by neuron (K = 6); 3 x 0.5 ms stays within the delay
        period = 1 + np.arange(c.n) % 3
        b.set_clocks(period)
    b.record_activity = True
    orn = c.select(type="ORN_DM1")
    jo = c.select(type="~^JO-")
    b.set_poisson(orn, torch.tensor([[120.0], [40.0]]))
    b.set_poisson(jo, torch.tensor([[90.0, 10.0], [0.0, 150.0]]))
    b.set_drive(c.select(type="DNp01"), torch.tensor([[12.0], [0.0]]))
    gen = torch.Generator().manual_seed(seed)
    U = np.stack([torch.rand((B, c.n), generator=gen).numpy() for _ in range(steps)])
    ras = np.zeros((steps, B, c.n), bool)
    for s in range(steps):
        b.step(1)
        ras[s] = b.spikes.numpy() > 0
    W = b._W_cpu.tocsr()
    out = _table(c.neurons) | {"W_data": c.W.data, "W_indices": c.W.indices, "W_indptr": c.W.indptr,
                               "shaped_data": W.data, "shaped_indices": W.indices, "shaped_indptr": W.indptr,
                               "frozen": frozen, "orn": orn, "jo": jo, "dnp01": c.select(type="DNp01"),
                               "raster": ras, "uniform_sha": np.array(sha(U)), "seed": np.int64(seed),
                               "steps": np.int64(steps), "batch": np.int64(B)}
    for key in ("v", "g", "refrac", "adapt", "res", "rate", "spike_counts", "spikes"):
        out[f"final_{key}"] = getattr(b, key).numpy().copy()
    if period is not None:
        out["clock_period"] = period
    if adapt_by_type:
        out["adapt_jump_vec"] = b.adapt_jump_vec.numpy().copy()
        out["adapt_patterns"] = np.array(list(adapt_by_type), dtype="U")
        out["adapt_values"] = np.array(list(adapt_by_type.values()), np.float32)
    print(f"lif_19cell (adapt_by_type={adapt_by_type}, clocks={clocks}): {int(ras.sum())} spikes, {W.nnz} shaped entries")
    return out


def optic_hex(ref) -> dict:
    optic, rt = ref["optic"], ref["retina"]
    th = ref["test_optic_hooks"]
    c = th.hex_graph()
    r = rt.build_retina(c)
    B = 2
    ol = optic.OpticLobe(c, r, optic.OpticParams(), device="cpu", batch=B)
    ol.relax()
    gen = torch.Generator().manual_seed(3)
    out = _table(c.neurons) | {"W_data": c.W.data, "W_indices": c.W.indices, "W_indptr": c.W.indptr,
                               "hex1": c.neurons.hex1.to_numpy(np.float64), "hex2": c.neurons.hex2.to_numpy(np.float64),
                               "hex_side": c.neurons.hex_side.fillna("").astype(str).to_numpy().astype("U"),
                               "pr_index": r.pr_index, "pr_column": r.pr_column, "pr_sens": r.pr_sens,
                               "n_columns": np.int64(r.n_columns), "rate_idx": ol.rate_idx, "spk_idx": ol.spk_idx}
    for f in range(3):
        rad = torch.rand(B, r.n_columns, 4, generator=gen)
        spk = torch.rand(B, c.n, generator=gen) * 80.0
        drive = ol.step_frame(rad, spk, 10.0)
        out[f"frame{f}_rad"], out[f"frame{f}_spk"] = rad.numpy(), spk.numpy()
        for key in ("v", "adapt", "delta_rate", "contrast", "I_lp", "I_mean"):
            out[f"frame{f}_{key}"] = getattr(ol, key).numpy().copy()
        out[f"frame{f}_drive"] = drive.numpy().copy()
    print("optic_hex: 3 frames")
    return out


def optic_hex_slow(ref, mode: str) -> dict:
    """The hex patch's optic lobe under the receptor model's slow tone (classical class at scale 2,
    built from connectome.receptor_signs) in one slow_mode, batch 2, three frames from a displaced
    start."""
    optic, rt, brain, cn = ref["optic"], ref["retina"], ref["brain"], ref["connectome"]
    th = ref["test_optic_hooks"]
    c = th.hex_graph()
    r = rt.build_retina(c)
    p = brain.LIFParams(receptor_model="full", slow_gain_by_class={"metabotropic_classical": 2.0}, slow_mode=mode)
    rec = cn.receptor_signs(c, net_rule=p.receptor_net_rule, with_counts=True)
    B = 2
    ol = optic.OpticLobe(c, r, optic.OpticParams(), device="cpu", batch=B, receptor=rec,
                         receptor_gain=brain._receptor_gain(p), slow=brain._slow_spec(p))
    ol.relax()
    gen = torch.Generator().manual_seed(4)
    # the receptor model silences the patch's histamine photoreceptor synapses, so the lobe starts
    # from a displaced state (public state, as a caller may set it) whose decay drives the tone
    v0 = torch.rand(B, ol.n_rate, generator=gen) * 0.8 - 0.3
    ol.v.copy_(v0)
    out = {"rec_fast_sign": rec.fast_sign, "rec_slow_sign": rec.slow_sign, "rec_fast_gain": rec.fast_gain,
           "rec_slow_gain": rec.slow_gain, "rec_slow_class": rec.slow_class, "rec_count": rec.count,
           "slow_mode": np.array(mode), "slow_entries": np.array(repr(ol.slow_entries)), "v0": v0.numpy()}
    for f in range(3):
        rad = torch.rand(B, r.n_columns, 4, generator=gen)
        spk = torch.rand(B, c.n, generator=gen) * 80.0
        drive = ol.step_frame(rad, spk, 10.0)
        out[f"frame{f}_rad"], out[f"frame{f}_spk"] = rad.numpy(), spk.numpy()
        for key in ("v", "adapt", "delta_rate", "g_slow"):
            out[f"frame{f}_{key}"] = getattr(ol, key).numpy().copy()
        out[f"frame{f}_g_slow_cls"] = ol.g_slow_cls.numpy().copy()
        out[f"frame{f}_drive"] = drive.numpy().copy()
    print(f"optic_hex_slow ({mode}): slow entries {ol.slow_entries}, max tone {float(ol.g_slow.abs().max()):.4f}")
    return out


HOOK_CASES = {
    "rectify": dict(stream_rectify=[("Mi1", "T3", "pos"), ("Mi1", "Pm1", "abs")]),
    "adapt": dict(stream_adapt=[("Mi1", "T3|Pm1", 15.0, 0.8)]),
    "suppress": dict(spatial_suppress=[("Mi1", 0.6, 6.0)]),
    "all": dict(stream_rectify=[("Mi1", "T3", "neg"), ("T3", "LC11", "abs")], stream_adapt=[("Mi1", ".*", 25.0, 0.5)],
                spatial_suppress=[("Mi1", 0.4, 6.0)]),
}


def optic_hex_hooks(ref, case: str) -> dict:
    """The hex patch's OpticLobe with the per-stream hooks of HOOK_CASES[case], batch 2, three frames."""
    optic, rt = ref["optic"], ref["retina"]
    th = ref["test_optic_hooks"]
    c = th.hex_graph()
    r = rt.build_retina(c)
    B = 2
    ol = optic.OpticLobe(c, r, optic.OpticParams(**HOOK_CASES[case]), device="cpu", batch=B)
    ol.relax()
    gen = torch.Generator().manual_seed(6)
    out = {"case": np.array(case), "hook_info": np.array(repr(ol.hook_info))}
    for f in range(3):
        rad = torch.rand(B, r.n_columns, 4, generator=gen)
        spk = torch.rand(B, c.n, generator=gen) * 80.0
        drive = ol.step_frame(rad, spk, 10.0)
        out[f"frame{f}_rad"], out[f"frame{f}_spk"] = rad.numpy(), spk.numpy()
        for key in ("v", "adapt", "delta_rate", "stream_adapt_state"):
            out[f"frame{f}_{key}"] = getattr(ol, key).numpy().copy()
        out[f"frame{f}_drive"] = drive.numpy().copy()
    print(f"optic_hex_hooks ({case}): {ol.hook_info.get('entries_rr_matched')} rr / "
          f"{ol.hook_info.get('entries_sr_matched')} sr entries in streams, |v| max {float(ol.v.abs().max()):.4f}")
    return out


def optic_synth(ref) -> dict:
    """The reference's substep expressions on a synthetic lobe, called on the reference class."""
    optic = ref["optic"]
    cfg = synthetic.optic_config3(seed=1, m=3000, nnz=200_000, n_pr=300, n_types=60, n_spk=500)
    W = cfg.W_rr()
    B, steps = 2, 60
    rng = np.random.default_rng(5)
    v0 = (rng.standard_normal((B, cfg.m)) * 0.2).astype(np.float32)
    ad0 = (rng.standard_normal((B, cfg.m)) * 0.05).astype(np.float32)
    pr = (rng.standard_normal((B, cfg.m)) * 0.3).astype(np.float32)
    spk = (rng.standard_normal((B, cfg.m)) * 0.1).astype(np.float32)
    lobe = object.__new__(optic.OpticLobe)
    lobe.p = optic.OpticParams(adapt_tau_ms=cfg.adapt_tau_ms, dt_ms=cfg.dt_ms)
    lobe.slow, lobe._hooks = None, False
    lobe.W_rr = torch.sparse_csr_tensor(torch.from_numpy(W.indptr.astype(np.int64)), torch.from_numpy(W.indices.astype(np.int64)),
                                        torch.from_numpy(W.data), size=W.shape)
    lobe._a = torch.from_numpy(cfg.a)
    lobe.b_vec = torch.from_numpy(cfg.b)
    lobe._a_ad = cfg.aad
    lobe.v, lobe.adapt = torch.from_numpy(v0.copy()), torch.from_numpy(ad0.copy())
    vs = []
    for _ in range(steps):
        optic.OpticLobe._substep(lobe, torch.from_numpy(pr), torch.from_numpy(spk))
        vs.append(lobe.v.numpy().copy())
    print("optic_synth: 60 substeps")
    snap = np.array([0, 9, 19, 29, 39, 49, 59])
    return {"seed": np.int64(1), "m": np.int64(cfg.m), "nnz": np.int64(200_000), "n_pr": np.int64(300),
            "n_types": np.int64(60), "n_spk": np.int64(500), "W_sha": np.array(sha(W.data) + sha(W.indices)),
            "v0": v0, "adapt0": ad0, "pr": pr, "spk": spk, "snap": snap, "v": np.stack(vs)[snap],
            "adapt": lobe.adapt.numpy().copy(), "aad": np.float64(cfg.aad)}


def eye_grid(radius: int = 6) -> pd.DataFrame:
    """One R1-R6 photoreceptor per column of a hex patch on each side (ids 1000 + k)."""
    cells = [(h1, h2) for h1 in range(-radius, radius + 1) for h2 in range(-radius, radius + 1) if abs(h1 - h2) <= radius]
    sites = [(side, h1, h2) for side in ("L", "R") for h1, h2 in cells]
    return pd.DataFrame([dict(bodyId=1000 + k, type="R1-R6", superclass="ol_sensory", nt="histamine", hex1=h1, hex2=h2,
                              hex_side=side) for k, (side, h1, h2) in enumerate(sites)])


def tracer(ref) -> dict:
    world, bworld, rt, cn = ref["world"], ref["batch_world"], ref["retina"], ref["connectome"]
    out = {}
    # known answers of the reference's tests (tests/test_world.py:18-28)
    w = world.World(spheres=[world.Sphere((1, 0, 0), (.2, .2, .2), "apple")], device="cpu", detail=0,
                    ambient=(1, 1, 1, 1), light_color=(0, 0, 0, 0))
    out["known_apple"] = w.trace(torch.zeros(1, 3), torch.tensor([[1., 0, 0]])).numpy()
    # the room and the reference tests' rays (test_world.py:9-14, 43-50)
    room, _ = world.make_room(0)
    room.device = "cpu"

    def rays(n, seed):
        g = torch.Generator().manual_seed(seed)
        d = torch.randn(n, 3, generator=g)
        d /= d.norm(dim=-1, keepdim=True)
        return torch.tensor([-.5, .05, .7512]).expand_as(d).contiguous(), d

    o1, d1 = rays(67, 0)
    o2, d2 = rays(134, 8)
    o2, d2 = (o2[::2] + .03).contiguous(), d2[::2].contiguous()
    for k, (o, d) in enumerate(((o1, d1), (o2, d2))):
        out[f"room_o{k}"], out[f"room_d{k}"] = o.numpy(), d.numpy()
        out[f"room_rad{k}"] = room.trace(o, d).numpy()
    # the same room without texture detail, and seen from a camera
    room.detail = 0
    room.invalidate()
    out["room_flat_rad0"] = room.trace(o1, d1).numpy()
    room.detail = 1.4
    room.invalidate()
    out["camera"] = room.render_camera((0, 0, 1), (1, 0, 0), (0, 0, 1), width=48, height=32).numpy()
    # three batched rooms (tests/test_batch_sim.py:141-161)
    scenes = [world.make_room(i)[0] for i in range(3)]
    for sc in scenes:
        sc.device = "cpu"
    scenes[1].spheres[0].material = "black"
    scenes[2].light_pos = (1, 0, 2)
    batched = bworld.BatchWorld(scenes, "cpu")
    gen = torch.Generator().manual_seed(12)
    dirs = torch.randn(3, 74, 3, generator=gen)[:, ::2]
    dirs = (dirs / dirs.norm(dim=-1, keepdim=True)).contiguous()
    org = torch.tensor([-.5, .05, .7512]).expand_as(dirs).contiguous()
    out["batch_o"], out["batch_d"] = org.numpy(), dirs.numpy()
    out["batch_rad"] = batched.trace(org, dirs).numpy()
    batched.move_sphere(0, (-.45, .05, .77), (.05,) * 3, rows=[1])
    out["batch_rad_moved"] = batched.trace(org, dirs).numpy()
    # the eye: the reference's retina geometry on a two-eye hex grid, traced from four poses
    n = eye_grid()
    n["class"] = ""; n["subclass"] = ""; n["somaSide"] = n.hex_side; n["instance"] = n.type + "_x"
    n["sign"] = np.array([cn.NT_SIGN[x] for x in n.nt], dtype=np.float32)
    c = cn.Connectome(n, sp.csr_matrix((len(n), len(n)), dtype=np.float32), pd.Series(np.arange(len(n)), index=n.bodyId.to_numpy()))
    r = rt.build_retina(c)
    eye_dirs, wts = r.ray_directions()
    out.update({"eye_hex1": n.hex1.to_numpy(np.float64), "eye_hex2": n.hex2.to_numpy(np.float64),
                "eye_side": n.hex_side.to_numpy().astype("U"), "eye_col_dir": r.col_dir, "eye_col_az_el": r.col_az_el,
                "eye_dirs": eye_dirs, "eye_w": wts, "eye_pr_column": r.pr_column})
    B = 4
    rooms = [world.make_room(i)[0] for i in range(B)]
    for sc in rooms:
        sc.device = "cpu"
    rooms[3].spheres[0].material = "lamp"
    eyes = bworld.BatchWorld(rooms, "cpu")
    rng = np.random.default_rng(21)
    heading = rng.uniform(-np.pi, np.pi, B)
    pitch = rng.uniform(-0.3, 0.3, B)
    eye = np.c_[rng.uniform(-0.5, 0.5, B), rng.uniform(-0.3, 0.3, B), 0.76 + rng.uniform(0, 0.1, B)]
    f = np.c_[np.cos(pitch) * np.cos(heading), np.cos(pitch) * np.sin(heading), np.sin(pitch)]
    left = np.c_[-np.sin(heading), np.cos(heading), np.zeros(B)]
    up = np.cross(f, left)
    # BatchSim.column_radiance (batch_sim.py:192-201)
    rotation = np.stack([f, left, up], axis=2)
    directions = eye_dirs.reshape(1, -1, 3) @ rotation.transpose(0, 2, 1)
    origins = np.broadcast_to(eye[:, None], directions.shape)
    rad = eyes.trace(torch.from_numpy(np.ascontiguousarray(origins, dtype=np.float32)),
                     torch.from_numpy(np.ascontiguousarray(directions, dtype=np.float32)))
    wts_t = torch.as_tensor(wts, dtype=torch.float32)
    out["eye_rad"] = rad.numpy()
    out["eye_columns"] = (rad.reshape(B, *eye_dirs.shape[:2], 4) * wts_t[None, None, :, None]).sum(2).numpy()
    out.update({"eye_pos": eye, "eye_f": f, "eye_left": left, "eye_up": up,
                "eye_ray_d": np.ascontiguousarray(directions, dtype=np.float32)})
    print(f"tracer: {r.n_columns} columns x {eye_dirs.shape[1]} rays, {B} poses")
    return out


def _full_table(n: pd.DataFrame) -> dict:
    """Every column of a neuron table: strings as unicode arrays, numbers as they are."""
    out = {}
    for col in n.columns:
        v = n[col]
        if v.dtype == object or pd.api.types.is_string_dtype(v):
            out[f"tbl_{col}"] = v.fillna("").astype(str).to_numpy().astype("U")
        else:
            out[f"tbl_{col}"] = v.to_numpy()
    return out


FLY_RADIANCE = np.array([[.10, .20, .30, .40], [.90, .10, .55, .05], [.33, .66, .11, .77], [.50, .50, .50, .50]],
                        np.float32)


def fly_frames(ref) -> dict:
    """The reference's FlyBrain (CPU) on the 19-cell graph of tests/test_bit_identity.py, batch 2,
    seed 7, frame by frame, in the manner of that file's scenario: two held Poisson inputs and a
    radiance frame for three 10 ms frames; then a 300 Hz pulse on LC4 for 7 ms (it ends inside the
    next frame), a 12 mV drive on DNp01 and the mirrored radiance for two 13.3 ms frames (the
    fractional milliseconds carry over); a reset of fly 0 and a frame; a full reset, one input and
    a 20 ms frame. Recorded: every LIF step's spikes and the uniforms the brain drew for it (zeros
    when it drew none), and the state at each frame end."""
    fly, brain, tb = ref["fly"], ref["brain"], ref["test_bit_identity"]
    c = tb.graph()
    fb = fly.FlyBrain(c, batch=2, device="cpu", seed=7, lif_params=brain.LIFParams(receptor_model=None))
    b = fb.brain
    B, N = b.B, b.n
    U, R = [], []
    plain_step = b.step

    def recording_step(n=1):
        for _ in range(int(n)):
            if b._poisson_on:
                state = b.gen.get_state()
                U.append(torch.rand((B, N), generator=b.gen).numpy().copy())
                b.gen.set_state(state)
            else:
                U.append(np.zeros((B, N), np.float32))
            plain_step(1)
            R.append(b.spikes.numpy() > 0)

    b.step = recording_step
    orn, jo = c.select(type="ORN_DM1"), c.select(type="~^JO-")
    out = _full_table(c.neurons) | {"W_data": c.W.data, "W_indices": c.W.indices, "W_indptr": c.W.indptr,
                                    "orn": orn, "jo": jo, "radiance": FLY_RADIANCE}
    frames = []

    def frame(ms):
        fb.step(ms)
        k = len(frames)
        for key in ("v", "g", "refrac", "rate", "spike_counts", "adapt", "res", "drive", "poisson_p"):
            out[f"f{k}_brain_{key}"] = getattr(b, key).numpy().copy()
        for key in ("v", "adapt", "delta_rate"):
            out[f"f{k}_optic_{key}"] = getattr(fb.optic, key).numpy().copy()
        out[f"f{k}_steps"] = np.int64(len(R))
        out[f"f{k}_pending_ms"] = np.float64(fb._pending_ms)
        frames.append(ms)

    fb._input("smell", orn, np.array([[120.0], [40.0]], np.float32))
    fb._input("wind", jo, np.array([[90.0, 10.0], [0.0, 150.0]], np.float32))
    fb.vision(FLY_RADIANCE)
    for _ in range(3):
        frame(10.0)
    fb.stimulate([9], 300.0, 7.0)
    fb.brain.set_drive([15], np.float32(12.0))
    fb.vision(FLY_RADIANCE[::-1].copy())
    for _ in range(2):
        frame(13.3)
    fb.reset([0])
    frame(10.0)
    fb.reset()
    fb._input("smell", orn, np.float32(75.0))
    fb.vision(FLY_RADIANCE)
    frame(20.0)
    assert len(R) == sum(int(np.floor(x / b.p.dt + 1e-9)) for x in (10, 10, 10, 26.6, 10, 20)), len(R)
    out["frames_ms"] = np.array(frames)
    out["raster"] = np.stack(R)
    out["uniforms"] = np.stack(U)
    print(f"fly_frames: {len(frames)} frames, {len(R)} LIF steps, {int(np.stack(R).sum())} spikes")
    return out


def ref_cache(ref) -> dict:
    """A graph cache written by the reference's own `connectome.save` (a subset of the 19-cell graph,
    so the reference_* files are written too) into tests/golden/ref_cache/, and what the
    reference's `connectome.load` reads back from it; plus the digest of what the reference reads
    from a cache that flyb200.connectome.save wrote for the same graph."""
    import hashlib
    import json
    import shutil
    cn, tb = ref["connectome"], ref["test_bit_identity"]
    full = tb.graph()
    sub = full.subset(np.arange(4, 19))
    folder = HERE / "ref_cache"
    shutil.rmtree(folder, ignore_errors=True)
    cn.save(sub, folder)
    back = cn.load(folder, verbose=False)

    def digest(c) -> str:
        h = hashlib.sha256()
        for part in (c.W.data, c.W.indices, c.W.indptr, c.reference.W.data, c.reference.W.indices,
                     c.reference.W.indptr, c.neurons.bodyId.to_numpy(), c.neurons["in_syn"].to_numpy(),
                     c.neurons["in_syn_l2"].to_numpy(), c.reference.neurons.bodyId.to_numpy()):
            h.update(np.ascontiguousarray(part).tobytes())
        h.update(json.dumps([list(c.neurons.columns), c.neurons.type.tolist()]).encode())
        return h.hexdigest()

    from flyb200 import connectome as ours
    mine = ours.Connectome(sub.neurons.copy(), sub.W.copy(), sub.body_to_index,
                           ours.Connectome(full.neurons.copy(), full.W.copy(), full.body_to_index))
    tmp = HERE / "_ours_cache_tmp"
    shutil.rmtree(tmp, ignore_errors=True)
    ours.save(mine, tmp)
    back_ours = cn.load(tmp, verbose=False)
    shutil.rmtree(tmp)
    print(f"ref_cache: {sub.n} neurons, {sub.W.nnz} entries; reference reads its own cache and ours alike:",
          digest(back) == digest(back_ours))
    return {"n": np.int64(back.n), "nnz": np.int64(back.W.nnz), "ref_n": np.int64(back.reference.n),
            "W_data": back.W.data, "W_indices": back.W.indices, "W_indptr": back.W.indptr,
            "in_syn": back.neurons["in_syn"].to_numpy(), "in_syn_l2": back.neurons["in_syn_l2"].to_numpy(),
            "body": back.neurons.bodyId.to_numpy(), "ref_body": back.reference.neurons.bodyId.to_numpy(),
            "columns": np.array(list(back.neurons.columns), dtype="U"),
            "digest_reference_cache": np.array(digest(back)), "digest_flyb200_cache": np.array(digest(back_ours))}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("FLYVERSE_REFERENCE"),
                    help="the flyverse checkout whose CPU path records the fixtures (or FLYVERSE_REFERENCE)")
    ap.add_argument("--only", default=None, help="regenerate one fixture (its file stem)")
    args = ap.parse_args()
    if not args.reference:
        ap.error("give the reference checkout with --reference or FLYVERSE_REFERENCE")
    sys.path.insert(1, args.reference)
    sys.path.insert(2, str(Path(args.reference) / "tests"))
    import importlib
    ref = {k: importlib.import_module(m) for k, m in (("connectome", "flyverse.connectome"), ("brain", "flyverse.brain"),
                                                      ("optic", "flyverse.optic"), ("retina", "flyverse.retina"),
                                                      ("test_bit_identity", "test_bit_identity"),
                                                      ("test_optic_hooks", "test_optic_hooks"),
                                                      ("world", "flyverse.world"), ("batch_world", "flyverse.batch_world"),
                                                      ("fly", "flyverse.fly"))}
    torch.set_num_threads(1)
    fixtures = {"lif_c1": lambda: lif_c1(ref), "lif_19cell": lambda: lif_19cell(ref),
                "lif_19cell_adapt_by_type": lambda: lif_19cell(ref, ADAPT_BY_TYPE),
                "lif_19cell_clocks": lambda: lif_19cell(ref, clocks=True),
                "lif_c1_clocks": lambda: lif_c1_clocks(ref),
                **{f"lif_19cell_slow_{m}": (lambda m=m: lif_19cell_slow(ref, m)) for m in ("additive", "gain", "threshold")},
                **{f"lif_19cell_clocks_slow_{m}": (lambda m=m: lif_19cell_slow(ref, m, clocks=True))
                   for m in ("additive", "gain", "threshold")},
                "optic_hex": lambda: optic_hex(ref), "optic_synth": lambda: optic_synth(ref),
                "tracer": lambda: tracer(ref), "fly_frames": lambda: fly_frames(ref),
                "ref_cache": lambda: ref_cache(ref),
                **{f"optic_hex_slow_{m}": (lambda m=m: optic_hex_slow(ref, m)) for m in ("additive", "gain", "threshold")},
                **{f"optic_hex_hooks_{k}": (lambda k=k: optic_hex_hooks(ref, k)) for k in HOOK_CASES}}
    for name, make in fixtures.items():
        if args.only in (None, name):
            np.savez_compressed(HERE / f"{name}.npz", **make())


if __name__ == "__main__":
    main()
