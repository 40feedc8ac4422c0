"""Parity at the benchmark sizes: the configurations the bench times, compared with the oracle at
their stated size (the reference's own full-connectome checks, tests/test_cuda.py:185-231, have
the same purpose on the real graph, which is not shipped).

  C2  71,618 LIF neurons, 15 M edges, Poisson 100 Hz on 2,000 cells, B = 1, 10,000 steps (1 s):
      rasters of every step and every state word bit-exact, through the Brain drop-in and through
      the C ABI (flyb_lif_run) with its full raster.
  C3  89,390 graded units, 6 M nnz, grating-driven photoreceptor input, 200 substeps: every kernel
      shape within 1e-5 relative of the FP32 oracle; the max |FP32 - FP64| is printed and bounded.
  C4  64 flies on C2's graph, per-fly Poisson rates in 20-200 Hz, uneven episodes ended by row
      resets: rasters and state bit-exact.
  C5  the whole fly (167,106 neurons) at 64 and 256 flies in the bench's engine setup (settled to
      steady firing, autotuned, overlapped stages, pull delivery beside the next step, replayed
      from a CUDA graph): every step's raster and the LIF state bit-exact, the optic state within
      1e-5. The LIF is fed the device's drive each step (the drive is an FP32 product within
      tolerance of the oracle's; a neuron within an ulp of threshold would otherwise flip).
"""
import numpy as np
import pytest
import torch

import oracle
from flyb200 import _abi, autotune, synthetic
from flyb200.brain import Brain, LIFParams, lif_coefficients, out_edges
from flyb200.weights import lif_weights
from flyb200.whole import WholeFly
from gpu_helpers import native_lif_run
from helpers import unpack

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-5, 1e-6
LIF_STATE = (("v", "v"), ("g", "g"), ("refrac", "refrac"), ("rate", "rate"), ("spike_counts", "counts"),
             ("spikes", "spikes"), ("adapt", "adapt"), ("res", "res"), ("drive", "drive"))


# ------------------------------------------------------------------ C2 and C4: the spiking tier
@pytest.fixture(scope="module")
def c2():
    cfg = synthetic.lif_config2(seed=0)
    p = LIFParams(**cfg.params)
    W, _ = lif_weights(cfg.c, p)
    ptr, edges, mode = out_edges(W, p.w_syn)
    assert mode == _abi.RING_COUNT and edges.shape[0] == 15_000_000
    return cfg, p, ptr, edges


C2_CHUNK, C2_STEPS = 1000, 10_000


@pytest.fixture(scope="module")
def c2_oracle(c2):
    """The oracle's C2 trajectory: per 1,000-step chunk the raster and the state at its end."""
    cfg, p, ptr, edges = c2
    st = oracle.LifState(cfg.c.n, 1, 19, _abi.RING_COUNT, p.v_rest)
    st.poisson_p[cfg.poisson_idx, :] = np.float32(cfg.poisson_hz) * np.float32(p.dt / 1000.0)
    P = lif_coefficients(p, False)
    chunks = []
    for _ in range(C2_STEPS // C2_CHUNK):
        r, ev = oracle.lif_run(st, ptr, edges, P, n_delay=18, flags=_abi.LIF_POISSON | _abi.LIF_COUNTS,
                               nsteps=C2_CHUNK, seed=1, raster=True)
        chunks.append((r, ev, st.copy()))
    assert chunks[-1][2].counts.sum() > 100_000          # ~10 Hz mean over 1 s
    return chunks


@pytest.mark.parametrize("launch", ["step", "persistent"])
def test_c2_brain_full_size_bit_exact(c2, c2_oracle, launch):
    """The Brain drop-in on the full C2 graph for 10,000 steps: after every 1,000 steps all state
    words, the pending-input ring, the last 18 steps' rasters (the spike history) and the synaptic
    event count equal the oracle's."""
    cfg, p, ptr, edges = c2
    b = Brain(cfg.c, p, device="cuda", seed=1, batch=1, launch=launch)
    b.record_activity = True
    b.set_poisson(cfg.poisson_idx, cfg.poisson_hz)
    events = 0
    for k, (r, ev, st) in enumerate(c2_oracle):
        b.step(C2_CHUNK)
        torch.cuda.synchronize()
        b.check()
        events += ev
        for name, oname in LIF_STATE:
            np.testing.assert_array_equal(b._st[name].cpu().numpy(), getattr(st, oname), err_msg=f"{name} @ {k}")
        pos = int(b._clock[1].item())
        assert pos == st.ring_pos
        np.testing.assert_array_equal(b.ring.cpu().numpy(), st.ring)
        hist = b._hist.cpu().numpy().view(np.uint32)
        hp = int(b._clock[2].item())
        D = b.n_delay
        last = np.stack([hist[(hp - D + j) % D] for j in range(D)])
        np.testing.assert_array_equal(last[:, : r.shape[1]], r[-D:])
        assert b.synaptic_events == events


def test_c2_c_abi_full_raster_bit_exact(c2, c2_oracle):
    """flyb_lif_run through the C ABI (persistent launch, 1,000 steps per call) reproduces the
    oracle's raster of all 10,000 steps bit for bit."""
    cfg, p, ptr, edges = c2
    st = oracle.LifState(cfg.c.n, 1, 19, _abi.RING_COUNT, p.v_rest)
    st.poisson_p[cfg.poisson_idx, :] = np.float32(cfg.poisson_hz) * np.float32(p.dt / 1000.0)
    P = lif_coefficients(p, False)
    total = 0
    for r_want, ev_want, st_want in c2_oracle:
        r, ev = native_lif_run(st, ptr, edges, P, n_delay=18, flags=_abi.LIF_POISSON | _abi.LIF_COUNTS,
                               nsteps=C2_CHUNK, seed=1, raster=True, launch=_abi.LAUNCH_PERSISTENT)
        np.testing.assert_array_equal(r, r_want)
        assert ev == ev_want
        total += int(unpack(r, cfg.c.n).sum())
        for name in oracle.LifState.NAMES:
            np.testing.assert_array_equal(getattr(st, name), getattr(st_want, name), err_msg=name)
    assert total > 100_000


def _reset_oracle_rows(st, rows, v_rest):
    """Brain.reset(rows) on the oracle state: rest, no pending input."""
    st.v[:, rows] = v_rest
    for name in ("g", "refrac", "drive", "poisson_p", "rate", "spikes", "adapt", "counts"):
        getattr(st, name)[:, rows] = 0.0
    st.res[:, rows] = 1.0
    st.ring[:, :, rows] = 0


def test_c4_uneven_episodes_full_graph_bit_exact(c2):
    """C4: 64 flies on C2's graph, each with its own Poisson rate (20-200 Hz on the 2,000 sensory
    cells), episodes of uneven length (drawn per fly; a finished fly is reset on its own row and
    starts a new episode with a new rate while the others run on). The Brain under the autotuner's
    launch choice and under the staged update with pull delivery against the oracle: rasters of
    every step (spike history) and every state word bit-exact. Episodes are 30-150 steps here so
    that many rows reset within the 300 compared steps; the bench times 500-4,000."""
    cfg, p, ptr, edges = c2
    B, T = 64, 300
    rng = np.random.default_rng(44)
    rates0 = rng.uniform(20.0, 200.0, B).astype(np.float32)
    plan, left, t, rates = [], rng.integers(30, 151, B), 0, rates0.copy()
    while t < T:                                           # (steps, rows reset after them, new rates)
        k = int(min(left.min(), T - t))
        t += k
        left -= k
        done = np.flatnonzero(left <= 0)
        new = rng.uniform(20.0, 200.0, len(done)).astype(np.float32)
        plan.append((k, done, new))
        left[done] = rng.integers(30, 151, len(done))
    assert sum(len(d) for _, d, _ in plan) >= 64
    P = lif_coefficients(p, False)
    st = oracle.LifState(cfg.c.n, B, 19, _abi.RING_COUNT, p.v_rest)
    st.poisson_p[cfg.poisson_idx, :] = rates0[None, :] * np.float32(p.dt / 1000.0)
    want = []
    for k, done, new in plan:
        r, ev = oracle.lif_run(st, ptr, edges, P, n_delay=18, flags=_abi.LIF_POISSON | _abi.LIF_COUNTS, nsteps=k,
                               seed=5, raster=True)
        want.append((r, ev, st.copy()))
        _reset_oracle_rows(st, done, p.v_rest)
        st.poisson_p[cfg.poisson_idx[:, None], done[None, :]] = new[None, :] * np.float32(p.dt / 1000.0)
    for delivery in ("tuned", "staged-pull"):
        b = Brain(cfg.c, p, device="cuda", seed=5, batch=B, launch="step")
        b.record_activity = True
        b.set_poisson(cfg.poisson_idx, torch.from_numpy(rates0)[:, None].expand(B, len(cfg.poisson_idx)))
        if delivery == "tuned":
            autotune.tune_lif(b, steps=5)
        else:
            b.pull, b.staged = True, True
            b._make_args()
            assert b._pull_active()
        for (k, done, new), (r, ev, st_want) in zip(plan, want):
            b.step(k)
            torch.cuda.synchronize()
            b.check()
            for name, oname in LIF_STATE:
                np.testing.assert_array_equal(b._st[name].cpu().numpy(), getattr(st_want, oname),
                                              err_msg=f"{delivery}: {name}")
            np.testing.assert_array_equal(b.ring.cpu().numpy(), st_want.ring)
            D = min(k, b.n_delay)
            hist = b._hist.cpu().numpy().view(np.uint32)
            hp = int(b._clock[2].item())
            last = np.stack([hist[(hp - D + j) % b.n_delay] for j in range(D)])
            np.testing.assert_array_equal(last[:, : r.shape[1]], r[-D:])
            if len(done):
                b.reset(done)
                rate = torch.from_numpy(new)[:, None].expand(len(done), len(cfg.poisson_idx))
                b.poisson_p[torch.as_tensor(done)[:, None].cuda(), torch.as_tensor(cfg.poisson_idx)[None, :].cuda()] = \
                    (rate * np.float32(p.dt / 1000.0)).cuda()


# ------------------------------------------------------------------ C3: the optic lobe
def grating_input(o, B, t_ms=0.0):
    """Held photoreceptor input of the drifting grating: channel-weighted intensity per
    photoreceptor, contrast against the frame mean, clipped to [-1, 2], through gain_in * W_rp."""
    rad = o.grating(t_ms, B, seed=0)
    ip = (rad[:, o.pr_column, :] * o.sens[None]).sum(-1)
    mean = ip.mean(1, keepdims=True)
    a_pr = np.clip((ip - mean) / (mean + 0.02), -1.0, 2.0).T.astype(np.float32)
    M = o.W_rp.tocsr()
    return oracle.spmm(M.indptr, M.indices, M.data, a_pr, B, rows=o.m, alpha=o.gain_in)


@pytest.fixture(scope="module")
def c3():
    cfg = synthetic.optic_config3(seed=3)
    assert cfg.m == 89_390 and cfg.W0.nnz == 6_000_000
    return cfg


@pytest.mark.parametrize("batch,steps,variants", [(1, 200, (0, 1, 2, 3, 4)), (4, 200, (0,)),
                                                  (64, 40, (0, 1, 2, 3, 4, 5))])
def test_c3_full_lobe_every_shape_within_1e5(c3, batch, steps, variants):
    """C3 at full size from rest under the grating input: every kernel shape, per-substep and
    persistent launches, within 1e-5 relative of the FP32 oracle after `steps` substeps; the FP32
    result against the FP64 oracle is printed (max |dv| and max |d rate|) and bounded by 1e-4."""
    from flyb200.optic import OpticCore
    cfg = c3
    W = cfg.W_rr()
    pr = grating_input(cfg, batch)
    spk = np.zeros((cfg.m, batch), np.float32)
    v = np.zeros((cfg.m, batch), np.float32)
    ad = np.zeros((cfg.m, batch), np.float32)
    oracle.optic_run(v, ad, W.indptr, W.indices, W.data, pr, spk, cfg.a, cfg.b, cfg.gain_rr, cfg.adapt_gain, cfg.aad,
                     steps)
    v64, ad64 = np.zeros((cfg.m, batch)), np.zeros((cfg.m, batch))
    oracle.optic_run_f64(v64, ad64, W.indptr, W.indices, W.data, pr, spk, cfg.a, cfg.b, cfg.gain_rr,
                         cfg.adapt_gain, cfg.aad, steps)
    assert np.abs(v).max() > 0.05                        # the grating moves the lobe
    for launch in ("step", "persistent"):
        for variant in variants:
            core = OpticCore(W, cfg.a, cfg.b, batch=batch, device="cuda", gain_rr=cfg.gain_rr,
                             adapt_gain=cfg.adapt_gain, aad=cfg.aad, launch=launch)
            core.variant = variant
            core.pr_in.copy_(torch.from_numpy(pr))
            core.substeps(steps)
            torch.cuda.synchronize()
            core.check()
            gv, ga = core.v_s.cpu().numpy(), core.adapt_s.cpu().numpy()
            np.testing.assert_allclose(gv, v, rtol=RTOL, atol=ATOL, err_msg=f"{launch}/{variant}")
            np.testing.assert_allclose(ga, ad, rtol=RTOL, atol=ATOL, err_msg=f"{launch}/{variant}")
            dv = float(np.abs(gv - v64).max())
            drate = float(np.abs(np.clip(gv + cfg.b[:, None], 0, 1) - np.clip(v64 + cfg.b[:, None], 0, 1)).max())
            print(f"C3 B={batch} {launch}/{variant}: {steps} substeps, max|v32-v64| = {dv:.3e}, "
                  f"max|rate32-rate64| = {drate:.3e}")
            assert dv < 1e-4 and drate < 1e-4


# ------------------------------------------------------------------ C5: the whole fly
@pytest.fixture(scope="module")
def c5():
    return synthetic.whole_fly_config5(seed=0)


def settled_whole_fly(cfg, B, settle=3000, chunk=20):
    """The bench's engine: seed 1, the grating's photoreceptor stage, steady firing after `settle`
    steps replayed from CUDA graphs, then both autotuners at that firing density."""
    eng = WholeFly(cfg, B, device="cuda", seed=1, launch="step")
    eng.set_radiance(torch.from_numpy(cfg.optic.grating(0.0, B, seed=0)).cuda(), 0.1)
    eng.step(3)
    g = _capture(eng, chunk)
    for _ in range(settle // chunk):
        g.replay()
    torch.cuda.synchronize()
    del g
    eng.tuned = {"lif": autotune.tune_lif(eng.lif, steps=10), "optic": autotune.tune_optic(eng.optic, steps=10)}
    eng.step(2)
    torch.cuda.synchronize()
    eng.lif.check()
    return eng


def _capture(eng, steps):
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            eng.step(steps)
    torch.cuda.current_stream().wait_stream(s)
    return g


def oracle_from_engine(eng):
    """The engine's whole state copied into oracle arrays (LIF in the stored neuron order)."""
    lif = eng.lif
    n, B = lif.n, lif.B
    st = oracle.LifState(n, B, lif.R, lif.ring_mode, lif.p.v_rest)
    for name, oname in LIF_STATE + (("poisson_p", "poisson_p"),):
        getattr(st, oname)[...] = lif._st[name].cpu().numpy()
    st.active[...] = lif.active.cpu().numpy()
    st.ring[...] = lif.ring.cpu().numpy()
    clock = lif._clock.cpu().numpy()
    st.step, st.ring_pos = int(clock[0]), int(clock[1]) % lif.R
    o = eng.optic
    return st, o.v_s.cpu().numpy(), o.adapt_s.cpu().numpy(), o.pr_in.cpu().numpy()


@pytest.mark.parametrize("B,steps", [(64, 40), (256, 8)])
def test_c5_whole_fly_steady_state_bit_exact(c5, B, steps):
    cfg = c5
    eng = settled_whole_fly(cfg, B)
    print(f"C5 B={B}: tuned LIF {({k: v for k, v in eng.tuned['lif'].items() if k != 'all'})}, "
          f"optic {({k: v for k, v in eng.tuned['optic'].items() if k != 'all'})}")
    o = cfg.optic
    lif = eng.lif
    p = lif.p
    W, _ = lif_weights(eng.lif_connectome, p)
    ptr, edges, mode = out_edges(W, p.w_syn)
    assert mode == lif.ring_mode
    st, v, ad, pr = oracle_from_engine(eng)
    rate0 = float(st.rate.mean())
    assert rate0 > 100.0, rate0                       # steady firing (~220 Hz mean)
    Wr, Wrs, Wsr = o.W_rr(), eng.W_rs_host, eng.W_sr_host
    a = np.exp(-0.1 / o.tau_of_type[o.type_of].astype(np.float32)).astype(np.float32)
    aad = float(np.exp(-0.1 / o.adapt_tau_ms))
    P = lif_coefficients(p, False)
    flags = _abi.LIF_POISSON | _abi.LIF_COUNTS
    g1 = _capture(eng, 1)                             # the bench's graph replay, one step per replay
    words = (lif.n * B + 31) // 32
    ev_gpu0, ev_ora = lif.synaptic_events, 0
    max_drive = 0.0
    for k in range(steps):
        g1.replay()
        torch.cuda.synchronize()
        gpu_drive = lif._st["drive"].cpu().numpy()
        gpu_spk = lif._st["spikes"].cpu().numpy()
        spk = oracle.spmm(Wrs.indptr, Wrs.indices, Wrs.data, st.rate, B, rows=o.m, x_div=100.0, x_lo=0.0, x_hi=3.0,
                          alpha=o.gain_fb)
        oracle.optic_run(v, ad, Wr.indptr, Wr.indices, Wr.data, pr, spk, a, o.b, o.gain_rr, o.adapt_gain, aad, 1)
        dr = (np.clip(v + o.b[:, None], 0, 1) - o.b[:, None]).astype(np.float32)
        oracle.spmm(Wsr.indptr, Wsr.indices, Wsr.data, dr, B, rows=lif.n, y=st.drive, alpha=o.gain_out_mv,
                    y_lo=-o.drive_clip_mv, y_hi=o.drive_clip_mv)
        np.testing.assert_allclose(gpu_drive, st.drive, rtol=1e-4, atol=1e-3)
        max_drive = max(max_drive, float(np.abs(gpu_drive - st.drive).max()))
        st.drive[...] = gpu_drive                     # the LIF sees the same drive on both sides
        r, ev = oracle.lif_run(st, ptr, edges, P, n_delay=lif.n_delay, flags=flags, nsteps=1, seed=1, raster=True)
        ev_ora += ev
        np.testing.assert_array_equal(unpack(r, lif.n * B)[0], gpu_spk.ravel() != 0, err_msg=f"raster @ step {k}")
        assert r.shape[1] == words
    del g1
    eng.lif.check()
    eng.optic.check()
    for name, oname in LIF_STATE:
        np.testing.assert_array_equal(lif._st[name].cpu().numpy(), getattr(st, oname), err_msg=name)
    np.testing.assert_array_equal(lif.ring.cpu().numpy(), st.ring)
    assert lif.synaptic_events - ev_gpu0 == ev_ora > 1_000_000 * steps
    np.testing.assert_allclose(eng.optic.v_s.cpu().numpy(), v, rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(eng.optic.adapt_s.cpu().numpy(), ad, rtol=RTOL, atol=ATOL)
    print(f"C5 B={B}: {steps} steps at {rate0:.0f} Hz mean, {ev_ora / steps:.3e} synaptic events per step, "
          f"max |drive_gpu - drive_oracle| = {max_drive:.3e} mV")
