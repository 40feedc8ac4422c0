"""The slow receptor tone (receptor_model "full") on the GPU: the extended LIF kernel against the
oracle bit for bit (state, rings, per-class and summed tone, rasters) on a random graph in every
slow_mode, and the Brain drop-in against the reference's rasters."""
import math

import numpy as np
import pytest
import scipy.sparse as sp
import torch

import oracle
from flyb200 import _abi
from flyb200.brain import Brain, LIFParams, out_edges
from gpu_helpers import LIF_ARRAYS, native_lif_run
from helpers import torch_uniforms, unpack
from test_gpu_lif import case_random
from test_oracle_golden import slow_case

pytestmark = pytest.mark.gpu


def random_slow(n, mode, seed=5, entries=40_000):
    """Two slow classes over random synapses (signed, 0.01-0.2 mV per spike), decays of 100 and
    200 ms at dt 0.1 ms, the reference's normalisation and clip."""
    rng = np.random.default_rng(seed)
    classes = []
    for c, tau in enumerate((100.0, 200.0)):
        pre, post = rng.integers(0, n, entries), rng.integers(0, n, entries)
        w = (rng.uniform(0.01, 0.2, entries) * np.where(rng.random(entries) < 0.7, 1, -1)).astype(np.float32)
        S = sp.csr_matrix((w, (post, pre)), shape=(n, n))
        ptr, edges, _ = out_edges(S, 0.275, "fixed")
        classes.append((ptr, edges, math.exp(-0.1 / tau)))
    return {"mode": mode, "norm": 7.0, "clip": (0.0, 4.0), "th_max": float(np.float32(0.9 * 7.0)), "classes": classes}


@pytest.mark.parametrize("mode", ["additive", "gain", "threshold"])
@pytest.mark.parametrize("kind", ["count", "fixed-std"])
def test_slow_tone_kernel_equals_oracle(mode, kind):
    case = case_random(batch=8, n=3000, edges=60_000, steps=100, fixed=kind == "fixed-std", std=kind == "fixed-std")
    slow = random_slow(3000, mode)
    s_ref, s_gpu = case["state"].copy(), case["state"].copy()
    for chunk in (40, 60):
        kw = dict(n_delay=case["n_delay"], flags=case["flags"], nsteps=chunk, seed=case["seed"], raster=True,
                  slow=slow)
        r_ref, ev_ref = oracle.lif_run(s_ref, case["ptr"], case["edges"], case["P"], **kw)
        r_gpu, ev_gpu = native_lif_run(s_gpu, case["ptr"], case["edges"], case["P"], launch=_abi.LAUNCH_PERSISTENT,
                                       **kw)
        np.testing.assert_array_equal(r_gpu, r_ref)
        for k in LIF_ARRAYS:
            np.testing.assert_array_equal(getattr(s_gpu, k), getattr(s_ref, k), err_msg=k)
        np.testing.assert_array_equal(s_gpu.ring, s_ref.ring)
        np.testing.assert_array_equal(s_gpu.slow_ring, s_ref.slow_ring)
        np.testing.assert_array_equal(s_gpu.slow_g, s_ref.slow_g)
        np.testing.assert_array_equal(s_gpu.g_slow, s_ref.g_slow)
        assert ev_gpu == ev_ref
    assert unpack(r_ref, s_ref.n * s_ref.batch).sum() > 0
    assert np.abs(s_ref.g_slow).max() > 0.1


@pytest.mark.parametrize("mode", ["additive", "gain", "threshold"])
@pytest.mark.parametrize("kind", ["count", "fixed-std"])
def test_clocked_slow_tone_kernel_equals_oracle(mode, kind):
    """Clocks and the slow tone together: per-class phase decays and per-class pending input, bit
    for bit against the oracle over two calls (the held slow input carries over)."""
    from flyb200.brain import clock_coefficients
    case = case_random(batch=8, n=3000, edges=60_000, steps=100, fixed=kind == "fixed-std", std=kind == "fixed-std")
    slow = random_slow(3000, mode)
    p = LIFParams(adapt_jump=1.5, dt=0.1)
    period = np.random.default_rng(3).choice([1, 2, 3, 6], 3000).astype(np.int64)
    clocks = (period, clock_coefficients(p, kind == "fixed-std", 6, (100.0, 200.0)))
    s_ref, s_gpu = case["state"].copy(), case["state"].copy()
    for chunk in (41, 59):
        kw = dict(n_delay=case["n_delay"], flags=case["flags"], nsteps=chunk, seed=case["seed"], raster=True,
                  slow=slow, clocks=clocks)
        r_ref, ev_ref = oracle.lif_run(s_ref, case["ptr"], case["edges"], case["P"], **kw)
        r_gpu, ev_gpu = native_lif_run(s_gpu, case["ptr"], case["edges"], case["P"], launch=_abi.LAUNCH_STEP, **kw)
        np.testing.assert_array_equal(r_gpu, r_ref)
        for k in LIF_ARRAYS:
            np.testing.assert_array_equal(getattr(s_gpu, k), getattr(s_ref, k), err_msg=k)
        for k in ("ring", "clock_acc", "slow_ring", "slow_g", "g_slow", "slow_clock_acc"):
            np.testing.assert_array_equal(getattr(s_gpu, k), getattr(s_ref, k), err_msg=k)
        assert ev_gpu == ev_ref
    assert np.abs(s_ref.slow_clock_acc).sum() > 0        # slow input held between updates
    assert np.abs(s_ref.g_slow).max() > 0.1


@pytest.mark.parametrize("clocks", [False, True], ids=["plain", "clocked"])
@pytest.mark.parametrize("mode", ["additive", "gain", "threshold"])
def test_brain_slow_tone_drop_in_equals_reference_golden(mode, clocks):
    z, c, p, rec, W_ref, S_ref = slow_case(mode, clocks)
    B, T = int(z["batch"]), int(z["steps"])
    b = Brain(c, p, device="cuda", seed=int(z["seed"]), batch=B, launch="step", receptor=rec)
    b.freeze(z["frozen"])
    b.prune(z["frozen"])
    if clocks:
        b.set_clocks(z["clock_period"])
    np.testing.assert_array_equal(b._W_cpu.data, z["shaped_data"])
    for k, Sk in S_ref.items():
        np.testing.assert_array_equal(b._W_slow_cpu[k].toarray(), Sk.toarray(), err_msg=k)
    b.record_activity = True
    b.set_poisson(z["orn"], torch.tensor([[120.0], [40.0]]))
    b.set_poisson(z["jo"], torch.tensor([[90.0, 10.0], [0.0, 150.0]]))
    b.set_drive(z["dnp01"], torch.tensor([[12.0], [0.0]]))
    U = torch.from_numpy(torch_uniforms(int(z["seed"]), T, (B, c.n))).cuda()
    ras = []
    for s in range(T):
        b.step(1, uniforms=U[s:s + 1])
        ras.append((b.spikes > 0).cpu().numpy())
    np.testing.assert_array_equal(np.stack(ras), z["raster"])
    for key in ("v", "g", "adapt", "res", "rate", "spike_counts", "g_slow"):
        np.testing.assert_allclose(getattr(b, key).cpu().numpy(), z[f"final_{key}"], rtol=1e-5, atol=1e-4, err_msg=key)
    # checkpoint round trip and a row reset with the tone
    saved = b.state_dict()
    b.step(20)
    after = {k: getattr(b, k).clone() for k in ("v", "g_slow", "rate")}
    b.load_state_dict(saved)
    b.step(20)
    for k, v in after.items():
        assert torch.equal(getattr(b, k), v), k
    if clocks:
        assert "slow_clock_acc" in saved
    b.reset([1])
    assert float(b.g_slow[1].abs().sum()) == 0.0 and float(b.g_slow_cls[:, 1].abs().sum()) == 0.0
    if clocks:
        assert int(b.slow_clock_acc[:, :, 1].abs().sum()) == 0


@pytest.mark.parametrize("mode", ["additive", "gain", "threshold"])
def test_optic_slow_tone_equals_reference_golden(mode):
    """OpticLobe with the slow receptor tone (the unit update kernel after the recurrent and slow
    products) against the reference's frames, and the state survives a FlyBrain-style checkpoint
    of its tensors."""
    from flyb200.optic import OpticLobe
    from flyb200.weights import receptor_gain, slow_spec
    from test_oracle_golden import optic_slow_case
    z, c, r, rec, lp, p, L, slow = optic_slow_case(mode)
    ol = OpticLobe(c, r, p, device="cuda", batch=2, receptor=rec, receptor_gain=receptor_gain(lp), slow=slow_spec(lp),
                   launch="step")
    ol.relax()
    ol.v = torch.from_numpy(z["v0"]).cuda()
    for f in range(3):
        drive = ol.step_frame(torch.from_numpy(z[f"frame{f}_rad"]), torch.from_numpy(z[f"frame{f}_spk"]).cuda(), 10.0)
        for key in ("v", "adapt", "g_slow", "delta_rate"):
            np.testing.assert_allclose(getattr(ol, key).cpu().numpy(), z[f"frame{f}_{key}"], rtol=1e-5, atol=1e-6,
                                       err_msg=f"{key} frame {f}")
        np.testing.assert_allclose(ol.g_slow_cls.cpu().numpy(), z[f"frame{f}_g_slow_cls"], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(drive.cpu().numpy(), z[f"frame{f}_drive"], rtol=1e-5, atol=1e-4)
    assert float(ol.g_slow.abs().max()) > 0.5
    ol.reset([1])
    assert float(ol.g_slow[1].abs().sum()) == 0.0 and float(ol.g_slow_cls[:, 1].abs().sum()) == 0.0


def test_flybrain_full_receptor_model_runs_both_tones():
    """FlyBrain under receptor_model="full": the brain and the optic lobe both carry the tone, and a
    checkpoint restores it."""
    from flyb200.fly import FlyBrain
    from test_oracle_golden import optic_slow_case
    z, c, r, rec, lp, p, L, slow = optic_slow_case("additive")
    lp = LIFParams(receptor_model="full", slow_gain_by_class={"metabotropic_classical": 2.0}, dt=0.5)
    fb = FlyBrain(c, batch=2, device="cuda", seed=3, retina=r, lif_params=lp, optic_params=p, receptor=rec)
    assert fb.brain.slow is not None and fb.optic.slow is not None
    fb.optic.v = torch.from_numpy(z["v0"]).cuda()
    fb.vision(z["frame0_rad"][0])
    fb.step(10.0)
    saved = fb.state_dict()
    fb.step(10.0)
    after = (fb.optic.g_slow.clone(), fb.optic.v.clone(), fb.brain.v.clone())
    fb.load_state_dict(saved)
    fb.step(10.0)
    assert torch.equal(fb.optic.g_slow, after[0]) and torch.equal(fb.optic.v, after[1]) and torch.equal(fb.brain.v, after[2])
    assert float(fb.optic.g_slow.abs().max()) > 0
