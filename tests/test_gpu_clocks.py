"""Per-neuron clocks on the GPU: the clocked LIF kernel against the oracle bit for bit (state,
ring, pending input, rasters), the Brain drop-in against the reference's clocked rasters, and the
host bookkeeping (checkpoints, row resets, graph replay, FlyBrain's dt_by_module)."""
import numpy as np
import pytest
import torch

import oracle
from flyb200 import _abi, synthetic
from flyb200.brain import Brain, LIFParams, clock_coefficients
from gpu_helpers import LIF_ARRAYS, native_lif_run
from helpers import connectome_from_fixture, golden, torch_uniforms, unpack
from test_gpu_lif import _abt, case_random

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["count", "fixed-std", "episodes"])
@pytest.mark.parametrize("periods", [(1, 2, 3, 4), (3, 6), (1,)])
def test_clocked_kernel_equals_oracle(kind, periods):
    case = case_random(batch=16, n=3000, edges=60_000, steps=120, fixed=kind == "fixed-std", std=kind == "fixed-std",
                       episodes=kind == "episodes", ext_uniform=kind == "count")
    rng = np.random.default_rng(len(periods))
    period = rng.choice(periods, case["state"].n).astype(np.int64)
    p = LIFParams(adapt_jump=1.5, dt=0.1)
    clocks = (period, clock_coefficients(p, kind == "fixed-std", int(period.max())))
    s_ref, s_gpu = case["state"].copy(), case["state"].copy()
    fs_ref = None if case["fly_steps"] is None else case["fly_steps"].copy()
    fs_gpu = None if fs_ref is None else fs_ref.copy()
    done = 0
    for chunk in (50, 70):                       # two calls: the held input carries over
        kw = dict(n_delay=case["n_delay"], flags=case["flags"], nsteps=chunk, seed=case["seed"], raster=True,
                  clocks=clocks, uniforms=None if case["uniforms"] is None else
                  np.ascontiguousarray(case["uniforms"][done:done + chunk]))
        done += chunk
        r_ref, ev_ref = oracle.lif_run(s_ref, case["ptr"], case["edges"], case["P"], fly_steps=fs_ref, **kw)
        r_gpu, ev_gpu = native_lif_run(s_gpu, case["ptr"], case["edges"], case["P"], fly_steps=fs_gpu,
                                       launch=_abi.LAUNCH_STEP, **kw)
        np.testing.assert_array_equal(r_gpu, r_ref)
        for k in LIF_ARRAYS:
            np.testing.assert_array_equal(getattr(s_gpu, k), getattr(s_ref, k), err_msg=k)
        np.testing.assert_array_equal(s_gpu.ring, s_ref.ring)
        np.testing.assert_array_equal(s_gpu.clock_acc, s_ref.clock_acc)
        assert ev_gpu == ev_ref
    assert unpack(r_ref, s_ref.n * s_ref.batch).sum() > 0
    if max(periods) > 1:
        assert np.abs(s_ref.clock_acc).sum() > 0          # some slow neurons hold input


def test_clocks_reject_deferred_delivery():
    case = case_random(batch=4, n=500, edges=5000, steps=5)
    period = np.full(500, 2, np.int64)
    with pytest.raises(RuntimeError):
        native_lif_run(case["state"].copy(), case["ptr"], case["edges"], case["P"], n_delay=case["n_delay"],
                       flags=case["flags"], nsteps=5, launch=_abi.LAUNCH_STEP, defer=True,
                       clocks=(period, clock_coefficients(LIFParams(), False, 2)))


def test_brain_config1_clocked_equals_reference_golden():
    z = golden("lif_c1_clocks")
    cfg = synthetic.lif_config1(seed=0)
    b = Brain(cfg.c, LIFParams(**cfg.params), device="cuda", seed=0, launch="persistent")
    b.set_clocks(z["clock_period"])
    b.record_activity = True
    b.set_poisson(cfg.poisson_idx, cfg.poisson_hz)
    b.set_drive(np.arange(cfg.c.n), float(z["drive"]))
    U = torch.from_numpy(torch_uniforms(int(z["seed"]), cfg.steps, (1, cfg.c.n))).cuda()
    ras = torch.zeros(cfg.steps, cfg.c.n, dtype=torch.bool, device="cuda")
    for s in range(cfg.steps):
        b.step(1, uniforms=U[s:s + 1])
        ras[s] = b.spikes[0] > 0
    ref = np.unpackbits(z["raster"], axis=1, bitorder="little")[:, : cfg.c.n].astype(bool)
    np.testing.assert_array_equal(ras.cpu().numpy(), ref)
    np.testing.assert_array_equal(b.spike_counts[0].cpu().numpy(), z["spike_counts"])
    np.testing.assert_allclose(b.v[0].cpu().numpy(), z["v"], rtol=0, atol=2e-5)
    b.check()


def test_brain_19cell_clocked_drop_in_equals_reference_golden():
    z = golden("lif_19cell_clocks")
    c = connectome_from_fixture(z)
    B, T = int(z["batch"]), int(z["steps"])
    b = Brain(c, LIFParams(receptor_model=None, adapt_by_type=_abt(z)), device="cuda", seed=int(z["seed"]), batch=B,
              launch="step")
    b.freeze(z["frozen"])
    b.prune(z["frozen"])
    b.set_clocks(z["clock_period"])
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
    for key in ("v", "g", "refrac", "adapt", "res", "rate", "spike_counts"):
        np.testing.assert_allclose(getattr(b, key).cpu().numpy(), z[f"final_{key}"], rtol=1e-5, atol=1e-4, err_msg=key)


def _clocked_brain(batch=4):
    cfg = synthetic.lif_config1(seed=2, n=1500, edges=30_000)
    b = Brain(cfg.c, LIFParams(**cfg.params), device="cuda", seed=9, batch=batch, launch="step")
    b.set_clocks(np.array([1, 2, 3, 6])[np.arange(cfg.c.n) % 4])
    b.record_activity = True
    b.set_poisson(cfg.poisson_idx, 400.0)
    b.set_drive(np.arange(cfg.c.n), 6.9)
    return b


def test_clocked_checkpoint_reset_and_graph_replay():
    a, b = _clocked_brain(), _clocked_brain()
    a.step(41)                 # the last step (40) updates periods 1 and 2 only: 3 and 6 hold input
    saved = a.state_dict()
    assert "clock_acc" in saved and int(saved["clock_acc"].abs().sum()) > 0
    a.step(25)
    b.load_state_dict(saved)
    b.step(25)
    torch.cuda.synchronize()
    for k in ("v", "g", "rate", "spike_counts"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k
    assert torch.equal(a.clock_acc, b.clock_acc)
    a.reset([1])
    assert int(a.clock_acc[:, 1].abs().sum()) == 0 and int(a.clock_acc[:, 0].abs().sum()) > 0
    # a captured chunk of clocked steps replays like eager steps (the phase comes from the device clock)
    c, d = _clocked_brain(), _clocked_brain()
    c.step(3)
    d.step(3)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            c.step(5)
    torch.cuda.current_stream().wait_stream(s)
    for _ in range(4):
        g.replay()
    d.step(20)
    torch.cuda.synchronize()
    for k in ("v", "g", "rate", "spike_counts", "adapt"):
        assert torch.equal(getattr(c, k), getattr(d, k)), k
    assert torch.equal(c.clock_acc, d.clock_acc)
    del g


def test_flybrain_dt_by_module_sets_the_clocks():
    from flyb200.fly import FlyBrain
    from flyb200.optic import OpticParams
    from flyb200.regions import clock_periods, labels
    from test_oracle_golden import hex_lobe
    _, c, r = hex_lobe()
    lp = LIFParams(receptor_model=None, dt=0.5, dt_by_module={"visual_projection": 1.0})
    fb = FlyBrain(c, batch=2, device="cuda", seed=1, retina=r, lif_params=lp, optic_params=OpticParams())
    expect = clock_periods(c, 0.5, {"visual_projection": 1.0})
    np.testing.assert_array_equal(fb.brain._kvec, expect)
    assert set(expect[labels(c) == "visual_projection"]) == {2} and expect.max() == 2
    fb.vision(np.random.default_rng(0).random((r.n_columns, 4)).astype(np.float32))
    fb.step(10.0)
    fb.brain.check()
    with pytest.raises(ValueError, match="unknown module"):
        clock_periods(c, 0.5, {"cortex": 1.0})
