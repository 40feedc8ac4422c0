"""GPU parity of the fused LIF step: the native kernel against the oracle, bit for bit, and the
Brain drop-in against the reference's golden rasters. All calls go through the C ABI."""
import ctypes as ct

import numpy as np
import pytest
import scipy.sparse as sp
import torch

import oracle
from flyb200 import _abi, synthetic
from flyb200.brain import Brain, LIFParams, lif_coefficients, out_edges
from flyb200.weights import DEFAULT_STD_U_BY_TYPE, lif_weights, per_type
from gpu_helpers import LIF_ARRAYS, native_lif_run, native_lif_run_split
from helpers import connectome_from_fixture, golden, torch_uniforms, unpack

pytestmark = pytest.mark.gpu

STEP, PERS = _abi.LAUNCH_STEP, _abi.LAUNCH_PERSISTENT


def case_c1(ring="auto", regime_seed=1, drive=6.5):
    cfg = synthetic.lif_config1(seed=0)
    p = LIFParams(**cfg.params)
    W, _ = lif_weights(cfg.c, p)
    ptr, edges, mode = out_edges(W, p.w_syn, ring)
    st = oracle.LifState(cfg.c.n, 1, 19, mode, p.v_rest)
    st.poisson_p[cfg.poisson_idx, 0] = np.float32(cfg.poisson_hz) * np.float32(p.dt / 1000.0)
    st.drive[:] = np.float32(drive)
    U = torch_uniforms(regime_seed, cfg.steps, (1, cfg.c.n)).transpose(0, 2, 1)
    flags = _abi.LIF_POISSON | _abi.LIF_EXT_UNIFORM | _abi.LIF_COUNTS
    return dict(state=st, ptr=ptr, edges=edges, P=lif_coefficients(p, False), n_delay=18, flags=flags,
                nsteps=cfg.steps, uniforms=np.ascontiguousarray(U))


def _abt(z):
    """The fixture's adapt_by_type map, or None."""
    return dict(zip(z["adapt_patterns"].tolist(), z["adapt_values"].tolist())) if "adapt_patterns" in z else None


def case_19cell(fixture="lif_19cell"):
    z = golden(fixture)
    c = connectome_from_fixture(z)
    p = LIFParams(receptor_model=None, adapt_by_type=_abt(z))
    W = sp.csr_matrix((z["shaped_data"], z["shaped_indices"], z["shaped_indptr"]), shape=(c.n, c.n))
    ptr, edges, mode = out_edges(W, p.w_syn, "auto", std_on=True)
    B, T = int(z["batch"]), int(z["steps"])
    st = oracle.LifState(c.n, B, 5, mode, p.v_rest)
    st.active[z["frozen"]] = 0
    st.std_u[:] = per_type(c, DEFAULT_STD_U_BY_TYPE, p.std_u)
    dtp = np.float32(p.dt / 1000.0)
    st.poisson_p[z["orn"], 0], st.poisson_p[z["orn"], 1] = np.float32(120.0) * dtp, np.float32(40.0) * dtp
    st.poisson_p[z["jo"], 0] = np.array([90.0, 10.0], np.float32) * dtp
    st.poisson_p[z["jo"], 1] = np.array([0.0, 150.0], np.float32) * dtp
    st.drive[z["dnp01"], 0] = 12.0
    U = torch_uniforms(int(z["seed"]), T, (B, c.n)).transpose(0, 2, 1)
    flags = (_abi.LIF_POISSON | _abi.LIF_EXT_UNIFORM | _abi.LIF_COUNTS | _abi.LIF_ADAPT | _abi.LIF_STD |
             _abi.LIF_SKIP_FROZEN)
    jumps = per_type(c, p.adapt_by_type, p.adapt_jump) if p.adapt_by_type else None
    return dict(state=st, ptr=ptr, edges=edges, P=lif_coefficients(p, True, True), n_delay=4, flags=flags, nsteps=T,
                uniforms=np.ascontiguousarray(U), adapt_jump=jumps)


def case_random(batch=64, n=3000, edges=60_000, steps=200, episodes=False, fixed=False, seed=3, std=False,
                ext_uniform=False):
    rng = np.random.default_rng(seed)
    pre, post = rng.integers(0, n, edges), rng.integers(0, n, edges)
    sign = np.where(rng.random(n) < 0.65, 1.0, -1.0).astype(np.float32)
    W = sp.csr_matrix((rng.geometric(0.25, edges).astype(np.float32) * sign[pre] * np.float32(0.275), (post, pre)),
                      shape=(n, n), dtype=np.float32)
    p = LIFParams(conn_cap=0.0, input_norm_alpha=0.0, path_gain=[], type_path_gain=[], same_type_gain=1.0,
                  adapt_jump=1.5, receptor_model=None, dt=0.1)
    ptr, e, mode = out_edges(W, p.w_syn, "fixed" if (fixed or std) else "auto", std_on=std)
    st = oracle.LifState(n, batch, 19, mode, p.v_rest)
    st.poisson_p[rng.choice(n, n // 10, replace=False), :] = rng.uniform(0.002, 0.02, (n // 10, batch)).astype(np.float32)
    st.drive[:] = rng.uniform(5.0, 7.5, (n, batch)).astype(np.float32)
    st.active[rng.choice(n, n // 20, replace=False)] = 0.0
    flags = _abi.LIF_POISSON | _abi.LIF_COUNTS | _abi.LIF_ADAPT | _abi.LIF_SKIP_FROZEN
    fs = None
    if episodes:
        flags |= _abi.LIF_EPISODES
        fs = rng.integers(0, steps + 1, batch).astype(np.int32)
    if std:
        flags |= _abi.LIF_STD
        st.std_u[:] = rng.uniform(0.1, 0.5, n).astype(np.float32)
    uni = None
    if ext_uniform:
        flags |= _abi.LIF_EXT_UNIFORM
        uni = rng.random((steps, n, batch), dtype=np.float32)
    return dict(state=st, ptr=ptr, edges=e, P=lif_coefficients(p, std), n_delay=18, flags=flags, nsteps=steps,
                uniforms=uni, fly_steps=fs, seed=12345)


def _compare(case, launch, block, grid=0, ipt=0, with_sync=True, staged=0, defer=False):
    s_ref, s_gpu = case["state"].copy(), case["state"].copy()
    fs_ref = None if case.get("fly_steps") is None else case["fly_steps"].copy()
    fs_gpu = None if fs_ref is None else fs_ref.copy()
    kw = dict(n_delay=case["n_delay"], flags=case["flags"], nsteps=case["nsteps"], seed=case.get("seed", 0),
              uniforms=case["uniforms"], raster=True, adapt_jump=case.get("adapt_jump"))
    r_ref, ev_ref = oracle.lif_run(s_ref, case["ptr"], case["edges"], case["P"], fly_steps=fs_ref, **kw)
    r_gpu, ev_gpu = native_lif_run(s_gpu, case["ptr"], case["edges"], case["P"], fly_steps=fs_gpu, launch=launch,
                                   block=block, grid=grid, items_per_thread=ipt, with_sync=with_sync, staged=staged,
                                   defer=defer, **kw)
    assert unpack(r_ref, s_ref.n * s_ref.batch).sum() > 0
    np.testing.assert_array_equal(r_gpu, r_ref)                      # spike rasters
    for k in LIF_ARRAYS:
        np.testing.assert_array_equal(getattr(s_gpu, k), getattr(s_ref, k), err_msg=k)   # every state bit
    np.testing.assert_array_equal(s_gpu.ring, s_ref.ring)
    assert ev_gpu == ev_ref
    if fs_ref is not None:
        np.testing.assert_array_equal(fs_gpu, fs_ref)


@pytest.mark.parametrize("launch", [STEP, PERS])
@pytest.mark.parametrize("ring", ["auto", "fixed"])
def test_config1_native_equals_oracle(launch, ring):
    _compare(case_c1(ring), launch, 256)


@pytest.mark.parametrize("launch,block", [(STEP, 128), (PERS, 256), (PERS, 512)])
@pytest.mark.parametrize("fixture", ["lif_19cell", "lif_19cell_adapt_by_type"])
def test_19cell_depression_adaptation_native_equals_oracle(launch, block, fixture):
    _compare(case_19cell(fixture), launch, block)


@pytest.mark.parametrize("launch,block,grid", [(STEP, 256, 0), (PERS, 256, 0), (PERS, 128, 7), (PERS, 512, 0)])
def test_batched_philox_native_equals_oracle(launch, block, grid):
    _compare(case_random(batch=64), launch, block, grid)


@pytest.mark.parametrize("ipt", [1, 2, 4])
@pytest.mark.parametrize("launch,batch", [(STEP, 64), (PERS, 64), (STEP, 3)])
def test_items_per_thread_variants_equal_oracle(ipt, launch, batch):
    _compare(case_random(batch=batch, steps=100), launch, 256, ipt=ipt)


@pytest.mark.parametrize("block,ipt", [(256, 2), (256, 4), (128, 2), (512, 4)])
@pytest.mark.parametrize("kind", ["count", "fixed", "episodes"])
def test_staged_step_equals_oracle(block, ipt, kind):
    """The bulk-copy (staged) per-step kernel: every state bit, ring, raster and event count equal
    the oracle, in both ring modes and with uneven episodes; chunks end mid-array (n * batch is not
    a multiple of the chunk)."""
    case = case_random(batch=20, n=2999, steps=80, fixed=kind == "fixed", episodes=kind == "episodes")
    _compare(case, STEP, block, ipt=ipt, staged=1)


@pytest.mark.parametrize("block,ipt", [(256, 1), (256, 2), (128, 4), (512, 2)])
@pytest.mark.parametrize("kind", ["count", "fixed", "episodes"])
def test_deferred_delivery_equals_oracle(block, ipt, kind):
    """Spikes listed by the update kernel (one entry per 1024 out-edges) and delivered by the
    scatter kernel: every state bit, ring, raster and event count equal the oracle."""
    case = case_random(batch=20, n=2999, steps=80, fixed=kind == "fixed", episodes=kind == "episodes")
    _compare(case, STEP, block, ipt=ipt, defer=True)


@pytest.mark.parametrize("block,ipt", [(256, 2), (512, 2), (256, 4), (128, 2)])
@pytest.mark.parametrize("kind", ["count", "fixed", "episodes"])
def test_staged_deferred_delivery_equals_oracle(block, ipt, kind):
    """The staged (bulk-copy) update listing its spikers for the scatter kernel: every state bit,
    ring, raster and event count equal the oracle."""
    case = case_random(batch=20, n=2999, steps=80, fixed=kind == "fixed", episodes=kind == "episodes")
    _compare(case, STEP, block, ipt=ipt, staged=1, defer=True)


def test_deferred_delivery_splits_high_out_degree_spikers():
    """A hub with more out-edges than one list entry covers (and uneven batch 3) still delivers
    every edge once."""
    case = case_random(batch=3, n=3000, edges=60_000, steps=60)
    rng = np.random.default_rng(11)
    ptr, e = case["ptr"].copy(), case["edges"].copy()
    hub_extra = 5000                                   # neuron 0 gets 5000 more targets
    w = 1 if case["state"].ring_mode == _abi.RING_COUNT else int(np.float32(0.275).view(np.int32))
    extra = np.stack([rng.integers(0, 3000, hub_extra), np.full(hub_extra, w, np.int64)], 1).astype(np.int32)
    e = np.concatenate([e[: ptr[1]], extra, e[ptr[1]:]]).astype(np.int32)
    ptr = np.concatenate([[0], ptr[1:] + hub_extra]).astype(np.int32)
    case["ptr"], case["edges"] = ptr, e
    case["state"].poisson_p[0, :] = 0.5                # the hub fires often
    _compare(case, STEP, 256, ipt=1, defer=True)


def test_staged_request_falls_back_when_unaligned():
    """n * batch % 4 != 0: the staged request runs the register path, same results."""
    _compare(case_random(batch=3, n=2999, steps=60), STEP, 256, staged=1)


def test_staged_depression_and_external_uniforms():
    _compare(case_random(batch=8, n=2999, steps=60, std=True, ext_uniform=True), STEP, 256, ipt=2, staged=1)
    _compare(case_random(batch=8, n=2999, steps=60, std=True), STEP, 256, ipt=4, staged=1)


def test_depression_random_graph_register_paths():
    for launch in (STEP, PERS):
        _compare(case_random(batch=8, n=2999, steps=60, std=True, ext_uniform=True), launch, 256)


@pytest.mark.parametrize("staged,ipt,defer", [(0, 4, False), (0, 1, False), (1, 2, False), (1, 4, False),
                                              (0, 2, True)])
@pytest.mark.parametrize("kind", ["count", "fixed-episodes"])
def test_neuron_ranges_on_two_streams_equal_oracle(staged, ipt, defer, kind):
    """Each step as two neuron ranges launched on overlapping streams (FLYB_LIF_NO_ADVANCE), then
    flyb_lif_advance: every state bit, ring, raster and event count equal the oracle's whole steps."""
    case = case_random(batch=8, n=2999, steps=60, fixed=kind != "count", episodes=kind != "count")
    s_ref, s_gpu = case["state"].copy(), case["state"].copy()
    fs_ref = None if case.get("fly_steps") is None else case["fly_steps"].copy()
    fs_gpu = None if fs_ref is None else fs_ref.copy()
    kw = dict(n_delay=case["n_delay"], flags=case["flags"], nsteps=case["nsteps"], seed=case["seed"])
    r_ref, ev_ref = oracle.lif_run(s_ref, case["ptr"], case["edges"], case["P"], fly_steps=fs_ref, raster=True, **kw)
    r_gpu, ev_gpu = native_lif_run_split(s_gpu, case["ptr"], case["edges"], case["P"], split=1504, fly_steps=fs_gpu,
                                         items_per_thread=ipt, staged=staged, defer=defer, **kw)
    np.testing.assert_array_equal(r_gpu, r_ref)
    for k in LIF_ARRAYS:
        np.testing.assert_array_equal(getattr(s_gpu, k), getattr(s_ref, k), err_msg=k)
    np.testing.assert_array_equal(s_gpu.ring, s_ref.ring)
    assert ev_gpu == ev_ref
    if fs_ref is not None:
        np.testing.assert_array_equal(fs_gpu, fs_ref)


def test_neuron_range_must_start_on_a_raster_word():
    case = case_random(batch=3, n=200, steps=2)
    with pytest.raises(RuntimeError, match="1001"):
        native_lif_run_split(case["state"].copy(), case["ptr"], case["edges"], case["P"], split=7,
                             n_delay=case["n_delay"], flags=case["flags"], nsteps=1)


@pytest.mark.parametrize("batch", [1, 3, 33])
def test_uneven_batches_and_fixed_ring(batch):
    _compare(case_random(batch=batch, fixed=True, steps=120), PERS, 256)


@pytest.mark.parametrize("launch,with_sync", [(STEP, True), (STEP, False), (PERS, True)])
def test_uneven_episodes_native_equals_oracle(launch, with_sync):
    """Episode counters gate the update and are lowered after the run; per-step launches need no
    sync words."""
    _compare(case_random(batch=16, steps=150, episodes=True), launch, 256, with_sync=with_sync)


def test_sharded_flies_equal_one_batch():
    """Flies split across calls with fly0 offsets draw the same Philox streams as one batch."""
    whole = case_random(batch=8, steps=80)
    s_all = whole["state"].copy()
    r_all, _ = native_lif_run(s_all, whole["ptr"], whole["edges"], whole["P"], n_delay=18, flags=whole["flags"],
                              nsteps=80, seed=whole["seed"], raster=True)
    for lo, hi in ((0, 3), (3, 8)):
        part = whole["state"].copy()
        for k in LIF_ARRAYS:
            setattr(part, k, np.ascontiguousarray(getattr(part, k)[:, lo:hi]))
        part.batch = hi - lo
        part.ring = np.ascontiguousarray(part.ring[:, :, lo:hi])
        native_lif_run(part, whole["ptr"], whole["edges"], whole["P"], n_delay=18, flags=whole["flags"], nsteps=80,
                       seed=whole["seed"], fly0=lo)
        for k in LIF_ARRAYS:
            np.testing.assert_array_equal(getattr(part, k), getattr(s_all, k)[:, lo:hi], err_msg=k)


# ------------------------------------------------------------------ the Brain drop-in
def test_brain_config1_rasters_equal_reference_golden():
    z = golden("lif_c1")
    cfg = synthetic.lif_config1(seed=0)
    for regime in ("poisson", "drive65", "drive72"):
        b = Brain(cfg.c, LIFParams(**cfg.params), device="cuda", seed=0)
        assert b.ring_mode == _abi.RING_COUNT
        b.record_activity = True
        b.set_poisson(cfg.poisson_idx, cfg.poisson_hz)
        b.set_drive(np.arange(cfg.c.n), float(z[f"{regime}_drive"]))
        U = torch.from_numpy(torch_uniforms(int(z[f"{regime}_seed"]), cfg.steps, (1, cfg.c.n))).cuda()
        ras = torch.zeros(cfg.steps, cfg.c.n, dtype=torch.bool, device="cuda")
        for s in range(cfg.steps):
            b.step(1, uniforms=U[s:s + 1])
            ras[s] = b.spikes[0] > 0
        ref = np.unpackbits(z[f"{regime}_raster"], axis=1, bitorder="little")[:, : cfg.c.n].astype(bool)
        np.testing.assert_array_equal(ras.cpu().numpy(), ref, err_msg=regime)
        np.testing.assert_array_equal(b.spike_counts[0].cpu().numpy(), z[f"{regime}_spike_counts"])
        np.testing.assert_allclose(b.v[0].cpu().numpy(), z[f"{regime}_v"], rtol=0, atol=2e-5)
        b.check()


@pytest.mark.parametrize("fixture", ["lif_19cell", "lif_19cell_adapt_by_type"])
def test_brain_19cell_drop_in_equals_reference_golden(fixture):
    z = golden(fixture)
    c = connectome_from_fixture(z)
    B, T = int(z["batch"]), int(z["steps"])
    b = Brain(c, LIFParams(receptor_model=None, adapt_by_type=_abt(z)), device="cuda", seed=int(z["seed"]), batch=B,
              launch="step")
    b.freeze(z["frozen"])
    b.prune(z["frozen"])
    b.record_activity = True
    b.set_poisson(z["orn"], torch.tensor([[120.0], [40.0]]))
    b.set_poisson(z["jo"], torch.tensor([[90.0, 10.0], [0.0, 150.0]]))
    b.set_drive(z["dnp01"], torch.tensor([[12.0], [0.0]]))
    W = b._W_cpu
    np.testing.assert_array_equal(W.data, z["shaped_data"])
    U = torch.from_numpy(torch_uniforms(int(z["seed"]), T, (B, c.n))).cuda()
    ras = []
    for s in range(T):
        b.step(1, uniforms=U[s:s + 1])
        ras.append((b.spikes > 0).cpu().numpy())
    np.testing.assert_array_equal(np.stack(ras), z["raster"])
    for key in ("v", "g", "refrac", "adapt", "res", "rate", "spike_counts"):
        np.testing.assert_allclose(getattr(b, key).cpu().numpy(), z[f"final_{key}"], rtol=1e-5, atol=1e-4, err_msg=key)


def _fresh_brain(launch="persistent", batch=4):
    cfg = synthetic.lif_config1(seed=2, n=1500, edges=30_000)
    b = Brain(cfg.c, LIFParams(**cfg.params), device="cuda", seed=9, batch=batch, launch=launch)
    b.record_activity = True
    b.set_poisson(cfg.poisson_idx, 400.0)
    b.set_drive(np.arange(cfg.c.n), 6.9)
    return b


@pytest.mark.parametrize("launch", ["step", "persistent"])
def test_brain_cuda_graph_replay_equals_eager(launch):
    eager, graphed = _fresh_brain(launch), _fresh_brain(launch)
    eager.step(5)
    graphed.step(5)                              # warm
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            graphed.step(10)
    torch.cuda.current_stream().wait_stream(s)
    # capture does not run the kernels; the device clock still reads step 5
    for _ in range(3):
        g.replay()
        eager.step(10)
    torch.cuda.synchronize()
    for k in ("v", "g", "refrac", "rate", "spike_counts", "spikes", "adapt"):
        torch.testing.assert_close(getattr(graphed, k), getattr(eager, k), rtol=0, atol=0, msg=k)
    assert torch.equal(graphed.ring, eager.ring)
    assert int(graphed._clock[0]) == int(eager._clock[0]) == 35


def test_brain_spike_buf_round_trip_and_row_reset():
    a = _fresh_brain()
    a.step(23)
    sb = a.spike_buf.clone()
    b = _fresh_brain()
    b.load_state_dict(a.state_dict())
    b.load_spike_buf(sb, buf_pos=a.step_count % a.n_delay)      # rebuild the ring from the buffer
    a.step(17)
    b.step(17)
    torch.testing.assert_close(b.v, a.v, rtol=0, atol=0)
    assert torch.equal(b.ring, a.ring)
    a.reset([1, 3])
    assert torch.all(a.v[[1, 3]] == a.p.v_rest) and torch.all(a.ring[:, :, [1, 3]] == 0)
    assert torch.all(a.res[[1, 3]] == 1.0)


def test_set_weights_mid_run_reapplies_pending_spikes():
    """Pending deliveries follow the new weights, as the reference's spike buffer would."""
    a, b = _fresh_brain(), _fresh_brain()
    a.step(7)
    b.step(7)
    W = a._W_cpu.copy()
    W.data *= 2
    a.set_weights(W)
    assert a.ring_mode == _abi.RING_COUNT
    sb = b.spike_buf
    b.set_weights(W)
    assert torch.equal(a.ring, b.ring)
    c = _fresh_brain()
    c.load_state_dict(b.state_dict())
    c.set_weights(W)
    c.load_spike_buf(sb, buf_pos=b.step_count % b.n_delay)
    assert torch.equal(c.ring, b.ring)


def test_bounded_wait_reports_instead_of_hanging():
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    rc = _abi.lib().flyb_selftest_wait(flag.data_ptr(), status.data_ptr(), 20_000, torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    torch.cuda.synchronize()
    assert status[0].item() == _abi.EBARRIER and status[1].item() == 2


def test_invalid_arguments_rejected_without_launch():
    a = _abi.LifArgs(n=10, batch=1, n_delay=5, ring_slots=5)       # R must exceed D
    assert _abi.lib().flyb_lif_run(ct.byref(a), None) == _abi.EINVAL
    with pytest.raises(ValueError):
        Brain(synthetic.lif_config1(seed=0).c, LIFParams(receptor_model=None), device="cpu")
