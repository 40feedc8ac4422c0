"""The whole-fly step (LIF + optic coupled every step) on the GPU against the oracle's step in the
same order, on a reduced whole-fly graph; and the autotuner leaves the state untouched."""
import numpy as np
import pytest
import torch

import oracle
from flyb200 import _abi, autotune, synthetic
from flyb200.brain import LIFParams, lif_coefficients, out_edges
from flyb200.weights import lif_weights
from flyb200.whole import WholeFly

pytestmark = pytest.mark.gpu


def small_fly():
    return synthetic.whole_fly_config5(seed=2, n_rate=3000, n_lif=2500, n_sensory=300, edges=700_000,
                                       optic_nnz=200_000, n_pr=300)


@pytest.mark.parametrize("overlap,capped,defer", [(True, False, False), (False, False, False), (True, True, False),
                                                  (True, False, True), (True, False, "staged"), (True, False, "pull"),
                                                  (False, False, "pull"), (True, False, "staged-pull")])
def test_whole_fly_matches_oracle_step_order(overlap, capped, defer):
    """Bit-identical spikes every step whether the undriven LIF neurons update concurrently with
    the optic chain (overlap) or after it, also with a capped persistent optic grid beside capped
    staged LIF blocks, and with pull delivery (32 flies, the ranges' spikes pulled once per step);
    the oracle runs the stages serially on the engine's stored neuron order."""
    cfg = small_fly()
    pull = isinstance(defer, str) and "pull" in defer
    B, T = (32, 120) if pull else (4, 120)
    eng = WholeFly(cfg, B, device="cuda", seed=1, launch="step", overlap=overlap)
    if capped:
        eng.optic.launch, eng.optic.grid = "persistent", 20
        eng.lif.staged, eng.lif.grid = True, 7
        eng.lif._make_args()
    eng.lif.defer = bool(defer) and not pull
    eng.lif.pull = pull
    if defer in ("staged", "staged-pull"):
        eng.lif.staged = True
    eng.lif._make_args()
    assert eng.overlapping == overlap and eng.lif._pull_active() == pull
    a_pr = torch.from_numpy((np.random.default_rng(0).standard_normal((cfg.optic.n_pr, B)) * 0.5).astype(np.float32)).cuda()
    eng.set_photoreceptors(a_pr)
    pr = eng.optic.pr_in.cpu().numpy()
    counts = []
    for _ in range(T):
        eng.step(1)
        counts.append(eng.lif.spike_counts.sum().item())
    # the oracle, same order: spk_in, optic substep, drive, LIF step
    o = cfg.optic
    p = LIFParams(**{**cfg.lif.params, "dt": 0.1})
    W, _ = lif_weights(eng.lif_connectome, p)
    ptr, edges, mode = out_edges(W, p.w_syn)
    n, m = cfg.n_spiking, o.m
    st = oracle.LifState(n, B, 19, mode, p.v_rest)
    st.poisson_p[eng.sensory_idx, :] = np.float32(cfg.lif.poisson_hz) * np.float32(p.dt / 1000.0)
    Wr, Wrs, Wsr = o.W_rr(), eng.W_rs_host, eng.W_sr_host
    a = np.exp(-0.1 / o.tau_of_type[o.type_of].astype(np.float32)).astype(np.float32)
    aad = float(np.exp(-0.1 / o.adapt_tau_ms))
    v, ad = np.zeros((m, B), np.float32), np.zeros((m, B), np.float32)
    ocounts = []
    for _ in range(T):
        spk = oracle.spmm(Wrs.indptr, Wrs.indices, Wrs.data, st.rate, B, rows=m, x_div=100.0, x_lo=0.0, x_hi=3.0,
                          alpha=o.gain_fb)
        oracle.optic_run(v, ad, Wr.indptr, Wr.indices, Wr.data, pr, spk, a, o.b, o.gain_rr, o.adapt_gain, aad, 1)
        dr = (np.clip(v + o.b[:, None], 0, 1) - o.b[:, None]).astype(np.float32)
        oracle.spmm(Wsr.indptr, Wsr.indices, Wsr.data, dr, B, rows=n, y=st.drive, alpha=o.gain_out_mv,
                    y_lo=-o.drive_clip_mv, y_hi=o.drive_clip_mv)
        oracle.lif_run(st, ptr, edges, lif_coefficients(p, False), n_delay=18,
                       flags=_abi.LIF_POISSON | _abi.LIF_COUNTS, nsteps=1, seed=1)
        ocounts.append(float(st.counts.sum()))
    assert ocounts[-1] > 0
    np.testing.assert_array_equal(np.array(counts), np.array(ocounts))          # same spikes every step
    if pull:
        assert eng.lif.synaptic_events > 0
    np.testing.assert_array_equal(eng.lif.spike_counts.t().cpu().numpy(), st.counts)
    np.testing.assert_allclose(eng.optic.v_s.cpu().numpy(), v, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(eng.lif._st["v"].cpu().numpy(), st.v, rtol=0, atol=1e-4)


def test_stored_order_puts_driven_neurons_last():
    cfg = small_fly()
    eng = WholeFly(cfg, 3, device="cuda", seed=1)
    driven = np.unique(cfg.optic.W_sr.tocoo().row)
    assert eng.split % 32 == 0 and eng.split <= cfg.n_spiking - len(driven)
    assert set(eng.lif_position[driven]) <= set(range(eng.split, cfg.n_spiking))
    np.testing.assert_array_equal(np.sort(eng.lif_order), np.arange(cfg.n_spiking))
    np.testing.assert_array_equal(eng.lif_position[eng.lif_order], np.arange(cfg.n_spiking))


@pytest.mark.parametrize("chunk", [2, 3])
def test_graph_replay_equals_eager_steps(chunk):
    """A CUDA graph of `chunk` whole-fly steps replayed back to back gives the bits of eager steps:
    the carried optic dr ends each replay in the buffer it started from (an odd chunk adds a copy)
    and the LIF device clock gives every replay fresh Philox counters and ring slots."""
    cfg = small_fly()
    B = 4
    a_pr = torch.from_numpy((np.random.default_rng(5).standard_normal((cfg.optic.n_pr, B)) * 0.5).astype(np.float32)).cuda()
    engs = []
    for _ in range(2):
        eng = WholeFly(cfg, B, device="cuda", seed=7, launch="step")
        eng.set_photoreceptors(a_pr)
        eng.step(3)
        engs.append(eng)
    graphed, eager = engs
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            graphed.step(chunk)
    torch.cuda.current_stream().wait_stream(s)
    reps = 5
    for _ in range(reps):
        g.replay()
    eager.step(chunk * reps)
    torch.cuda.synchronize()
    graphed.lif.check()
    graphed.optic.check()
    for k in ("v", "g", "rate", "spike_counts", "spikes", "adapt"):
        assert torch.equal(graphed.lif._st[k], eager.lif._st[k]), k
    assert torch.equal(graphed.lif.ring, eager.lif.ring)
    assert torch.equal(graphed.optic.v_s, eager.optic.v_s)
    assert torch.equal(graphed.optic.adapt_s, eager.optic.adapt_s)
    assert torch.equal(graphed.optic.dr_out, eager.optic.dr_out)
    del g


def test_autotuner_keeps_state_and_installs_a_choice():
    cfg = small_fly()
    eng = WholeFly(cfg, 8, device="cuda", seed=3, launch="step")
    eng.step(5)
    before = {k: v.clone() for k, v in eng.lif._st.items()}
    ring = eng.lif.ring.clone()
    choice = autotune.tune_lif(eng.lif, steps=5)
    assert choice["launch"] in ("step", "persistent") and choice["block"] in (128, 256, 512)
    for k, v in before.items():
        assert torch.equal(v, eng.lif._st[k]), k
    assert torch.equal(ring, eng.lif.ring)
    assert autotune.tune_lif(eng.lif) is choice                   # cached per (graph, batch, activity)
    oc = autotune.tune_optic(eng.optic, steps=5)
    assert oc["launch"] in ("step", "persistent")


def test_fly_shards_equal_one_batch_after_argument_rebuilds():
    """The per-rank fly offset (Brain.fly0) keys the Poisson streams by the global fly index and
    survives argument rebuilds (the autotuner's): two 4-fly shards of the spiking population equal
    one 8-fly batch bit for bit."""
    from flyb200.brain import Brain
    cfg = small_fly()
    p = LIFParams(**{**cfg.lif.params, "dt": 0.1})
    hz = torch.as_tensor(cfg.lif.poisson_hz, dtype=torch.float32)
    whole = Brain(cfg.lif.c, p, device="cuda", seed=11, batch=8, launch="step")
    whole.record_activity = True
    whole.set_poisson(cfg.sensory_idx, hz)
    whole.step(80)
    for lo in (0, 4):
        part = Brain(cfg.lif.c, p, device="cuda", seed=11, batch=4, launch="step")
        part.record_activity = True
        part.set_poisson(cfg.sensory_idx, hz)
        part.fly0 = lo
        part._make_args()
        part.items_per_thread = 1                          # another rebuild, as the autotuner does
        part._make_args()
        part.step(80)
        torch.cuda.synchronize()
        assert whole.spike_counts.sum().item() > 0
        assert torch.equal(part.spike_counts, whole.spike_counts[lo:lo + 4])
        assert torch.equal(part._st["v"], whole._st["v"][:, lo:lo + 4])


def test_per_step_inputs_and_readouts_in_one_call():
    """step(n, before, after) installs each step's photoreceptor input and reads each step's rates
    exactly as n separate calls do."""
    cfg = small_fly()
    B = 4
    rng = np.random.default_rng(9)
    frames = torch.from_numpy((rng.standard_normal((5, cfg.optic.n_pr, B)) * 0.4).astype(np.float32)).cuda()
    a, b = (WholeFly(cfg, B, device="cuda", seed=4, launch="step") for _ in range(2))
    seen_a, seen_b = [], []
    a.step(5, before=lambda k: a.set_photoreceptors(frames[k]), after=lambda k: seen_a.append(a.lif.rate.clone()))
    for k in range(5):
        b.set_photoreceptors(frames[k])
        b.step(1)
        seen_b.append(b.lif.rate.clone())
    torch.cuda.synchronize()
    for x, y in zip(seen_a, seen_b):
        assert torch.equal(x, y)
    for k in ("v", "g", "rate", "spike_counts"):
        assert torch.equal(a.lif._st[k], b.lif._st[k]), k
    assert torch.equal(a.optic.v_s, b.optic.v_s)


def test_set_radiance_equals_oracle_photoreceptor_stage():
    """WholeFly.set_radiance: the native photoreceptor stage (its low-pass and adaptation states
    carried frame to frame, the first frame fresh) and the lamina-row product into pr_in, against
    the oracle's stage and a full-matrix product; pr_in stays zero off the lamina rows."""
    from types import SimpleNamespace
    from oracle import frame as oframe
    from flyb200.optic import OpticParams, photoreceptor_cells
    cfg = small_fly()
    o, B = cfg.optic, 4
    eng = WholeFly(cfg, B, device="cuda", seed=7, launch="step")
    has, avg, cell = photoreceptor_cells(o.pr_column, o.pr_family, o.n_col)
    L = SimpleNamespace(sens=o.sens, pr_column=o.pr_column, avg=avg, has=has, pr_cell=cell)
    st = {"I_lp": np.zeros((B, o.n_col * 5), np.float32), "I_mean": np.zeros((B, o.n_col * 5), np.float32),
          "fresh": np.ones(B, bool)}
    M = o.W_rp.tocsr()
    for f in range(4):
        rad = o.grating(7.0 * f, B, seed=f)
        eng.set_radiance(torch.from_numpy(rad).cuda(), 2.0)
        want = oframe.photoreceptor(L, st, rad, 2.0, OpticParams())
        np.testing.assert_allclose(eng.photo.a_pr.cpu().numpy(), want, rtol=1e-5, atol=1e-6)
        pr = oracle.spmm(M.indptr, M.indices, M.data, want, B, rows=M.shape[0], alpha=o.gain_in)
        np.testing.assert_allclose(eng.optic.pr_in.cpu().numpy(), pr, rtol=1e-5, atol=1e-6)
    assert np.abs(want).max() > 0.01
    assert not eng.optic.pr_in[np.flatnonzero(np.diff(M.indptr) == 0)].any()
    # a per-frame buffer leaves the installed input alone until set_photoreceptors
    held = eng.optic.pr_in.clone()
    buf = torch.empty(o.n_pr, B, device="cuda")
    eng.set_radiance(torch.from_numpy(o.grating(40.0, B, seed=9)).cuda(), 2.0, a_pr=buf)
    assert torch.equal(eng.optic.pr_in, held)
    eng.set_photoreceptors(buf)
    assert not torch.equal(eng.optic.pr_in, held)


@pytest.mark.parametrize("B", [32, 64, 128, 256])
@pytest.mark.parametrize("staged", [False, True, "128x2"])
def test_pull_delivery_equals_scatter_at_high_activity(B, staged):
    """Pull delivery against the scatter, bit for bit (state, ring, rasters, synaptic event count),
    on a graph driven into dense firing, at every supported batch width, after the register update,
    the staged update, and the staged update in blocks of 128 threads with 2 items each."""
    from flyb200.brain import Brain
    cfg = synthetic.lif_config2(seed=4, n=4000, edges=600_000, n_poisson=800, poisson_hz=400.0)
    p = LIFParams(**cfg.params)
    brains = []
    for pull in (False, True):
        b = Brain(cfg.c, p, device="cuda", seed=3, batch=B, launch="step")
        b.set_poisson(cfg.poisson_idx, 400.0)
        b.set_drive(np.arange(cfg.c.n), 5.0)
        b.record_activity = True
        b.pull, b.staged = pull, bool(staged)
        if staged == "128x2":
            b.block, b.items_per_thread = 128, 2
        b._make_args()
        assert b._pull_active() == pull
        brains.append(b)
    push, pull = brains
    for chunk in (1, 7, 40):
        push.step(chunk)
        pull.step(chunk)
        torch.cuda.synchronize()
        for k in ("v", "g", "refrac", "rate", "spike_counts", "spikes"):
            assert torch.equal(getattr(push, k), getattr(pull, k)), k
        assert torch.equal(push.ring, pull.ring)
        assert push.synaptic_events == pull.synaptic_events
    assert float(pull.spike_counts.sum()) / (48 * B * cfg.c.n) > 0.005     # dense firing


@pytest.mark.parametrize("B", [32, 64])
def test_pull_delivery_with_wide_count_ranges_equals_scatter(B):
    """Counts whose range inside a chunk needs more than 8 bits (up to +-3,000 synapses per edge)
    take the 16-plane input table instead of the packed entries: pull delivery against the
    scatter, bit for bit (state, ring, synaptic event count)."""
    import scipy.sparse as sp
    from flyb200.brain import Brain, pull_inputs
    cfg = synthetic.lif_config2(seed=5, n=3000, edges=200_000, n_poisson=600, poisson_hz=300.0)
    p = LIFParams(**cfg.params)
    n, w = cfg.c.n, np.float32(p.w_syn)
    rng = np.random.default_rng(7)
    W = sp.random(n, n, density=0.02, random_state=11, format="csr")
    W.data = (rng.integers(-3000, 3001, W.nnz) * w).astype(np.float32)
    W.eliminate_zeros()
    assert pull_inputs(W, w)[4] == 16
    brains = []
    for pull in (False, True):
        b = Brain(cfg.c, p, device="cuda", seed=3, batch=B, launch="step")
        b.set_weights(W)
        b.set_poisson(cfg.poisson_idx, 300.0)
        b.set_drive(np.arange(n), 3.0)
        b.pull, b.staged = pull, True
        b._make_args()
        assert b._pull_active() == pull
        brains.append(b)
    push, pull = brains
    for chunk in (1, 7, 24):
        push.step(chunk)
        pull.step(chunk)
        torch.cuda.synchronize()
        assert pull._pull_planes_n == 16                # the tables are built at the first step
        for k in ("v", "g", "refrac", "rate", "spikes"):
            assert torch.equal(getattr(push, k), getattr(pull, k)), k
        assert torch.equal(push.ring, pull.ring)
        assert push.synaptic_events == pull.synaptic_events
    assert push.synaptic_events > 0


def test_lagged_pull_beside_the_next_step_equals_one_step_per_call():
    """Under pull delivery the whole-fly step delivers each step's spikes on a side stream beside
    the next step (joined before that step's clock advance): ten steps per call, eager or from a
    captured graph, end bit-identical to one step per call (each call joins its last pull)."""
    cfg = small_fly()
    B = 32
    a_pr = torch.from_numpy((np.random.default_rng(2).standard_normal((cfg.optic.n_pr, B)) * 0.5)
                            .astype(np.float32)).cuda()
    engs = []
    for _ in range(3):
        eng = WholeFly(cfg, B, device="cuda", seed=3, launch="step")
        eng.lif.pull, eng.lif.staged = True, True
        eng.lif._make_args()
        eng.set_photoreceptors(a_pr)
        engs.append(eng)
    single, batched, graphed = engs
    for _ in range(40):
        single.step(1)
    for _ in range(4):
        batched.step(10)
    graphed.step(2)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            graphed.step(19)
    torch.cuda.current_stream().wait_stream(s)
    g.replay()
    graphed.step(19)
    torch.cuda.synchronize()
    for eng in (batched, graphed):
        for k in ("v", "g", "rate", "spike_counts", "refrac"):
            assert torch.equal(getattr(single.lif, k), getattr(eng.lif, k)), k
        assert torch.equal(single.lif.ring, eng.lif.ring)
        assert torch.equal(single.optic.v_s, eng.optic.v_s)
    assert single.lif.synaptic_events == batched.lif.synaptic_events > 0
    del g
