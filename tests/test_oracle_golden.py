"""The oracle pinned to the reference: its outputs against fixtures the reference's own CPU code
produced (tests/golden/make_golden.py), and Philox against published known-answer vectors."""
import numpy as np
import pytest

import oracle
from oracle import frame as oframe
from flyb200 import _abi, synthetic
from flyb200.brain import LIFParams, clock_coefficients, lif_coefficients, out_edges
from flyb200.optic import OpticParams, lobe_matrices
from flyb200.retina import build_retina
from flyb200.weights import lif_weights, per_type, DEFAULT_STD_U_BY_TYPE
from helpers import connectome_from_fixture, golden, sha, torch_uniforms, unpack


def test_philox_known_answer_vectors():
    # Random123 philox4x32-10 KAT vectors (counter, key) -> output
    assert list(oracle.philox(0, [0, 0, 0, 0])) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert list(oracle.philox(0xFFFFFFFFFFFFFFFF, [0xFFFFFFFF] * 4)) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert list(oracle.philox(0x299F31D0A4093822, [0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344])) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def _c1_run(regime_seed, drive, ring="auto", period=None):
    cfg = synthetic.lif_config1(seed=0)
    p = LIFParams(**cfg.params)
    W, _ = lif_weights(cfg.c, p)
    ptr, edges, mode = out_edges(W, p.w_syn, ring)
    st = oracle.LifState(cfg.c.n, 1, 19, mode, p.v_rest)
    st.poisson_p[cfg.poisson_idx, 0] = np.float32(cfg.poisson_hz) * np.float32(p.dt / 1000.0)
    st.drive[:] = np.float32(drive)
    U = torch_uniforms(regime_seed, cfg.steps, (1, cfg.c.n))
    flags = _abi.LIF_POISSON | _abi.LIF_EXT_UNIFORM | _abi.LIF_COUNTS
    clocks = None
    if period is not None:
        clocks = (period, clock_coefficients(p, False, int(period.max())))
    r, ev = oracle.lif_run(st, ptr, edges, lif_coefficients(p, False), n_delay=18, flags=flags, nsteps=cfg.steps,
                           uniforms=U.transpose(0, 2, 1), raster=True, clocks=clocks)
    return cfg, st, unpack(r, cfg.c.n), U, mode


def test_lif_config1_clocked_matches_reference():
    """Config 1 with per-neuron clocks of 1, 2 and 4 steps: the exact count ring against the
    reference's clocked sparse-matmul step, rasters bit for bit."""
    z = golden("lif_c1_clocks")
    cfg, st, ras, U, mode = _c1_run(int(z["seed"]), float(z["drive"]), period=z["clock_period"])
    assert mode == _abi.RING_COUNT
    assert sha(U) == str(z["uniform_sha"])
    ref = np.unpackbits(z["raster"], axis=1, bitorder="little")[:, : cfg.c.n].astype(bool)
    assert ras.sum() > 500
    np.testing.assert_array_equal(ras, ref)
    np.testing.assert_array_equal(st.counts[:, 0], z["spike_counts"])
    np.testing.assert_allclose(st.v[:, 0], z["v"], rtol=0, atol=2e-5)
    np.testing.assert_allclose(st.g[:, 0], z["g"], rtol=0, atol=2e-5)


@pytest.mark.parametrize("regime", ["poisson", "drive65", "drive72"])
def test_lif_config1_count_ring_matches_reference(regime):
    z = golden("lif_c1")
    cfg = synthetic.lif_config1(seed=0)
    assert sha(cfg.c.W.data) + sha(cfg.c.W.indices) + sha(cfg.c.W.indptr) == str(z["W_sha"])
    cfg, st, ras, U, mode = _c1_run(int(z[f"{regime}_seed"]), float(z[f"{regime}_drive"]))
    assert mode == _abi.RING_COUNT
    assert sha(U) == str(z[f"{regime}_uniform_sha"])
    ref = np.unpackbits(z[f"{regime}_raster"], axis=1, bitorder="little")[:, : cfg.c.n].astype(bool)
    assert ras.sum() > 0
    np.testing.assert_array_equal(ras, ref)                       # bit-exact spike rasters
    np.testing.assert_array_equal(st.counts[:, 0], z[f"{regime}_spike_counts"])
    # the integer ring sums counts exactly; the reference sums float products in event order
    np.testing.assert_allclose(st.v[:, 0], z[f"{regime}_v"], rtol=0, atol=2e-5)
    np.testing.assert_allclose(st.g[:, 0], z[f"{regime}_g"], rtol=0, atol=2e-5)
    np.testing.assert_allclose(st.rate[:, 0], z[f"{regime}_rate"], rtol=1e-6, atol=1e-3)


def test_lif_config1_fixed_ring_matches_reference():
    z = golden("lif_c1")
    cfg, st, ras, _, mode = _c1_run(int(z["drive65_seed"]), float(z["drive65_drive"]), ring="fixed")
    assert mode == _abi.RING_FIXED
    ref = np.unpackbits(z["drive65_raster"], axis=1, bitorder="little")[:, : cfg.c.n].astype(bool)
    np.testing.assert_array_equal(ras, ref)
    np.testing.assert_allclose(st.v[:, 0], z["drive65_v"], rtol=0, atol=2e-5)


def _nineteen(name="lif_19cell"):
    z = golden(name)
    c = connectome_from_fixture(z)
    abt = dict(zip(z["adapt_patterns"].tolist(), z["adapt_values"].tolist())) if "adapt_patterns" in z else None
    p = LIFParams(receptor_model=None, adapt_by_type=abt)
    return z, c, p


def test_lif_19cell_weights_identical_to_reference():
    z, c, p = _nineteen()
    W, _ = lif_weights(c, p)
    keep = np.ones(c.n, np.float32)
    keep[z["frozen"]] = 0
    import scipy.sparse as sp
    W = (sp.diags(keep) @ W @ sp.diags(keep)).tocsr()
    W.eliminate_zeros()
    np.testing.assert_array_equal(W.indptr, z["shaped_indptr"])
    np.testing.assert_array_equal(W.indices, z["shaped_indices"])
    np.testing.assert_array_equal(W.data, z["shaped_data"])        # float32 bit for bit


@pytest.mark.parametrize("fixture", ["lif_19cell", "lif_19cell_adapt_by_type"])
def test_lif_19cell_rasters_match_reference(fixture):
    """Default model constants: fan-in scale, cap, gains, adaptation, depression on ORNs -> Q32.32 ring;
    and the same with per-type adaptation jumps (adapt_by_type)."""
    z, c, p = _nineteen(fixture)
    import scipy.sparse as sp
    W = sp.csr_matrix((z["shaped_data"], z["shaped_indices"], z["shaped_indptr"]), shape=(c.n, c.n))
    u = per_type(c, DEFAULT_STD_U_BY_TYPE, p.std_u)
    ptr, edges, mode = out_edges(W, p.w_syn, "auto", std_on=True)
    assert mode == _abi.RING_FIXED
    B, T, n = int(z["batch"]), int(z["steps"]), c.n
    st = oracle.LifState(n, B, 5, mode, p.v_rest)        # dt 0.5: D = round(1.8 / 0.5) = 4
    st.active[z["frozen"]] = 0
    st.std_u[:] = u
    dtp = np.float32(p.dt / 1000.0)
    st.poisson_p[z["orn"], 0], st.poisson_p[z["orn"], 1] = np.float32(120.0) * dtp, np.float32(40.0) * dtp
    st.poisson_p[z["jo"], 0] = np.array([90.0, 10.0], np.float32) * dtp
    st.poisson_p[z["jo"], 1] = np.array([0.0, 150.0], np.float32) * dtp
    st.drive[z["dnp01"], 0] = 12.0
    U = torch_uniforms(int(z["seed"]), T, (B, n))
    assert sha(U) == str(z["uniform_sha"])
    flags = _abi.LIF_POISSON | _abi.LIF_EXT_UNIFORM | _abi.LIF_COUNTS | _abi.LIF_ADAPT | _abi.LIF_STD | _abi.LIF_SKIP_FROZEN
    jumps = None
    if p.adapt_by_type:
        jumps = per_type(c, p.adapt_by_type, p.adapt_jump)
        np.testing.assert_array_equal(jumps, z["adapt_jump_vec"])              # the reference's per-neuron jumps
    r, _ = oracle.lif_run(st, ptr, edges, lif_coefficients(p, True, True), n_delay=4, flags=flags, nsteps=T,
                          uniforms=U.transpose(0, 2, 1), raster=True, adapt_jump=jumps)
    ras = unpack(r, n * B).reshape(T, n, B).transpose(0, 2, 1)
    assert ras.sum() > 20
    np.testing.assert_array_equal(ras, z["raster"])
    for key, mine in (("v", st.v), ("g", st.g), ("refrac", st.refrac), ("adapt", st.adapt), ("res", st.res),
                      ("rate", st.rate), ("spike_counts", st.counts)):
        np.testing.assert_allclose(mine.T, z[f"final_{key}"], rtol=1e-5, atol=1e-4, err_msg=key)


def test_optic_substeps_match_reference_substep():
    """FP32 oracle vs the reference's own _substep on a synthetic lobe (1e-5 relative)."""
    z = golden("optic_synth")
    cfg = synthetic.optic_config3(seed=int(z["seed"]), m=int(z["m"]), nnz=int(z["nnz"]), n_pr=int(z["n_pr"]),
                                  n_types=int(z["n_types"]), n_spk=int(z["n_spk"]))
    W = cfg.W_rr()
    assert sha(W.data) + sha(W.indices) == str(z["W_sha"])
    v, ad = np.ascontiguousarray(z["v0"].T), np.ascontiguousarray(z["adapt0"].T)
    pr, spk = np.ascontiguousarray(z["pr"].T), np.ascontiguousarray(z["spk"].T)
    done = 0
    v64, ad64 = v.astype(np.float64), ad.astype(np.float64)
    for k, s in enumerate(z["snap"]):
        oracle.optic_run(v, ad, W.indptr, W.indices, W.data, pr, spk, cfg.a, cfg.b, 1.0, 1.0, float(z["aad"]), s + 1 - done)
        oracle.optic_run_f64(v64, ad64, W.indptr, W.indices, W.data, pr, spk, cfg.a, cfg.b, 1.0, 1.0, float(z["aad"]),
                             s + 1 - done)
        done = s + 1
        ref = z["v"][k].T
        np.testing.assert_allclose(v, ref, rtol=1e-5, atol=1e-6)
        assert np.abs(v64 - ref).max() < 1e-4                       # FP32 reference vs FP64 restatement
    np.testing.assert_allclose(ad, z["adapt"].T, rtol=1e-5, atol=1e-6)


def hex_lobe():
    z = golden("optic_hex")
    c = connectome_from_fixture(z, extra=())
    c.neurons["hex1"], c.neurons["hex2"], c.neurons["hex_side"] = z["hex1"], z["hex2"], z["hex_side"]
    c.neurons["hex_side"] = c.neurons.hex_side.replace("", None)
    r = build_retina(c)
    np.testing.assert_array_equal(r.pr_index, z["pr_index"])
    np.testing.assert_array_equal(r.pr_column, z["pr_column"])
    np.testing.assert_array_equal(r.pr_sens, z["pr_sens"])
    assert r.n_columns == int(z["n_columns"])
    return z, c, r


def test_optic_hex_frames_match_reference():
    z, c, r = hex_lobe()
    p = OpticParams()
    L = lobe_matrices(c, r, p)
    np.testing.assert_array_equal(L.rate_idx, z["rate_idx"])
    np.testing.assert_array_equal(L.spk_idx, z["spk_idx"])
    B = 2
    st = {"v": np.zeros((len(L.rate_idx), B), np.float32), "adapt": np.zeros((len(L.rate_idx), B), np.float32),
          "I_lp": np.zeros((B, r.n_columns * 5), np.float32), "I_mean": np.zeros((B, r.n_columns * 5), np.float32),
          "fresh": np.ones(B, bool), "pending": 0.0}
    for f in range(3):
        drive = oframe.frame(L, st, z[f"frame{f}_rad"], z[f"frame{f}_spk"], 10.0, p)
        np.testing.assert_allclose(st["contrast"], z[f"frame{f}_contrast"], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(st["v"].T, z[f"frame{f}_v"], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(st["adapt"].T, z[f"frame{f}_adapt"], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(st["delta"].T, z[f"frame{f}_delta_rate"], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(drive, z[f"frame{f}_drive"], rtol=1e-5, atol=1e-4)


def test_lif_19cell_clocked_rasters_match_reference():
    """Per-neuron clocks (periods 1/2/3 steps): the oracle's clocked step against the reference's
    Brain.set_clocks run (its sparse-matmul path), rasters bit for bit."""
    z, c, p = _nineteen("lif_19cell_clocks")
    import scipy.sparse as sp
    W = sp.csr_matrix((z["shaped_data"], z["shaped_indices"], z["shaped_indptr"]), shape=(c.n, c.n))
    u = per_type(c, DEFAULT_STD_U_BY_TYPE, p.std_u)
    ptr, edges, mode = out_edges(W, p.w_syn, "auto", std_on=True)
    B, T, n = int(z["batch"]), int(z["steps"]), c.n
    st = oracle.LifState(n, B, 5, mode, p.v_rest)
    st.active[z["frozen"]] = 0
    st.std_u[:] = u
    dtp = np.float32(p.dt / 1000.0)
    st.poisson_p[z["orn"], 0], st.poisson_p[z["orn"], 1] = np.float32(120.0) * dtp, np.float32(40.0) * dtp
    st.poisson_p[z["jo"], 0] = np.array([90.0, 10.0], np.float32) * dtp
    st.poisson_p[z["jo"], 1] = np.array([0.0, 150.0], np.float32) * dtp
    st.drive[z["dnp01"], 0] = 12.0
    U = torch_uniforms(int(z["seed"]), T, (B, n))
    assert sha(U) == str(z["uniform_sha"])
    flags = _abi.LIF_POISSON | _abi.LIF_EXT_UNIFORM | _abi.LIF_COUNTS | _abi.LIF_ADAPT | _abi.LIF_STD | _abi.LIF_SKIP_FROZEN
    period = z["clock_period"]
    table = clock_coefficients(p, True, int(period.max()))
    r, _ = oracle.lif_run(st, ptr, edges, lif_coefficients(p, True, True), n_delay=4, flags=flags, nsteps=T,
                          uniforms=U.transpose(0, 2, 1), raster=True, clocks=(period, table))
    ras = unpack(r, n * B).reshape(T, n, B).transpose(0, 2, 1)
    assert ras.sum() > 20
    np.testing.assert_array_equal(ras, z["raster"])
    for key, mine in (("v", st.v), ("g", st.g), ("refrac", st.refrac), ("adapt", st.adapt), ("res", st.res),
                      ("rate", st.rate), ("spike_counts", st.counts)):
        np.testing.assert_allclose(mine.T, z[f"final_{key}"], rtol=1e-5, atol=1e-4, err_msg=key)


def slow_case(mode, clocks=False):
    """The 19-cell slow-tone fixture (with `clocks`, the clocked one): connectome, parameters, the
    receptor record it was built from, and the shaped fast and slow matrices the reference held
    after pruning."""
    import scipy.sparse as sp
    from flyb200.weights import ReceptorSigns
    z = golden(f"lif_19cell_clocks_slow_{mode}" if clocks else f"lif_19cell_slow_{mode}")
    c = connectome_from_fixture(z)
    p = LIFParams(receptor_model="full", slow_gain_by_class={"metabotropic_classical": 0.5}, slow_mode=mode)
    rec = ReceptorSigns(fast_sign=z["rec_fast_sign"], slow_sign=z["rec_slow_sign"], fast_gain=z["rec_fast_gain"],
                        slow_gain=z["rec_slow_gain"], count=z["rec_count"], slow_class=z["rec_slow_class"])
    W = sp.csr_matrix((z["shaped_data"], z["shaped_indices"], z["shaped_indptr"]), shape=(c.n, c.n))
    S = {k: sp.csr_matrix((z[f"slow_{k}_data"], z[f"slow_{k}_indices"], z[f"slow_{k}_indptr"]), shape=(c.n, c.n))
         for k in z["slow_classes"].tolist()}
    return z, c, p, rec, W, S


@pytest.mark.parametrize("clocks", [False, True], ids=["plain", "clocked"])
@pytest.mark.parametrize("mode", ["additive", "gain", "threshold"])
def test_lif_19cell_slow_tone_matches_reference(mode, clocks):
    """receptor_model="full": the shaped fast and slow matrices are the reference's bit for bit, and
    the oracle's step with the slow tone reproduces its rasters in every slow_mode, also under
    per-neuron clocks of 1, 2 and 3 steps (the reference's clocked step, brain.py:898-957)."""
    import math
    import scipy.sparse as sp
    from flyb200.weights import slow_spec, slow_weights
    z, c, p, rec, W_ref, S_ref = slow_case(mode, clocks)
    W, scale = lif_weights(c, p, rec)
    keep = np.ones(c.n, np.float32)
    keep[z["frozen"]] = 0
    W = (sp.diags(keep) @ W @ sp.diags(keep)).tocsr()
    W.eliminate_zeros()
    np.testing.assert_array_equal(W.data, W_ref.data)
    spec = slow_spec(p)
    S = slow_weights(c, p, rec, spec, scale)
    assert list(S) == list(S_ref) == spec.classes
    for k in S:
        Sk = (sp.diags(keep) @ S[k] @ sp.diags(keep)).tocsr()
        Sk.eliminate_zeros()
        np.testing.assert_array_equal(Sk.toarray(), S_ref[k].toarray(), err_msg=k)
    assert sum(Sk.nnz for Sk in S_ref.values()) > 0
    u = per_type(c, DEFAULT_STD_U_BY_TYPE, p.std_u)
    ptr, edges, mode_r = out_edges(W_ref, p.w_syn, "auto", std_on=True)
    B, T, n = int(z["batch"]), int(z["steps"]), c.n
    st = oracle.LifState(n, B, 5, mode_r, p.v_rest)
    st.active[z["frozen"]] = 0
    st.std_u[:] = u
    dtp = np.float32(p.dt / 1000.0)
    st.poisson_p[z["orn"], 0], st.poisson_p[z["orn"], 1] = np.float32(120.0) * dtp, np.float32(40.0) * dtp
    st.poisson_p[z["jo"], 0] = np.array([90.0, 10.0], np.float32) * dtp
    st.poisson_p[z["jo"], 1] = np.array([0.0, 150.0], np.float32) * dtp
    st.drive[z["dnp01"], 0] = 12.0
    U = torch_uniforms(int(z["seed"]), T, (B, n))
    assert sha(U) == str(z["uniform_sha"])
    classes = []
    for k, Sk in S_ref.items():
        sptr, sedges, smode = out_edges(Sk, p.w_syn, "fixed")
        classes.append((sptr, sedges, math.exp(-p.dt / spec.tau[k])))
    slow = {"mode": mode, "norm": spec.norm_mv, "clip": spec.clip, "th_max": float(np.float32(0.9 * spec.norm_mv)),
            "classes": classes}
    flags = _abi.LIF_POISSON | _abi.LIF_EXT_UNIFORM | _abi.LIF_COUNTS | _abi.LIF_ADAPT | _abi.LIF_STD | _abi.LIF_SKIP_FROZEN
    ck = None
    if clocks:
        period = z["clock_period"]
        ck = (period, clock_coefficients(p, True, int(period.max()), [spec.tau[k] for k in S_ref]))
    r, _ = oracle.lif_run(st, ptr, edges, lif_coefficients(p, True, True), n_delay=4, flags=flags, nsteps=T,
                          uniforms=U.transpose(0, 2, 1), raster=True, slow=slow, clocks=ck)
    ras = unpack(r, n * B).reshape(T, n, B).transpose(0, 2, 1)
    np.testing.assert_array_equal(ras, z["raster"])
    for key, mine in (("v", st.v), ("g", st.g), ("adapt", st.adapt), ("res", st.res), ("rate", st.rate),
                      ("spike_counts", st.counts), ("g_slow", st.g_slow)):
        np.testing.assert_allclose(mine.T, z[f"final_{key}"], rtol=1e-5, atol=1e-4, err_msg=key)
    assert np.abs(st.g_slow).max() > 1.0


def optic_slow_case(mode):
    """The hex patch under the slow receptor tone: fixture, lobe matrices with the receptor record,
    the slow description for the oracle and its initial state."""
    from flyb200.optic import slow_blocks
    from flyb200.weights import ReceptorSigns, receptor_gain, slow_spec
    _, c, r = hex_lobe()
    z = golden(f"optic_hex_slow_{mode}")
    rec = ReceptorSigns(fast_sign=z["rec_fast_sign"], slow_sign=z["rec_slow_sign"], fast_gain=z["rec_fast_gain"],
                        slow_gain=z["rec_slow_gain"], count=z["rec_count"], slow_class=z["rec_slow_class"])
    lp = LIFParams(receptor_model="full", slow_gain_by_class={"metabotropic_classical": 2.0}, slow_mode=mode)
    p = OpticParams()
    L = lobe_matrices(c, r, p, rec, receptor_gain(lp))
    spec = slow_spec(lp)
    blocks, norm = slow_blocks(c, L.rate_idx, L.spk_idx, p, rec, receptor_gain(lp), spec)
    slow = {"mode": mode, "norm": norm, "clip": spec.clip, "classes": blocks}
    return z, c, r, rec, lp, p, L, slow


@pytest.mark.parametrize("mode", ["additive", "gain", "threshold"])
def test_optic_slow_tone_frames_match_reference(mode):
    """The optic lobe's slow receptor tone (optic.py:526-551): three frames from a displaced start,
    every state within 1e-5 of the reference's OpticLobe."""
    z, c, r, rec, lp, p, L, slow = optic_slow_case(mode)
    B, m, K = 2, len(L.rate_idx), len(slow["classes"])
    st = {"v": np.ascontiguousarray(z["v0"].T), "adapt": np.zeros((m, B), np.float32),
          "I_lp": np.zeros((B, r.n_columns * 5), np.float32), "I_mean": np.zeros((B, r.n_columns * 5), np.float32),
          "fresh": np.ones(B, bool), "pending": 0.0, "g_cls": np.zeros((K, m, B), np.float32),
          "g_slow": np.zeros((m, B), np.float32), "held": np.zeros((K, m, B), np.float32)}
    for f in range(3):
        drive = oframe.frame(L, st, z[f"frame{f}_rad"], z[f"frame{f}_spk"], 10.0, p, slow=slow)
        np.testing.assert_allclose(st["v"].T, z[f"frame{f}_v"], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(st["adapt"].T, z[f"frame{f}_adapt"], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(st["g_slow"].T, z[f"frame{f}_g_slow"], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(st["g_cls"].transpose(0, 2, 1), z[f"frame{f}_g_slow_cls"], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(st["delta"].T, z[f"frame{f}_delta_rate"], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(drive, z[f"frame{f}_drive"], rtol=1e-5, atol=1e-4)
    assert np.abs(st["g_slow"]).max() > 0.5


HOOK_CASES = {      # the OpticParams of tests/golden/make_golden.py's optic_hex_hooks_{case} fixtures
    "rectify": dict(stream_rectify=[("Mi1", "T3", "pos"), ("Mi1", "Pm1", "abs")]),
    "adapt": dict(stream_adapt=[("Mi1", "T3|Pm1", 15.0, 0.8)]),
    "suppress": dict(spatial_suppress=[("Mi1", 0.6, 6.0)]),
    "all": dict(stream_rectify=[("Mi1", "T3", "neg"), ("T3", "LC11", "abs")], stream_adapt=[("Mi1", ".*", 25.0, 0.5)],
                spatial_suppress=[("Mi1", 0.4, 6.0)]),
}


def optic_hooks_case(case):
    """The hex patch with the per-stream hooks of HOOK_CASES[case]: fixture, lobe matrices, hook blocks."""
    from flyb200.optic import stream_hooks
    _, c, r = hex_lobe()
    z = golden(f"optic_hex_hooks_{case}")
    p = OpticParams(**HOOK_CASES[case])
    L = lobe_matrices(c, r, p)
    return z, c, r, p, L, stream_hooks(c, r, L.rate_idx, L.spk_idx, p, L.M_rr, L.M_sr)


@pytest.mark.parametrize("case", list(HOOK_CASES))
def test_optic_hook_blocks_match_reference(case):
    """The stream split and the spatial operator: per stream the rule pair and its entry counts, the
    rest blocks and G's entries, against the reference lobe's own hook record."""
    z, c, r, p, L, h = optic_hooks_case(case)
    info = eval(str(z["hook_info"]), {"__builtins__": {}}, {"True": True, "False": False, "None": None})
    assert len(h.streams) == len(info["streams"])
    rect, adapt = p.stream_rectify or [], p.stream_adapt or []
    for s, ref in zip(h.streams, info["streams"]):
        assert s["mode"] == (ref["rect"][2] if ref["rect"] else None)
        assert (list(adapt[s["adapt_id"]]) if s["adapt_id"] >= 0 else None) == ref["adapt"]
        for which, key in (("W_rr", "rate_to_rate"), ("W_sr", "rate_to_spiking")):
            assert (s[which].nnz if s[which] is not None else None) == (ref[key]["entries"] if ref[key] else None)
            if s[which] is not None:
                assert abs(float(np.abs(s[which].data).sum()) - ref[key]["syn_eq"]) < 1e-5
    assert (h.matched("rr"), h.rest_rr.nnz) == (info["entries_rr_matched"], info["entries_rr_rest"])
    assert (h.matched("sr"), h.rest_sr.nnz) == (info["entries_sr_matched"], info["entries_sr_rest"])
    if "spatial" in info:
        assert h.G.nnz == info["spatial"]["G_nnz"]
        assert [(e["pre"], e["k"], e["radius_deg"]) for e in info["spatial"]["entries"]] == \
            [tuple(x) for x in p.spatial_suppress]
    else:
        assert h.G is None
    assert {tuple(x["rect"]) for x in info["streams"] if x["rect"]} <= {tuple(x) for x in rect}


@pytest.mark.parametrize("case", list(HOOK_CASES))
def test_optic_hook_frames_match_reference(case):
    """The per-stream hooks (optic.py:453-495, 526-551): three frames of the hex patch, every state
    within 1e-5 of the reference's OpticLobe, the drive within 1e-4 mV."""
    z, c, r, p, L, h = optic_hooks_case(case)
    B, m = 2, len(L.rate_idx)
    st = {"v": np.zeros((m, B), np.float32), "adapt": np.zeros((m, B), np.float32),
          "I_lp": np.zeros((B, r.n_columns * 5), np.float32), "I_mean": np.zeros((B, r.n_columns * 5), np.float32),
          "fresh": np.ones(B, bool), "pending": 0.0, "A": np.zeros((len(p.stream_adapt or []), m, B), np.float32)}
    for f in range(3):
        drive = oframe.frame(L, st, z[f"frame{f}_rad"], z[f"frame{f}_spk"], 10.0, p, hooks=h)
        np.testing.assert_allclose(st["v"].T, z[f"frame{f}_v"], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(st["adapt"].T, z[f"frame{f}_adapt"], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(st["A"].transpose(0, 2, 1), z[f"frame{f}_stream_adapt_state"], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(st["delta"].T, z[f"frame{f}_delta_rate"], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(drive, z[f"frame{f}_drive"], rtol=1e-5, atol=1e-4)
    assert np.abs(z["frame2_drive"]).max() > 0


def test_optic_hooks_reject_bad_rules():
    from flyb200.optic import stream_hooks
    _, c, r = hex_lobe()
    for kw in (dict(stream_rectify=[("Mi1", "T3", "half")]), dict(stream_adapt=[("Mi1", "T3", 0.0, 1.0)])):
        p = OpticParams(**kw)
        L = lobe_matrices(c, r, p)
        with pytest.raises(ValueError):
            stream_hooks(c, r, L.rate_idx, L.spk_idx, p, L.M_rr, L.M_sr)
