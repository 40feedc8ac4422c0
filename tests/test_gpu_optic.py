"""GPU parity of the optic lobe: fused substeps against the FP32 oracle (1e-5 relative), the
OpticLobe drop-in against the reference's frames, the held-input products, and the
reference-compatible launchers against the reference's own test expressions."""
from types import SimpleNamespace

import numpy as np
import pytest
import scipy.sparse as sp
import torch

import oracle
from flyb200 import cuda as fcuda
from flyb200 import synthetic
from flyb200.optic import DeviceCSR, OpticCore, OpticLobe, OpticParams, spmm
from helpers import golden
from test_oracle_golden import hex_lobe

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-5, 1e-6


def small_optic(seed=4, m=4000, nnz=300_000):
    return synthetic.optic_config3(seed=seed, m=m, nnz=nnz, n_pr=360, n_types=80, n_spk=700)


@pytest.mark.parametrize("batch", [1, 2, 5, 32, 64, 100, 256])
@pytest.mark.parametrize("launch", ["step", "persistent"])
def test_fused_substeps_match_oracle(batch, launch):
    cfg = small_optic()
    W = cfg.W_rr()
    rng = np.random.default_rng(batch)
    v = (rng.standard_normal((cfg.m, batch)) * 0.3).astype(np.float32)
    ad = (rng.standard_normal((cfg.m, batch)) * 0.05).astype(np.float32)
    pr = (rng.standard_normal((cfg.m, batch)) * 0.3).astype(np.float32)
    spk = (rng.standard_normal((cfg.m, batch)) * 0.1).astype(np.float32)
    core = OpticCore(W, cfg.a, cfg.b, batch=batch, device="cuda", gain_rr=cfg.gain_rr, adapt_gain=cfg.adapt_gain,
                     aad=cfg.aad, launch=launch)
    core.v_s.copy_(torch.from_numpy(v))
    core.adapt_s.copy_(torch.from_numpy(ad))
    core.pr_in.copy_(torch.from_numpy(pr))
    core.spk_in.copy_(torch.from_numpy(spk))
    T = 40
    vh = torch.zeros(T, cfg.m, batch, device="cuda")
    ih = torch.zeros(T, cfg.m, batch, device="cuda")
    core.substeps(T, vh, ih)
    torch.cuda.synchronize()
    core.check()
    ovh, oih = oracle.optic_run(v, ad, W.indptr, W.indices, W.data, pr, spk, cfg.a, cfg.b, cfg.gain_rr,
                                cfg.adapt_gain, cfg.aad, T, history=True)
    np.testing.assert_allclose(core.v_s.cpu().numpy(), v, rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(core.adapt_s.cpu().numpy(), ad, rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(vh.cpu().numpy(), ovh, rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(ih.cpu().numpy(), oih, rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("batch,variant", [(1, 1), (1, 2), (1, 3), (1, 4), (64, 1), (64, 2), (64, 3), (64, 4),
                                           (64, 5), (100, 1), (100, 3), (48, 3), (256, 1), (256, 3), (256, 5),
                                           (200, 3)])
@pytest.mark.parametrize("launch", ["step", "persistent"])
def test_kernel_shape_variants_match_oracle(batch, variant, launch):
    """Every kernel shape the autotuner may pick (flyb_optic_args.variant) against the FP32 oracle."""
    cfg = small_optic(seed=8)
    W = cfg.W_rr()
    rng = np.random.default_rng(variant)
    v = (rng.standard_normal((cfg.m, batch)) * 0.3).astype(np.float32)
    ad = (rng.standard_normal((cfg.m, batch)) * 0.05).astype(np.float32)
    pr = (rng.standard_normal((cfg.m, batch)) * 0.3).astype(np.float32)
    spk = (rng.standard_normal((cfg.m, batch)) * 0.1).astype(np.float32)
    core = OpticCore(W, cfg.a, cfg.b, batch=batch, device="cuda", gain_rr=cfg.gain_rr, adapt_gain=cfg.adapt_gain,
                     aad=cfg.aad, launch=launch)
    core.variant = variant
    core.v_s.copy_(torch.from_numpy(v))
    core.adapt_s.copy_(torch.from_numpy(ad))
    core.pr_in.copy_(torch.from_numpy(pr))
    core.spk_in.copy_(torch.from_numpy(spk))
    core.substeps(20)
    torch.cuda.synchronize()
    core.check()
    oracle.optic_run(v, ad, W.indptr, W.indices, W.data, pr, spk, cfg.a, cfg.b, cfg.gain_rr, cfg.adapt_gain, cfg.aad, 20)
    np.testing.assert_allclose(core.v_s.cpu().numpy(), v, rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(core.adapt_s.cpu().numpy(), ad, rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("batch", [1, 64])
@pytest.mark.parametrize("launch", ["step", "persistent"])
def test_every_long_row_threshold_matches_oracle(batch, launch):
    """The autotuner's long-row thresholds (and the extremes: every non-empty row split across a
    block, none split) against the FP32 oracle; changing the threshold keeps the row-order buffer."""
    from flyb200.autotune import OPTIC_LONG_ROWS
    cfg = small_optic(seed=12)
    W = cfg.W_rr()
    rng = np.random.default_rng(batch)
    v = (rng.standard_normal((cfg.m, batch)) * 0.3).astype(np.float32)
    ad = (rng.standard_normal((cfg.m, batch)) * 0.05).astype(np.float32)
    pr = (rng.standard_normal((cfg.m, batch)) * 0.3).astype(np.float32)
    spk = (rng.standard_normal((cfg.m, batch)) * 0.1).astype(np.float32)
    ov, oad = v.copy(), ad.copy()
    oracle.optic_run(ov, oad, W.indptr, W.indices, W.data, pr, spk, cfg.a, cfg.b, cfg.gain_rr, cfg.adapt_gain,
                     cfg.aad, 20)
    core = OpticCore(W, cfg.a, cfg.b, batch=batch, device="cuda", gain_rr=cfg.gain_rr, adapt_gain=cfg.adapt_gain,
                     aad=cfg.aad, launch=launch)
    rows = core.rows
    deg = np.diff(W.indptr)
    for long_row in (0, 16) + tuple(OPTIC_LONG_ROWS) + (1 << 30,):
        core.set_long_rows(long_row)
        assert core.rows is rows and core.n_long == int((deg > long_row).sum())
        core.v_s.copy_(torch.from_numpy(v))
        core.adapt_s.copy_(torch.from_numpy(ad))
        core.pr_in.copy_(torch.from_numpy(pr))
        core.spk_in.copy_(torch.from_numpy(spk))
        core.substeps(20)
        torch.cuda.synchronize()
        core.check()
        np.testing.assert_allclose(core.v_s.cpu().numpy(), ov, rtol=RTOL, atol=ATOL, err_msg=f"long_row {long_row}")
        np.testing.assert_allclose(core.adapt_s.cpu().numpy(), oad, rtol=RTOL, atol=ATOL)


def test_single_carried_persistent_substeps_with_a_block_cap_equal_step_launches():
    """One substep on a carried dr is an ordinary launch of a capped grid looping over the rows:
    bit-identical to one launch per substep."""
    cfg = small_optic(seed=9)
    W = cfg.W_rr()
    B = 64
    rng = np.random.default_rng(4)
    v0 = (rng.standard_normal((cfg.m, B)) * 0.3).astype(np.float32)
    pr = (rng.standard_normal((cfg.m, B)) * 0.3).astype(np.float32)
    cores = []
    for launch, grid in (("step", 0), ("persistent", 37)):
        core = OpticCore(W, cfg.a, cfg.b, batch=B, device="cuda", gain_rr=cfg.gain_rr, adapt_gain=cfg.adapt_gain,
                         aad=cfg.aad, launch=launch)
        core.grid = grid
        core.v_s.copy_(torch.from_numpy(v0))
        core.pr_in.copy_(torch.from_numpy(pr))
        for _ in range(7):
            core.substeps(1, carry=True)
        torch.cuda.synchronize()
        core.check()
        cores.append(core)
    assert torch.equal(cores[0].v_s, cores[1].v_s)
    assert torch.equal(cores[0].adapt_s, cores[1].adapt_s)
    assert torch.equal(cores[0].dr_out, cores[1].dr_out)


def test_unknown_kernel_shape_is_rejected():
    cfg = small_optic(seed=8)
    core = OpticCore(cfg.W_rr(), cfg.a, cfg.b, batch=8, device="cuda", gain_rr=cfg.gain_rr,
                     adapt_gain=cfg.adapt_gain, aad=cfg.aad, launch="step")
    core.variant = 3                     # batch widths 2-32 have one shape only
    with pytest.raises(RuntimeError, match="1001"):
        core.substeps(1)


def test_fp64_error_of_fp32_substeps_is_small():
    cfg = small_optic(seed=5)
    W = cfg.W_rr()
    rng = np.random.default_rng(0)
    B, T = 4, 200
    v = (rng.standard_normal((cfg.m, B)) * 0.3).astype(np.float32)
    ad = np.zeros((cfg.m, B), np.float32)
    pr = (rng.standard_normal((cfg.m, B)) * 0.3).astype(np.float32)
    spk = np.zeros((cfg.m, B), np.float32)
    core = OpticCore(W, cfg.a, cfg.b, batch=B, device="cuda", gain_rr=1.0, adapt_gain=1.0, aad=cfg.aad)
    core.v_s.copy_(torch.from_numpy(v))
    core.pr_in.copy_(torch.from_numpy(pr))
    core.substeps(T)
    v64, ad64 = v.astype(np.float64), ad.astype(np.float64)
    oracle.optic_run_f64(v64, ad64, W.indptr, W.indices, W.data, pr, spk, cfg.a, cfg.b, 1.0, 1.0, cfg.aad, T)
    r_gpu = np.clip(core.v_s.cpu().numpy() + cfg.b[:, None], 0, 1)
    r_64 = np.clip(v64 + cfg.b[:, None], 0, 1)
    assert np.abs(r_gpu - r_64).max() < 1e-4


@pytest.mark.parametrize("launch", ["step", "persistent"])
def test_carried_dr_equals_fresh_initialisation(launch):
    """Substeps that reuse the previous call's dr (FLYB_OPTIC_DR_VALID) give the same bits as calls
    that recompute it; a host write to v between calls is seen and forces the recompute."""
    cfg = small_optic(seed=7)
    W = cfg.W_rr()
    B = 8
    rng = np.random.default_rng(3)
    v0 = (rng.standard_normal((cfg.m, B)) * 0.3).astype(np.float32)
    pr = (rng.standard_normal((cfg.m, B)) * 0.3).astype(np.float32)
    v_mid = (rng.standard_normal((cfg.m, B)) * 0.3).astype(np.float32)
    cores = []
    for carry in (True, False):
        core = OpticCore(W, cfg.a, cfg.b, batch=B, device="cuda", gain_rr=cfg.gain_rr, adapt_gain=cfg.adapt_gain,
                         aad=cfg.aad, launch=launch)
        core.v_s.copy_(torch.from_numpy(v0))
        core.pr_in.copy_(torch.from_numpy(pr))
        for k, n in enumerate((1, 2, 1, 3, 1, 1)):
            if k == 3:
                core.v_s[: cfg.m // 2].copy_(torch.from_numpy(v_mid[: cfg.m // 2]))
            core.substeps(n, carry=carry)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(core.dr_out.cpu().numpy(), core.dr().cpu().numpy())
        core.check()
        cores.append(core)
    for name in ("v_s", "adapt_s"):
        np.testing.assert_array_equal(getattr(cores[0], name).cpu().numpy(), getattr(cores[1], name).cpu().numpy())
    # and both equal the oracle run the same way
    v, ad = v0.copy(), np.zeros_like(v0)
    spk = np.zeros_like(v0)
    for k, n in enumerate((1, 2, 1, 3, 1, 1)):
        if k == 3:
            v[: cfg.m // 2] = v_mid[: cfg.m // 2]
        oracle.optic_run(v, ad, W.indptr, W.indices, W.data, pr, spk, cfg.a, cfg.b, cfg.gain_rr, cfg.adapt_gain,
                         cfg.aad, n)
    np.testing.assert_allclose(cores[0].v_s.cpu().numpy(), v, rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("batch,wpr", [(1, None), (3, None), (64, None), (64, 1), (5, 2), (64, 4), (40, 8), (1, 8)])
def test_held_input_products_match_oracle(batch, wpr):
    """The held-input products with the warps-per-row split chosen from the mean row length, or
    forced to each allowed value."""
    cfg = small_optic(seed=6)
    rng = np.random.default_rng(1)
    rates = (rng.random((cfg.W_rs.shape[1] + 50, batch)) * 500).astype(np.float32)   # [N][B] Hz
    x_index = rng.permutation(cfg.W_rs.shape[1] + 50)[: cfg.W_rs.shape[1]].astype(np.int32)
    M = DeviceCSR(cfg.W_rs, "cuda")
    y = torch.zeros(cfg.m, batch, device="cuda")
    spmm(M, torch.from_numpy(rates).cuda(), y, x_index=torch.from_numpy(x_index).cuda(), x_div=100.0, x_lo=0.0,
         x_hi=3.0, alpha=0.5, warps_per_row=wpr)
    W = cfg.W_rs.tocsr()
    ref = oracle.spmm(W.indptr, W.indices, W.data, rates, batch, rows=W.shape[0], x_index=x_index, x_div=100.0,
                      x_lo=0.0, x_hi=3.0, alpha=0.5)
    np.testing.assert_allclose(y.cpu().numpy(), ref, rtol=RTOL, atol=ATOL)
    d = (rng.standard_normal((cfg.m, batch)) * 0.5).astype(np.float32)
    W = cfg.W_sr.tocsr()
    y_index = rng.permutation(W.shape[0] + 10)[: W.shape[0]].astype(np.int32)
    out = torch.zeros(W.shape[0] + 10, batch, device="cuda")
    spmm(DeviceCSR(W, "cuda"), torch.from_numpy(d).cuda(), out, y_index=torch.from_numpy(y_index).cuda(), alpha=100.0,
         y_lo=-35.0, y_hi=35.0, warps_per_row=wpr)
    ref = np.zeros((W.shape[0] + 10, batch), np.float32)
    oracle.spmm(W.indptr, W.indices, W.data, d, batch, rows=W.shape[0], y=ref, y_index=y_index, alpha=100.0,
                y_lo=-35.0, y_hi=35.0)
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=RTOL, atol=1e-4)


@pytest.mark.parametrize("launch", ["step", "persistent"])
def test_optic_lobe_drop_in_equals_reference_frames(launch):
    z, c, r = hex_lobe()
    ol = OpticLobe(c, r, OpticParams(), device="cuda", batch=2, launch=launch)
    ol.relax()
    for f in range(3):
        drive = ol.step_frame(torch.from_numpy(z[f"frame{f}_rad"]), torch.from_numpy(z[f"frame{f}_spk"]).cuda(), 10.0)
        for key in ("v", "adapt", "delta_rate", "contrast", "I_lp", "I_mean"):
            np.testing.assert_allclose(getattr(ol, key).cpu().numpy(), z[f"frame{f}_{key}"], rtol=RTOL, atol=ATOL,
                                       err_msg=f"{key} frame {f}")
        np.testing.assert_allclose(drive.cpu().numpy(), z[f"frame{f}_drive"], rtol=RTOL, atol=1e-4)
    ol.reset([1])
    assert torch.all(ol.v[1] == 0) and bool(ol._fresh[1]) and not bool(ol._fresh[0])


# ------------------------------------------------------------------ reference-compatible launchers
def test_compat_optic_update_is_exact():
    """The reference's own check (tests/test_cuda.py:42-63): torch expression vs kernel, atol=0."""
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        gen = torch.Generator(device="cuda").manual_seed(6)
        rand = lambda *shape: torch.rand(*shape, device="cuda", generator=gen)  # noqa: E731
        for batch in (1, 3):
            n = 259
            v, adapt = rand(batch, n) - .5, rand(batch, n)
            o = SimpleNamespace(v=v.clone(), adapt=adapt.clone(), B=batch, n_rate=n, p=OpticParams(), _a=rand(n),
                                b_vec=rand(n), _a_ad=.997, _cuda_dr=torch.empty_like(v))
            fcuda.optic_dr(o.v, o.b_vec, o._cuda_dr)
            for _ in range(10):
                y, pr, sk = rand(batch, n), rand(batch, n), rand(batch, n)
                dr = (v + o.b_vec).clamp(0, 1) - o.b_vec
                inp = o.p.gain_rr * y + pr - o.p.adapt_gain * adapt
                inp = inp + sk
                v = inp + (v - inp) * o._a
                adapt = dr + (adapt - dr) * o._a_ad
                fcuda.optic_update(o, y, pr, sk)
            torch.testing.assert_close(o.v, v, rtol=0, atol=0)
            torch.testing.assert_close(o.adapt, adapt, rtol=0, atol=0)
    stream.synchronize()


def test_compat_csr_and_events_against_dense():
    rng = np.random.default_rng(5)
    matrix = sp.random(277, 277, density=.04, random_state=rng, format="csr", dtype=np.float32)
    matrix.data -= .5
    for dtype in (torch.float32, torch.float16):
        for batch in (1, 8):
            csr = fcuda.CSR(matrix, "cuda", dtype)
            x = torch.as_tensor(rng.random((batch, 277), dtype=np.float32), device="cuda")
            x[:, ::3] = 0
            dense = torch.as_tensor(matrix.toarray(), device="cuda").to(dtype).float()
            refx = x.half().float() if dtype == torch.float16 else x
            torch.testing.assert_close(csr.matvec(x), refx @ dense.T, rtol=2e-5, atol=2e-6)
            csc = matrix.tocsc()
            ptr = torch.tensor(csc.indptr, dtype=torch.int32, device="cuda")
            idx = torch.tensor(csc.indices, dtype=torch.int32, device="cuda")
            w = torch.tensor(csc.data, dtype=dtype, device="cuda")
            g = torch.ones_like(x)
            fcuda.event_scatter(ptr, idx, w, x, g)
            torch.testing.assert_close(g, 1 + x @ dense.T, rtol=2e-5, atol=3e-6)
    csr = fcuda.CSR(sp.csr_matrix((3, 4)), "cuda")
    torch.testing.assert_close(csr.matvec(torch.zeros(2, 4, device="cuda")), torch.zeros(2, 3, device="cuda"))
    v = torch.empty(2, 0, device="cuda")
    fcuda.optic_dr(v, torch.zeros(0, device="cuda"), v)


def test_compat_group_means_double_order():
    rng = np.random.default_rng(2)
    rates = torch.as_tensor(rng.random((3, 50), dtype=np.float32) * 100, device="cuda")
    groups = [np.array([1, 4, 9]), np.array([], int), np.arange(50)]
    ptr = torch.tensor(np.r_[0, np.cumsum([len(g) for g in groups])], dtype=torch.int32, device="cuda")
    idx = torch.tensor(np.concatenate(groups), dtype=torch.int32, device="cuda")
    spikes = torch.as_tensor((rng.random((3, 50)) < 0.2).astype(np.float32), device="cuda")
    out = fcuda.group_means(ptr, idx, rates, spikes).cpu().numpy()
    r = rates.cpu().numpy().astype(np.float64)
    for k, gidx in enumerate(groups):
        expect = r[:, gidx].sum(1) / len(gidx) if len(gidx) else np.zeros(3)
        np.testing.assert_array_equal(out[:, k], expect)
    np.testing.assert_array_equal(out[:, -1], spikes.sum(1).cpu().numpy())


def test_compat_lif_update_matches_torch_step():
    """launch_lif against the reference's Torch update on a batch-major brain-like object."""
    rng = np.random.default_rng(0)
    B, N = 3, 500
    t = lambda a: torch.as_tensor(np.asarray(a, np.float32), device="cuda").contiguous()  # noqa: E731
    a_m, a_r, a_ad, a_std = np.exp(-0.5 / 20), np.exp(-0.5 / 100), np.exp(-0.5 / 200), np.exp(-0.5 / 300)
    P = t([-52, -52, -45, a_m, 0.5, 2.2, 1.5, a_ad, a_std, a_r, (1 - a_r) * 1000 / 0.5])
    br = SimpleNamespace(v=t(rng.uniform(-60, -40, (B, N))), g=t(rng.normal(0, 3, (B, N))), drive=t(rng.normal(5, 2, (B, N))),
                         adapt=t(rng.random((B, N))), refrac=t(rng.choice([0, 0, 0.7, 2.2], (B, N))),
                         active=t(rng.random(N) > 0.1), poisson_p=t(rng.random((B, N)) * 0.05), res=t(rng.random((B, N))),
                         std_u_vec=t(rng.random(N) * 0.3), spikes=t(np.zeros((B, N))), spike_buf=t(np.zeros((3, B, N))),
                         buf_pos=1, rate=t(rng.random((B, N)) * 10), spike_counts=t(np.zeros((B, N))), _cuda_P=P,
                         _poisson_on=True, _std_on=True, record_activity=True, p=SimpleNamespace(adapt_jump=1.5),
                         cuda_compact=False, B=B, n=N)
    before = {k: getattr(br, k).clone() for k in ("v", "g", "drive", "adapt", "refrac", "res", "rate", "spike_counts")}
    rnd = t(rng.random((B, N)))
    fcuda.lif_update(br, rnd)
    target = -52 + before["g"] + before["drive"] - before["adapt"]
    v = target + (before["v"] - target) * np.float32(a_m)
    v = torch.where(before["refrac"] > 0, torch.full_like(v, -52.0), v)
    spikes = (v >= -45).float() * br.active
    spikes = torch.maximum(spikes, (rnd < br.poisson_p).float())
    fired = spikes > 0
    v = torch.where(fired, torch.full_like(v, -52.0), v)
    torch.testing.assert_close(br.v, v, rtol=0, atol=0)
    torch.testing.assert_close(br.spikes, spikes, rtol=0, atol=0)
    torch.testing.assert_close(br.spike_buf[1], spikes * before["res"], rtol=0, atol=0)
    torch.testing.assert_close(br.spike_counts, before["spike_counts"] + spikes, rtol=0, atol=0)


def test_gather_probe_reads_every_row_once():
    """flyb_gather_probe (the L2 gather-rate measurement of bench.py): with every element 1 the
    thread sums add up to 64 per gathered row; out-of-range indices are skipped."""
    import ctypes as ct
    from flyb200 import _abi
    rows, n_idx = 1000, 100_003
    x = torch.ones(rows, 64, device="cuda")
    idx = torch.randint(0, rows, (n_idx,), dtype=torch.int32, device="cuda")
    idx[::1000] = rows + 5                                       # skipped
    skipped = int((idx >= rows).sum().item())
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    out = torch.zeros(sms * 16 * 256, device="cuda")
    lib = _abi.lib()
    for bps in (1, 16):
        out.zero_()
        rc = lib.flyb_gather_probe(ct.c_void_p(x.data_ptr()), rows, ct.c_void_p(idx.data_ptr()), n_idx,
                                   ct.c_void_p(out.data_ptr()), bps, ct.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 0
        torch.cuda.synchronize()
        assert out.double().sum().item() == 64.0 * (n_idx - skipped)
    assert lib.flyb_gather_probe(ct.c_void_p(x.data_ptr()), rows, ct.c_void_p(idx.data_ptr()), n_idx,
                                 ct.c_void_p(out.data_ptr()), 17, None) == _abi.EINVAL
