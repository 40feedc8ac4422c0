"""The hand-written optic adjoint against FP64: central finite differences and torch autograd
through the same expressions (oracle/optic64.py), plus the checkpointing and the autograd.Function."""
import numpy as np
import pytest
import torch

from oracle import optic64
from flyb200 import synthetic
from flyb200.adjoint import OpticAdjoint, OpticRollout

pytestmark = pytest.mark.gpu


def problem(batch=2, steps=60, seed=7):
    cfg = synthetic.optic_config3(seed=seed, m=400, nnz=9000, n_pr=40, n_types=16, n_spk=50)
    rng = np.random.default_rng(seed)
    v0 = (rng.standard_normal((cfg.m, batch)) * 0.25).astype(np.float32)
    ad0 = (rng.standard_normal((cfg.m, batch)) * 0.02).astype(np.float32)
    pr = (rng.standard_normal((cfg.m, batch)) * 0.2).astype(np.float32)
    spk = (rng.standard_normal((cfg.m, batch)) * 0.05).astype(np.float32)
    w = np.zeros(cfg.m)
    groups = rng.permutation(cfg.m)[:100]
    w[groups[:50]], w[groups[50:]] = 1 / 50, -1 / 50          # L - R difference of two 50-unit groups
    gains = cfg.gain0 * rng.uniform(0.8, 1.2, len(cfg.gain0))
    tau = cfg.tau_of_type * rng.uniform(0.9, 1.1, cfg.n_types)
    return cfg, v0, ad0, pr, spk, w, gains.astype(np.float64), tau.astype(np.float64), steps


def gpu_grads(cfg, v0, ad0, pr, spk, w, gains, tau, steps, checkpoint=20, launch="persistent"):
    B = v0.shape[1]
    eng = OpticAdjoint(cfg.W0, cfg.pair_id, len(cfg.gain0), cfg.type_of, cfg.n_types, cfg.b,
                       torch.from_numpy(pr).cuda(), torch.from_numpy(spk).cuda(), dt_ms=cfg.dt_ms, batch=B,
                       adapt_tau_ms=cfg.adapt_tau_ms, checkpoint=checkpoint, launch=launch)
    g = torch.tensor(gains, dtype=torch.float32, device="cuda", requires_grad=True)
    t = torch.tensor(tau, dtype=torch.float32, device="cuda", requires_grad=True)
    vT, _ = OpticRollout.apply(g, t, torch.from_numpy(v0).cuda(), torch.from_numpy(ad0).cuda(), eng, steps)
    b = torch.from_numpy(cfg.b).cuda()[:, None]
    L = ((vT + b).clamp(0, 1) * torch.from_numpy(w).float().cuda()[:, None]).sum()
    L.backward()
    eng.check()
    return g.grad.double().cpu().numpy(), t.grad.double().cpu().numpy(), float(L)


def fp64(cfg, v0, ad0, pr, spk, w, gains, tau, steps):
    kw = dict(dt=cfg.dt_ms, gr=cfg.gain_rr, ga=cfg.adapt_gain, adapt_tau=cfg.adapt_tau_ms, steps=steps)
    return optic64.torch_grads(cfg.W0, cfg.pair_id, gains, tau, cfg.type_of, cfg.b, v0, ad0, pr, spk, w, **kw), kw


@pytest.mark.parametrize("launch", ["step", "persistent"])
@pytest.mark.parametrize("batch", [1, 2, 40])
def test_adjoint_matches_fp64_autograd(launch, batch):
    prob = problem(batch=batch)
    cfg = prob[0]
    (g64, t64, L64), _ = fp64(*prob)
    g32, t32, L32 = gpu_grads(*prob, launch=launch)
    assert abs(L32 - L64) <= 1e-5 * max(1.0, abs(L64))
    assert np.linalg.norm(g32 - g64) <= 1e-4 * np.linalg.norm(g64)
    assert np.linalg.norm(t32 - t64) <= 1e-4 * np.linalg.norm(t64)
    big = np.abs(g64) > 1e-2 * np.abs(g64).max()
    np.testing.assert_allclose(g32[big], g64[big], rtol=1e-3, atol=1e-6 * np.abs(g64).max())
    assert cfg.W0.nnz > 0


def test_fp64_autograd_agrees_with_central_differences_and_gpu():
    """FD (h = 1e-4) pins the FP64 autograd comparator; the GPU adjoint then matches FD to 1e-4 relative."""
    cfg, v0, ad0, pr, spk, w, gains, tau, steps = problem(batch=2)
    (g64, t64, _), kw = fp64(cfg, v0, ad0, pr, spk, w, gains, tau, steps)
    g32, t32, _ = gpu_grads(cfg, v0, ad0, pr, spk, w, gains, tau, steps)

    def loss_gain(x):
        vT, _ = optic64.rollout(cfg.W0, cfg.pair_id, x, tau, cfg.type_of, cfg.b, v0, ad0, pr, spk, **kw)
        return optic64.readout(vT, cfg.b, w)

    def loss_tau(x):
        vT, _ = optic64.rollout(cfg.W0, cfg.pair_id, gains, x, cfg.type_of, cfg.b, v0, ad0, pr, spk, **kw)
        return optic64.readout(vT, cfg.b, w)

    top = np.argsort(-np.abs(g64))[:12]
    fd_g = optic64.central_differences(loss_gain, gains, top, h=1e-4)
    fd_t = optic64.central_differences(loss_tau, tau, np.arange(len(tau)), h=1e-4)
    smooth = np.abs(fd_g - g64[top]) <= 1e-6 + 1e-5 * np.abs(g64[top])      # no clip kink crossed by +-h
    assert smooth.sum() >= 8
    np.testing.assert_allclose(g32[top][smooth], fd_g[smooth], rtol=1e-4, atol=1e-4 * np.abs(fd_g).max())
    ok = np.abs(fd_t - t64) <= 1e-6 + 1e-5 * np.abs(t64)
    np.testing.assert_allclose(t32[ok], fd_t[ok], rtol=1e-4, atol=1e-4 * np.abs(fd_t).max())


def test_checkpoint_interval_does_not_change_gradients():
    prob = problem(batch=3, steps=57)
    g20, t20, _ = gpu_grads(*prob, checkpoint=20)
    g7, t7, _ = gpu_grads(*prob, checkpoint=7)
    np.testing.assert_allclose(g7, g20, rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(t7, t20, rtol=1e-6, atol=1e-9)


def test_c3_full_lobe_gradients_match_fp64_central_differences():
    """Config 3 at its stated size (89,390 units, 6 M nnz, 200 substeps, checkpoint 20), one fly,
    the readout L = sum of the rates of one fixed 50-unit group minus another's: the 20 largest
    pair-gain and the 10 largest time-constant gradients of the FP32 adjoint against FP64 central
    differences (h = 1e-4) of the C FP64 oracle, within 1e-4 relative. Components whose +-h and
    +-h/2 differences disagree (a clip kink inside the interval) are left out; most are smooth."""
    import oracle
    cfg = synthetic.optic_config3(seed=3)
    assert cfg.m == 89_390 and cfg.W0.nnz == 6_000_000
    B, steps = 1, 200
    rng = np.random.default_rng(3)
    v0 = (rng.standard_normal((cfg.m, B)) * 0.2).astype(np.float32)
    ad0 = np.zeros((cfg.m, B), np.float32)
    pr = (rng.standard_normal((cfg.m, B)) * 0.2).astype(np.float32)
    spk = np.zeros((cfg.m, B), np.float32)
    w = np.zeros(cfg.m)
    groups = rng.permutation(cfg.m)[:100]
    w[groups[:50]], w[groups[50:]] = 1 / 50, -1 / 50
    gains, tau = cfg.gain0.astype(np.float64), cfg.tau_of_type.astype(np.float64)
    g32, t32, L32 = gpu_grads(cfg, v0, ad0, pr, spk, w, gains, tau, steps)
    W = cfg.W0.tocsr()
    aad = float(np.exp(-cfg.dt_ms / cfg.adapt_tau_ms))

    def loss(g, t):
        v, ad = v0.astype(np.float64), ad0.astype(np.float64)
        a = np.exp(-cfg.dt_ms / t[cfg.type_of])
        oracle.optic_run_f64(v, ad, W.indptr, W.indices, W.data.astype(np.float64) * g[cfg.pair_id], pr, spk, a, cfg.b,
                             cfg.gain_rr, cfg.adapt_gain, aad, steps)
        return optic64.readout(v, cfg.b, w)

    L64 = loss(gains, tau)
    assert abs(L32 - L64) <= 1e-5 * max(1.0, abs(L64))

    def fd(which, k, h):
        xp, xm = (gains.copy(), tau.copy()), (gains.copy(), tau.copy())
        xp[which][k] += h
        xm[which][k] -= h
        return (loss(*xp) - loss(*xm)) / (2 * h)

    for which, grad, count in ((0, g32, 20), (1, t32, 10)):
        top = np.argsort(-np.abs(grad))[:count]
        h1 = np.array([fd(which, k, 1e-4) for k in top])
        h2 = np.array([fd(which, k, 5e-5) for k in top])
        smooth = np.abs(h1 - h2) <= 1e-6 * np.abs(h1).max() + 1e-5 * np.abs(h1)
        assert smooth.sum() >= 0.75 * count, (which, smooth)
        err = np.abs(grad[top] - h1) / np.abs(h1)
        print(f"C3 adjoint {'gains' if which == 0 else 'tau'}: {int(smooth.sum())}/{count} smooth components, "
              f"max relative error {err[smooth].max():.2e} against FP64 central differences")
        np.testing.assert_allclose(grad[top][smooth], h1[smooth], rtol=1e-4, atol=1e-6 * np.abs(h1).max())
