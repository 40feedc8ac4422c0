"""The optic lobe's per-stream hooks on the GPU (stream_rectify, stream_adapt, spatial_suppress;
optic.py:50-70, 378-495): OpticLobe against the reference's frames, the hooks under the slow
receptor tone against the oracle, and FlyBrain's graph replay and checkpoints of the hook state."""
import numpy as np
import pytest
import torch

from oracle import frame as oframe
from flyb200.brain import LIFParams
from flyb200.optic import OpticLobe, OpticParams, lobe_matrices, slow_blocks, stream_hooks
from flyb200.weights import receptor_gain, slow_spec
from test_oracle_golden import HOOK_CASES, optic_hooks_case, optic_slow_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", list(HOOK_CASES))
def test_optic_hooks_equal_reference_golden(case):
    z, c, r, p, L, h = optic_hooks_case(case)
    ol = OpticLobe(c, r, p, device="cuda", batch=2, launch="step")
    ol.relax()
    for f in range(3):
        drive = ol.step_frame(torch.from_numpy(z[f"frame{f}_rad"]), torch.from_numpy(z[f"frame{f}_spk"]).cuda(), 10.0)
        for key in ("v", "adapt", "delta_rate", "stream_adapt_state"):
            np.testing.assert_allclose(getattr(ol, key).cpu().numpy(), z[f"frame{f}_{key}"], rtol=1e-5, atol=1e-6,
                                       err_msg=f"{key} frame {f}")
        np.testing.assert_allclose(drive.cpu().numpy(), z[f"frame{f}_drive"], rtol=1e-5, atol=1e-4)
    if p.stream_adapt:
        assert float(ol.stream_adapt_state.abs().max()) > 0
        ol.reset([1])
        assert float(ol.stream_adapt_state[:, 1].abs().sum()) == 0.0
        assert float(ol.stream_adapt_state[:, 0].abs().sum()) > 0.0


@pytest.mark.parametrize("mode", ["additive", "gain", "threshold"])
def test_optic_hooks_under_the_slow_tone_equal_oracle(mode):
    """Both extensions at once (the slow products beside the hooked recurrent product), against the
    oracle, which each reference golden pins separately."""
    z, c, r, rec, lp, _, _, _ = optic_slow_case(mode)
    p = OpticParams(**HOOK_CASES["all"])
    L = lobe_matrices(c, r, p, rec, receptor_gain(lp))
    spec = slow_spec(lp)
    blocks, norm = slow_blocks(c, L.rate_idx, L.spk_idx, p, rec, receptor_gain(lp), spec)
    slow = {"mode": mode, "norm": norm, "clip": spec.clip, "classes": blocks}
    h = stream_hooks(c, r, L.rate_idx, L.spk_idx, p, L.M_rr, L.M_sr)
    B, m, K = 2, len(L.rate_idx), len(blocks)
    st = {"v": np.ascontiguousarray(z["v0"].T), "adapt": np.zeros((m, B), np.float32),
          "I_lp": np.zeros((B, r.n_columns * 5), np.float32), "I_mean": np.zeros((B, r.n_columns * 5), np.float32),
          "fresh": np.ones(B, bool), "pending": 0.0, "g_cls": np.zeros((K, m, B), np.float32),
          "g_slow": np.zeros((m, B), np.float32), "held": np.zeros((K, m, B), np.float32),
          "A": np.zeros((1, m, B), np.float32)}
    ol = OpticLobe(c, r, p, device="cuda", batch=2, receptor=rec, receptor_gain=receptor_gain(lp), slow=spec,
                   launch="step")
    ol.relax()
    ol.v = torch.from_numpy(z["v0"]).cuda()
    for f in range(3):
        want = oframe.frame(L, st, z[f"frame{f}_rad"], z[f"frame{f}_spk"], 10.0, p, slow=slow, hooks=h)
        drive = ol.step_frame(torch.from_numpy(z[f"frame{f}_rad"]), torch.from_numpy(z[f"frame{f}_spk"]).cuda(), 10.0)
        for key, ref in (("v", st["v"].T), ("adapt", st["adapt"].T), ("g_slow", st["g_slow"].T),
                         ("delta_rate", st["delta"].T), ("stream_adapt_state", st["A"].transpose(0, 2, 1))):
            np.testing.assert_allclose(getattr(ol, key).cpu().numpy(), ref, rtol=1e-5, atol=1e-6, err_msg=f"{key} {f}")
        np.testing.assert_allclose(drive.cpu().numpy(), want, rtol=1e-5, atol=1e-4)
    assert float(ol.g_slow.abs().max()) > 0 and float(ol.stream_adapt_state.abs().max()) > 0


def _hooked_fly(graphs):
    from flyb200.fly import FlyBrain
    z, c, r, p, L, h = optic_hooks_case("all")
    fb = FlyBrain(c, batch=2, device="cuda", seed=3, retina=r, lif_params=LIFParams(receptor_model=None, dt=0.5),
                  optic_params=p, cuda_graphs=graphs)
    fb.vision(z["frame0_rad"][0])
    return fb


def test_flybrain_hooks_graph_replay_and_checkpoint():
    """A FlyBrain whose optic lobe runs the hooks: captured frames replay like eager ones, and a
    checkpoint carries the stream adaptation state."""
    eager, graphed = _hooked_fly(False), _hooked_fly(True)
    for _ in range(4):
        eager.step(10.0)
        graphed.step(10.0)
    torch.cuda.synchronize()
    for key in ("v", "adapt", "stream_adapt_state"):
        assert torch.equal(getattr(eager.optic, key), getattr(graphed.optic, key)), key
    assert torch.equal(eager.brain.v, graphed.brain.v)
    saved = eager.state_dict()
    assert "stream_adapt_state" in saved["optic"]
    eager.step(10.0)
    after = (eager.optic.stream_adapt_state.clone(), eager.optic.v.clone(), eager.brain.v.clone())
    eager.load_state_dict(saved)
    eager.step(10.0)
    assert torch.equal(eager.optic.stream_adapt_state, after[0]) and torch.equal(eager.optic.v, after[1])
    assert torch.equal(eager.brain.v, after[2])
    assert float(eager.optic.stream_adapt_state.abs().max()) > 0
