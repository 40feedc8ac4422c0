"""The frame loop on the GPU: graph-captured frames equal eager frames bit for bit, checkpoints
round-trip, pulses split frames, and uneven batched episodes reset only their own rows."""
import numpy as np
import pytest
import torch

from flyb200.batch_sim import BatchSim
from flyb200.brain import LIFParams
from flyb200.fly import FlyBrain
from flyb200.optic import OpticParams
from test_oracle_golden import hex_lobe

pytestmark = pytest.mark.gpu


def make(cuda_graphs=False, batch=3, seed=5):
    z, c, r = hex_lobe()
    fb = FlyBrain(c, batch=batch, device="cuda", seed=seed, retina=r, cuda_graphs=cuda_graphs,
                  lif_params=LIFParams(receptor_model=None, dt=0.5), optic_params=OpticParams())
    rad = np.random.default_rng(1).random((batch, r.n_columns, 4)).astype(np.float32)
    fb.vision(rad)
    fb.set_input("drive", [int(fb.optic.spk_idx[0])], np.array([[300.0], [150.0], [0.0]][:batch], np.float32))
    return fb


def state(fb):
    out = {k: getattr(fb.brain, k).clone() for k in FlyBrain.BRAIN_TENSORS}
    out.update({f"optic_{k}": getattr(fb.optic, k).clone() for k in FlyBrain.OPTIC_TENSORS})
    out["ring"] = fb.brain.ring.clone()
    return out


def assert_same(a, b):
    for k in a:
        assert torch.equal(a[k], b[k]), k


def test_graph_frames_equal_eager_frames():
    eager, graphed = make(False), make(True)
    for ms in (10.0, 10.0, 13.3, 10.0, 6.7, 10.0):
        eager.step(ms)
        graphed.step(ms)
    torch.cuda.synchronize()
    assert len(graphed._graphs) >= 2
    assert_same(state(eager), state(graphed))
    assert eager.brain.step_count == graphed.brain.step_count
    assert int(graphed.brain._clock[0]) == graphed.brain.step_count


def test_pulses_split_frames_and_expire():
    fb = make(True)
    fb.stimulate([int(fb.optic.spk_idx[0])], 500.0, 7.0)
    fb.step(10.0)
    assert not fb.poisson.pulses
    assert float(fb.brain.spike_counts.sum()) > 0


def test_state_dict_round_trip():
    fb = make(True)
    fb.step(10.0)
    saved = fb.state_dict()
    fb.step(10.0)
    after = state(fb)
    fb.load_state_dict(saved)
    fb.step(10.0)
    assert_same(after, state(fb))


def test_batch_sim_uneven_episodes_reset_their_rows():
    z, c, r = hex_lobe()
    rad = np.random.default_rng(2).random((r.n_columns, 4)).astype(np.float32)
    lc = np.flatnonzero(c.neurons.type.to_numpy() == "LC11")

    def stimulus(frame, fb):
        return rad, {"drive": (lc, np.full((fb.B, len(lc)), 200.0, np.float32))}

    sim = BatchSim(4, c=c, retina=r, seed=3, cuda_graphs=True, episode_frames=(2, 5), groups={"lc": lc},
                   stimulus=stimulus, lif_params=LIFParams(receptor_model=None, dt=0.5))
    resets = 0
    for _ in range(12):
        out = sim.step()
        for row in out["reset_rows"]:
            assert float(sim.fb.brain.v[row].max()) == sim.fb.brain.p.v_rest
            assert float(sim.fb.brain.spike_counts[row].sum()) == 0.0
            resets += 1
        assert out["lc"].shape == (4,)
    assert resets == sim.stats.finished > 0


def _member_order_means(rates, groups):
    out = {}
    for k, idx in groups.items():
        acc = np.zeros(rates.shape[0])
        for i in idx:
            acc += rates[:, i]
        out[k] = acc / len(idx) if len(idx) else acc
    return out


def test_motor_readout_inside_captured_frames():
    """Registered groups are reduced inside every (captured or eager) frame and copied to pinned
    memory; the result equals a member-order double sum of the rates on the host, the reference's
    launcher on the batch-major copy, and a fresh reduction after a reset."""
    from flyb200 import cuda as fcuda
    for graphs in (True, False):
        fb = make(graphs)
        rng = np.random.default_rng(4)
        groups = {"spk": [int(i) for i in fb.optic.spk_idx[:7]], "rand": rng.integers(0, fb.brain.n, 40).tolist(),
                  "empty": [], "one": [int(fb.optic.spk_idx[0])]}
        fb.set_motor(groups)
        first = fb.motor()                                  # before any frame: reduced on demand
        assert all(np.all(v == 0) or np.all(np.isfinite(v)) for v in first.values())
        for ms in (10.0, 10.0, 13.3, 10.0):
            fb.step(ms)
            got = fb.motor()
            rates = fb.brain.rate.double().cpu().numpy()
            want = _member_order_means(rates, groups)
            for k in groups:
                np.testing.assert_array_equal(got[k], want[k], err_msg=k)
            ptr = torch.tensor(np.r_[0, np.cumsum([len(groups[k]) for k in groups])], dtype=torch.int32, device="cuda")
            flat = torch.tensor(sum((groups[k] for k in groups), []), dtype=torch.int32, device="cuda")
            ref = fcuda.group_means(ptr, flat, fb.brain.rate.contiguous()).cpu().numpy()
            np.testing.assert_array_equal(np.stack([got[k] for k in groups], 1), ref)
            assert fb.motor(dict(groups)) .keys() == got.keys()
            other = fb.motor({"x": groups["rand"][:5]})     # unregistered groups: one explicit reduction
            np.testing.assert_array_equal(other["x"], _member_order_means(rates, {"x": groups["rand"][:5]})["x"])
        assert float(np.abs(got["spk"]).sum()) > 0
        fb.reset([0])
        after = fb.motor()
        np.testing.assert_array_equal(after["spk"][0], 0.0)
        if graphs:
            assert len(fb._graphs) >= 1


def fly_frames_connectome(z):
    import pandas as pd
    import scipy.sparse as sp
    from flyb200.connectome import Connectome
    n = pd.DataFrame({k[4:]: z[k] for k in z if k.startswith("tbl_")})
    W = sp.csr_matrix((z["W_data"], z["W_indices"], z["W_indptr"]), shape=(len(n), len(n)))
    return Connectome(n, W, pd.Series(np.arange(len(n)), index=n.bodyId.to_numpy()))


@pytest.mark.parametrize("launch", ["step", "persistent"])
def test_flybrain_frames_equal_reference_golden(launch):
    """The FlyBrain drop-in against the reference's FlyBrain frame by frame (tests/golden
    fly_frames: the 19-cell graph at 2 flies, held inputs and vision, a pulse ending inside a frame,
    an injected drive, 13.3 ms frames carrying fractional milliseconds, a row reset, a full reset),
    fed the uniforms the reference's generator drew: every LIF step's spikes bit-exact; at every
    frame end the LIF state within 1e-4 (the reference sums float weights in event order, the
    native ring sums exact integers), the optic state within 1e-5, the Poisson forcing exact."""
    from helpers import golden
    z = golden("fly_frames")
    c = fly_frames_connectome(z)
    fb = FlyBrain(c, batch=2, device="cuda", seed=7, lif_params=LIFParams(receptor_model=None), launch=launch)
    assert fb.optic is not None
    U = torch.from_numpy(z["uniforms"])
    cursor = [0]

    def uniforms(n):
        out = U[cursor[0]:cursor[0] + n]
        cursor[0] += n
        return out

    fb.uniform_source = uniforms
    raster = []
    plain_step = fb.brain.step

    def recording_step(n=1, uniforms=None):
        for k in range(int(n)):
            plain_step(1, uniforms=None if uniforms is None else uniforms[k:k + 1])
            raster.append(fb.brain.spikes.cpu().numpy() > 0)

    fb.brain.step = recording_step
    frames = iter(range(100))

    def frame(ms):
        fb.step(ms)
        k = next(frames)
        assert len(raster) == int(z[f"f{k}_steps"])
        np.testing.assert_array_equal(np.stack(raster), z["raster"][:len(raster)], err_msg=f"raster by frame {k}")
        for key in ("v", "g", "refrac", "rate", "spike_counts", "adapt", "res", "drive"):
            np.testing.assert_allclose(getattr(fb.brain, key).cpu().numpy(), z[f"f{k}_brain_{key}"], rtol=0, atol=1e-4,
                                       err_msg=f"brain {key} frame {k}")
        np.testing.assert_array_equal(fb.brain.poisson_p.cpu().numpy(), z[f"f{k}_brain_poisson_p"])
        for key in ("v", "adapt", "delta_rate"):
            np.testing.assert_allclose(getattr(fb.optic, key).cpu().numpy(), z[f"f{k}_optic_{key}"], rtol=1e-5,
                                       atol=1e-6, err_msg=f"optic {key} frame {k}")
        assert abs(fb._pending_ms - float(z[f"f{k}_pending_ms"])) < 1e-9

    rad = z["radiance"]
    fb.set_input("smell", z["orn"], np.array([[120.0], [40.0]], np.float32))
    fb.set_input("wind", z["jo"], np.array([[90.0, 10.0], [0.0, 150.0]], np.float32))
    fb.vision(rad)
    for _ in range(3):
        frame(10.0)
    fb.stimulate([9], 300.0, 7.0)
    fb.brain.set_drive([15], np.float32(12.0))
    fb.vision(rad[::-1].copy())
    for _ in range(2):
        frame(13.3)
    fb.reset([0])
    frame(10.0)
    fb.reset()
    fb.set_input("smell", z["orn"], np.float32(75.0))
    fb.vision(rad)
    frame(20.0)
    assert cursor[0] == len(U) and z["raster"].sum() > 0


def test_batch_sim_takes_the_reference_brain_arguments():
    """BatchSim accepts the reference's brain-step keywords (batch_sim.py:89-94) and refuses room,
    body and program settings by name."""
    z, c, r = hex_lobe()
    lp = LIFParams(receptor_model=None, dt=0.5)
    sim = BatchSim(2, c=c, seed=1, device="cuda", brain_dt=0.5, cuda_kernels=True, event_driven=True,
                   cuda_sparse="warp", cuda_compact=False, weight_dtype="float32", prune_frozen=True, lif_params=lp,
                   wind_speed=0.3, program="none", preset="raw")
    assert sim.fb.brain.cuda_sparse == "warp" and not sim.fb.brain.cuda_compact
    sim.step()
    with pytest.raises(ValueError, match="program"):
        BatchSim(2, c=c, device="cuda", lif_params=lp, program="walk")
    with pytest.raises(TypeError, match="bogus"):
        BatchSim(2, c=c, device="cuda", lif_params=lp, bogus=1)
    with pytest.raises(ValueError, match="cuda_kernels"):
        BatchSim(2, c=c, device="cuda", lif_params=lp, cuda_kernels=False)
