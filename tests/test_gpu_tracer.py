"""The eye's ray tracer on the GPU (flyb_trace) against the reference tracer's own outputs and the
C oracle, bit for bit: the reference tests' rays and scene edits, batched rooms with per-row sphere
moves, the fused eye (pose turn, shared origin, column sums), larger random poses, graph capture,
and traced vision driving a FlyBrain frame."""
from pathlib import Path

import numpy as np
import pytest
import torch

import oracle
from flyb200 import world as W
from flyb200.batch_world import BatchWorld

pytestmark = pytest.mark.gpu
GOLDEN = np.load(Path(__file__).parent / "golden" / "tracer.npz")


def t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_move_and_invalidate_scene():
    """tests/test_world.py:18-28 of the reference."""
    w = W.World(spheres=[W.Sphere((1, 0, 0), (.2, .2, .2), "apple")], detail=0, ambient=(1, 1, 1, 1),
                light_color=(0, 0, 0, 0))
    o, d = torch.zeros(1, 3), torch.tensor([[1., 0, 0]])
    np.testing.assert_array_equal(w.trace(o, d).cpu().numpy(), GOLDEN["known_apple"])
    scene = w._scene
    w.move_sphere(0, (1, 1, 0))
    assert w._scene is scene                                   # moved in place, no repack
    assert torch.equal(w.trace(o, d).cpu(), torch.zeros(1, 4))
    w.spheres[0].center = (1, 0, 0)
    w.spheres[0].material = "lamp"
    w.invalidate()
    torch.testing.assert_close(w.trace(o, d).cpu(), torch.tensor([[.6, 1., 1., 1.]]))


@pytest.mark.parametrize("k", [0, 1])
def test_room_rays_match_reference(k):
    room = W.make_room(0)[0]
    got = room.trace(GOLDEN[f"room_o{k}"], GOLDEN[f"room_d{k}"])
    np.testing.assert_array_equal(got.cpu().numpy(), GOLDEN[f"room_rad{k}"])
    room.detail = 0
    room.invalidate()
    np.testing.assert_array_equal(room.trace(GOLDEN["room_o0"], GOLDEN["room_d0"]).cpu().numpy(),
                                  GOLDEN["room_flat_rad0"])


def test_results_own_storage_and_camera_matches_reference():
    room = W.make_room(0)[0]
    first = room.trace(GOLDEN["room_o0"], GOLDEN["room_d0"])
    snap = first.clone()
    img = room.render_camera((0, 0, 1), (1, 0, 0), (0, 0, 1), width=48, height=32)
    assert torch.equal(first, snap)
    ref = GOLDEN["camera"]
    got = img.cpu().numpy()
    # the camera's rays are built on the device (linspace, cross, norm), so a pixel on an edge may
    # round to the other side; every other pixel matches within the reference's own batched/scalar
    # tracer tolerance (tests/test_batch_sim.py:153)
    close = np.isclose(got, ref, rtol=3e-5, atol=2e-5).all(-1)
    assert close.mean() >= 0.995, close.mean()


def test_batched_rooms_and_row_moves_match_reference():
    scenes = [W.make_room(i)[0] for i in range(3)]
    scenes[1].spheres[0].material = "black"
    scenes[2].light_pos = (1, 0, 2)
    b = BatchWorld(scenes)
    org, dirs = GOLDEN["batch_o"], GOLDEN["batch_d"]
    first = b.trace(org, dirs)
    np.testing.assert_array_equal(first.cpu().numpy(), GOLDEN["batch_rad"])
    saved = first.clone()
    b.move_sphere(0, (-.45, .05, .77), (.05,) * 3, rows=[1])
    moved = b.trace(org, dirs)
    np.testing.assert_array_equal(moved.cpu().numpy(), GOLDEN["batch_rad_moved"])
    assert torch.equal(moved[0], first[0]) and torch.equal(moved[2], first[2]) and not torch.equal(moved[1], first[1])
    assert torch.equal(first, saved)


def test_empty_scenes_and_bad_shapes():
    b = BatchWorld([W.World(), W.World()])
    assert torch.equal(b.trace(torch.zeros(2, 3, 3), torch.ones(2, 3, 3)).cpu(), torch.zeros(2, 3, 4))
    with pytest.raises(ValueError):
        b.trace(torch.zeros(3, 3), torch.zeros(3, 3))
    b.worlds[1].spheres.append(W.Sphere((1, 0, 0), (.1,) * 3, "apple"))
    with pytest.raises(ValueError):
        b.trace(torch.zeros(2, 3, 3), torch.ones(2, 3, 3))
    assert W.World().trace(torch.zeros(0, 3), torch.zeros(0, 3)).shape == (0, 4)


def eye_world(n=4):
    scenes = [W.make_room(i)[0] for i in range(n)]
    scenes[3 % n].spheres[0].material = "lamp"
    return BatchWorld(scenes)


def test_eye_columns_match_reference():
    """Pose turn in double, shared origin, weighted sums in sample order: BatchSim.column_radiance
    over the reference tracer, bit for bit."""
    b = eye_world()
    b.set_eye(GOLDEN["eye_dirs"], GOLDEN["eye_w"])
    got = b.column_radiance(GOLDEN["eye_pos"], GOLDEN["eye_f"], GOLDEN["eye_left"], GOLDEN["eye_up"])
    np.testing.assert_array_equal(got.cpu().numpy(), GOLDEN["eye_columns"])
    rays = b.trace(np.broadcast_to(GOLDEN["eye_pos"][:, None], GOLDEN["eye_ray_d"].shape), GOLDEN["eye_ray_d"])
    np.testing.assert_array_equal(rays.cpu().numpy(), GOLDEN["eye_rad"])


def random_poses(B, seed):
    rng = np.random.default_rng(seed)
    heading, pitch = rng.uniform(-np.pi, np.pi, B), rng.uniform(-0.5, 0.5, B)
    eye = np.c_[rng.uniform(-1.8, 1.8, B), rng.uniform(-1.8, 1.8, B), rng.uniform(0.05, 2.4, B)]
    f = np.c_[np.cos(pitch) * np.cos(heading), np.cos(pitch) * np.sin(heading), np.sin(pitch)]
    left = np.c_[-np.sin(heading), np.cos(heading), np.zeros(B)]
    return eye, f, left, np.cross(f, left)


@pytest.mark.parametrize("k", [1, 7, 19])
def test_random_poses_match_oracle(k):
    """Sixteen flies anywhere in the room (inside the table, under it, at the lamp), k samples per
    column, against the C oracle bit for bit."""
    B, n_col = 16, 300
    rng = np.random.default_rng(k)
    az, el = rng.uniform(-np.pi, np.pi, (n_col, k)), rng.uniform(-1.2, 1.2, (n_col, k))
    dirs = np.stack([np.cos(el) * np.cos(az), np.cos(el) * np.sin(az), np.sin(el)], -1)
    w = rng.random(k)
    w /= w.sum()
    b = eye_world(B)
    b.set_eye(dirs, w)
    pose = random_poses(B, 100 + k)
    got = b.column_radiance(*pose).cpu().numpy()
    blob = np.stack([W.pack_scene(s) for s in b.worlds])
    ref = oracle.trace(blob, b._scene_shape, b.detail, origins=pose[0], eye_dirs=dirs.reshape(-1, 3),
                       pose=np.concatenate(pose[1:], 1), weights=w, shared_origin=True, batch=B)
    np.testing.assert_array_equal(got, ref)
    assert (got > 0).mean() > 0.5


def test_per_ray_origins_match_oracle():
    rng = np.random.default_rng(3)
    B, M = 5, 4000
    o = np.c_[rng.uniform(-1.9, 1.9, (B * M, 2)), rng.uniform(0.01, 2.5, B * M)].reshape(B, M, 3).astype(np.float32)
    d = rng.standard_normal((B, M, 3))
    d = (d / np.linalg.norm(d, axis=-1, keepdims=True)).astype(np.float32)
    d[0, :10] = [[1, 0, 0], [0, 1, 0], [0, 0, 1], [-1, 0, 0], [0, -1, 0], [0, 0, -1], [0.6, 0.8, 0], [0, 0.6, 0.8],
                 [0.8, 0, 0.6], [0, 0, 1]]                      # axis-parallel rays: the slab guards
    b = eye_world(B)
    got = b.trace(o, d).cpu().numpy()
    ref = oracle.trace(np.stack([W.pack_scene(s) for s in b.worlds]), b._scene_shape, b.detail, origins=o, dirs=d,
                       batch=B)
    np.testing.assert_array_equal(got, ref)


def test_captured_trace_follows_moves():
    """The eye trace in a CUDA graph reads the packed scenes and pose buffers in place: a replay
    after a sphere move and a new pose equals an eager trace."""
    b = eye_world()
    b.set_eye(GOLDEN["eye_dirs"], GOLDEN["eye_w"])
    out = torch.zeros(4, GOLDEN["eye_dirs"].shape[0], 4, device="cuda")
    pose = (GOLDEN["eye_pos"], GOLDEN["eye_f"], GOLDEN["eye_left"], GOLDEN["eye_up"])
    b.column_radiance(*pose, out=out)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            b.trace_eye(out)
    torch.cuda.current_stream().wait_stream(s)
    b.move_sphere(0, (-.45, .05, .77), (.3,) * 3)
    b.set_pose(GOLDEN["eye_pos"] + 0.01, *pose[1:])
    g.replay()
    torch.cuda.synchronize()
    eager = b.column_radiance(GOLDEN["eye_pos"] + 0.01, *pose[1:])
    assert torch.equal(out, eager)
    assert not np.array_equal(out.cpu().numpy(), GOLDEN["eye_columns"])
    del g


def test_traced_vision_drives_the_frame():
    """FlyBrain.look traces into the held radiance: the frame equals one fed the same radiance
    through vision()."""
    from flyb200.brain import LIFParams
    from flyb200.fly import FlyBrain
    from flyb200.optic import OpticParams
    from test_oracle_golden import hex_lobe
    _, c, r = hex_lobe()
    B = 4
    fbs = [FlyBrain(c, batch=B, device="cuda", seed=2, retina=r, lif_params=LIFParams(receptor_model=None, dt=0.5),
                    optic_params=OpticParams()) for _ in range(2)]
    world = eye_world(B)
    pose = random_poses(B, 7)
    fbs[0].look(world, *pose)
    rad = world.column_radiance(*pose).clone()
    assert float(rad.sum()) > 0
    fbs[1].vision(rad)
    for fb in fbs:
        fb.step(10.0)
    torch.cuda.synchronize()
    assert torch.equal(fbs[0]._radiance, fbs[1]._radiance)
    for k in ("v", "rate"):
        assert torch.equal(getattr(fbs[0].brain, k), getattr(fbs[1].brain, k))
    assert torch.equal(fbs[0].optic.v, fbs[1].optic.v)
