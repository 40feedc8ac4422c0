"""The eye's ray tracer on the CPU: the C oracle against the reference tracer's own outputs
(tests/golden/tracer.npz, made by tests/golden/make_golden.py from flyverse.world and
flyverse.batch_world), bit for bit; the retina's viewing directions and sample rays against the
reference's build_retina; scene packing rules."""
from pathlib import Path

import numpy as np
import pandas as pd
import pytest
import scipy.sparse as sp

import oracle
from flyb200 import world as W
from flyb200.connectome import Connectome
from flyb200.retina import build_retina

GOLDEN = np.load(Path(__file__).parent / "golden" / "tracer.npz")


def rooms(n):
    return [W.make_room(i)[0] for i in range(n)]


def test_oracle_known_answers():
    apple = W.World(spheres=[W.Sphere((1, 0, 0), (.2, .2, .2), "apple")], detail=0, ambient=(1, 1, 1, 1),
                    light_color=(0, 0, 0, 0))
    got = oracle.trace(W.pack_scene(apple), apple._shape(), 0.0, origins=np.zeros((1, 3)), dirs=np.array([[1., 0, 0]]))
    np.testing.assert_array_equal(got[0], GOLDEN["known_apple"])
    np.testing.assert_allclose(got[0, 0], [.05, .08, .20, .85], rtol=1e-6)
    lamp = W.World(spheres=[W.Sphere((1, 0, 0), (.2, .2, .2), "lamp")], detail=0, ambient=(1, 1, 1, 1),
                   light_color=(0, 0, 0, 0))
    got = oracle.trace(W.pack_scene(lamp), lamp._shape(), 0.0, origins=np.zeros((1, 3)), dirs=np.array([[1., 0, 0]]))
    np.testing.assert_allclose(got[0, 0], [.6, 1., 1., 1.], rtol=1e-6)
    miss = oracle.trace(W.pack_scene(apple), apple._shape(), 0.0, origins=np.zeros((1, 3)), dirs=np.array([[0., 1, 0]]))
    assert np.all(miss == 0)


@pytest.mark.parametrize("k", [0, 1])
def test_oracle_room_rays_match_reference(k):
    room = W.make_room(0)[0]
    got = oracle.trace(W.pack_scene(room), room._shape(), room.detail, origins=GOLDEN[f"room_o{k}"],
                       dirs=GOLDEN[f"room_d{k}"])
    np.testing.assert_array_equal(got[0], GOLDEN[f"room_rad{k}"])
    flat = oracle.trace(W.pack_scene(room), room._shape(), 0.0, origins=GOLDEN["room_o0"], dirs=GOLDEN["room_d0"])
    np.testing.assert_array_equal(flat[0], GOLDEN["room_flat_rad0"])


def test_oracle_batched_rooms_and_moved_sphere_match_reference():
    scenes = rooms(3)
    scenes[1].spheres[0].material = "black"
    scenes[2].light_pos = (1, 0, 2)
    shape = scenes[0]._shape()
    got = oracle.trace(np.stack([W.pack_scene(s) for s in scenes]), shape, 1.4, origins=GOLDEN["batch_o"],
                       dirs=GOLDEN["batch_d"], batch=3)
    np.testing.assert_array_equal(got, GOLDEN["batch_rad"])
    scenes[1].spheres[0].center, scenes[1].spheres[0].radii = (-.45, .05, .77), (.05,) * 3
    got = oracle.trace(np.stack([W.pack_scene(s) for s in scenes]), shape, 1.4, origins=GOLDEN["batch_o"],
                       dirs=GOLDEN["batch_d"], batch=3)
    np.testing.assert_array_equal(got, GOLDEN["batch_rad_moved"])


def eye_rooms():
    scenes = rooms(4)
    scenes[3].spheres[0].material = "lamp"
    return scenes


def test_oracle_eye_columns_match_reference():
    """Pose turn in double, the shared eye origin and the weighted column sums in sample order
    reproduce BatchSim.column_radiance over the reference tracer."""
    scenes = eye_rooms()
    blob, shape, B = np.stack([W.pack_scene(s) for s in scenes]), scenes[0]._shape(), 4
    rays = GOLDEN["eye_ray_d"].shape[1]
    origins = np.broadcast_to(GOLDEN["eye_pos"][:, None].astype(np.float32), (B, rays, 3))
    got = oracle.trace(blob, shape, 1.4, origins=origins, dirs=GOLDEN["eye_ray_d"], batch=B)
    np.testing.assert_array_equal(got, GOLDEN["eye_rad"])
    pose = np.concatenate([GOLDEN["eye_f"], GOLDEN["eye_left"], GOLDEN["eye_up"]], 1)
    got = oracle.trace(blob, shape, 1.4, origins=GOLDEN["eye_pos"], eye_dirs=GOLDEN["eye_dirs"].reshape(-1, 3),
                       pose=pose, weights=GOLDEN["eye_w"], shared_origin=True, batch=B)
    np.testing.assert_array_equal(got, GOLDEN["eye_columns"])


def test_retina_directions_match_reference():
    side = GOLDEN["eye_side"]
    n = pd.DataFrame({"bodyId": 1000 + np.arange(len(side)), "type": "R1-R6", "superclass": "ol_sensory",
                      "nt": "histamine", "hex1": GOLDEN["eye_hex1"], "hex2": GOLDEN["eye_hex2"], "hex_side": side})
    c = Connectome(n, sp.csr_matrix((len(n), len(n)), dtype=np.float32), pd.Series(np.arange(len(n)), index=n.bodyId))
    r = build_retina(c)
    np.testing.assert_array_equal(r.pr_column, GOLDEN["eye_pr_column"])
    np.testing.assert_allclose(r.col_dir, GOLDEN["eye_col_dir"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(r.col_az_el, GOLDEN["eye_col_az_el"], rtol=0, atol=1e-12)
    dirs, w = r.ray_directions()
    np.testing.assert_allclose(dirs, GOLDEN["eye_dirs"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(w, GOLDEN["eye_w"], rtol=0, atol=1e-15)
    # a subset keeps the full eye's directions for the columns it keeps
    keep = np.flatnonzero(n.hex_side.to_numpy() == "R")[:30]
    sub = build_retina(c.subset(keep))
    assert sub.n_columns == 30
    np.testing.assert_array_equal(sub.col_dir, r.col_dir[r.pr_column[keep]])


def test_scene_packing_rules():
    room = W.make_room(0)[0]
    blob = W.pack_scene(room)
    ns, nb, npl = room._shape()
    assert blob.dtype == np.float32 and blob.size == W.scene_floats(ns, nb, npl)
    assert (ns, nb, npl) == (20, 8, 6)
    pn = blob[6 * (ns + nb):6 * (ns + nb + npl)].reshape(npl, 6)[:, 3:]
    np.testing.assert_allclose(np.linalg.norm(pn, axis=1), 1, rtol=1e-6)
    bad = W.World(planes=[W.Plane((0, 0, 0), (0, 0, 1), "floor")], ambient=(-1, 0, 0, 0))
    with pytest.raises(ValueError):
        W.pack_scene(bad)
    with pytest.raises(ValueError):
        W.scene_floats(300, 300, 0)
    with pytest.raises(ValueError, match="unknown fruit set"):
        W.make_room(0, "pear")
    assert len(W.make_room(0, "apple")[0].spheres) == 2


def test_graph_request_requires_cuda():
    with pytest.raises(ValueError, match="CUDA device"):
        W.World(device="cpu").trace(np.zeros((2, 3)), np.ones((2, 3)), cuda_graphs=True)
    with pytest.raises(ValueError, match="CUDA device"):
        W.World(device="cpu").trace(np.zeros((2, 3)), np.ones((2, 3)))
