"""Multi-process fly sharding on CPU (gloo, world size 2): shards stepped on separate ranks with
global-fly Philox keys equal one rank stepping every fly; gradient sums and readout gathers."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from flyb200 import _abi
from flyb200.adjoint import parameter_grads_over_ranks
from flyb200.parallel import allreduce_gradients, gather_rows, shard
from gpu_helpers import LIF_ARRAYS
from test_gpu_lif import case_random

TOTAL = 7


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_covers_every_fly_once():
    for total in (0, 1, 7, 64, 257):
        for world in (1, 2, 3, 8):
            spans = [shard(total, world, r) for r in range(world)]
            flat = [i for f, c in spans for i in range(f, f + c)]
            assert flat == list(range(total))
            assert max(c for _, c in spans) - min(c for _, c in spans) <= 1


def _worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        case = case_random(batch=TOTAL, n=800, edges=12_000, steps=60, seed=11)
        fly0, count = shard(TOTAL, world, rank)
        st = case["state"].copy()
        for k in LIF_ARRAYS:
            setattr(st, k, np.ascontiguousarray(getattr(st, k)[:, fly0:fly0 + count]))
        st.batch = count
        st.ring = np.ascontiguousarray(st.ring[:, :, fly0:fly0 + count])
        oracle.lif_run(st, case["ptr"], case["edges"], case["P"], n_delay=18, flags=case["flags"], nsteps=60,
                       seed=case["seed"], fly0=fly0)
        v = gather_rows(torch.from_numpy(st.v.T.copy()), TOTAL)            # (flies, n) on every rank
        g = torch.full((5,), float(rank + 1), dtype=torch.float64)
        allreduce_gradients([g])
        # the adjoint's reduction of the shared parameters' gradients (OpticAdjoint.backward)
        d_gains, d_tau = torch.full((3,), float(rank + 1)), torch.full((2,), 10.0 * (rank + 1))
        parameter_grads_over_ranks([d_gains, d_tau])
        np.save(os.path.join(out_dir, f"p{rank}.npy"), torch.cat([d_gains, d_tau]).numpy())
        np.save(os.path.join(out_dir, f"v{rank}.npy"), v.numpy())
        np.save(os.path.join(out_dir, f"g{rank}.npy"), g.numpy())
    finally:
        dist.destroy_process_group()


def test_two_rank_shards_equal_single_batch(tmp_path):
    world = 2
    mp.spawn(_worker, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True)
    case = case_random(batch=TOTAL, n=800, edges=12_000, steps=60, seed=11)
    st = case["state"].copy()
    oracle.lif_run(st, case["ptr"], case["edges"], case["P"], n_delay=18, flags=case["flags"], nsteps=60,
                   seed=case["seed"])
    for r in range(world):
        np.testing.assert_array_equal(np.load(tmp_path / f"v{r}.npy"), st.v.T)
        np.testing.assert_array_equal(np.load(tmp_path / f"g{r}.npy"), np.full(5, 3.0))
        np.testing.assert_array_equal(np.load(tmp_path / f"p{r}.npy"), np.array([3, 3, 3, 30, 30], np.float32))
    assert _abi.LIF_POISSON & case["flags"]
