"""Shared builders for the tests: fixtures, graphs rebuilt from fixtures, raster unpacking."""
from __future__ import annotations

import hashlib
from pathlib import Path

import numpy as np
import pandas as pd
import scipy.sparse as sp
import torch

from flyb200.connectome import Connectome

GOLDEN = Path(__file__).resolve().parent / "golden"


def golden(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz", allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def torch_uniforms(seed: int, steps: int, shape) -> np.ndarray:
    """The reference's Poisson draws: torch.rand(shape) per step from a seeded CPU generator."""
    gen = torch.Generator().manual_seed(seed)
    return np.stack([torch.rand(shape, generator=gen).numpy() for _ in range(steps)])


def connectome_from_fixture(z: dict, extra: tuple = ()) -> Connectome:
    cols = {"bodyId": z["nrn_bodyId"], "type": z["nrn_type"], "superclass": z["nrn_superclass"], "nt": z["nrn_nt"],
            "class": z["nrn_class"]}
    for name in extra:
        cols[name] = z[name]
    n = pd.DataFrame(cols)
    W = sp.csr_matrix((z["W_data"], z["W_indices"], z["W_indptr"]), shape=(len(n), len(n)))
    return Connectome(n, W, pd.Series(np.arange(len(n)), index=n.bodyId.to_numpy()))


def unpack(words: np.ndarray, total: int) -> np.ndarray:
    """[steps][words] uint32 raster -> [steps][total] bool, bit t = i * batch + b."""
    w = np.ascontiguousarray(words).view(np.uint32)
    return np.unpackbits(w.view(np.uint8), bitorder="little").reshape(w.shape[0], -1)[:, :total].astype(bool)
