"""Graph container and cache I/O, interface-compatible with flyverse/connectome.py.

`Connectome(neurons, W, body_to_index)` holds the neuron table (row i = neuron i) and
W[post, pre] = signed synapse count as a float32 scipy CSR matrix (connectome.py:394-399). The
in-degree totals `in_syn` (sum |W| per row) and `in_syn_l2` (L2 norm per row) are filled in as the
reference does (connectome.py:439-446), since the LIF fan-in scale and the optic normalisation
read them. `load(cache_dir)` reads the reference's cache layout (`neurons.parquet`,
`W_post_pre.npz`, and `reference_neurons.parquet` / `reference_W.npz` for a saved subset;
connectome.py:870-895); compiling the raw MaleCNS feather tables is not part of this package.
"""
from __future__ import annotations

import json
import re
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
import pandas as pd
import scipy.sparse as sp

# Fast-synapse sign of each transmitter (the data convention of flyverse/connectome.py:44-50).
NT_SIGN = {"acetylcholine": 1.0, "gaba": -1.0, "glutamate": -1.0, "histamine": -1.0,
           "dopamine": 0.0, "octopamine": 0.0, "serotonin": 0.0, "tyramine": 0.0, "unknown": 0.0}
PHOTORECEPTOR_TYPES = ["R1-R6", "R7y", "R7p", "R7d", "R7_unclear", "R8y", "R8p", "R8d", "R8_unclear", "R7R8_unclear"]


@dataclass
class Connectome:
    neurons: pd.DataFrame
    W: sp.csr_matrix
    body_to_index: pd.Series
    _reference: "Connectome | None" = field(default=None, repr=False)
    _norm_cache: dict = field(default_factory=dict, repr=False)
    dataset: str = "malecns"
    release: str = "v1.0"

    def __post_init__(self):
        self.W = sp.csr_matrix(self.W, dtype=np.float32)
        missing = [k for k in ("in_syn", "in_syn_l2") if k not in self.neurons]
        if missing:
            l1, l2 = row_norms(self.W)
            fill = {"in_syn": l1, "in_syn_l2": l2}
            for k in missing:
                self.neurons[k] = fill[k]

    @property
    def n(self) -> int:
        return len(self.neurons)

    @property
    def reference(self) -> "Connectome":
        """The original graph a subset was cut from (fan-in normalisation reads it)."""
        return self if self._reference is None else self._reference

    @property
    def has_optic_columns(self) -> bool:
        return "hex1" in self.neurons

    def require(self, capability: str) -> None:
        if capability == "optic_columns" and not self.has_optic_columns:
            raise ValueError("this connectome has no optic column map")

    def index_of(self, body_ids) -> np.ndarray:
        return self.body_to_index.loc[np.asarray(body_ids)].to_numpy()

    def indices(self, selection) -> np.ndarray:
        """Row numbers of a selection (connectome.py:453-467): a dict of `select` criteria, a boolean
        mask with one entry per neuron, or distinct in-range integer rows in the caller's order.
        Anything else raises ValueError."""
        if isinstance(selection, dict):
            return self.select(**selection)
        arr = np.asarray(selection)
        if arr.dtype == np.bool_:
            if arr.shape != (self.n,):
                raise ValueError(f"a boolean selection needs shape ({self.n},), got {arr.shape}")
            return np.nonzero(arr)[0]
        if arr.ndim != 1:
            raise ValueError(f"a row selection must be one-dimensional, got {arr.ndim} dimensions")
        if arr.size == 0:
            return np.zeros(0, np.int64)
        if not np.issubdtype(arr.dtype, np.integer):
            raise ValueError(f"row numbers must be integers, got {arr.dtype}")
        rows = arr.astype(np.int64)
        if rows.min() < 0 or rows.max() >= self.n:
            raise ValueError(f"row numbers must lie in [0, {self.n})")
        if np.unique(rows).size != rows.size:
            raise ValueError("row numbers must not repeat")
        return rows

    def select(self, **criteria) -> np.ndarray:
        """Rows meeting every criterion column=value (connectome.py:604-616): a list, tuple, set or
        array is a set of accepted values, a string starting with '~' a regular expression searched
        in the column's text (missing values read as ''), anything else an exact value."""
        keep = np.ones(self.n, dtype=bool)
        for column, wanted in criteria.items():
            keep &= _column_matches(self.neurons[column], wanted)
        return np.nonzero(keep)[0]

    def subset(self, selection) -> "Connectome":
        """Induced subgraph in selection order; normalisation keeps reading the original graph."""
        idx = self.indices(selection)
        neurons = self.neurons.iloc[idx].copy().reset_index(drop=True)
        return Connectome(neurons, self.W[idx][:, idx].tocsr(), pd.Series(np.arange(len(idx)), index=neurons.bodyId.to_numpy()),
                          self.reference, dataset=self.dataset, release=self.release)

    def describe(self, idx) -> pd.DataFrame:
        cols = [c for c in ("bodyId", "type", "instance", "superclass", "somaSide", "nt") if c in self.neurons]
        return self.neurons.iloc[np.asarray(idx)][cols]


def row_norms(W: sp.csr_matrix) -> tuple[np.ndarray, np.ndarray]:
    """Per postsynaptic row the L1 norm (sum |w|) and the L2 norm of W, as float32: the in-degree
    totals `in_syn` / `in_syn_l2` that the fan-in scale and the optic normalisation read. Summed
    in float64 (exact for integer synapse counts), then rounded once to float32."""
    W = sp.csr_matrix(W)
    row = np.repeat(np.arange(W.shape[0]), np.diff(W.indptr))
    w = W.data.astype(np.float64)
    l1 = np.bincount(row, weights=np.abs(w), minlength=W.shape[0])
    sq = np.bincount(row, weights=w * w, minlength=W.shape[0])
    return l1.astype(np.float32), np.sqrt(sq).astype(np.float32)


def _column_matches(column: pd.Series, wanted) -> np.ndarray:
    if isinstance(wanted, str) and wanted[:1] == "~":
        pattern = re.compile(wanted[1:])
        text = column.fillna("").astype(str)
        return np.fromiter((pattern.search(t) is not None for t in text), dtype=bool, count=len(text))
    if isinstance(wanted, (list, tuple, set, np.ndarray)):
        return column.isin(list(wanted)).to_numpy()
    return (column == wanted).to_numpy()


def from_arrays(neurons: pd.DataFrame, W) -> Connectome:
    """A connectome whose rows are the table's rows, body ids from its `bodyId` column."""
    neurons = neurons.reset_index(drop=True)
    return Connectome(neurons, sp.csr_matrix(W, dtype=np.float32), pd.Series(np.arange(len(neurons)), index=neurons.bodyId.to_numpy()))


def save(c: Connectome, cache_dir) -> None:
    """Write the reference cache layout (connectome.py:751-804, graph files only)."""
    cache_dir = Path(cache_dir)
    cache_dir.mkdir(parents=True, exist_ok=True)
    (cache_dir / "manifest.json").write_text(json.dumps({"dataset": c.dataset, "release": c.release}), encoding="utf-8")
    c.neurons.to_parquet(cache_dir / "neurons.parquet")
    sp.save_npz(cache_dir / "W_post_pre.npz", c.W, compressed=False)
    if c.reference is not c:
        c.reference.neurons.to_parquet(cache_dir / "reference_neurons.parquet")
        sp.save_npz(cache_dir / "reference_W.npz", c.reference.W, compressed=False)
    else:
        for name in ("reference_neurons.parquet", "reference_W.npz"):
            (cache_dir / name).unlink(missing_ok=True)


def load(cache_dir=None, rebuild: bool = False, verbose: bool = True, type_nt_override=None, *, dataset=None,
         **_ignored) -> Connectome:
    """Read a compiled graph cache (the reference's `load`, connectome.py:820-895, read path).

    `cache_dir` is the directory holding `neurons.parquet` and `W_post_pre.npz` (a cache written by
    the reference or by `save`). Rebuilding from the raw dataset tables is not available here."""
    if cache_dir is None:
        raise ValueError("flyb200.connectome.load needs cache_dir: the directory of a compiled graph cache")
    if rebuild:
        raise ValueError("compiling the raw connectome tables is not part of flyb200; load a compiled cache")
    cache_dir = Path(cache_dir)
    manifest = {}
    if (cache_dir / "manifest.json").exists():
        manifest = json.loads((cache_dir / "manifest.json").read_text(encoding="utf-8"))
    ds = dataset or manifest.get("dataset", "malecns")
    neurons = pd.read_parquet(cache_dir / "neurons.parquet")
    W = sp.load_npz(cache_dir / "W_post_pre.npz").tocsr()
    reference = None
    if (cache_dir / "reference_W.npz").exists():
        rn = pd.read_parquet(cache_dir / "reference_neurons.parquet")
        reference = Connectome(rn, sp.load_npz(cache_dir / "reference_W.npz").tocsr(),
                               pd.Series(np.arange(len(rn)), index=rn.bodyId.to_numpy()), dataset=ds)
    if verbose:
        print(f"flyb200: loaded {len(neurons):,} neurons, {W.nnz:,} synapse entries from {cache_dir}")
    return Connectome(neurons, W, pd.Series(np.arange(len(neurons)), index=neurons.bodyId.to_numpy()), reference,
                      dataset=ds, release=manifest.get("release", "v1.0"))
