"""The graph cache interchange (connectome.py:751-896): a cache the reference's own `save` wrote is
read by flyb200.connectome.load as the reference reads it; a cache flyb200 writes round-trips and
the reference reads it as its own (recorded by tests/golden/make_golden.py, `ref_cache`)."""
import numpy as np
import pandas as pd
import pytest

from flyb200 import connectome
from helpers import GOLDEN, golden


def test_reference_written_cache_loads_as_the_reference_reads_it():
    z = golden("ref_cache")
    c = connectome.load(GOLDEN / "ref_cache", verbose=False)
    assert c.n == int(z["n"]) and c.W.nnz == int(z["nnz"])
    np.testing.assert_array_equal(c.W.data, z["W_data"])
    np.testing.assert_array_equal(c.W.indices, z["W_indices"])
    np.testing.assert_array_equal(c.W.indptr, z["W_indptr"])
    np.testing.assert_array_equal(c.neurons.bodyId.to_numpy(), z["body"])
    np.testing.assert_array_equal(c.neurons["in_syn"].to_numpy(), z["in_syn"])
    np.testing.assert_array_equal(c.neurons["in_syn_l2"].to_numpy(), z["in_syn_l2"])
    assert list(c.neurons.columns) == list(z["columns"])
    assert c.reference is not c and c.reference.n == int(z["ref_n"])      # the saved subset keeps its origin
    np.testing.assert_array_equal(c.reference.neurons.bodyId.to_numpy(), z["ref_body"])
    np.testing.assert_array_equal(c.index_of(z["body"][[2, 0]]), [2, 0])


def test_row_norms_equal_the_references_in_degree_columns():
    """in_syn / in_syn_l2, recomputed when a table lacks them, equal the columns the reference stored
    for its full graph (a subset keeps the values of the graph it was cut from)."""
    z = golden("ref_cache")
    c = connectome.load(GOLDEN / "ref_cache", verbose=False)
    full = c.reference
    l1, l2 = connectome.row_norms(full.W)
    np.testing.assert_array_equal(l1, full.neurons["in_syn"].to_numpy())
    np.testing.assert_array_equal(l2, full.neurons["in_syn_l2"].to_numpy())
    rows = full.index_of(z["body"])
    np.testing.assert_array_equal(l1[rows], z["in_syn"])
    bare = connectome.Connectome(full.neurons.drop(columns=["in_syn", "in_syn_l2"]), full.W, full.body_to_index)
    np.testing.assert_array_equal(bare.neurons["in_syn_l2"].to_numpy(), full.neurons["in_syn_l2"].to_numpy())


def test_flyb200_cache_round_trips_and_the_reference_reads_it_alike(tmp_path):
    z = golden("ref_cache")
    assert str(z["digest_flyb200_cache"]) == str(z["digest_reference_cache"])
    c = connectome.load(GOLDEN / "ref_cache", verbose=False)
    connectome.save(c, tmp_path / "cache")
    d = connectome.load(tmp_path / "cache", verbose=False)
    assert (d.W != c.W).nnz == 0 and (d.reference.W != c.reference.W).nnz == 0
    pd.testing.assert_frame_equal(d.neurons, c.neurons)
    full = c.reference
    connectome.save(full, tmp_path / "full")                  # no subset: no reference_* files
    assert not (tmp_path / "full" / "reference_W.npz").exists()
    assert connectome.load(tmp_path / "full", verbose=False).reference.n == full.n


def test_selection_rules():
    c = connectome.load(GOLDEN / "ref_cache", verbose=False)
    t = c.neurons.type.to_numpy()
    np.testing.assert_array_equal(c.select(type="Mi1"), np.flatnonzero(t == "Mi1"))
    np.testing.assert_array_equal(c.select(type="~^DNa0"), np.flatnonzero(np.char.startswith(t.astype(str), "DNa0")))
    np.testing.assert_array_equal(c.select(type=["Mi1", "Pm1"]), np.flatnonzero(np.isin(t, ["Mi1", "Pm1"])))
    np.testing.assert_array_equal(c.indices({"type": "LC4"}), c.select(type="LC4"))
    mask = np.zeros(c.n, bool)
    mask[[1, 3]] = True
    np.testing.assert_array_equal(c.indices(mask), [1, 3])
    np.testing.assert_array_equal(c.indices([3, 1]), [3, 1])
    assert c.indices(np.zeros(0, np.float32)).size == 0
    for bad in ([1, 1], [c.n], [-1], [[1]], [0.5], np.ones(c.n + 1, bool)):
        with pytest.raises(ValueError):
            c.indices(np.asarray(bad))
