"""The host tables of pull delivery (brain.pull_inputs): decoded back, they give W x spikes exactly
for signed counts whose chunk ranges fit the packed entries (8 bits) and those that need the
16-plane table, empty rows and padding included."""
import numpy as np
import scipy.sparse as sp

from flyb200.brain import PULL_PAD, pull_inputs


def _decode_product(ptr, pre, planes, meta, S, x):
    n = len(ptr) - 1
    out = np.zeros((n, x.shape[1]), np.int64)
    if S == 0:                                        # packed: pre | excess << 24
        e = pre.view(np.uint32).astype(np.int64)
        pre, exc = np.where((e & PULL_PAD) == PULL_PAD, -1, e & PULL_PAD), e >> 24
    else:
        pl = planes.reshape(-1, S).astype(np.int64)
    for r in range(n):
        for c in range(ptr[r], ptr[r + 1]):
            base, used = int(meta[c]) >> 5, int(meta[c]) & 31
            for lane in range(32):
                j = pre[c * 32 + lane]
                if j < 0:
                    continue
                if S == 0:
                    d = int(exc[c * 32 + lane])
                    assert d < (1 << used)
                else:
                    d = sum(((pl[c, q] >> lane) & 1) << q for q in range(used))
                out[r] += (base + d) * x[j]
    return out


def test_pull_tables_reproduce_the_product():
    rng = np.random.default_rng(0)
    w = np.float32(0.275)
    for lim, want_s in ((100, 0), (3000, 16)):
        n = 200
        W = sp.random(n, n, density=0.15, random_state=int(lim), format="csr")
        W.data = (rng.integers(-lim, lim, W.nnz) * w).astype(np.float32)
        W = W.tolil()
        W[5, :] = 0                                   # an empty row
        W = W.tocsr()
        W.eliminate_zeros()
        ptr, pre, planes, meta, S = pull_inputs(W, w)
        assert S == want_s and ptr[6] == ptr[5]
        x = (rng.random((n, 64)) < 0.3).astype(np.int64)
        C = np.round(W.toarray() / w).astype(np.int64)
        np.testing.assert_array_equal(_decode_product(ptr, pre, planes, meta, S, x), C @ x)
        assert (meta & 31).mean() < (S or 8)          # sorted chunks need fewer planes than the stride
        assert planes.size == (0 if S == 0 else (ptr[-1] * S))


def test_pull_tables_refuse_non_integer_weights():
    W = sp.csr_matrix(np.array([[0.0, 0.3], [0.1, 0.0]], np.float32))
    assert pull_inputs(W, 0.275) is None
