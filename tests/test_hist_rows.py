"""Brain._clear_hist_rows (the spike-history part of Brain.reset(rows)) on CPU tensors: the per-fly-
group mask used when the batch is a multiple of 32 clears exactly the bits the full (neuron, fly)
mask clears, and the full mask still serves other batch widths."""
from types import SimpleNamespace

import numpy as np
import torch

from flyb200.brain import Brain


def _full_mask_clear(h0, n, B, words, rows):
    flat = (np.arange(n)[:, None] * B + np.asarray(rows)[None, :]).ravel()
    mask = np.zeros(words * 32, bool)
    mask[flat] = True
    keep = ~np.packbits(mask, bitorder="little").view(np.uint32)
    return h0 & torch.from_numpy(keep.view(np.int32))


def test_group_mask_clears_the_same_bits_as_the_full_mask():
    rng = np.random.default_rng(0)
    for B in (32, 64, 256):
        n, D = 37, 5
        words = n * B // 32
        h0 = torch.from_numpy(rng.integers(-2**31, 2**31, (D, words), dtype=np.int64).astype(np.int32))
        for rows in (rng.choice(B, size=7, replace=False), np.array([0, B - 1, 0]), np.arange(B)):
            fake = SimpleNamespace(n=n, B=B, n_delay=D, words=words, device="cpu", _hist=h0.clone())
            Brain._clear_hist_rows(fake, rows)
            assert torch.equal(fake._hist, _full_mask_clear(h0, n, B, words, rows)), (B, rows)


def test_other_batch_widths_use_the_full_mask():
    rng = np.random.default_rng(1)
    n, D, B = 41, 3, 5
    words = -(-n * B // 32)
    h0 = torch.from_numpy(rng.integers(-2**31, 2**31, (D, words), dtype=np.int64).astype(np.int32))
    fake = SimpleNamespace(n=n, B=B, n_delay=D, words=words, device="cpu", _hist=h0.clone())
    Brain._clear_hist_rows(fake, np.array([1, 4]))
    assert torch.equal(fake._hist, _full_mask_clear(h0, n, B, words, [1, 4]))
