"""ORACLE (test infrastructure): the optic rate dynamics in FP64, parameterised by per-type-pair
gains and per-type time constants, for checking the hand-written adjoint.

  W_ij = gain[pair(j -> i)] * W0_ij      a_i = exp(-dt / tau[type(i)])      aad = exp(-dt / adapt_tau)
  dr = clip(v + b, 0, 1) - b;  inp = gr * W dr + pr - ga * adapt;  inp = inp + spk
  v <- inp + (v - inp) * a;    adapt <- dr + (adapt - dr) * aad        (flyverse/optic.py:644-669)

`rollout` (numpy FP64) feeds central finite differences; `torch_grads` runs the same expressions
through torch autograd in float64 (the reference's differentiable spelling, optic.py:606-676).
The reference has no adjoint, so these are the pin ("parity" of the gradients is against FP64).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import torch


def rollout(W0: sp.csr_matrix, pair_id, gains, tau, type_of, b, v0, ad0, pr, spk, *, dt, gr, ga, adapt_tau, steps):
    """FP64 rollout on [m][B] state; returns (v_T, adapt_T)."""
    W = W0.astype(np.float64).copy()
    W.data = W.data * np.asarray(gains, np.float64)[pair_id]
    a = np.exp(-dt / np.asarray(tau, np.float64)[type_of])[:, None]
    aad = np.exp(-dt / adapt_tau)
    b = np.asarray(b, np.float64)[:, None]
    v, ad = np.array(v0, np.float64), np.array(ad0, np.float64)
    for _ in range(steps):
        dr = np.clip(v + b, 0.0, 1.0) - b
        inp = gr * (W @ dr) + pr - ga * ad
        inp = inp + spk
        v = inp + (v - inp) * a
        ad = dr + (ad - dr) * aad
    return v, ad


def readout(v, b, weights) -> float:
    """L = sum_i,b weights_i * clip(v_ib + b_i, 0, 1)."""
    return float((np.clip(v + np.asarray(b, np.float64)[:, None], 0, 1) * np.asarray(weights, np.float64)[:, None]).sum())


def central_differences(loss, x0: np.ndarray, idx, h: float = 1e-4) -> np.ndarray:
    """d loss / d x0[k] for k in idx by (L(x + h) - L(x - h)) / 2h in FP64."""
    out = np.zeros(len(idx))
    for n, k in enumerate(idx):
        xp, xm = x0.copy(), x0.copy()
        xp[k] += h
        xm[k] -= h
        out[n] = (loss(xp) - loss(xm)) / (2 * h)
    return out


def torch_grads(W0: sp.csr_matrix, pair_id, gains, tau, type_of, b, v0, ad0, pr, spk, weights, *, dt, gr, ga,
                adapt_tau, steps):
    """(dL/dgains, dL/dtau) by torch autograd in float64 through the same expressions."""
    d = torch.float64
    pid = torch.from_numpy(np.asarray(pair_id, np.int64))            # pair of each CSR entry of W0
    g = torch.tensor(np.asarray(gains, np.float64), requires_grad=True)
    t = torch.tensor(np.asarray(tau, np.float64), requires_grad=True)
    vals = torch.from_numpy(W0.data.astype(np.float64)) * g[pid]
    rows = torch.from_numpy(np.repeat(np.arange(W0.shape[0]), np.diff(W0.indptr)))
    Wd = torch.zeros(W0.shape, dtype=d).index_put((rows, torch.from_numpy(W0.indices.astype(np.int64))), vals,
                                                  accumulate=True)
    a = torch.exp(-dt / t[torch.from_numpy(np.asarray(type_of, np.int64))])[:, None]
    aad = float(np.exp(-dt / adapt_tau))
    bb = torch.from_numpy(np.asarray(b, np.float64))[:, None]
    v, ad = torch.from_numpy(np.array(v0, np.float64)), torch.from_numpy(np.array(ad0, np.float64))
    prt, spkt = torch.from_numpy(np.asarray(pr, np.float64)), torch.from_numpy(np.asarray(spk, np.float64))
    for _ in range(steps):
        dr = (v + bb).clamp(0, 1) - bb
        inp = gr * (Wd @ dr) + prt - ga * ad
        inp = inp + spkt
        v = inp + (v - inp) * a
        ad = dr + (ad - dr) * aad
    L = ((v + bb).clamp(0, 1) * torch.from_numpy(np.asarray(weights, np.float64))[:, None]).sum()
    L.backward()
    return g.grad.numpy(), t.grad.numpy(), float(L)
