"""The reference's module-level kernel wrappers (names of flyverse/cuda.py), bound to this
library's reference-compatible launchers: launch_lif, launch_optic_dr, launch_optic, launch_csr,
launch_events and launch_means (include/flyb200.h).

Each wrapper describes its launcher's operands as a list of `Operand`s (the tensor and the dtype
and shape it must have); `_launch` checks the whole list before anything runs, packs the device
pointers in the launcher's order and issues the call on the current stream of the operands'
device. Operands are batch-major (B, N) like the reference's tensors. A bad operand raises
ValueError, a launcher status other than 0 raises RuntimeError. The fly-minor engine itself does
not go through this module; `group_means_native` is the readout it does use.
"""
from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp
import torch

from . import _abi

_MAX_ELEMENTS = 2**31          # the launchers index with 32-bit integers


def lib(device=None):
    return _abi.lib()


@dataclass
class Operand:
    """One pointer argument: `shape` None accepts any shape; `dtypes` None accepts any dtype."""
    tensor: torch.Tensor
    shape: tuple | None = None
    dtypes: tuple | None = (torch.float32,)

    def problem(self) -> str | None:
        t = self.tensor
        if self.dtypes is not None and t.dtype not in self.dtypes:
            return f"dtype {t.dtype} (wanted {' or '.join(map(str, self.dtypes))})"
        if self.shape is not None and tuple(t.shape) != tuple(self.shape):
            return f"shape {tuple(t.shape)} (wanted {tuple(self.shape)})"
        if t.numel() >= _MAX_ELEMENTS:
            return f"{t.numel()} elements (the launchers take fewer than 2**31)"
        return None


def _launch(name: str, operands: list[Operand], *scalars) -> None:
    device = operands[0].tensor.device
    if device.type != "cuda":
        raise ValueError(f"{name}: operands must live on a CUDA device, not {device}")
    for k, op in enumerate(operands):
        if op.tensor.device != device:
            raise ValueError(f"{name}: operand {k} is on {op.tensor.device}, operand 0 on {device}")
        if not op.tensor.is_contiguous():
            raise ValueError(f"{name}: operand {k} is not contiguous")
        bad = op.problem()
        if bad:
            raise ValueError(f"{name}: operand {k} has {bad}")
    table = (ct.c_void_p * len(operands))(*[op.tensor.data_ptr() for op in operands])
    with torch.cuda.device(device):
        status = getattr(_abi.lib(), name)(table, *scalars, torch.cuda.current_stream(device).cuda_stream)
    if status:
        raise RuntimeError(f"{name} returned status {status}")


def lif_update(brain, rnd, phase=None):
    """launch_lif on a batch-major brain-like object carrying the reference's field names
    (v, g, drive, adapt, refrac, active, poisson_p, res, std_u_vec, spikes, spike_buf, buf_pos,
    rate, spike_counts, _cuda_P and the flag sources)."""
    B, N = brain.B, brain.n
    bn, n = (B, N), (N,)
    ops = [Operand(brain.v, bn), Operand(brain.g, bn), Operand(brain.drive, bn), Operand(brain.adapt, bn),
           Operand(brain.refrac, bn), Operand(brain.active, n), Operand(brain.poisson_p, bn), Operand(rnd, bn),
           Operand(brain.res, bn), Operand(brain.std_u_vec, n), Operand(brain.spikes, bn),
           Operand(brain.spike_buf[brain.buf_pos], bn), Operand(brain.rate, bn), Operand(brain.spike_counts, bn),
           Operand(brain._cuda_P, (11,)),
           Operand(phase, (8, N)) if phase is not None else Operand(brain._cuda_P, (11,))]
    flags = sum(bit for bit, on in ((1, brain._poisson_on), (2, brain._std_on), (4, brain.record_activity),
                                    (8, brain.p.adapt_jump > 0), (16, phase is not None), (32, brain.cuda_compact))
                if on)
    _launch("launch_lif", ops, N, B, flags)


def optic_dr(v, b, dr):
    """dr = clip(v + b, 0, 1) - b on batch-major (B, n) tensors."""
    if v.ndim != 2:
        raise ValueError(f"optic_dr: v must be a (batch, units) matrix, got {v.ndim} dimensions")
    B, n = v.shape
    _launch("launch_optic_dr", [Operand(v, (B, n)), Operand(b, (n,)), Operand(dr, (B, n))], n, B)


def optic_update(optic, y, pr, sk):
    """The fused rate update of an optic-lobe-like object (v, adapt, _cuda_dr, _a, b_vec, _a_ad, p)."""
    bn, n = (optic.B, optic.n_rate), (optic.n_rate,)
    ops = [Operand(optic.v, bn), Operand(optic.adapt, bn), Operand(optic._cuda_dr, bn), Operand(y.contiguous(), bn),
           Operand(pr.contiguous(), bn), Operand(sk.contiguous(), bn), Operand(optic._a, n), Operand(optic.b_vec, n)]
    _launch("launch_optic", ops, optic.n_rate, optic.B, optic.p.gain_rr, optic.p.adapt_gain, optic._a_ad)


class CSR:
    """A CSR matrix for launch_csr: y (batch, rows) = x (batch, cols) @ M^T, one warp per row."""

    def __init__(self, matrix, device, dtype=torch.float32):
        if dtype not in (torch.float32, torch.float16):
            raise ValueError(f"CSR weights are float32 or float16, not {dtype}")
        m = sp.csr_matrix(matrix, copy=True)
        m.sum_duplicates()
        m.sort_indices()
        m.check_format(full_check=True)
        if m.nnz >= _MAX_ELEMENTS or any(s >= _MAX_ELEMENTS for s in m.shape):
            raise ValueError("CSR dimensions and entry count must fit 32-bit indices")
        self.shape = m.shape
        self.ptr = torch.as_tensor(m.indptr.astype(np.int32), device=device)
        self.idx = torch.as_tensor(m.indices.astype(np.int32), device=device)
        self.values = torch.as_tensor(m.data, dtype=dtype, device=device)

    def matvec(self, x):
        rows, cols = self.shape
        if x.dtype != torch.float32 or x.ndim != 2 or x.shape[1] != cols:
            raise ValueError(f"matvec input must be float32 of shape (batch, {cols})")
        if x.shape[0] * max(rows, cols) >= _MAX_ELEMENTS:
            raise ValueError("matvec batch too large for 32-bit indexing")
        y = torch.empty(x.shape[0], rows, dtype=torch.float32, device=x.device)
        ops = [Operand(self.ptr, dtypes=(torch.int32,)), Operand(self.idx, dtypes=(torch.int32,)),
               Operand(self.values, dtypes=(torch.float32, torch.float16)), Operand(x.contiguous()), Operand(y)]
        _launch("launch_csr", ops, rows, cols, x.shape[0], int(self.values.dtype == torch.float16))
        return y


def event_scatter(ptr, idx, weights, x, g, pre_ids=None):
    """g (B, N) += W x with W given pre-major (CSC ptr / idx / weights); float atomics as the
    reference's event kernel. `pre_ids`: the compact list of presynaptic columns to visit."""
    if x.ndim != 2:
        raise ValueError("event_scatter: x must be a (batch, neurons) matrix")
    B, N = x.shape
    ops = [Operand(ptr, (N + 1,), (torch.int32,)), Operand(idx, None, (torch.int32,)),
           Operand(weights, None, (torch.float32, torch.float16)), Operand(x, (B, N)), Operand(g, (B, N))]
    if idx.ndim != 1 or tuple(weights.shape) != tuple(idx.shape):
        raise ValueError("event_scatter: idx and weights must be vectors of one length")
    if pre_ids is not None and (pre_ids.ndim != 1):
        raise ValueError("event_scatter: pre_ids must be a vector")
    ops.append(Operand(pre_ids if pre_ids is not None else ptr, None, (torch.int32,)))
    _launch("launch_events", ops, N, B, int(weights.dtype == torch.float16), -1 if pre_ids is None else pre_ids.numel())


def group_means_native(ptr, idx, rates_nb, out):
    """out (B, groups) float64 = group means of the fly-minor rates [N][B] (flyb_group_means: the
    reduction of `group_means` without a batch-major copy of the rates)."""
    if rates_nb.ndim != 2:
        raise ValueError("group_means_native: rates must be a fly-minor (N, B) matrix")
    groups, batch = ptr.numel() - 1, rates_nb.shape[1]
    checks = [Operand(ptr, None, (torch.int32,)), Operand(idx, None, (torch.int32,)), Operand(rates_nb),
              Operand(out, (batch, groups), (torch.float64,))]
    for k, op in enumerate(checks):
        bad = op.problem()
        if bad or op.tensor.device != out.device or out.device.type != "cuda" or not op.tensor.is_contiguous():
            raise ValueError(f"group_means_native: operand {k} ({bad or 'device or layout'})")
    if groups <= 0:
        return out
    with torch.cuda.device(out.device):
        status = _abi.lib().flyb_group_means(ptr.data_ptr(), idx.data_ptr(), rates_nb.data_ptr(), out.data_ptr(),
                                             groups, batch, torch.cuda.current_stream(out.device).cuda_stream)
    if status:
        raise RuntimeError(f"flyb_group_means returned status {status}")
    return out


def group_means(ptr, idx, rates, spikes=None):
    """(B, groups [+ 1]) float64: group means of batch-major rates, summed in double in member
    order, plus the per-fly spike totals as a last column when `spikes` is given."""
    if rates.ndim != 2 or ptr.ndim != 1 or idx.ndim != 1:
        raise ValueError("group_means: ptr and idx are vectors, rates a (batch, neurons) matrix")
    groups = ptr.numel() - 1
    if groups < 0 or rates.shape[0] * max(groups, 0) >= _MAX_ELEMENTS:
        raise ValueError("group_means: empty or oversized group table")
    out = torch.empty(rates.shape[0], groups + (spikes is not None), dtype=torch.float64, device=rates.device)
    _launch("launch_means", [Operand(ptr, None, (torch.int32,)), Operand(idx, None, (torch.int32,)), Operand(rates),
                             Operand(out, None, (torch.float64,))], rates.shape[1], groups, rates.shape[0], out.shape[1])
    if spikes is not None:
        bad = Operand(spikes, tuple(rates.shape)).problem()
        if bad:
            raise ValueError(f"group_means: spikes have {bad}")
        torch.sum(spikes, dim=1, out=out[:, -1])
    return out
