"""Module-level wrappers with the reference's names and argument rules (flyverse/cuda.py:82-184),
bound to this library's reference-compatible launchers (launch_lif, launch_optic_dr, launch_optic,
launch_csr, launch_events, launch_means). Tensors are batch-major (B, N), contiguous, on one CUDA
device; launches go on the current stream; a non-zero status raises RuntimeError."""
from __future__ import annotations

import ctypes as ct

import numpy as np
import scipy.sparse as sp
import torch

from . import _abi


def lib(device=None):
    return _abi.lib()


def _call(name, tensors, *args):
    device = tensors[0].device
    for t in tensors:
        if t.device != device or device.type != "cuda" or not t.is_contiguous():
            raise ValueError("CUDA kernels require contiguous tensors on the same CUDA device")
    pointers = (ct.c_void_p * len(tensors))(*(t.data_ptr() for t in tensors))
    with torch.cuda.device(device):
        error = getattr(_abi.lib(), name)(pointers, *args, torch.cuda.current_stream(device).cuda_stream)
    if error:
        raise RuntimeError(f"{name}: CUDA error {error}")


def _float_shapes(tensors, shapes):
    for t, shape in zip(tensors, shapes, strict=True):
        if t.dtype != torch.float32 or tuple(t.shape) != tuple(shape):
            raise ValueError(f"expected float32 tensor of shape {tuple(shape)}, got {t.dtype} {tuple(t.shape)}")
        if t.numel() >= 2**31:
            raise ValueError("CUDA kernels require fewer than 2**31 elements")


def lif_update(brain, rnd, phase=None):
    """One fused LIF update of a batch-major brain-like object (the reference's field names)."""
    tensors = [brain.v, brain.g, brain.drive, brain.adapt, brain.refrac, brain.active, brain.poisson_p, rnd, brain.res,
               brain.std_u_vec, brain.spikes, brain.spike_buf[brain.buf_pos], brain.rate, brain.spike_counts,
               brain._cuda_P]
    flags = int(brain._poisson_on) | (2 * brain._std_on) | (4 * brain.record_activity) | (8 * (brain.p.adapt_jump > 0))
    tensors.append(phase if phase is not None else brain._cuda_P)
    flags |= 16 if phase is not None else 0
    flags |= 32 if brain.cuda_compact else 0
    B, N = brain.B, brain.n
    _float_shapes(tensors, [(B, N)] * 5 + [(N,), (B, N), (B, N), (B, N), (N,)] + [(B, N)] * 4 +
                  [(11,), (8, N) if phase is not None else (11,)])
    _call("launch_lif", tensors, N, B, flags)


def optic_dr(v, b, dr):
    if v.ndim != 2:
        raise ValueError("optic voltage must have shape (batch, neurons)")
    _float_shapes([v, b, dr], [v.shape, (v.shape[1],), v.shape])
    _call("launch_optic_dr", [v, b, dr], v.shape[1], v.shape[0])


def optic_update(optic, y, pr, sk):
    p = optic.p
    tensors = [optic.v, optic.adapt, optic._cuda_dr, y.contiguous(), pr.contiguous(), sk.contiguous(), optic._a,
               optic.b_vec]
    _float_shapes(tensors, [(optic.B, optic.n_rate)] * 6 + [(optic.n_rate,)] * 2)
    _call("launch_optic", tensors, optic.n_rate, optic.B, p.gain_rr, p.adapt_gain, optic._a_ad)


class CSR:
    """Warp-per-row CSR product, batch-major x (batch, cols) -> (batch, rows)."""

    def __init__(self, matrix, device, dtype=torch.float32):
        if dtype not in (torch.float32, torch.float16):
            raise ValueError("CUDA CSR weights must be float32 or float16")
        matrix = sp.csr_matrix(matrix, copy=True)
        matrix.sum_duplicates()
        matrix.sort_indices()
        matrix.check_format(full_check=True)
        if max(matrix.shape, default=0) >= 2**31 or matrix.nnz >= 2**31:
            raise ValueError("CUDA CSR requires 32-bit dimensions and indices")
        self.shape = matrix.shape
        self.ptr = torch.as_tensor(matrix.indptr.astype(np.int32), device=device)
        self.idx = torch.as_tensor(matrix.indices.astype(np.int32), device=device)
        self.values = torch.as_tensor(matrix.data, dtype=dtype, device=device)

    def matvec(self, x):
        if x.ndim != 2 or x.shape[1] != self.shape[1] or x.dtype != torch.float32:
            raise ValueError("CSR input must be float32 (batch, columns)")
        if max(x.numel(), x.shape[0] * self.shape[0]) >= 2**31:
            raise ValueError("CUDA CSR batch is too large")
        y = torch.empty(x.shape[0], self.shape[0], dtype=torch.float32, device=x.device)
        _call("launch_csr", [self.ptr, self.idx, self.values, x.contiguous(), y], *self.shape, x.shape[0],
              int(self.values.dtype == torch.float16))
        return y


def event_scatter(ptr, idx, weights, x, g, pre_ids=None):
    if ptr.dtype != torch.int32 or idx.dtype != torch.int32:
        raise ValueError("CUDA events require int32 indices")
    if x.ndim != 2 or ptr.shape != (x.shape[1] + 1,) or idx.ndim != 1 or weights.shape != idx.shape:
        raise ValueError("invalid CSC buffers or input shape")
    if weights.dtype not in (torch.float16, torch.float32):
        raise ValueError("CUDA event weights must be float32 or float16")
    _float_shapes([x, g], [x.shape, x.shape])
    if pre_ids is not None and (pre_ids.dtype != torch.int32 or pre_ids.ndim != 1):
        raise ValueError("compact presynaptic indices must be an int32 vector")
    _call("launch_events", [ptr, idx, weights, x, g, ptr if pre_ids is None else pre_ids], x.shape[1], x.shape[0],
          int(weights.dtype == torch.float16), -1 if pre_ids is None else pre_ids.numel())


def group_means_native(ptr, idx, rates_nb, out):
    """out (B, groups) float64 = group means of the fly-minor rates [N][B] (flyb_group_means: the
    reduction of `group_means` without a batch-major copy of the rates)."""
    if ptr.dtype != torch.int32 or idx.dtype != torch.int32 or rates_nb.dtype != torch.float32 or rates_nb.ndim != 2:
        raise ValueError("group indices must be int32 vectors; rates must be a float32 (N, B) matrix")
    groups, batch = ptr.numel() - 1, rates_nb.shape[1]
    if out.dtype != torch.float64 or tuple(out.shape) != (batch, groups):
        raise ValueError(f"out must be float64 of shape ({batch}, {groups})")
    for t in (ptr, idx, rates_nb, out):
        if t.device != out.device or t.device.type != "cuda" or not t.is_contiguous():
            raise ValueError("CUDA kernels require contiguous tensors on the same CUDA device")
    if groups <= 0:
        return out
    with torch.cuda.device(out.device):
        error = _abi.lib().flyb_group_means(ptr.data_ptr(), idx.data_ptr(), rates_nb.data_ptr(), out.data_ptr(),
                                            groups, batch, torch.cuda.current_stream(out.device).cuda_stream)
    if error:
        raise RuntimeError(f"flyb_group_means: CUDA error {error}")
    return out


def group_means(ptr, idx, rates, spikes=None):
    """(B, groups [+1]) float64 means of rates over index groups (+ spike totals)."""
    if ptr.dtype != torch.int32 or idx.dtype != torch.int32 or ptr.ndim != 1 or idx.ndim != 1 or rates.ndim != 2:
        raise ValueError("group indices must be int32 vectors; rates must be a matrix")
    _float_shapes([rates], [rates.shape])
    if ptr.numel() < 1 or rates.shape[0] * (ptr.numel() - 1) >= 2**31:
        raise ValueError("invalid or oversized group table")
    groups = ptr.numel() - 1
    result = torch.empty(rates.shape[0], groups + int(spikes is not None), dtype=torch.float64, device=rates.device)
    _call("launch_means", [ptr, idx, rates, result], rates.shape[1], groups, rates.shape[0], result.shape[1])
    if spikes is not None:
        _float_shapes([spikes], [rates.shape])
        torch.sum(spikes, dim=1, out=result[:, -1])
    return result
