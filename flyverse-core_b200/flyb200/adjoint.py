"""Gradients of the optic-lobe rate dynamics through a hand-written adjoint (flyb_optic_adjoint).

The reference differentiates the lobe with torch autograd through its functional frame
(flyverse/optic.py:606-676), which keeps every substep's graph in memory. Here the forward pass
keeps only a checkpoint of (v, adapt) every `checkpoint` substeps; the backward pass recomputes
each segment with its histories (v_t, inp_t) and runs the reverse recurrence on the device:
W_rr^T products with the rectifier masks, per-edge accumulation for the pair gains and per-unit
accumulation for the time constants (the equations are in csrc/adjoint.cu). Gradients are FP32;
FP64 is used only by the check (oracle/optic64.py).

Parameters: per-type-pair gains g (W_ij = g[pair(j -> i)] * W0_ij) and per-type time constants tau
(a_i = exp(-dt / tau[type(i)])). `OpticRollout.apply` wraps one checkpointed rollout as a
torch.autograd.Function from (gains, tau, v0, adapt0) to (v_T, adapt_T). The parameter gradients
are segmented FP32 sums on the device (flyb_segment_sum). Under torch.distributed each rank
rolls out its own flies and the parameter gradients are summed over ranks.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import scipy.sparse as sp
import torch

from . import _abi
from .optic import DeviceCSR, OpticCore
from .parallel import allreduce_gradients


class OpticAdjoint:
    def __init__(self, W0: sp.csr_matrix, pair_id: np.ndarray, n_pairs: int, type_of: np.ndarray, n_types: int,
                 b: np.ndarray, pr: torch.Tensor, spk: torch.Tensor, *, dt_ms: float, gain_rr: float = 1.0,
                 adapt_gain: float = 1.0, adapt_tau_ms: float = 400.0, batch: int = 1, device="cuda",
                 checkpoint: int = 20, launch: str = "persistent"):
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.B, self.C, self.dt = int(batch), int(checkpoint), float(dt_ms)
        self.gr, self.ga = float(gain_rr), float(adapt_gain)
        self.aad = float(np.exp(-dt_ms / adapt_tau_ms))
        self.n_pairs, self.n_types = int(n_pairs), int(n_types)
        W0 = sp.csr_matrix(W0, dtype=np.float32)
        W0.sort_indices()
        dev = self.device
        self.core = OpticCore(W0, np.ones(W0.shape[0], np.float32), b, batch=self.B, device=dev, gain_rr=self.gr,
                              adapt_gain=self.ga, aad=self.aad, launch=launch)
        self.m = self.core.m
        self.W0 = torch.from_numpy(W0.data.astype(np.float32)).to(dev)
        self.pair_id = torch.from_numpy(np.asarray(pair_id, np.int64)).to(dev)
        self.type_of = torch.from_numpy(np.asarray(type_of, np.int64)).to(dev)
        self.core.pr_in.copy_(pr)
        self.core.spk_in.copy_(spk)
        self.WT, self.perm = self.core.W.transpose(dev)
        # the per-edge accumulator is kept in the transposed order the reverse pass walks (coalesced,
        # single writer); the pair reduction reads W0 and the pair ids in that order too
        perm = self.perm.long()
        self.W0_t, self.pair_t = self.W0[perm].contiguous(), self.pair_id[perm].contiguous()
        # the parameter gradients are segmented sums (flyb_segment_sum): the accumulator's edges
        # grouped by pair, the units grouped by type
        self._pair_seg = self._segments(self.pair_t.cpu().numpy(), self.n_pairs)
        self._type_seg = self._segments(np.asarray(type_of, np.int64), self.n_types)
        self._d_gains = torch.zeros(self.n_pairs, device=dev)
        self._d_tau = torch.zeros(self.n_types, device=dev)
        self.launch = launch
        # with a process group, each rank holds its own shard of flies and the parameters are shared:
        # their gradients are summed over ranks (NCCL over NVLink between GPUs)
        self.reduce_over_ranks = True
        M, B = self.m, self.B
        self.lam_v = torch.zeros(M, B, device=dev)
        self.lam_a = torch.zeros(M, B, device=dev)
        self.mu0 = torch.zeros(M, B, device=dev)
        self.mu1 = torch.zeros(M, B, device=dev)
        self.g_edge = torch.zeros(W0.nnz, device=dev)
        self.g_a = torch.zeros(M, device=dev)
        self.v_hist = torch.zeros(self.C, M, B, device=dev)
        self.inp_hist = torch.zeros(self.C, M, B, device=dev)
        self._status = torch.zeros(4, dtype=torch.int32, device=dev)
        self._sync = torch.zeros(64, dtype=torch.int32, device=dev)
        self.ckpt = []

    def _segments(self, key: np.ndarray, count: int):
        """(ptr [count + 1], positions grouped by key) as int32 device tensors."""
        order = np.argsort(key, kind="stable").astype(np.int32)
        ptr = np.concatenate([[0], np.cumsum(np.bincount(key, minlength=count))]).astype(np.int32)
        return torch.from_numpy(ptr).to(self.device), torch.from_numpy(order).to(self.device)

    def _segment_sum(self, seg, x: torch.Tensor, w: torch.Tensor | None, alpha: float, out: torch.Tensor) -> None:
        ptr, idx = seg
        with torch.cuda.device(self.device):
            rc = _abi.lib().flyb_segment_sum(ptr.data_ptr(), idx.data_ptr(), x.data_ptr(),
                                             None if w is None else w.data_ptr(), alpha, out.data_ptr(),
                                             out.numel(), torch.cuda.current_stream(self.device).cuda_stream)
        if rc:
            raise RuntimeError(f"flyb_segment_sum: error {rc}")

    # ------------------------------------------------------------------ parameters
    def set_params(self, gains: torch.Tensor, tau: torch.Tensor) -> None:
        g = gains.to(self.device, torch.float32)
        self.core.W.w.copy_(g[self.pair_id] * self.W0)
        self.core.W.refresh_cw()
        self.WT.w.copy_(self.core.W.w[self.perm.long()])
        self.tau = tau.to(self.device, torch.float32)
        self.core.a.copy_(torch.exp(-self.dt / self.tau[self.type_of]))

    # ------------------------------------------------------------------ passes
    def forward(self, v0: torch.Tensor, adapt0: torch.Tensor, steps: int):
        """Run `steps` substeps from (v0, adapt0) [m][B]; keeps a checkpoint every C substeps."""
        self.core.v_s.copy_(v0)
        self.core.adapt_s.copy_(adapt0)
        self.steps, self.ckpt = int(steps), []
        done = 0
        while done < self.steps:
            n = min(self.C, self.steps - done)
            self.ckpt.append((self.core.v_s.clone(), self.core.adapt_s.clone(), n))
            self.core.substeps(n)
            done += n
        return self.core.v_s.clone(), self.core.adapt_s.clone()

    def backward(self, dv_T: torch.Tensor, dadapt_T: torch.Tensor | None = None):
        """Adjoints at the end -> (d gains, d tau, d v0, d adapt0)."""
        self.lam_v.copy_(dv_T)
        if dadapt_T is None:
            self.lam_a.zero_()
        else:
            self.lam_a.copy_(dadapt_T)
        self.g_edge.zero_()
        self.g_a.zero_()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        for v_c, a_c, n in reversed(self.ckpt):
            self.core.v_s.copy_(v_c)
            self.core.adapt_s.copy_(a_c)
            self.core.substeps(n, self.v_hist, self.inp_hist)       # recompute with histories
            args = _abi.AdjointArgs(m=self.m, batch=self.B, nsteps=n, launch=_abi.LAUNCHES_BY_NAME[self.launch],
                                    t_ptr=self.WT.ptr.data_ptr(), t_col=self.WT.col.data_ptr(), t_w=self.WT.w.data_ptr(),
                                    t_perm=None, v_hist=self.v_hist.data_ptr(),
                                    inp_hist=self.inp_hist.data_ptr(), a=self.core.a.data_ptr(), b=self.core.b.data_ptr(),
                                    gr=self.gr, ga=self.ga, aad=self.aad, lam_v=self.lam_v.data_ptr(),
                                    lam_a=self.lam_a.data_ptr(), lam_tmp=self.mu1.data_ptr(), mu=self.mu0.data_ptr(),
                                    g_edge=self.g_edge.data_ptr(), g_a=self.g_a.data_ptr(),
                                    status=self._status.data_ptr(), sync=self._sync.data_ptr())
            with torch.cuda.device(self.device):
                rc = _abi.lib().flyb_optic_adjoint(ct.byref(args), stream)
            if rc:
                raise RuntimeError(f"flyb_optic_adjoint: error {rc}")
        # dL/dgain_p = gr * sum over the pair's edges of W0_e * g_edge[e];
        # dL/dtau_k = dt / tau_k^2 * sum over the type's units of g_a[i] * a_i   (all FP32)
        self._segment_sum(self._pair_seg, self.g_edge, self.W0_t, self.gr, self._d_gains)
        self._segment_sum(self._type_seg, self.g_a, self.core.a, 1.0, self._d_tau)
        d_tau = self._d_tau * (self.dt / (self.tau * self.tau))
        d_gains = self._d_gains.clone()
        if self.reduce_over_ranks:
            parameter_grads_over_ranks([d_gains, d_tau])
        return d_gains, d_tau, self.lam_v.clone(), self.lam_a.clone()

    def check(self) -> None:
        s = self._status.cpu().tolist()
        if s[0]:
            raise RuntimeError(f"flyb200 adjoint kernel status {s[0]} (where {s[1]}, step {s[2]})")


def parameter_grads_over_ranks(grads) -> None:
    """Sum the shared parameters' gradients over the ranks of the default process group, in place
    (each rank's loss covers its own flies); nothing without a group of more than one rank."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        allreduce_gradients(grads)


class OpticRollout(torch.autograd.Function):
    """(gains, tau, v0 [m][B], adapt0 [m][B]) -> (v_T, adapt_T) with the hand-written adjoint."""

    @staticmethod
    def forward(ctx, gains, tau, v0, adapt0, engine: OpticAdjoint, steps: int):
        engine.set_params(gains.detach(), tau.detach())
        vT, aT = engine.forward(v0.detach(), adapt0.detach(), steps)
        ctx.engine = engine
        return vT, aT

    @staticmethod
    def backward(ctx, g_v, g_a):
        e = ctx.engine
        if g_v is None:
            g_v = torch.zeros(e.m, e.B, device=e.device)
        d_gains, d_tau, d_v0, d_a0 = e.backward(g_v.contiguous(), None if g_a is None else g_a.contiguous())
        return d_gains, d_tau, d_v0, d_a0, None, None
