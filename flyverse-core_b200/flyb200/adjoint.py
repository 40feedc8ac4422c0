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
torch.autograd.Function from (gains, tau, v0, adapt0) to (v_T, adapt_T).
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import scipy.sparse as sp
import torch

from . import _abi
from .optic import DeviceCSR, OpticCore


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
        self.launch = launch
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
        contrib = (self.gr * self.W0_t.double()) * self.g_edge.double()
        d_gains = torch.zeros(self.n_pairs, dtype=torch.float64, device=self.device).index_add_(0, self.pair_t, contrib)
        a = self.core.a.double()
        tau_i = self.tau.double()[self.type_of]
        d_tau = torch.zeros(self.n_types, dtype=torch.float64, device=self.device).index_add_(
            0, self.type_of, self.g_a.double() * a * self.dt / tau_i**2)
        return d_gains.float(), d_tau.float(), self.lam_v.clone(), self.lam_a.clone()

    def check(self) -> None:
        s = self._status.cpu().tolist()
        if s[0]:
            raise RuntimeError(f"flyb200 adjoint kernel status {s[0]} (where {s[1]}, step {s[2]})")


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
