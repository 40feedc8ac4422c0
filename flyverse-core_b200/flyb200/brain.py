"""Batched Shiu-style LIF brain on the B200 native step: the drop-in for flyverse/brain.py.

`Brain(c, params, device, seed, batch, ...)` keeps the reference constructor (brain.py:373-376),
`step(n)` / `run_ms` / `set_drive` / `set_poisson` / `freeze` / `reset(rows)` / `prune` /
`set_weights` and the public (B, N) state tensors (v, g, refrac, drive, poisson_p, rate, spikes,
spike_counts, adapt, res). Differences that follow from the design:

  * every step runs the fused native kernel (include/flyb200.h: flyb_lif_run); there is no Torch
    or CPU path, and a missing library or a non-CUDA device raises;
  * state is stored neuron-major, fly-minor ([N][B]); the public attributes are (B, N) views of that
    storage, so in-place edits (`brain.v[:, 3] = -40`) reach the kernel and assignment copies in;
  * the delay is an exact ring of pending synaptic input (`ring`, [R][N][B]) rather than a float
    spike buffer: int32 synapse counts when W is w_syn x integer counts (the model of the
    benchmark graphs), Q32.32 millivolts otherwise. `spike_buf` is rebuilt on demand from a
    1-bit spike history, and `load_spike_buf` converts a reference checkpoint's buffer;
  * Poisson draws come from Philox4x32-10 keyed by (seed, step, neuron, fly); `step(n, uniforms=)`
    takes external uniforms instead (parity runs feed the reference generator's draws).
"""
from __future__ import annotations

import ctypes as ct
import math
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp
import torch

from . import _abi
from .weights import (DEFAULT_ADAPT_BY_TYPE, DEFAULT_STD_U_BY_TYPE, SLOW_THRESHOLD_MAX_FRAC, integer_counts,
                      lif_weights, per_type, slow_spec, slow_weights)


@dataclass
class LIFParams:
    """The reference's LIF parameters (brain.py:29-158), same names and defaults."""
    v_rest: float = -52.0
    v_reset: float = -52.0
    v_th: float = -45.0
    tau_m: float = 20.0
    tau_syn: float = 5.0
    t_ref: float = 2.2
    delay: float = 1.8
    w_syn: float = 0.275
    dt: float = 0.5
    rate_tau: float = 100.0
    adapt_jump: float = 1.5
    adapt_tau: float = 200.0
    adapt_by_type: dict | None = None
    std_u: float = 0.0
    std_tau: float = 300.0
    std_u_by_type: dict = None
    input_norm_alpha: float = 1.0
    input_norm_ref: float = 5000.0
    same_type_gain: float = 0.1
    conn_cap: float = 60.0
    path_gain: list = None
    type_path_gain: list = None
    event_driven: bool | None = None
    weight_dtype: str = "float32"
    dt_by_module: dict | None = None
    prune_frozen: bool = True
    receptor_model: str | None = "sign"
    receptor_net_rule: str = "abs"
    receptor_nt_class_fallback: bool = False
    receptor_table: str | None = None
    receptor_gain: dict | None = None
    slow_tau_ms: float = 200.0
    slow_gain: float = 0.02
    slow_gain_by_class: dict | None = None
    slow_tau_by_class: dict | None = None
    slow_mode: str = "additive"
    slow_gain_clip: tuple = (0.0, 4.0)
    w_syn_by_nt: dict | None = None
    surrogate_grad: bool = False


_STATE = ("v", "g", "refrac", "drive", "poisson_p", "rate", "spikes", "spike_counts", "adapt", "res")


def upload(x, device, dtype=None) -> torch.Tensor:
    """A small host array on `device` without waiting for the device: staged through pinned memory
    and copied asynchronously on the current stream, so a caller between two launches (a reset
    between graph replays) does not wait for the work already queued. Plain copy off CUDA."""
    t = torch.as_tensor(x, dtype=dtype)
    device = torch.device(device)
    if device.type != "cuda":
        return t.to(device)
    return t.pin_memory().to(device, non_blocking=True)
LAUNCHES = {"step": _abi.LAUNCH_STEP, "persistent": _abi.LAUNCH_PERSISTENT}


def lif_coefficients(p: LIFParams, std_on: bool, adapt_on: bool | None = None) -> np.ndarray:
    """The float32 coefficient vector of the native step (the reference's `_cuda_P`, brain.py:493-520,
    plus tau_syn's decay and w_syn), with the exponentials taken in double as the reference does."""
    a_r = math.exp(-p.dt / p.rate_tau)
    P = np.zeros(_abi.LIF_NPARAM, np.float32)
    P[_abi.P_V_REST], P[_abi.P_V_RESET], P[_abi.P_V_TH] = p.v_rest, p.v_reset, p.v_th
    P[_abi.P_A_M], P[_abi.P_A_S] = math.exp(-p.dt / p.tau_m), math.exp(-p.dt / p.tau_syn)
    P[_abi.P_DT], P[_abi.P_T_REF] = p.dt, p.t_ref
    P[_abi.P_ADAPT_JUMP] = p.adapt_jump
    adapt_on = p.adapt_jump > 0 if adapt_on is None else adapt_on       # per-type jumps keep the decay on
    P[_abi.P_A_AD] = math.exp(-p.dt / p.adapt_tau) if adapt_on else 0.0
    P[_abi.P_A_STD] = math.exp(-p.dt / p.std_tau) if std_on else 1.0
    P[_abi.P_A_R], P[_abi.P_RATE_GAIN] = a_r, (1 - a_r) * 1000.0 / p.dt
    P[_abi.P_W_SYN] = p.w_syn
    return P


def clock_coefficients(p: LIFParams, std_on: bool, max_period: int, slow_tau=()) -> np.ndarray:
    """[max_period + 1][CLOCK_NCOEF] float32 phase coefficients of per-neuron clocks (brain.py:
    627-637): row k those of an update of a period-k neuron (a step of k * dt), row 0 those of a
    step without update (no decay, no refractory time, no spike, no Poisson). `slow_tau`: the time
    constants of the slow tone's classes, in class order (their decays fill CLOCK_A_SLOW0 on).
    Evaluated with the reference's float32 tensor expressions on the CPU, so they carry its bits."""
    kt = torch.arange(max_period + 1, dtype=torch.float32)
    kt[0] = 1.0
    u = torch.ones(max_period + 1)
    u[0] = 0.0
    one = torch.ones_like(u)

    def coef(tau):
        return torch.where(u > 0, torch.exp(-p.dt * kt / tau), one)

    out = torch.zeros(max_period + 1, _abi.CLOCK_NCOEF)
    out[:, _abi.CLOCK_A_M], out[:, _abi.CLOCK_A_S], out[:, _abi.CLOCK_A_R] = coef(p.tau_m), coef(p.tau_syn), coef(p.rate_tau)
    out[:, _abi.CLOCK_A_AD] = coef(p.adapt_tau) if p.adapt_jump > 0 else torch.zeros_like(u)
    out[:, _abi.CLOCK_A_STD] = coef(p.std_tau) if std_on else one
    out[:, _abi.CLOCK_DT] = u * kt * p.dt
    out[:, _abi.CLOCK_RATE_GAIN] = u * (1 - torch.exp(-p.dt * kt / p.rate_tau)) * 1000.0 / (kt * p.dt)
    out[:, _abi.CLOCK_U] = u
    out[:, _abi.CLOCK_POIS] = u * kt
    if len(slow_tau) > _abi.SLOW_MAX_CLASSES:
        raise ValueError("more slow classes than the native step holds")
    out[:, _abi.CLOCK_A_SLOW0:_abi.CLOCK_A_SLOW0 + _abi.SLOW_MAX_CLASSES] = 1.0
    for c, tau in enumerate(slow_tau):
        out[:, _abi.CLOCK_A_SLOW0 + c] = coef(tau)
    return out.numpy()


PULL_PAD = 0xFFFFFF           # packed pull entry without an input


def pull_inputs(W, w_syn: float):
    """The inputs of every neuron for FLYB_LIF_PULL_DELIVERY, from W[post, pre] = w_syn x signed
    integer counts: (pull_ptr int32 [N+1] in 32-entry chunks, pull_pre int32 [chunks * 32],
    pull_planes uint32 [chunks * S], pull_meta int32 [chunks], S). A row's inputs are sorted by
    count, so a chunk's counts lie close together: it stores its smallest count as the base and
    each entry's excess over it (meta = base << 5 | planes, the bits that range needs).

    When every excess fits 8 bits (and N < 2^24 - 1) the tables are packed, S = 0: an entry is
    pre | excess << 24, 0xFFFFFF padding the last chunk of a row, and pull_planes is empty (the
    kernel rebuilds the planes with warp ballots). Otherwise S = 16: entries are pre with -1
    padding, and pull_planes holds each chunk's excesses as 16 bit planes (bit l of plane p = bit p
    of entry l's excess). None when the weights are not such counts or a chunk's range needs more
    than 16 bits."""
    Wr = sp.csr_matrix(W, dtype=np.float32)
    Wr.sum_duplicates()
    Wr.sort_indices()
    counts = integer_counts(Wr, w_syn)
    if counts is None:
        return None
    counts = counts.astype(np.int64)
    n = Wr.shape[0]
    deg = np.diff(Wr.indptr).astype(np.int64)
    row = np.repeat(np.arange(n), deg)
    order = np.lexsort((counts, row))                 # by row, then by count
    pre_sorted, cnt_sorted = Wr.indices[order], counts[order]
    ptr = np.concatenate([[0], np.cumsum((deg + 31) // 32)])
    chunks = int(ptr[-1])
    pos = ptr[row] * 32 + (np.arange(Wr.nnz) - np.repeat(Wr.indptr[:-1].astype(np.int64), deg))
    chunk_of = pos // 32
    pre = np.full(chunks * 32, -1, np.int32)
    pre[pos] = pre_sorted
    base = np.zeros(chunks, np.int64)
    if Wr.nnz:
        base_min = np.full(chunks, np.iinfo(np.int64).max)
        np.minimum.at(base_min, chunk_of, cnt_sorted)
        base = np.where(base_min == np.iinfo(np.int64).max, 0, base_min)
    excess = np.zeros(chunks * 32, np.int64)
    excess[pos] = cnt_sorted - base[chunk_of]
    top = excess.reshape(chunks, 32).max(axis=1) if chunks else np.zeros(0, np.int64)
    planes_needed = np.array([int(t).bit_length() for t in top], np.int64)
    if planes_needed.size and planes_needed.max() > 16:
        return None
    if base.size and (base.min() < -(1 << 26) or base.max() >= (1 << 26)):
        return None
    meta = ((base << 5) | planes_needed).astype(np.int32)
    if (not planes_needed.size or planes_needed.max() <= 8) and max(Wr.shape) < PULL_PAD:
        packed = np.where(pre >= 0, pre.astype(np.int64) | (excess << 24), PULL_PAD).astype(np.uint32)
        return ptr.astype(np.int32), packed.view(np.int32), np.zeros(0, np.uint32), meta, 0
    S = 16
    u = excess.astype(np.uint64).reshape(chunks, 32)
    lanes = np.arange(32, dtype=np.uint64)
    planes = np.zeros((chunks, S), np.uint64)
    for q in range(S):
        planes[:, q] = (((u >> np.uint64(q)) & np.uint64(1)) << lanes).sum(axis=1)
    return ptr.astype(np.int32), pre, planes.astype(np.uint32).ravel(), meta, S


def out_edges(W, w_syn: float, prefer: str = "auto", std_on: bool = False):
    """Pre-major (CSC) outgoing synapses of W[post, pre] for the native step.

    Returns (out_ptr int32 [N+1], out_edge int32 [nnz][2], ring mode): {post, signed count} on the
    int32 count ring when every weight is w_syn x an integer count and depression is off (unless
    prefer='fixed'), else {post, float32 bits of w} on the Q32.32 ring."""
    Wc = sp.csc_matrix(W, dtype=np.float32)
    Wc.sum_duplicates()
    Wc.sort_indices()
    if max(*Wc.shape, Wc.nnz) >= 2**31:
        raise ValueError("the native step needs 32-bit dimensions and indices")
    counts = None if (std_on or prefer == "fixed") else integer_counts(Wc, w_syn)
    if prefer == "count" and counts is None:
        raise ValueError("ring='count' needs weights that are w_syn x integer synapse counts and no depression")
    mode = _abi.RING_COUNT if counts is not None else _abi.RING_FIXED
    second = counts if counts is not None else Wc.data.astype(np.float32).view(np.int32)
    edges = np.ascontiguousarray(np.stack([Wc.indices.astype(np.int32), second.astype(np.int32)], axis=1))
    return Wc.indptr.astype(np.int32), edges, mode


def _unsupported(p: LIFParams, metal_kernels, cuda_kernels, cuda_sparse) -> None:
    if metal_kernels:
        raise ValueError("flyb200 runs on B200 CUDA kernels only; the Metal backend is not provided")
    if cuda_kernels is False:
        raise ValueError("flyb200 has no Torch path: cuda_kernels=False is not available")
    if cuda_sparse not in ("torch", "warp"):
        raise ValueError("cuda_sparse must be torch or warp")
    if p.surrogate_grad:
        raise NotImplementedError("surrogate_grad (Torch autograd through the LIF) is not part of the native step; "
                                  "the spiking path is left undifferentiated")
    if p.weight_dtype not in ("float32", "float16"):
        raise ValueError("weight_dtype must be float32 or float16")
    if p.event_driven is False:
        pass   # the native step is event driven for every activity level; the flag is accepted for compatibility


class Brain:
    def __init__(self, c, params: LIFParams | None = None, device=None, seed: int = 0, batch: int = 1,
                 metal_kernels=None, cuda_kernels=None, cuda_sparse: str = "torch", cuda_compact: bool = True,
                 receptor=None, *, launch: str = "persistent", ring: str = "auto", block: int = 256,
                 ring_slots: int | None = None):
        p = params or LIFParams()
        _unsupported(p, metal_kernels, cuda_kernels, cuda_sparse)
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        if self.device.type != "cuda":
            raise ValueError("flyb200.Brain runs on a CUDA device only; there is no CPU path")
        if int(batch) < 1 or not math.isfinite(p.dt) or p.dt <= 0:
            raise ValueError("batch must be positive and dt must be positive and finite")
        if launch not in LAUNCHES:
            raise ValueError(f"launch must be one of {sorted(LAUNCHES)}")
        if ring not in ("auto", "count", "fixed"):
            raise ValueError("ring must be 'auto', 'count' or 'fixed'")
        self._lib = _abi.lib()
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.c, self.p, self.n, self.B = c, p, c.n, int(batch)
        self.seed, self.launch, self.block, self.ring_pref = int(seed), launch, int(block), ring
        self.cuda, self.metal, self.event_driven = True, False, True
        self.cuda_sparse, self.cuda_compact = cuda_sparse, bool(cuda_compact)
        self.receptor = receptor
        W, self.input_scale = lif_weights(c, p, receptor)
        if p.weight_dtype == "float16":
            W.data = W.data.astype(np.float16).astype(np.float32)
        N, B, dev = self.n, self.B, self.device
        self.n_delay = max(1, int(round(p.delay / p.dt)))
        self.R = int(ring_slots) if ring_slots else self.n_delay + 1
        if self.R < self.n_delay + 1:
            raise ValueError("ring_slots must exceed the delay in steps")
        std_map = DEFAULT_STD_U_BY_TYPE if p.std_u_by_type is None else p.std_u_by_type
        u = per_type(c, std_map, p.std_u)
        self._std_on = bool((u > 0).any())
        self.std_u_vec = torch.from_numpy(u).to(dev)
        self._a_m = math.exp(-p.dt / p.tau_m)
        self._a_s = math.exp(-p.dt / p.tau_syn)
        self._a_r = math.exp(-p.dt / p.rate_tau)
        # per-type adaptation (brain.py:497-506): a per-neuron jump, and the decay always on
        adapt_map = DEFAULT_ADAPT_BY_TYPE if p.adapt_by_type is None else p.adapt_by_type
        self.adapt_jump_vec = torch.from_numpy(per_type(c, adapt_map, p.adapt_jump)).to(dev) if adapt_map else None
        self._adapt_on = p.adapt_jump > 0 or self.adapt_jump_vec is not None
        self._a_ad = math.exp(-p.dt / p.adapt_tau) if self._adapt_on else 0.0
        self._a_std = math.exp(-p.dt / p.std_tau) if self._std_on else 1.0
        self._P = lif_coefficients(p, self._std_on, self._adapt_on)
        # state: [N][B] storage, (B, N) public views
        self._st = {k: torch.zeros(N, B, device=dev) for k in _STATE}
        self._st["v"].fill_(p.v_rest)
        self._st["res"].fill_(1.0)
        self.active = torch.ones(N, device=dev)
        # slow receptor tone (receptor_model "full"): per class [K][N][B] and the sum [N][B], (B, N) views
        self.slow = slow_spec(p)
        self.slow_classes = self.slow.classes if self.slow is not None else []
        K = len(self.slow_classes)
        self._slow_g = torch.zeros(K, N, B, device=dev)
        self._g_slow = torch.zeros(N, B, device=dev)
        self.g_slow = self._g_slow.t()
        self.g_slow_cls = self._slow_g.transpose(1, 2)
        self._W_slow_cpu = slow_weights(c, p, receptor, self.slow, self.input_scale) if self.slow is not None else None
        self._slow_rings = []
        self.gen = torch.Generator(device=dev).manual_seed(seed)
        self.words = (N * B + 31) // 32
        self._hist = torch.zeros(self.n_delay, self.words, dtype=torch.int32, device=dev)   # 1-bit spike history
        self._clock = torch.zeros(3, dtype=torch.int64, device=dev)        # {step, ring_pos, hist_pos}
        # pull delivery: {first undelivered step, its ring position, block counter}; equal to the
        # clock's first two words whenever nothing is pending (between calls)
        self._pull_state = torch.zeros(3, dtype=torch.int64, device=dev)
        self._pull_pending = 0                  # steps updated but not yet pulled (host count)
        self._pull_bits = None
        self._status = torch.zeros(4, dtype=torch.int32, device=dev)
        self._sync = torch.zeros(_abi.LIF_SYNC_WORDS, dtype=torch.int32, device=dev)
        self._events = torch.zeros(1, dtype=torch.int64, device=dev)
        self.ring = None
        self.record_activity = False
        self._poisson_on = False
        self.t, self.step_count, self.buf_pos = 0.0, 0, 0
        self._rate_np, self._rate_np_key = None, None
        self._weights_version = 0
        self._kvec = None                       # per-neuron clocks (set_clocks)
        self._W_cpu = W
        self.set_weights(W)

    # ------------------------------------------------------------------ public state views
    def __getattr__(self, name):
        st = self.__dict__.get("_st")
        if st is not None and name in st:
            return st[name].t()
        raise AttributeError(name)

    def __setattr__(self, name, value):
        st = self.__dict__.get("_st")
        if st is not None and name in st:
            st[name].t().copy_(torch.as_tensor(value, dtype=torch.float32, device=self.device))
            return
        object.__setattr__(self, name, value)

    # ------------------------------------------------------------------ weights
    def set_weights(self, W) -> None:
        """Install W[post, pre] in mV per transmitted spike (brain.py:525-545); pending deliveries
        are rebuilt with the new weights from the spike history, as the reference's buffer would."""
        indptr, edges, mode = out_edges(W, self.p.w_syn, self.ring_pref, self._std_on)
        had_ring = self.ring is not None
        spike_buf = None
        if had_ring and self.step_count and not self._std_on:
            spike_buf = self.spike_buf
        self._W_cpu = sp.csr_matrix(W, dtype=np.float32)
        self._set_slow_lists()
        self._weights_version += 1
        self.ring_mode = mode
        self.nnz = int(edges.shape[0])
        self._out_ptr = torch.from_numpy(indptr).to(self.device)
        self._out_edge = torch.from_numpy(edges).to(self.device)
        dtype = torch.int32 if mode == _abi.RING_COUNT else torch.int64
        if getattr(self, "_kvec", None) is not None and had_ring and self.ring.dtype != dtype:
            self.clock_acc.zero_()          # held input is in the units of the previous ring
        self.ring = torch.zeros(self.R, self.n, self.B, dtype=dtype, device=self.device)
        self._make_args()
        if had_ring and spike_buf is not None:
            self.load_spike_buf(spike_buf)

    def _set_slow_lists(self) -> None:
        """Pre-major synapse lists of the slow classes, and their rings (kept across rebuilds)."""
        self._slow_lists = []
        if self._W_slow_cpu is None:
            return
        for S in self._W_slow_cpu.values():
            ptr, edges, _ = out_edges(S, self.p.w_syn, "fixed")
            if not len(edges):                  # a class without synapses still needs an address
                edges = np.zeros((1, 2), np.int32)
            self._slow_lists.append((torch.from_numpy(ptr).to(self.device), torch.from_numpy(edges).to(self.device)))
        if not self._slow_rings:
            self._slow_rings = [torch.zeros(self.R, self.n, self.B, dtype=torch.int64, device=self.device)
                                for _ in self._W_slow_cpu]

    def prune(self, idx) -> None:
        """Drop every synapse from and onto neurons `idx` (brain.py:602-616)."""
        keep = np.ones(self.n, np.float32)
        keep[np.asarray(idx)] = 0.0
        if self._W_slow_cpu is not None:
            S = {}
            for k, Sk in self._W_slow_cpu.items():
                Sk = (sp.diags(keep) @ Sk @ sp.diags(keep)).tocsr()
                Sk.eliminate_zeros()
                S[k] = Sk
            self._W_slow_cpu = S
        W = (sp.diags(keep) @ self._W_cpu @ sp.diags(keep)).tocsr()
        W.eliminate_zeros()
        self.set_weights(W)

    # ------------------------------------------------------------------ native call
    def _make_args(self) -> None:
        st, a = self._st, _abi.LifArgs()
        a.n, a.batch, a.n_delay, a.ring_slots, a.ring_mode = self.n, self.B, self.n_delay, self.R, self.ring_mode
        a.launch, a.block = LAUNCHES[self.launch], self.block
        a.grid = int(getattr(self, "grid", 0))        # persistent / staged launches: block cap
        a.items_per_thread = getattr(self, "items_per_thread", 0)
        a.staged = int(bool(getattr(self, "staged", False)))
        a.fly0 = int(getattr(self, "fly0", 0))       # global index of local fly 0 (Philox key when sharded)
        a.raster_slots = self.n_delay
        a.seed = self.seed & 0xFFFFFFFFFFFFFFFF
        a.out_ptr, a.out_edge = self._out_ptr.data_ptr(), self._out_edge.data_ptr()
        for name, field_ in (("v", "v"), ("g", "g"), ("refrac", "refrac"), ("adapt", "adapt"), ("res", "res"),
                             ("rate", "rate"), ("spike_counts", "counts"), ("spikes", "spikes"), ("drive", "drive"),
                             ("poisson_p", "poisson_p")):
            setattr(a, field_, st[name].data_ptr())
        a.active, a.std_u = self.active.data_ptr(), self.std_u_vec.data_ptr()
        a.params = self._P.ctypes.data
        a.ring, a.clock, a.raster = self.ring.data_ptr(), self._clock.data_ptr(), self._hist.data_ptr()
        a.events, a.status, a.sync = self._events.data_ptr(), self._status.data_ptr(), self._sync.data_ptr()
        a.adapt_jump = None if self.adapt_jump_vec is None else self.adapt_jump_vec.data_ptr()
        if self._kvec is not None:
            a.clock_k, a.clock_coef = self._clock_k.data_ptr(), self._clock_coef.data_ptr()
            a.clock_acc = self.clock_acc.data_ptr()
            if self.slow is not None:
                for c in range(len(self.slow_classes)):
                    a.slow_clock_acc[c] = self.slow_clock_acc[c].data_ptr()
        if self.slow is not None:
            spec = self.slow
            a.slow_classes, a.slow_mode = len(self.slow_classes), _abi.SLOW_MODE_CODES[spec.mode]
            a.slow_norm, a.slow_clip_lo, a.slow_clip_hi = spec.norm_mv, spec.clip[0], spec.clip[1]
            a.slow_th_max = float(np.float32(SLOW_THRESHOLD_MAX_FRAC * spec.norm_mv))
            for c, name in enumerate(self.slow_classes):
                a.slow_decay[c] = math.exp(-self.p.dt / spec.tau[name])
                a.slow_out_ptr[c] = self._slow_lists[c][0].data_ptr()
                a.slow_out_edge[c] = self._slow_lists[c][1].data_ptr()
                a.slow_ring[c], a.slow_g[c] = self._slow_rings[c].data_ptr(), self._slow_g[c].data_ptr()
            a.g_slow = self._g_slow.data_ptr()
        self._args = a
        self._lists = {}          # deferred-delivery lists per neuron range, sized on first use

    def _defer_active(self) -> bool:
        """Deferred delivery (FLYB_LIF_DEFER_DELIVERY) applies to per-step launches (register or staged
        path) without clocks or the slow tone."""
        return bool(getattr(self, "defer", False)) and self.launch == "step" and self._kvec is None \
            and self.slow is None and not self._pull_active()

    def can_pull(self) -> bool:
        """Whether pull delivery (FLYB_LIF_PULL_DELIVERY) fits this brain: the int32 count ring (no
        depression), 32, 64, 128 or 256 flies, no clocks or slow tone."""
        return self.ring_mode == _abi.RING_COUNT and self.B in (32, 64, 128, 256) and self._kvec is None \
            and self.slow is None and not self._std_on

    def _pull_active(self) -> bool:
        """Pull delivery runs: requested (`pull`), per-step launches, and `can_pull`."""
        return bool(getattr(self, "pull", False)) and self.launch == "step" and self.can_pull()

    def _set_pull(self, a) -> None:
        """Point the arguments at the pull tables (built from the shaped weights on first use)."""
        if not self._pull_active():
            a.pull_ptr = a.pull_pre = a.pull_planes = a.pull_meta = None
            a.pull_nplanes = 0
            return
        key = self._weights_version
        if getattr(self, "_pull_key", None) != key:
            t = pull_inputs(self._W_cpu, self.p.w_syn)
            if t is None:
                raise ValueError("pull delivery needs weights of w_syn x counts within 16 bits")
            ptr, pre, planes, meta, S = t
            self._pull_t = tuple(torch.from_numpy(x).to(self.device) if x.size else None
                                 for x in (ptr, pre, planes.view(np.int32), meta))
            self._pull_planes_n, self._pull_key = S, key
        a.pull_ptr, a.pull_pre, a.pull_planes, a.pull_meta = (None if x is None else x.data_ptr()
                                                              for x in self._pull_t)
        a.pull_nplanes = self._pull_planes_n
        L = self.pull_group
        if self._pull_bits is None or self._pull_bits.numel() != 2 * L * self.words:
            self._pull_bits = torch.zeros(2 * L * self.words, dtype=torch.int32, device=self.device)
        a.pull_group, a.pull_bits, a.pull_state = L, self._pull_bits.data_ptr(), self._pull_state.data_ptr()
        a.pull_grid = int(getattr(self, "pull_grid", 0))      # pull launch block cap (0: one wave)
        a.pull_phase = self.step_count % L

    @property
    def pull_group(self) -> int:
        """Steps a pull delivers together (flyb_lif_args.pull_group): 8 / (B / 32), so that one
        gather per input fetches a 32-byte sector of spike words, when the delay allows a group's
        pull to run beside the next group (2 L <= n_delay); else 1."""
        L = 8 // max(1, self.B // 32)
        return L if 2 * L <= self.n_delay else 1

    # ------------------------------------------------------------------ per-neuron clocks
    def set_clocks(self, multiplier) -> None:
        """Integrate neuron i every multiplier[i] base steps (dt_i = multiplier[i] * dt), the
        reference's Brain.set_clocks (brain.py:618-640): on other steps a neuron holds its state and
        the input that reaches it waits for its next update. The native step then runs one launch
        per step through the clocked kernel. Input already held for a slow neuron stays in the
        units of the ring it arrived on (it is dropped if set_weights changes the ring mode). With
        the slow receptor tone each class decays by its phase coefficient and its input waits
        for the update too (brain.py:905-917)."""
        k = np.asarray(multiplier, dtype=np.int64)
        if k.shape != (self.n,) or (k < 1).any():
            raise ValueError("multiplier must be an (N,) array of positive integers")
        p = self.p
        if int(k.max()) * p.dt > p.delay + 1e-9:
            raise ValueError("the slowest clock must not exceed the synaptic delay")
        if int(k.max()) > 255:
            raise ValueError("clock periods above 255 steps are not supported")
        self._kvec = k
        self.K = int(np.lcm.reduce(np.unique(k)))
        self._clock_k = torch.from_numpy(k.astype(np.uint8)).to(self.device)
        slow_tau = [self.slow.tau[name] for name in self.slow_classes] if self.slow is not None else []
        self._clock_coef = torch.from_numpy(clock_coefficients(p, self._std_on, int(k.max()), slow_tau)).to(self.device)
        self.clock_acc = torch.zeros(self.n, self.B, dtype=torch.int64, device=self.device)
        self.slow_clock_acc = torch.zeros(len(slow_tau), self.n, self.B, dtype=torch.int64, device=self.device)
        self._weights_version += 1
        self._make_args()

    def _set_delivery(self, a, n_first: int, n_count: int) -> None:
        """Point the arguments at the spike list of this neuron range (one list per range, so
        ranges running on different streams never share one), or at none."""
        if not self._defer_active():
            a.spike_list, a.spike_n, a.spike_cap = None, None, 0
            return
        key = (int(n_first), int(n_count))
        lst = self._lists.get(key)
        if lst is None:
            a.n_first, a.n_count = key
            cap = int(self._lib.flyb_lif_spike_capacity(ct.byref(a)))
            if cap <= 0:
                raise RuntimeError("flyb_lif_spike_capacity failed")
            lst = (torch.empty(cap, 4, dtype=torch.int32, device=self.device),
                   torch.zeros(1, dtype=torch.int32, device=self.device), cap)
            self._lists[key] = lst
        a.spike_list, a.spike_n, a.spike_cap = lst[0].data_ptr(), lst[1].data_ptr(), lst[2]

    def _flags(self, external: bool) -> int:
        f = 0
        if self._defer_active():
            f |= _abi.LIF_DEFER_DELIVERY
        if self._pull_active():
            f |= _abi.LIF_PULL_DELIVERY
        if self._poisson_on:
            f |= _abi.LIF_POISSON
        if self._std_on:
            f |= _abi.LIF_STD
        if self.record_activity:
            f |= _abi.LIF_COUNTS
        if self._adapt_on:
            f |= _abi.LIF_ADAPT
        if self.cuda_compact:
            f |= _abi.LIF_SKIP_FROZEN
        if external:
            f |= _abi.LIF_EXT_UNIFORM
        return f

    def step(self, n_steps: int = 1, *, uniforms: torch.Tensor | None = None) -> None:
        """Advance n_steps of dt. `uniforms` (n_steps, B, N): external Poisson draws."""
        n_steps = int(n_steps)
        if n_steps <= 0:
            return
        a = self._args
        ext = None
        if uniforms is not None:
            if tuple(uniforms.shape) != (n_steps, self.B, self.n):
                raise ValueError(f"uniforms must have shape ({n_steps}, {self.B}, {self.n})")
            ext = uniforms.to(self.device, torch.float32).transpose(1, 2).contiguous()
        a.flags = self._flags(ext is not None)
        a.nsteps = n_steps
        a.uniforms = ext.data_ptr() if ext is not None else None
        self._set_delivery(a, 0, 0)
        self._set_pull(a)
        a.n_first, a.n_count = 0, 0
        stream = torch.cuda.current_stream(self.device).cuda_stream
        with torch.cuda.device(self.device):
            rc = self._lib.flyb_lif_run(ct.byref(a), stream)
        if rc:
            raise RuntimeError(f"flyb_lif_run: error {rc}")
        self.buf_pos = (self.buf_pos + n_steps) % self.R
        self.t += n_steps * self.p.dt
        self.step_count += n_steps

    def step_range(self, n_first: int, n_count: int) -> None:
        """Update neurons [n_first, n_first + n_count) by one step on the current stream, leaving
        the device clock where it is (FLYB_LIF_NO_ADVANCE): the ranges of one step may run on
        different streams, after which `advance(1)` ends the step. n_first * B must be a multiple
        of 32. Spikes of the range are delivered to every postsynaptic neuron as in `step`."""
        a = self._args
        a.flags = self._flags(False) | _abi.LIF_NO_ADVANCE
        a.nsteps, a.uniforms = 1, None
        self._set_delivery(a, n_first, n_count)
        self._set_pull(a)
        a.n_first, a.n_count = int(n_first), int(n_count)
        try:
            with torch.cuda.device(self.device):
                rc = self._lib.flyb_lif_run(ct.byref(a), torch.cuda.current_stream(self.device).cuda_stream)
        finally:
            a.n_first, a.n_count = 0, 0
        if rc:
            raise RuntimeError(f"flyb_lif_run: error {rc}")

    def deliver(self, steps: int | None = None) -> None:
        """Pull delivery of the first `steps` (default: all) steps updated but not yet delivered
        (after `advance(n, pull=False)`), on the current stream, in launches that end at group
        boundaries. A delivery may run on another stream beside the updates of the next group of
        steps; the caller orders it before the next delivery and before the updates of the group
        after that (their spike words reuse its half of the pull buffer)."""
        left = self._pull_pending if steps is None else int(steps)
        if left <= 0:
            return
        if left > self._pull_pending:
            raise ValueError(f"only {self._pull_pending} steps are pending")
        a = self._args
        a.flags, a.nsteps = self._flags(False) & ~_abi.LIF_DEFER_DELIVERY, 1
        self._set_pull(a)
        L = self.pull_group
        first = self.step_count - self._pull_pending            # the first undelivered step
        stream = torch.cuda.current_stream(self.device).cuda_stream
        while left:
            a.pull_steps = min(left, L - first % L)
            with torch.cuda.device(self.device):
                rc = self._lib.flyb_lif_pull(ct.byref(a), stream)
            if rc:
                raise RuntimeError(f"flyb_lif_pull: error {rc}")
            first += a.pull_steps
            left -= a.pull_steps
            self._pull_pending -= a.pull_steps

    def advance(self, n_steps: int = 1, *, pull: bool = True) -> None:
        """End `n_steps` steps run by ranges: move the device clock (ring and history positions,
        Philox step) on, as the end of `step` does. Under pull delivery the steps become pending;
        with `pull` they are delivered at once, else `deliver` delivers them later (at most a
        group's worth may be pending)."""
        a = self._args
        a.flags = self._flags(False) & ~_abi.LIF_DEFER_DELIVERY
        a.nsteps = int(n_steps)
        stream = torch.cuda.current_stream(self.device).cuda_stream
        with torch.cuda.device(self.device):
            rc = self._lib.flyb_lif_advance(ct.byref(a), stream)
        if rc:
            raise RuntimeError(f"flyb_lif_advance: error {rc}")
        self.buf_pos = (self.buf_pos + n_steps) % self.R
        self.t += n_steps * self.p.dt
        self.step_count += n_steps
        if self._pull_active():
            self._pull_pending += int(n_steps)
            if self._pull_pending > self.pull_group and not pull:
                raise ValueError("more than one group of steps is waiting for its pull")
            if pull:
                self.deliver()

    def restart_clock(self) -> None:
        """Step counter, ring and history positions back to 0 (a full reset), nothing pending."""
        self._clock.zero_()
        self._pull_state.zero_()
        self._pull_pending = 0
        self.t, self.step_count, self.buf_pos = 0.0, 0, 0

    def run_ms(self, ms: float) -> None:
        self.step(int(round(ms / self.p.dt)))

    def check(self) -> None:
        """Raise if a kernel recorded an error (bounded barrier wait ran out); host sync."""
        s = self._status.cpu().tolist()
        if s[0]:
            raise RuntimeError(f"flyb200 LIF kernel status {s[0]} (where {s[1]}, step {s[2]})")

    # ------------------------------------------------------------------ inputs
    def _idx(self, idx) -> torch.Tensor:
        return torch.as_tensor(idx, device=self.device, dtype=torch.long)

    def set_drive(self, idx, mv) -> None:
        """Injected current (mV) of neurons `idx`: scalar, (len(idx),) or (B, len(idx))."""
        self.drive[:, self._idx(idx)] = torch.as_tensor(mv, dtype=torch.float32, device=self.device)

    def set_poisson(self, idx, rate_hz) -> None:
        """Poisson forcing at rate_hz on neurons `idx` (brain.py:707-713)."""
        r = torch.as_tensor(rate_hz, dtype=torch.float32, device=self.device)
        self.poisson_p[:, self._idx(idx)] = r * (self.p.dt / 1000.0)
        self._poisson_on = bool((r > 0).any()) or bool(self._st["poisson_p"].count_nonzero() > 0)

    def freeze(self, idx) -> None:
        self.active[self._idx(idx)] = 0.0

    def reset(self, rows=None) -> None:
        """Reset brains `rows` (all if None) to rest, their pending input included."""
        sel = slice(None) if rows is None else upload(np.asarray(rows, dtype=np.int64), self.device)
        st = self._st
        st["v"][:, sel] = self.p.v_rest
        for k in ("g", "refrac", "drive", "poisson_p", "rate", "spikes", "adapt", "spike_counts"):
            st[k][:, sel] = 0.0
        st["res"][:, sel] = 1.0
        self.g_slow[sel] = 0.0
        self.g_slow_cls[:, sel] = 0.0
        for r in self._slow_rings:
            r[:, :, sel] = 0
        self.ring[:, :, sel] = 0
        if self._kvec is not None:
            self.clock_acc[:, sel] = 0
            self.slow_clock_acc[:, :, sel] = 0
        if rows is None:
            self._hist.zero_()
        else:
            self._clear_hist_rows(np.asarray(rows))
        self._rate_np_key = None

    def _clear_hist_rows(self, rows: np.ndarray) -> None:
        """Clear the spike-history bits of flies `rows`. Item (neuron i, fly b) is bit i * B + b; with
        B a multiple of 32 a word holds one neuron's flies 32 g .. 32 g + 31, so the bits to keep
        depend only on the word's fly group g: one word per group, applied on the device."""
        rows = np.asarray(rows, dtype=np.int64)
        if self.B % 32 == 0:
            keep = np.full(self.B // 32, 0xFFFFFFFF, np.uint32)
            np.bitwise_and.at(keep, rows // 32, ~(np.uint32(1) << (rows % 32).astype(np.uint32)))
            k = upload(keep.view(np.int32), self.device)
            self._hist.view(self.n_delay, self.n, self.B // 32).bitwise_and_(k)
            return
        flat = (np.arange(self.n)[:, None] * self.B + rows[None, :]).ravel()
        mask = np.zeros(self.words * 32, bool)
        mask[flat] = True
        keep = ~np.packbits(mask, bitorder="little").view(np.uint32)
        self._hist &= torch.from_numpy(keep.view(np.int32)).to(self.device)

    # ------------------------------------------------------------------ spike buffer interchange
    @property
    def spike_buf(self) -> torch.Tensor:
        """(D, B, N) transmitted spikes in the reference's buffer order (brain.py:486, 858-865):
        slot (buf + k) % D holds the spikes delivered k steps from now. Depression makes the
        transmitted amount fractional, which the 1-bit history does not keep."""
        if self._std_on:
            raise NotImplementedError("spike_buf export needs the transmitted amounts; depression is on")
        D, N, B = self.n_delay, self.n, self.B
        words = self._hist.cpu().numpy().view(np.uint32)
        bits = np.unpackbits(words.view(np.uint8), bitorder="little").reshape(D, -1)[:, : N * B]
        hist = bits.reshape(D, N, B).transpose(0, 2, 1).astype(np.float32)     # hist slot -> (B, N)
        pos = int(self._clock[2].item()) % D           # next history slot = oldest entry = due now
        out = np.empty((D, B, N), np.float32)
        for k in range(D):
            out[(self.step_count + k) % D] = hist[(pos + k) % D]
        return torch.from_numpy(out).to(self.device)

    def load_spike_buf(self, spike_buf, buf_pos: int | None = None) -> None:
        """Rebuild the pending-input ring from a (D, B, N) spike buffer (a reference checkpoint's
        `spike_buf` with its `buf_pos`): slot (buf_pos + k) % D is delivered k steps from now."""
        sb = torch.as_tensor(spike_buf, dtype=torch.float32, device=self.device)
        D = self.n_delay
        if tuple(sb.shape) != (D, self.B, self.n):
            raise ValueError(f"spike_buf must have shape ({D}, {self.B}, {self.n})")
        buf_pos = self.step_count % D if buf_pos is None else int(buf_pos)
        if self.ring_mode == _abi.RING_COUNT and not bool(((sb == 0) | (sb == 1)).all()):
            raise ValueError("a count ring needs 0/1 spikes; rebuild the brain with ring='fixed'")
        self.ring.zero_()
        rpos = int(self._clock[1].item()) % self.R
        stream = torch.cuda.current_stream(self.device).cuda_stream
        hist = np.zeros((D, self.words), np.uint32)
        hpos = int(self._clock[2].item()) % D
        for k in range(D):
            x = sb[(buf_pos + k) % D].t().contiguous()
            slot = self.ring[(rpos + k) % self.R]
            rc = self._lib.flyb_ring_deposit(self.n, self.B, self.ring_mode, self._out_ptr.data_ptr(),
                                             self._out_edge.data_ptr(), x.data_ptr(), slot.data_ptr(), stream)
            if rc:
                raise RuntimeError(f"flyb_ring_deposit: error {rc}")
            bits = np.packbits((x.cpu().numpy().ravel() != 0), bitorder="little")
            bits = np.concatenate([bits, np.zeros(self.words * 4 - bits.size, np.uint8)])
            hist[(hpos + k) % D] = bits.view(np.uint32)
        self._hist.copy_(torch.from_numpy(hist.view(np.int32)))

    # ------------------------------------------------------------------ checkpoint
    def state_dict(self) -> dict:
        out = {k: getattr(self, k).detach().cpu().clone() for k in _STATE}
        out.update(ring=self.ring.cpu().clone(), hist=self._hist.cpu().clone(), clock=self._clock.cpu().clone(),
                   scalars=dict(t=self.t, step_count=self.step_count, buf_pos=self.buf_pos, _poisson_on=self._poisson_on))
        if self._kvec is not None:
            out.update(clock_period=self._kvec.copy(), clock_acc=self.clock_acc.cpu().clone(),
                       slow_clock_acc=self.slow_clock_acc.cpu().clone())
        if self.slow is not None:
            out.update(g_slow=self._g_slow.cpu().clone(), g_slow_cls=self._slow_g.cpu().clone(),
                       slow_rings=[r.cpu().clone() for r in self._slow_rings])
        return out

    def load_state_dict(self, state: dict) -> None:
        for k in _STATE:
            getattr(self, k).copy_(state[k].to(self.device))
        if state["ring"].dtype != self.ring.dtype or state["ring"].shape != self.ring.shape:
            raise ValueError("checkpoint ring does not match this brain's ring")
        self.ring.copy_(state["ring"].to(self.device))
        self._hist.copy_(state["hist"].to(self.device))
        self._clock.copy_(state["clock"].to(self.device))
        self._pull_state[:2].copy_(self._clock[:2])         # a checkpoint has nothing pending
        self._pull_state[2] = 0
        self._pull_pending = 0
        if "clock_period" in state:
            if self._kvec is None or not np.array_equal(state["clock_period"], self._kvec):
                self.set_clocks(state["clock_period"])
            self.clock_acc.copy_(state["clock_acc"].to(self.device))
            if "slow_clock_acc" in state:
                self.slow_clock_acc.copy_(state["slow_clock_acc"].to(self.device))
        elif self._kvec is not None:
            raise ValueError("checkpoint has no per-neuron clocks but this brain runs them")
        if (self.slow is not None) != ("g_slow_cls" in state):
            raise ValueError("checkpoint and brain disagree on the slow receptor tone")
        if self.slow is not None:
            self._g_slow.copy_(state["g_slow"].to(self.device))
            self._slow_g.copy_(state["g_slow_cls"].to(self.device))
            for r, saved in zip(self._slow_rings, state["slow_rings"]):
                r.copy_(saved.to(self.device))
        for k, v in state["scalars"].items():
            setattr(self, k, v)
        self._rate_np_key = None

    # ------------------------------------------------------------------ readouts (brain.py:963-992)
    def rate_np(self) -> np.ndarray:
        key = (self.step_count, self.t)
        if self._rate_np_key != key:
            self._rate_np = self.rate[0].detach().cpu().numpy()
            self._rate_np_key = key
        return self._rate_np

    def rates(self, idx) -> np.ndarray:
        if self.B == 1:
            return self.rate_np()[np.asarray(idx)]
        return self.rate[:, self._idx(idx)].detach().cpu().numpy()

    def mean_rate(self, idx):
        if len(idx) == 0:
            return 0.0 if self.B == 1 else np.zeros(self.B)
        if self.B == 1:
            return float(self.rate_np()[np.asarray(idx)].mean())
        return self.rate[:, self._idx(idx)].mean(dim=1).detach().cpu().numpy()

    def total_spikes(self):
        s = self.spikes.sum(dim=1)
        return float(s[0]) if self.B == 1 else s.cpu().numpy()

    @property
    def synaptic_events(self) -> int:
        """Edges delivered since construction (sum over spikes of the out-degree); host sync."""
        return int(self._events.item())
