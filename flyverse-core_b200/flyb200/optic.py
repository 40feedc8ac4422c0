"""Graded rate-model optic lobe on the B200 native substep: the drop-in for flyverse/optic.py.

`OpticLobe(c, retina, params, device, batch, ...)` keeps the reference constructor
(optic.py:169-172), `step_frame(col_radiance, spk_rate_hz, frame_ms) -> drive (B, N)`,
`photoreceptor_activity`, `rates`, `relax`, `reset(rows)` and the state tensors of
FlyBrain.OPTIC_TENSORS (fly.py:39). The matrices are built by the reference's rules
(optic.py:238-348: per-target L1 / L2 normalisation, pair gains matched with re.match,
per-type time constants and operating points) and run on:

  flyb_photoreceptor  the photoreceptor stage (optic.py:496-517)
  flyb_spmm           the held inputs gain_in * W_rp a_pr and gain_fb * W_rs s (optic.py:579-580),
                      s = clamp(rate / 100, 0, 3) gathered straight from the brain's rate storage,
                      and the drive gain_out * W_sr dr clipped to +-drive_clip (optic.py:599-602)
  flyb_optic_run      the fused substeps: W_rr SpMV/SpMM + rate update (optic.py:525-551)

State is stored unit-major, fly-minor ([n][B]); the (B, n) attributes are views of it. The
opt-in per-stream hooks and the slow receptor term are Torch-only in the reference and are not
provided here (they raise).
"""
from __future__ import annotations

import ctypes as ct
import math
import re
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp
import torch

from . import _abi
from .connectome import PHOTORECEPTOR_TYPES

FAMILY_OF_TYPE = {"R1-R6": 0, "R7p": 1, "R7y": 2, "R7d": 1, "R7_unclear": 2, "R8p": 3, "R8y": 4,
                  "R8d": 1, "R8_unclear": 4, "R7R8_unclear": 2}
# Model constants of the reference's optic lobe (optic.py:126-146), needed for identical weights.
DEFAULT_TAU_BY_TYPE = {"Mi4": 150.0, "Mi9": 150.0, "CT1": 150.0, "Tm9": 150.0, "L3": 40.0, "Mi1": 8.0, "Tm3": 8.0,
                       "Tm1": 8.0, "Tm2": 8.0, "Tm4": 8.0, "L1": 6.0, "L2": 6.0, "T4a": 10.0, "T4b": 10.0, "T4c": 10.0,
                       "T4d": 10.0, "T5a": 10.0, "T5b": 10.0, "T5c": 10.0, "T5d": 10.0}
T4T5 = ["T4a", "T4b", "T4c", "T4d", "T5a", "T5b", "T5c", "T5d"]
DEFAULT_BASELINE_BY_TYPE = {t: 0.0 for t in T4T5}
DEFAULT_PAIR_GAIN = [(r"^(Mi4|Mi9|CT1|C3)$", r"^T4[abcd]$", 5.0), (r"^(Tm4|Tm9|CT1|TmY15)$", r"^T5[abcd]$", 5.0),
                     (r"^LPi(34|43)$", r"^LPLC2$", 4.0), (r"^T[45][abcd]$", r".*", 2.0)]


@dataclass
class OpticParams:
    """The reference's optic-lobe parameters (optic.py:47-123), same names and defaults."""
    tau_ms: float = 10.0
    dt_ms: float = 1.0
    baseline: float = 0.5
    gain_rr: float = 1.0
    gain_in: float = 3.0
    norm: str = "l2"
    gain_fb: float = 0.5
    adapt_tau_ms: float = 400.0
    adapt_gain: float = 1.0
    tau_by_type: dict = None
    baseline_by_type: dict = None
    pair_gain: list = None
    gain_out_mv: float = 100.0
    out_norm: str = "l1"
    drive_clip_mv: float = 35.0
    tau_lp_ms: float = 10.0
    tau_adapt_ms: float = 300.0
    contrast_clip: float = 2.0
    eps: float = 0.02
    stream_rectify: list = None
    stream_adapt: list = None
    spatial_suppress: list = None
    fb_hold: list = None


# ------------------------------------------------------------------ device CSR and the products
class DeviceCSR:
    """A scipy CSR copied to the device as int32 row pointers / columns and float32 values."""

    def __init__(self, M: sp.spmatrix, device):
        M = sp.csr_matrix(M, dtype=np.float32)
        M.sum_duplicates()
        M.sort_indices()
        if max(*M.shape, M.nnz) >= 2**31:
            raise ValueError("the native products need 32-bit dimensions and indices")
        self.shape, self.nnz = M.shape, int(M.nnz)
        self.ptr = torch.from_numpy(M.indptr.astype(np.int32)).to(device)
        self.col = torch.from_numpy(M.indices.astype(np.int32)).to(device)
        self.w = torch.from_numpy(M.data.astype(np.float32)).to(device)
        self._cw = None

    @property
    def cw(self) -> torch.Tensor:
        """[nnz][2] int32 {column, float bits of the weight}: one 8-byte load per entry."""
        if self._cw is None:
            self._cw = torch.stack([self.col, self.w.view(torch.int32)], dim=1).contiguous()
        return self._cw

    def refresh_cw(self) -> None:
        """Copy changed weights into the interleaved entries."""
        if self._cw is not None:
            self._cw[:, 1].copy_(self.w.view(torch.int32))

    def transpose(self, device):
        """(CSR of M^T, perm) with perm[e'] = index in M's CSR order of transposed entry e'."""
        rows = np.repeat(np.arange(self.shape[0], dtype=np.int64), np.diff(self.ptr.cpu().numpy()))
        cols = self.col.cpu().numpy().astype(np.int64)
        order = np.lexsort((rows, cols))
        T = sp.csr_matrix((self.w.cpu().numpy()[order], (cols[order], rows[order])), shape=self.shape[::-1])
        t = DeviceCSR.__new__(DeviceCSR)
        t.shape, t.nnz, t._cw = T.shape, int(T.nnz), None
        t.ptr = torch.from_numpy(np.concatenate([[0], np.cumsum(np.bincount(cols, minlength=self.shape[1]))]).astype(np.int32)).to(device)
        t.col = torch.from_numpy(rows[order].astype(np.int32)).to(device)
        t.w = torch.from_numpy(self.w.cpu().numpy()[order]).to(device)
        return t, torch.from_numpy(order.astype(np.int32)).to(device)


_SMS: dict = {}


def _sm_count(device) -> int:
    if device not in _SMS:
        _SMS[device] = torch.cuda.get_device_properties(device).multi_processor_count
    return _SMS[device]


def spmm_warps_per_row(nnz: int, rows: int, batch: int, sms: int = 148) -> int:
    """Warps sharing one row of flyb_spmm (1, 2, 4, 8; a block holds 8 warps): the fewest that
    still give about two blocks per SM, or that keep a warp within 16 passes of U entries per lane
    group over a row of mean length (F, FPL as the library picks them for the batch). Measured at
    64 flies on the whole-fly coupling blocks: 3,885 rows of 50 entries run best at 1 warp per row,
    1,787 rows of 20 at 2."""
    if rows <= 0:
        return 1
    lanes = {1: 1, 2: 2, 4: 4, 8: 8, 16: 16}
    f, fpl = next(((f, 1) for b, f in lanes.items() if batch <= b), None) or \
        ((8, 4) if batch <= 32 else (16, 4) if batch <= 64 else (32, 4) if batch <= 128 else (32, 8))
    unroll = 8 if fpl <= 2 else (4 if fpl == 4 else 2)
    per_pass = unroll * (32 // f)
    mean = -(-nnz // rows)
    wpr = 1
    while wpr < 8 and (rows * wpr / 8 < 2 * sms or mean > wpr * per_pass * 16):
        wpr *= 2
    return wpr


def spmm(M: DeviceCSR, x: torch.Tensor, y: torch.Tensor, *, x_index=None, x_div=1.0, x_lo=-math.inf,
         x_hi=math.inf, y_index=None, alpha=1.0, y_lo=-math.inf, y_hi=math.inf, accumulate=False,
         warps_per_row: int | None = None) -> None:
    """y[ymap(i)][b] (+)= clamp(alpha * sum_e w_e * clamp(x[xmap(col_e)][b] / x_div, x_lo, x_hi), y_lo, y_hi).

    x, y: contiguous fly-minor storage [rows][B] on the device (include/flyb200.h: flyb_spmm)."""
    B = x.shape[1]
    if x.dtype != torch.float32 or y.dtype != torch.float32 or not x.is_contiguous() or not y.is_contiguous():
        raise ValueError("spmm needs contiguous float32 [rows][batch] tensors")
    if y.shape[1] != B:
        raise ValueError("x and y batch widths differ")
    a = _abi.SpmmArgs(rows=M.shape[0], cols=M.shape[1], batch=B, accumulate=int(accumulate), ptr=M.ptr.data_ptr(),
                      col=M.col.data_ptr(), w=M.w.data_ptr(), x=x.data_ptr(),
                      x_index=None if x_index is None else x_index.data_ptr(), x_rows=x.shape[0], x_div=x_div,
                      x_lo=x_lo, x_hi=x_hi, y=y.data_ptr(), y_index=None if y_index is None else y_index.data_ptr(),
                      y_rows=y.shape[0], alpha=alpha, y_lo=y_lo, y_hi=y_hi,
                      warps_per_row=warps_per_row or spmm_warps_per_row(M.nnz, M.shape[0], B, _sm_count(x.device)))
    rc = _abi.lib().flyb_spmm(ct.byref(a), torch.cuda.current_stream(x.device).cuda_stream)
    if rc:
        raise RuntimeError(f"flyb_spmm: error {rc}")


LONG_ROW = 192      # rows with more entries than this are split across a whole block


class OpticCore:
    """The rate-unit recurrence on the device: W_rr, per-unit a / b, state [M][B], held inputs.

    Rows run longest first (so the tail of a substep is short rows) and rows longer than
    `long_row` entries are each shared by all warps of a block (flyb_optic_args.rows / n_long)."""

    def set_long_rows(self, long_row: int) -> None:
        """Rows with more than `long_row` entries are split across a block. The row order (longest
        first) is built once and kept in the same device buffer, so captured graphs stay valid;
        only the count of long rows (a launch argument) changes."""
        if getattr(self, "_deg", None) is None:
            self._deg = np.diff(self.W.ptr.cpu().numpy())
            order = np.argsort(-self._deg, kind="stable").astype(np.int32)
            self.rows = torch.from_numpy(order).to(self.device)
        self.n_long = int((self._deg > long_row).sum())
        self.long_row = int(long_row)

    def __init__(self, W_rr: sp.spmatrix, a: np.ndarray, b: np.ndarray, *, batch: int, device, gain_rr: float,
                 adapt_gain: float, aad: float, launch: str = "persistent"):
        self.device, self.B = torch.device(device), int(batch)
        if self.device.type != "cuda":
            raise ValueError("the optic lobe runs on a CUDA device only; there is no CPU path")
        self._lib = _abi.lib()
        self.W = DeviceCSR(W_rr, self.device)
        self.m = self.W.shape[0]
        self.a = torch.from_numpy(np.asarray(a, np.float32)).to(self.device)
        self.b = torch.from_numpy(np.asarray(b, np.float32)).to(self.device)
        self.gain_rr, self.adapt_gain, self.aad = float(gain_rr), float(adapt_gain), float(aad)
        self.launch = launch
        self.variant = 0                 # kernel shape (flyb_optic_args.variant), set by the autotuner
        self.grid = 0                    # persistent launches: block cap (0 = every resident block)
        self.set_long_rows(LONG_ROW)
        M, B, dev = self.m, self.B, self.device
        self.v_s = torch.zeros(M, B, device=dev)
        self.adapt_s = torch.zeros(M, B, device=dev)
        self.pr_in = torch.zeros(M, B, device=dev)
        self.spk_in = torch.zeros(M, B, device=dev)
        # dr ping-pong: _bufs[_cur] holds clip(v + b, 0, 1) - b of the current state after every call;
        # _dr_key records (v, b) versions then, so a later call can skip recomputing it (carry=True)
        self._bufs = (torch.zeros(M, B, device=dev), torch.zeros(M, B, device=dev))
        self._cur = 0
        self._dr_key = None
        self._status = torch.zeros(4, dtype=torch.int32, device=dev)
        self._sync = torch.zeros(64, dtype=torch.int32, device=dev)
        self._WT = None

    def _state_key(self):
        return (self.v_s._version, self.b._version, self.v_s.data_ptr(), self.b.data_ptr())

    def substeps(self, nsteps: int, v_hist: torch.Tensor | None = None, inp_hist: torch.Tensor | None = None,
                 carry: bool = False) -> None:
        """Run `nsteps` substeps. `carry`: reuse the dr the previous call left (FLYB_OPTIC_DR_VALID)
        when v and b have not been written since (tensor version counters), saving one pass over
        the state; the kernels themselves never bump the counters."""
        if nsteps <= 0:
            return
        flags = _abi.OPTIC_HISTORY if v_hist is not None else 0
        if carry and self._dr_key == self._state_key():
            flags |= _abi.OPTIC_DR_VALID
        dr, dr_tmp = self._bufs[self._cur], self._bufs[1 - self._cur]
        a = _abi.OpticArgs(m=self.m, batch=self.B, nsteps=int(nsteps), launch=_abi.LAUNCHES_BY_NAME[self.launch],
                           grid=int(self.grid), ptr=self.W.ptr.data_ptr(), cw=self.W.cw.data_ptr(), variant=self.variant,
                           rows=self.rows.data_ptr(), n_long=self.n_long,
                           v=self.v_s.data_ptr(), adapt=self.adapt_s.data_ptr(), dr=dr.data_ptr(),
                           dr_tmp=dr_tmp.data_ptr(), pr=self.pr_in.data_ptr(), spk=self.spk_in.data_ptr(),
                           a=self.a.data_ptr(), b=self.b.data_ptr(), gr=self.gain_rr, ga=self.adapt_gain, aad=self.aad,
                           flags=flags, v_hist=None if v_hist is None else v_hist.data_ptr(),
                           inp_hist=None if inp_hist is None else inp_hist.data_ptr(),
                           status=self._status.data_ptr(), sync=self._sync.data_ptr())
        with torch.cuda.device(self.device):
            rc = self._lib.flyb_optic_run(ct.byref(a), torch.cuda.current_stream(self.device).cuda_stream)
        if rc:
            raise RuntimeError(f"flyb_optic_run: error {rc}")
        self._cur ^= int(nsteps) & 1
        self._dr_key = self._state_key()

    @property
    def dr_out(self) -> torch.Tensor:
        """The device buffer holding clip(v + b, 0, 1) - b of the state the last call left, [M][B]."""
        return self._bufs[self._cur]

    def pin_dr(self, cur: int) -> None:
        """Move the current dr into buffer `cur` (stream-ordered copy when it is elsewhere): a CUDA
        graph of an odd number of substeps must end with dr where it started."""
        if self._cur != cur:
            self._bufs[cur].copy_(self._bufs[self._cur])
            self._cur = cur
            self._dr_key = self._state_key()

    def dr(self) -> torch.Tensor:
        """clip(v + b, 0, 1) - b, [M][B]."""
        return (self.v_s + self.b[:, None]).clamp(0.0, 1.0) - self.b[:, None]

    def check(self) -> None:
        s = self._status.cpu().tolist()
        if s[0]:
            raise RuntimeError(f"flyb200 optic kernel status {s[0]} (where {s[1]}, step {s[2]})")


# ------------------------------------------------------------------ the reference-API lobe
def _mask(regex: str, labels: np.ndarray) -> np.ndarray:
    rx = re.compile(regex)
    cache = {t: bool(rx.match(t)) for t in np.unique(labels)}
    return np.fromiter((cache[t] for t in labels), bool, len(labels))


def _full_mask(regex: str, labels: np.ndarray) -> np.ndarray:
    rx = re.compile(str(regex))
    cache = {t: bool(rx.fullmatch(t)) for t in np.unique(labels)}
    return np.fromiter((cache[t] for t in labels), bool, len(labels))


@dataclass
class LobeMatrices:
    """Everything the optic lobe derives from the connectome once (host side, scipy)."""
    rate_idx: np.ndarray
    pr_idx: np.ndarray
    spk_idx: np.ndarray
    M_rr: sp.csr_matrix
    M_rp: sp.csr_matrix
    M_rs: sp.csr_matrix
    M_sr: sp.csr_matrix
    a: np.ndarray
    b: np.ndarray
    aad: float
    pr_family: np.ndarray
    has: np.ndarray
    avg: sp.csr_matrix
    pr_cell: np.ndarray
    pr_column: np.ndarray
    sens: np.ndarray


def photoreceptor_cells(pr_column, pr_family, n_col: int):
    """The column x family cells of the photoreceptor stage (optic.py:343-348): which cells have
    members (n_col, 5), the averaging matrix (n_col * 5, n_pr) with 1 / members per entry, and each
    photoreceptor's cell (column * 5 + family)."""
    pr_column, pr_family = np.asarray(pr_column, np.int64), np.asarray(pr_family, np.int64)
    has = np.zeros((n_col, 5), bool)
    np.add.at(has, (pr_column, pr_family), True)
    cnt = np.zeros((n_col, 5), np.float32)
    np.add.at(cnt, (pr_column, pr_family), 1.0)
    cell = pr_column * 5 + pr_family
    avg = sp.csr_matrix((1.0 / cnt[pr_column, pr_family], (cell, np.arange(len(cell)))), shape=(n_col * 5, len(cell)))
    return has, avg, cell


class PhotoreceptorStage:
    """The photoreceptor stage on the device (optic.py:496-517, `flyb_photoreceptor`): per fly and
    column x family cell the channel-weighted intensity averaged over the cell's photoreceptors, its
    low-pass (tau_lp_ms) and adaptation (tau_adapt_ms) states, the clipped contrast, gathered back
    to the photoreceptors as a_pr [n_pr][B]. The first frame after construction or `reset` starts
    both states at the frame's intensity. State: I_lp, I_mean, contrast (B, n_col * 5), fresh (B)."""

    def __init__(self, pr_column, pr_family, sens, n_col: int, batch: int, device, p: OpticParams | None = None):
        self.p = p or OpticParams()
        dev = torch.device(device)
        self.device, self.B, self.n_col = dev, int(batch), int(n_col)
        self.has, avg, cell = photoreceptor_cells(pr_column, pr_family, n_col)
        self.n_pr = len(cell)
        self.avg = DeviceCSR(avg, dev)
        self.sens = torch.from_numpy(np.ascontiguousarray(sens, np.float32).reshape(-1, 4)).to(dev)
        self.pr_column_t = torch.as_tensor(np.asarray(pr_column, np.int32), device=dev)
        self.pr_cell_t = torch.as_tensor(cell.astype(np.int32), device=dev)
        self.has_t = torch.from_numpy(self.has.reshape(-1).astype(np.uint8)).to(dev)
        self.I_lp = torch.zeros(self.B, n_col * 5, device=dev)
        self.I_mean = torch.zeros(self.B, n_col * 5, device=dev)
        self.contrast = torch.zeros(self.B, n_col * 5, device=dev)
        self.fresh_u8 = torch.ones(self.B, dtype=torch.uint8, device=dev)
        self.a_pr = torch.zeros(self.n_pr, self.B, device=dev)

    def reset(self, rows=None) -> None:
        sel = slice(None) if rows is None else torch.as_tensor(rows, device=self.device)
        for t in (self.I_lp, self.I_mean, self.contrast):
            t[sel] = 0.0
        self.fresh_u8[sel] = 1

    def __call__(self, rad: torch.Tensor, dt_ms: float, out: torch.Tensor | None = None) -> torch.Tensor:
        """rad: contiguous float32 (B, n_col, 4) on the device -> a_pr [n_pr][B] (`out` or the
        stage's own buffer), on the current stream."""
        if rad.dtype != torch.float32 or not rad.is_contiguous() or tuple(rad.shape) != (self.B, self.n_col, 4):
            raise ValueError("radiance must be a contiguous float32 (batch, columns, 4) tensor")
        out = self.a_pr if out is None else out
        if out.dtype != torch.float32 or not out.is_contiguous() or tuple(out.shape) != (self.n_pr, self.B):
            raise ValueError("out must be a contiguous float32 [n_pr][batch] tensor")
        p = self.p
        a_lp, a_ad = float(np.exp(-dt_ms / p.tau_lp_ms)), float(np.exp(-dt_ms / p.tau_adapt_ms))
        args = _abi.PhotoArgs(n_pr=self.n_pr, n_col=self.n_col, batch=self.B, rad=rad.data_ptr(),
                              pr_column=self.pr_column_t.data_ptr(), sens=self.sens.data_ptr(),
                              avg_ptr=self.avg.ptr.data_ptr(), avg_idx=self.avg.col.data_ptr(), avg_w=self.avg.w.data_ptr(),
                              pr_cell=self.pr_cell_t.data_ptr(), has=self.has_t.data_ptr(), I_lp=self.I_lp.data_ptr(),
                              I_mean=self.I_mean.data_ptr(), contrast=self.contrast.data_ptr(),
                              fresh=self.fresh_u8.data_ptr(), a_lp=a_lp, c_lp=1 - a_lp, a_ad=a_ad, c_ad=1 - a_ad,
                              eps=p.eps, clip_hi=p.contrast_clip, a_pr=out.data_ptr())
        rc = _abi.lib().flyb_photoreceptor(ct.byref(args), torch.cuda.current_stream(self.device).cuda_stream)
        if rc:
            raise RuntimeError(f"flyb_photoreceptor: error {rc}")
        return out


def lobe_matrices(c, retina, p: OpticParams, receptor=None, receptor_gain=None) -> LobeMatrices:
    """The reference's optic-lobe construction (optic.py:229-348): unit selection, normalised and
    gain-shaped blocks, per-type constants and the photoreceptor averaging matrix."""
    nrn = c.neurons
    types = nrn.type.fillna("").to_numpy()
    is_pr = nrn.type.isin(PHOTORECEPTOR_TYPES).to_numpy()
    rate_idx = np.flatnonzero((nrn.superclass == "ol_intrinsic").to_numpy() & ~is_pr)
    pr_idx = np.asarray(retina.pr_index)
    is_rate = np.zeros(c.n, bool)
    is_rate[rate_idx] = True
    spk_idx = np.flatnonzero(~is_rate & ~is_pr)
    W = c.W.tocsr()
    if receptor is not None:
        if len(receptor.fast_sign) != W.nnz:
            raise ValueError("receptor signs are not aligned with this connectome's W")
        W = W.copy()
        W.data = np.abs(W.data) * receptor.fast_factor(receptor_gain)
    tot = c.neurons.in_syn.to_numpy()
    Wn = (sp.diags(1.0 / np.maximum(tot, 1.0)) @ W).tocsr()
    if p.norm == "l2":
        Wn_ol = (sp.diags(1.0 / np.maximum(c.neurons.in_syn_l2.to_numpy(), 1.0)) @ W).tocsr()
    else:
        Wn_ol = Wn
    pair_gain = DEFAULT_PAIR_GAIN if p.pair_gain is None else p.pair_gain

    def gains(M, pre_types, post_types):
        if not pair_gain:
            return M
        M = M.tocoo()
        for pre_re, post_re, f in pair_gain:
            sel = _mask(pre_re, pre_types)[M.col] & _mask(post_re, post_types)[M.row]
            M.data[sel] *= f
        return M.tocsr()

    rt, st = types[rate_idx], types[spk_idx]
    M_rr = gains(Wn_ol[rate_idx][:, rate_idx], rt, rt)
    M_rs = Wn_ol[rate_idx][:, spk_idx].tocsr()
    M_sr = gains((Wn_ol if p.out_norm == "l2" else Wn)[spk_idx][:, rate_idx], rt, st)
    if p.fb_hold:
        C = M_rs.tocsr()
        rows = np.repeat(np.arange(C.shape[0]), np.diff(C.indptr))
        keep = np.ones(C.nnz, bool)
        for pre_re, post_re in p.fb_hold:
            keep &= ~(_full_mask(pre_re, st)[C.indices] & _full_mask(post_re, rt)[rows])
        indptr = np.concatenate([[0], np.cumsum(np.bincount(rows[keep], minlength=C.shape[0]))])
        M_rs = sp.csr_matrix((C.data[keep], C.indices[keep], indptr), shape=C.shape)
    M_rp = Wn_ol[rate_idx][:, pr_idx].tocsr()
    tau_map = DEFAULT_TAU_BY_TYPE if p.tau_by_type is None else p.tau_by_type
    tau = np.array([tau_map.get(t, p.tau_ms) for t in rt], dtype=np.float32)
    a = np.exp(-p.dt_ms / tau)
    bl_map = DEFAULT_BASELINE_BY_TYPE if p.baseline_by_type is None else p.baseline_by_type
    b = np.array([bl_map.get(t, p.baseline) for t in rt], dtype=np.float32)
    pr_family = np.array([FAMILY_OF_TYPE[t] for t in types[pr_idx]], dtype=np.int64)
    has, avg, rows = photoreceptor_cells(retina.pr_column, pr_family, retina.n_columns)
    return LobeMatrices(rate_idx, pr_idx, spk_idx, M_rr, M_rp, M_rs, M_sr, a.astype(np.float32), b,
                        float(np.exp(-p.dt_ms / p.adapt_tau_ms)), pr_family, has, avg, rows,
                        np.asarray(retina.pr_column, np.int64), np.asarray(retina.pr_sens, np.float32).reshape(-1, 4))


def _adopt_strongest(W: sp.csr_matrix, cells, known: np.ndarray, out: np.ndarray) -> None:
    """For each i of `cells`, visited in order: out[i] = known[j] of the input j of row i of W with the
    largest weight among the inputs whose known[j] >= 0 (the first of equal ones); a row with no such
    input keeps out[i]. With out = known a later cell sees the result of an earlier one."""
    for i in cells:
        lo, hi = W.indptr[i], W.indptr[i + 1]
        pre = W.indices[lo:hi]
        good = known[pre] >= 0
        if good.any():
            out[i] = known[pre[good][np.argmax(W.data[lo:hi][good])]]


def column_of_cells(c, retina, rate_idx) -> np.ndarray:
    """Retinal column of every cell (-1: none), as the reference assigns it for spatial suppression
    (interp/trace.py:945-971): a rate cell from its hex annotation; three passes then give an
    unannotated rate cell the column of its strongest rate input, and a last pass does the same for
    every cell still without one, spiking cells included."""
    lookup = {(str(side), int(h[0]), int(h[1])): k for k, (side, h) in enumerate(zip(retina.col_side, retina.col_hex))}
    ridx = np.asarray(rate_idx)
    ann = c.neurons.iloc[ridx]

    def annotated(side, h1, h2) -> int:
        return -1 if (h1 != h1 or h2 != h2) else lookup.get((str(side), int(h1), int(h2)), -1)

    col_rate = np.fromiter((annotated(*t) for t in zip(ann["hex_side"].fillna("").to_numpy(), ann["hex1"].to_numpy(),
                                                        ann["hex2"].to_numpy())), np.int64, len(ridx))
    absW = sp.csr_matrix(abs(c.W))
    rate_in = absW[ridx][:, ridx].tocsr()
    for _ in range(3):
        _adopt_strongest(rate_in, np.flatnonzero(col_rate < 0), col_rate, col_rate)
    col = np.full(c.n, -1, np.int64)
    col[ridx] = col_rate
    _adopt_strongest(absW[:, ridx].tocsr(), np.flatnonzero(col < 0), col_rate, col)
    return col


def _csr_select(C: sp.csr_matrix, keep: np.ndarray) -> sp.csr_matrix:
    """The entries of C flagged by `keep`, in C's order (each row sums its survivors in C's order)."""
    C = C.tocsr()
    rows = np.repeat(np.arange(C.shape[0]), np.diff(C.indptr))
    indptr = np.concatenate([[0], np.cumsum(np.bincount(rows[keep], minlength=C.shape[0]))])
    return sp.csr_matrix((C.data[keep], C.indices[keep], indptr), shape=C.shape)


def _first_rule(n: int, holds: list) -> np.ndarray:
    """Per item, the index of the first rule that holds for it (`holds`: one boolean mask per rule), -1 for none."""
    owner = np.full(n, -1, np.int64)
    for k in range(len(holds) - 1, -1, -1):
        owner[holds[k]] = k
    return owner


@dataclass
class StreamHooks:
    """The per-stream hooks (optic.py:50-70, 378-451): W_rr and W_sr split into the rest and one
    block per (rectify entry, adapt entry) stream, each block multiplying its stream's signal
    x = rectify(u - gain A), u = dr - G dr (G: the spatial suppression operator, or None)."""
    rest_rr: sp.csr_matrix
    rest_sr: sp.csr_matrix
    streams: list          # [{"mode": None|"pos"|"neg"|"abs", "adapt_id": int, "W_rr": csr|None, "W_sr": csr|None}]
    adapt_decay: list      # exp(-dt / tau) per stream_adapt entry
    adapt_gain: list
    G: sp.csr_matrix | None

    def matched(self, which: str) -> int:
        """Entries of W_rr ("rr") or W_sr ("sr") that belong to a stream."""
        return sum(s[f"W_{which}"].nnz for s in self.streams if s[f"W_{which}"] is not None)


def stream_hooks(c, retina, rate_idx, spk_idx, p: OpticParams, M_rr, M_sr) -> StreamHooks | None:
    """The blocks of OpticParams.stream_rectify / stream_adapt / spatial_suppress, or None when all
    three are off. An entry of W belongs to the first rectify and the first adapt rule whose pre and
    post patterns full-match its cells' types; it is in a stream when either rule, or a suppression
    rule on its presynaptic cell, matched. Streams are ordered by (rectify rule, adapt rule)."""
    rect, adapt, supp = list(p.stream_rectify or []), list(p.stream_adapt or []), list(p.spatial_suppress or [])
    if not (rect or adapt or supp):
        return None
    for k, rule in enumerate(rect):
        if rule[2] not in ("pos", "neg", "abs"):
            raise ValueError(f"stream_rectify[{k}]: mode must be pos, neg or abs, got {rule[2]!r}")
    for k, rule in enumerate(adapt):
        if not (np.isfinite(rule[2]) and rule[2] > 0):
            raise ValueError(f"stream_adapt[{k}]: tau_ms must be positive and finite")
    types = c.neurons.type.fillna("").to_numpy()
    rate_t, spk_t = types[rate_idx], types[spk_idx]
    n_rate = len(rate_idx)
    supp_of = _first_rule(n_rate, [_full_mask(rule[0], rate_t) for rule in supp])

    def blocks_of(M, post_t):
        C = M.tocsr()
        post, pre = np.repeat(np.arange(C.shape[0]), np.diff(C.indptr)), C.indices
        rect_of = _first_rule(C.nnz, [_full_mask(r[0], rate_t)[pre] & _full_mask(r[1], post_t)[post] for r in rect])
        adapt_of = _first_rule(C.nnz, [_full_mask(r[0], rate_t)[pre] & _full_mask(r[1], post_t)[post] for r in adapt])
        hooked = (rect_of >= 0) | (adapt_of >= 0) | (supp_of[pre] >= 0)
        keys = sorted(set(zip(rect_of[hooked].tolist(), adapt_of[hooked].tolist())))
        return ({k: _csr_select(C, hooked & (rect_of == k[0]) & (adapt_of == k[1])) for k in keys},
                _csr_select(C, ~hooked))

    blk_rr, rest_rr = blocks_of(M_rr, rate_t)
    blk_sr, rest_sr = blocks_of(M_sr, spk_t)
    streams = [{"mode": rect[k[0]][2] if k[0] >= 0 else None, "adapt_id": k[1], "W_rr": blk_rr.get(k),
                "W_sr": blk_sr.get(k)} for k in sorted(set(blk_rr) | set(blk_sr))]
    G = None
    if supp:
        # G[j, j'] = k / n_j over the n_j cells j' of j's type whose column lies within the rule's
        # radius of j's column (j itself included): u = dr - G dr is dr less k x the local type mean.
        col = column_of_cells(c, retina, rate_idx)[rate_idx]
        cd = np.asarray(retina.col_dir, dtype=np.float64)
        cos_cc = np.clip(cd @ cd.T, -1.0, 1.0)
        ii, jj, vv = [np.zeros(0, np.int64)], [np.zeros(0, np.int64)], [np.zeros(0)]
        for k, (_, strength, radius) in enumerate(supp):
            near_cc = cos_cc >= np.cos(np.radians(float(radius)))
            cells = np.flatnonzero((supp_of == k) & (col >= 0))
            for t in np.unique(rate_t[cells]):
                ct = cells[rate_t[cells] == t]
                near = near_cc[np.ix_(col[ct], col[ct])]
                r_, c_ = np.nonzero(near)
                ii.append(ct[r_]), jj.append(ct[c_]), vv.append(float(strength) / near.sum(1)[r_])
        G = sp.csr_matrix((np.concatenate(vv).astype(np.float32), (np.concatenate(ii), np.concatenate(jj))),
                          shape=(n_rate, n_rate))
    return StreamHooks(rest_rr, rest_sr, streams, [float(np.exp(-p.dt_ms / float(r[2]))) for r in adapt],
                       [float(r[3]) for r in adapt], G)


def slow_blocks(c, rate_idx, spk_idx, p: OpticParams, receptor, receptor_gain, spec) -> tuple[list, float]:
    """The optic lobe's slow-tone blocks (optic.py:285-309): per active class of `spec` the
    spiking -> rate and rate -> rate matrices (count x slow sign x gain class, normalised by the same
    denominators as the fast blocks; None where empty), the relaxation scale gain tau / tau_syn and
    factor exp(-dt / tau); and the tone's normalisation 1 - baseline."""
    if getattr(receptor, "count", None) is None:
        raise ValueError("the optic lobe's slow term needs the receptor record's synapse counts")
    denom = c.neurons.in_syn_l2.to_numpy() if p.norm == "l2" else c.neurons.in_syn.to_numpy()
    out = []
    for cls in spec.classes:
        S = c.W.tocsr().copy()
        S.data = receptor.count * receptor.slow_factor(receptor_gain, slow_class=cls)
        S.eliminate_zeros()
        Sn = (sp.diags(1.0 / np.maximum(denom, 1.0)) @ S).tocsr()
        rs = Sn[rate_idx][:, spk_idx].tocsr()
        rr = Sn[rate_idx][:, rate_idx].tocsr()
        out.append((rs if rs.nnz else None, rr if rr.nnz else None, float(spec.gain[cls] * spec.tau[cls] / spec.tau_syn),
                    float(np.exp(-p.dt_ms / spec.tau[cls]))))
    norm = float(1.0 - p.baseline)
    if norm <= 0:
        raise ValueError("the optic slow term needs baseline < 1")
    return out, norm


class OpticLobe:
    def __init__(self, c, retina, params: OpticParams | None = None, device=None, batch: int = 1,
                 metal_kernels=None, cuda_kernels=None, cuda_sparse: str = "torch", receptor=None,
                 receptor_gain=None, slow=None, surrogate_grad: bool = False, *, launch: str = "persistent"):
        c.require("optic_columns")
        self.c, self.r, self.p = c, retina, params or OpticParams()
        p = self.p
        if metal_kernels:
            raise ValueError("flyb200 runs on B200 CUDA kernels only; the Metal backend is not provided")
        if cuda_kernels is False:
            raise ValueError("flyb200 has no Torch path: cuda_kernels=False is not available")
        if surrogate_grad:
            raise NotImplementedError("use flyb200.adjoint (hand-written optic adjoint) for gradients")
        if not np.isfinite(p.dt_ms) or p.dt_ms <= 0:
            raise ValueError("optic dt_ms must be positive and finite")
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        if self.device.type != "cuda":
            raise ValueError("flyb200.OpticLobe runs on a CUDA device only; there is no CPU path")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.B = int(batch)
        # the slow receptor tone (optic.py:203, 285-309) is active with a receptor record and a scale
        self.slow = slow if (slow is not None and receptor is not None and getattr(slow, "gain", None)) else None
        self.receptor, self.surrogate_grad = receptor, False
        self._pending_ms = 0.0
        L = lobe_matrices(c, retina, p, receptor, receptor_gain)
        self.L = L
        self.rate_idx, self.pr_idx, self.spk_idx = L.rate_idx, L.pr_idx, L.spk_idx
        self.n_rate, self.n_pr, self.n_spk = len(self.rate_idx), len(self.pr_idx), len(self.spk_idx)
        self.M_rr, self.M_rp, self.M_rs, self.M_sr = L.M_rr, L.M_rp, L.M_rs, L.M_sr
        M_rr, M_rp, M_rs, M_sr, a, b = L.M_rr, L.M_rp, L.M_rs, L.M_sr, L.a, L.b
        self._a_ad = L.aad
        self.core = OpticCore(M_rr, a, b, batch=self.B, device=self.device, gain_rr=p.gain_rr,
                              adapt_gain=p.adapt_gain, aad=self._a_ad, launch=launch)
        dev = self.device
        self.W_rp, self.W_rs, self.W_sr = DeviceCSR(M_rp, dev), DeviceCSR(M_rs, dev), DeviceCSR(M_sr, dev)
        self.rate_idx_t = torch.as_tensor(self.rate_idx, device=dev)
        self.spk_idx_t = torch.as_tensor(self.spk_idx, device=dev)
        self._spk_idx32 = self.spk_idx_t.to(torch.int32)
        self._a, self.b_vec = self.core.a, self.core.b
        self.pr_family = L.pr_family
        self.photo = PhotoreceptorStage(retina.pr_column, L.pr_family, retina.pr_sens, retina.n_columns, self.B, dev, p)
        self.has = self.photo.has
        # the stage's state tensors, under the reference's names (FlyBrain checkpoints them)
        self.I_lp, self.I_mean, self.contrast = self.photo.I_lp, self.photo.I_mean, self.photo.contrast
        self._fresh_u8, self._a_pr = self.photo.fresh_u8, self.photo.a_pr
        B = self.B
        self._delta = torch.zeros(self.n_rate, B, device=dev)
        self._drive = torch.zeros(c.n, B, device=dev)
        self.slow_classes = list(self.slow.classes) if self.slow is not None else []
        K = len(self.slow_classes)
        self._g_cls_s = torch.zeros(K, self.n_rate, B, device=dev)        # [K][m][B] storage
        self._g_slow_s = torch.zeros(self.n_rate, B, device=dev)
        self._held_s = torch.zeros(K, self.n_rate, B, device=dev)
        self.g_slow_cls = self._g_cls_s.transpose(1, 2)                   # (K, B, m) views
        self.g_slow = self._g_slow_s.t()
        self._slow_in_s = self._held_s.transpose(1, 2)
        K_a = len(p.stream_adapt or [])
        self._stream_A_s = torch.zeros(K_a, self.n_rate, B, device=dev)     # [K_a][m][B] storage
        self.stream_adapt_state = self._stream_A_s.transpose(1, 2)
        self.hooks = stream_hooks(c, retina, self.rate_idx, self.spk_idx, p, self.M_rr, self.M_sr)
        if self.slow is not None or self.hooks is not None:
            self._setup_ext(c, receptor, receptor_gain)
        self.r0 = None
        self.last = {}
        self.diagnostics = False

    # public (B, n) views of the fly-minor storage
    @property
    def v(self):
        return self.core.v_s.t()

    @v.setter
    def v(self, value):
        self.core.v_s.t().copy_(value)

    @property
    def adapt(self):
        return self.core.adapt_s.t()

    @adapt.setter
    def adapt(self, value):
        self.core.adapt_s.t().copy_(value)

    @property
    def delta_rate(self):
        return self._delta.t()

    @property
    def _fresh(self):
        return self._fresh_u8.view(torch.bool)

    # ------------------------------------------------------------------ photoreceptors
    @torch.no_grad()
    def photoreceptor_activity(self, col_radiance, dt_ms: float, *, intensity=None) -> torch.Tensor:
        """(B, n_col, 4) radiance -> (B, n_pr) contrast activity (a view of [n_pr][B] storage)."""
        if intensity is not None:
            raise NotImplementedError("an intensity override is an extension-module input, not provided here")
        rad = torch.as_tensor(col_radiance, dtype=torch.float32, device=self.device)
        if rad.dim() == 2:
            rad = rad[None]
        self.photo(rad.expand(self.B, -1, -1).contiguous(), dt_ms)
        return self._a_pr.t()

    # ------------------------------------------------------------------ the slow receptor tone
    def _setup_ext(self, c, receptor, receptor_gain) -> None:
        """Device copies of the slow-tone blocks (`slow_blocks`), the hook blocks (`stream_hooks`)
        and the buffers of the extended substep."""
        p, dev = self.p, self.device
        m, B = self.n_rate, self.B
        self._rec = torch.zeros(m, B, device=dev)
        self._dr_ext = torch.zeros(m, B, device=dev)
        self._slow_rs, self._slow_rr, self._rec_slow = [], [], []
        h = self.hooks
        if h is not None:
            self._h_rest_rr, self._h_rest_sr = DeviceCSR(h.rest_rr, dev), DeviceCSR(h.rest_sr, dev)
            self._h_rr = [DeviceCSR(s_["W_rr"], dev) if s_["W_rr"] is not None else None for s_ in h.streams]
            self._h_sr = [DeviceCSR(s_["W_sr"], dev) if s_["W_sr"] is not None else None for s_ in h.streams]
            self._h_G = DeviceCSR(h.G, dev) if h.G is not None else None
            self._h_tmp = torch.zeros(m, B, device=dev)
            self._h_out = torch.zeros(len(self.spk_idx), B, device=dev)
        else:
            self._W_rr_plain = DeviceCSR(self.M_rr, dev)
        if self.slow is None:
            return
        blocks, self._slow_norm = slow_blocks(c, self.rate_idx, self.spk_idx, p, receptor, receptor_gain, self.slow)
        self._slow_rs = [DeviceCSR(rs, dev) if rs is not None else None for rs, _, _, _ in blocks]
        self._slow_rr = [DeviceCSR(rr, dev) if rr is not None else None for _, rr, _, _ in blocks]
        self._slow_scale = [scale for _, _, scale, _ in blocks]
        self._a_slow = [decay for _, _, _, decay in blocks]
        self.slow_entries = {cls: {"spiking_to_rate": 0 if rs is None else int(rs.nnz),
                                   "rate_to_rate": 0 if rr is None else int(rr.nnz)}
                             for cls, (rs, rr, _, _) in zip(self.slow_classes, blocks)}
        self._rec_slow = [torch.zeros(m, B, device=dev) if W is not None else None for W in self._slow_rr]

    def _stream_signals(self, dr: torch.Tensor, update: bool) -> list:
        """x per hook stream from dr [m][B] (optic.py:453-472): u = dr - G dr, y = u - gain A,
        x = rectify(y); with `update` each adaptation state then relaxes towards u."""
        h = self.hooks
        u = dr
        if self._h_G is not None:
            spmm(self._h_G, dr, self._h_tmp)
            u = dr - self._h_tmp
        xs = []
        for s_ in h.streams:
            a_id = s_["adapt_id"]
            y = u if a_id < 0 else u - h.adapt_gain[a_id] * self._stream_A_s[a_id]
            mode = s_["mode"]
            xs.append(y if mode is None else (y.clamp(min=0.0) if mode == "pos" else
                                              ((-y).clamp(min=0.0) if mode == "neg" else y.abs())))
        if update:
            for k, decay in enumerate(h.adapt_decay):
                torch.add(u, (self._stream_A_s[k] - u) * decay, out=self._stream_A_s[k])
        return xs

    def _hook_output(self, dr: torch.Tensor) -> torch.Tensor:
        """W_sr dr through the hook blocks (optic.py:485-495), [n_spk][B]."""
        xs = self._stream_signals(dr, False)
        spmm(self._h_rest_sr, dr, self._h_out)
        for W, x in zip(self._h_sr, xs):
            if W is not None:
                spmm(W, x, self._h_out, accumulate=True)
        return self._h_out

    def _ext_substeps(self, steps: int) -> None:
        """The substeps with the slow tone and / or the per-stream hooks (optic.py:526-551): dr
        (shifted by the tone in the threshold mode), the recurrent product (with the hooks, the rest
        block on dr plus each stream block on its signal), the slow products, then the native unit
        update."""
        p = self.p
        core = self.core
        b = self.b_vec[:, None]
        K = len(self.slow_classes)
        args = _abi.OpticUnitArgs(m=self.n_rate, batch=self.B, classes=K,
                                  mode=_abi.SLOW_MODE_CODES[self.slow.mode] if K else 0, adapt_gain=p.adapt_gain,
                                  a_ad=self._a_ad, norm=self._slow_norm if K else 1.0,
                                  clip_lo=self.slow.clip[0] if K else 0.0, clip_hi=self.slow.clip[1] if K else 0.0,
                                  v=core.v_s.data_ptr(), adapt=core.adapt_s.data_ptr(),
                                  g_slow=self._g_slow_s.data_ptr() if K else None, rec=self._rec.data_ptr(),
                                  pr=core.pr_in.data_ptr(), spk=core.spk_in.data_ptr(), dr=self._dr_ext.data_ptr(),
                                  a=self.core.a.data_ptr())
        for c in range(K):
            args.scale[c], args.decay[c] = self._slow_scale[c], self._a_slow[c]
            args.g_cls[c] = self._g_cls_s[c].data_ptr()
            args.held[c] = self._held_s[c].data_ptr() if self._slow_rs[c] is not None else None
            args.rec_slow[c] = self._rec_slow[c].data_ptr() if self._rec_slow[c] is not None else None
        stream = torch.cuda.current_stream(self.device).cuda_stream
        for _ in range(steps):
            r = core.v_s + b
            if K and self.slow.mode == "threshold":
                r = r + self._g_slow_s.clamp(max=0.9 * self._slow_norm)
            torch.sub(r.clamp(0.0, 1.0), b, out=self._dr_ext)
            if self.hooks is None:
                spmm(self._W_rr_plain, self._dr_ext, self._rec, alpha=p.gain_rr)
            else:
                xs = self._stream_signals(self._dr_ext, True)
                spmm(self._h_rest_rr, self._dr_ext, self._h_tmp)
                for W, x in zip(self._h_rr, xs):        # acc + (W x), the reference's rounding
                    if W is not None:
                        spmm(W, x, self._h_tmp, accumulate=True)
                torch.mul(self._h_tmp, p.gain_rr, out=self._rec)
            for W, y in zip(self._slow_rr, self._rec_slow):
                if W is not None:
                    spmm(W, self._dr_ext, y, alpha=p.gain_rr)
            rc = _abi.lib().flyb_optic_unit_step(ct.byref(args), stream)
            if rc:
                raise RuntimeError(f"flyb_optic_unit_step: error {rc}")

    # ------------------------------------------------------------------ rate dynamics
    def rates(self) -> torch.Tensor:
        if self.slow is not None and self.slow.mode == "threshold":
            return (self.v + self.b_vec[None] + self.g_slow.clamp(max=0.9 * self._slow_norm)).clamp(0.0, 1.0)
        return (self.v + self.b_vec[None]).clamp(0.0, 1.0)

    def relax(self, ms: float = 0.0) -> None:
        self.core.v_s.zero_()
        self.r0 = self.b_vec[None].clone()

    @staticmethod
    def _fly_minor(x: torch.Tensor) -> torch.Tensor:
        """[n][B] contiguous storage behind a (B, n) tensor (no copy for a Brain's state view)."""
        t = x.t()
        return t if t.is_contiguous() else t.contiguous()

    @torch.no_grad()
    def step_frame(self, col_radiance, spk_rate_hz, frame_ms: float, *, intensity=None,
                   out: torch.Tensor | None = None) -> torch.Tensor:
        """Advance one frame; returns the drive (B, N) in mV (optic.py:563-604).

        `out` ([N][B] float32 storage, e.g. a Brain's drive storage) receives the drive in place."""
        if self.r0 is None:
            self.relax()
        p = self.p
        a_pr = self.photoreceptor_activity(col_radiance, frame_ms, intensity=intensity)
        if spk_rate_hz.dim() == 1:
            spk_rate_hz = spk_rate_hz[None]
        rates_s = self._fly_minor(spk_rate_hz.to(self.device, torch.float32).expand(self.B, -1))
        total = self._pending_ms + frame_ms
        steps = int(np.floor((total + 1e-9) / p.dt_ms))
        self._pending_ms = max(0.0, total - steps * p.dt_ms)
        if steps:
            spmm(self.W_rp, self._fly_minor(a_pr), self.core.pr_in, alpha=p.gain_in)
            spmm(self.W_rs, rates_s, self.core.spk_in, x_index=self._spk_idx32, x_div=100.0, x_lo=0.0, x_hi=3.0,
                 alpha=p.gain_fb)
            if self.slow is None and self.hooks is None:
                self.core.substeps(steps)
            else:                       # the spiking part of the slow input, held for the frame too
                for W, h in zip(self._slow_rs, self._held_s):
                    if W is not None:
                        spmm(W, rates_s, h, x_index=self._spk_idx32, x_div=100.0, x_lo=0.0, x_hi=3.0, alpha=p.gain_fb)
                self._ext_substeps(steps)
        torch.sub(self.rates(), self.r0, out=self.delta_rate)
        drive = out if out is not None else self._drive
        drive.zero_()
        if self.hooks is None:
            spmm(self.W_sr, self._delta, drive, y_index=self._spk_idx32, alpha=p.gain_out_mv, y_lo=-p.drive_clip_mv,
                 y_hi=p.drive_clip_mv)
        else:                           # the drive through the hook blocks (optic.py:602)
            acc = self._hook_output(self._delta)
            drive[self.spk_idx_t] = (p.gain_out_mv * acc).clamp(-p.drive_clip_mv, p.drive_clip_mv)
        self.last["dr"] = self.delta_rate
        return drive.t() if out is not None else drive.t().clone()

    def reset(self, rows=None) -> None:
        if rows is None:
            self._fresh_u8.fill_(1)
            self.core.v_s.zero_()
            self.core.adapt_s.zero_()
            self._g_slow_s.zero_()
            self._g_cls_s.zero_()
            self._held_s.zero_()
            self._stream_A_s.zero_()
            self._pending_ms = 0.0
        else:
            sel = torch.as_tensor(np.asarray(rows), device=self.device, dtype=torch.long)
            self._fresh_u8[sel] = 1
            self.core.v_s[:, sel] = 0.0
            self.core.adapt_s[:, sel] = 0.0
            self._g_slow_s[:, sel] = 0.0
            self._g_cls_s[:, :, sel] = 0.0
            self._held_s[:, :, sel] = 0.0
            self._stream_A_s[:, :, sel] = 0.0

