"""The whole-fly brain step: spiking LIF population and graded optic lobe, coupled every step.

One step of dt advances every neuron once, in the order of the reference's frame
(flyverse/fly.py:477-498 -> optic.py:563-604 -> brain.py:819-870) with the optic <-> LIF coupling
refreshed every step instead of every 10 ms frame:

  1. spk_in = gain_fb * W_rs clamp(rate / 100, 0, 3)     (flyb_spmm, gathers the LIF rate storage)
  2. one optic substep: W_rr SpMV/SpMM + rate update      (flyb_optic_run)
  3. drive[vpn] = clip(gain_out * W_sr dr, +-35 mV)       (flyb_spmm into the LIF drive storage)
  4. one fused LIF step over the spiking population       (flyb_lif_run)
and, every `frame_steps` steps, the photoreceptor stage and pr_in = gain_in * W_rp a_pr. All
buffers are allocated at construction, so `capture(k)` records k steps into one CUDA graph.

Only the LIF neurons that receive the VPN drive (rows of W_sr) need stage 3 before their update;
the others depend on the previous step alone. The spiking population is therefore stored in an
order (`lif_order`) whose tail, from a multiple of 32 on, holds the driven neurons, and with
`overlap` the LIF update of the head runs on a second stream concurrently with stages 2-3; the
tail follows stage 3, and the device clock advances once both are done. Every neuron sees the same
inputs as in the serial order and the ring sums are exact, so the result is bit-identical.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _abi
from .brain import Brain, LIFParams, upload
from .optic import DeviceCSR, OpticCore, PhotoreceptorStage, spmm
from .synthetic import WholeFlyConfig


class WholeFly:
    def __init__(self, cfg: WholeFlyConfig, batch: int, *, device="cuda", seed: int = 0, dt_ms: float = 0.1,
                 launch: str = "step", poisson_hz=None, record_activity: bool = True, overlap: bool = True):
        self.cfg, self.B = cfg, int(batch)
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        o = cfg.optic
        self.dt_ms = dt_ms
        params = dict(cfg.lif.params)
        params["dt"] = dt_ms
        # spiking population order: undriven neurons, then (from a multiple of 32) the driven ones
        n = cfg.n_spiking
        driven = np.unique(o.W_sr.tocoo().row)
        head = np.setdiff1d(np.arange(n), driven)
        self.lif_order = np.concatenate([head, driven]).astype(np.int64)
        self.split = len(head) - len(head) % 32           # neurons [split, n) update after the drive
        self.lif_position = np.empty(n, np.int64)         # original spiking index -> stored position
        self.lif_position[self.lif_order] = np.arange(n)
        self.lif_connectome = cfg.lif.c.subset(self.lif_order)
        self.sensory_idx = self.lif_position[np.asarray(cfg.sensory_idx)]
        self.lif = Brain(self.lif_connectome, LIFParams(**params), device=self.device, seed=seed, batch=self.B,
                         launch=launch)
        self.lif.record_activity = record_activity
        hz = cfg.lif.poisson_hz if poisson_hz is None else poisson_hz
        self.lif.set_poisson(self.sensory_idx, torch.as_tensor(hz, dtype=torch.float32))
        self.overlap = bool(overlap)
        tau = o.tau_of_type[o.type_of].astype(np.float32)
        a = np.exp(-dt_ms / tau).astype(np.float32)
        aad = float(np.exp(-dt_ms / o.adapt_tau_ms))
        self.optic = OpticCore(o.W_rr(), a, o.b, batch=self.B, device=self.device, gain_rr=o.gain_rr,
                               adapt_gain=o.adapt_gain, aad=aad, launch="step")
        dev = self.device
        # the coupling blocks keep only their non-empty rows (+ the row map): the other rows of spk_in
        # and of the drive are never written and stay zero
        self.W_rs_host = o.W_rs.tocsc()[:, self.lif_order].tocsr()    # columns in stored LIF order
        self.W_sr_host = o.W_sr.tocsr()[self.lif_order]                # rows in stored LIF order
        self.W_rs, self.rs_rows = self._rows_with_entries(self.W_rs_host, dev)
        self.W_sr, self.sr_rows = self._rows_with_entries(self.W_sr_host, dev)
        # pr_in has input on the lamina rows alone: the product writes those and the rest stay zero
        self.W_rp, self.rp_rows = self._rows_with_entries(o.W_rp, dev)
        self.photo = PhotoreceptorStage(o.pr_column, o.pr_family, o.sens, o.n_col, self.B, dev)
        self.a_pr = self.photo.a_pr                       # [n_pr][B]: the stage's output
        self.steps_taken = 0
        self._fork = (torch.cuda.Stream(self.device, priority=-1), torch.cuda.Stream(self.device))
        self._pull_stream = torch.cuda.Stream(self.device)

    def launches(self, steps: int) -> int:
        """Kernels launched by `steps` steps in one call once running: per step two coupling
        products, the optic substep (its dr carried over), the LIF update (two ranges when
        overlapped; each followed by its scatter under deferred delivery) and the device-clock
        advance (or one persistent launch); under pull delivery one pull per group of
        `pull_group` steps (one per step without the overlap) and one for a group the call ends
        inside."""
        n = 6 if self.overlapping else (5 if self.lif.launch == "step" else 4)
        if self.lif._defer_active():
            n += 2 if self.overlapping else 1          # the scatter kernel of each LIF launch
        total = n * steps
        if self.lif._pull_active():
            L = self.lif.pull_group if self.overlapping else 1
            total += -(-steps // L)
        return total

    @property
    def overlapping(self) -> bool:
        """Whether steps fork the undriven LIF update onto a second stream. The LIF must use
        per-step launches (a persistent cooperative launch owns the device); the optic substep may
        be persistent, since one substep on a carried dr is an ordinary launch (with
        `optic.grid` blocks, leaving SMs room for the LIF blocks)."""
        return self.overlap and self.lif.launch == "step" and 0 < self.split

    @staticmethod
    def _rows_with_entries(M, dev):
        M = M.tocsr()
        rows = np.flatnonzero(np.diff(M.indptr)).astype(np.int32)
        return DeviceCSR(M[rows], dev), torch.from_numpy(rows).to(dev)

    @property
    def n_neurons(self) -> int:
        return self.cfg.n_rate + self.cfg.n_spiking

    def set_poisson_rates(self, hz) -> None:
        """Poisson drive of the sensory cells: a rate for all, or per fly (B,) or (B, cells)."""
        r = torch.as_tensor(hz, dtype=torch.float32)
        if r.ndim == 1:
            r = r[:, None].expand(self.B, len(self.sensory_idx))
        self.lif.set_poisson(self.sensory_idx, r)

    def reset(self, rows, poisson_hz=None) -> None:
        """Start new episodes in fly rows `rows`: their LIF state, pending input and spike history
        back to rest (Brain.reset), their optic state to the operating point (v = adapt = 0, and
        the carried dr to match), then their Poisson drive set to `poisson_hz` (per row, or one
        rate). The other flies and the held photoreceptor input are untouched. Between calls
        only (nothing is pending then)."""
        rows = np.asarray(rows, dtype=np.int64)
        if not rows.size:
            return
        sel = upload(rows, self.device)
        self.lif.reset(rows)
        o = self.optic
        o.v_s[:, sel] = 0.0
        o.adapt_s[:, sel] = 0.0
        o.dr_out[:, sel] = o.b.clamp(0.0, 1.0)[:, None] - o.b[:, None]     # clip(0 + b, 0, 1) - b
        o._dr_key = o._state_key()
        if poisson_hz is not None:
            hz = np.broadcast_to(np.asarray(poisson_hz, np.float32).reshape(-1, 1), (len(rows), 1))
            if getattr(self, "_sensory_dev", None) is None:
                self._sensory_dev = torch.as_tensor(self.sensory_idx, device=self.device)
            cols = self._sensory_dev
            p = upload(np.ascontiguousarray(hz * np.float32(self.lif.p.dt / 1000.0)), self.device)
            self.lif.poisson_p[sel[:, None], cols[None, :]] = p.expand(len(rows), len(self.sensory_idx))
            self.lif._poisson_on = True

    def set_photoreceptors(self, a_pr: torch.Tensor) -> None:
        """Photoreceptor activity [n_pr][B] (contiguous, on the device) -> held pr_in =
        gain_in * W_rp a_pr (a frame's input), read from `a_pr` where it lies."""
        spmm(self.W_rp, a_pr, self.optic.pr_in, alpha=self.cfg.optic.gain_in, y_index=self.rp_rows)

    def set_radiance(self, rad: torch.Tensor, frame_ms: float, a_pr: torch.Tensor | None = None) -> None:
        """A radiance frame (B, n_col, 4) on the device -> the photoreceptor stage (optic.py:496-517,
        its low-pass and adaptation advanced by frame_ms) -> held pr_in (optic.py:575). With `a_pr`
        the stage's output lands there (for instance a per-frame buffer on an input stream) and only
        the stage runs; `set_photoreceptors(a_pr)` installs it later."""
        if a_pr is not None:
            self.photo(rad, frame_ms, out=a_pr)
            return
        self.set_photoreceptors(self.photo(rad, frame_ms))

    def step(self, n: int = 1, before=None, after=None) -> None:
        """Advance every fly n steps. Each optic substep reuses the dr the previous one wrote. Under
        CUDA-graph capture the recorded steps end with that dr in the buffer they started from, so
        the graph replays back to back; a graph replay assumes nothing else wrote the optic state
        since the capture (a write is seen at capture time only). `before(k)` / `after(k)` run on
        the current stream around step k (new inputs, a readout), inside the same call, so n steps
        with per-step inputs and outputs stay one call."""
        o = self.cfg.optic
        lif_rate = self.lif._st["rate"]
        drive = self.lif._st["drive"]
        cur0 = self.optic._cur
        overlap = self.overlapping
        main = torch.cuda.current_stream(self.device)
        hi, side = self._fork
        # under pull delivery each group of L steps (Brain.pull_group) is pulled on its own stream
        # beside the next group's steps; the main stream joins it before the next group's pull
        # (and so before the updates of the group after, whose spike words reuse its half of the
        # pull buffer), and the call ends with the pull of a group it stops inside
        lag = overlap and self.lif._pull_active() and self.lif.n_delay >= 2
        L = self.lif.pull_group if lag else 1
        pulling = False
        for k in range(int(n)):
            if before is not None:
                before(k)
            spmm(self.W_rs, lif_rate, self.optic.spk_in, x_div=100.0, x_lo=0.0, x_hi=3.0, alpha=o.gain_fb,
                 y_index=self.rs_rows)
            if overlap:
                # the optic chain on a high-priority stream, the undriven LIF neurons beside it
                hi.wait_stream(main)
                side.wait_stream(main)
                with torch.cuda.stream(side):
                    self.lif.step_range(0, self.split)
                with torch.cuda.stream(hi):
                    self._optic_and_drive(drive)
                    self.lif.step_range(self.split, self.cfg.n_spiking - self.split)
                main.wait_stream(hi)
                main.wait_stream(side)
                if lag:
                    self.lif.advance(1, pull=False)
                    if self.lif.step_count % L == 0:          # a group is complete
                        self._pull_beside(main, pulling)
                        pulling = True
                else:
                    self.lif.advance(1)
            else:
                self._optic_and_drive(drive)
                self.lif.step(1)
            if after is not None:
                after(k)
        if lag and self.lif._pull_pending:
            self._pull_beside(main, pulling)
            pulling = True
        if pulling:
            main.wait_stream(self._pull_stream)
        if torch.cuda.is_current_stream_capturing():
            self.optic.pin_dr(cur0)
        self.steps_taken += int(n)

    def _pull_beside(self, main, pulling: bool) -> None:
        """Deliver the pending steps on the pull stream, after the previous pull and after the
        main stream's work so far."""
        if pulling:
            main.wait_stream(self._pull_stream)
        self._pull_stream.wait_stream(main)
        with torch.cuda.stream(self._pull_stream):
            self.lif.deliver()

    def _optic_and_drive(self, drive: torch.Tensor) -> None:
        o = self.cfg.optic
        self.optic.substeps(1, carry=True)
        spmm(self.W_sr, self.optic.dr_out, drive, y_index=self.sr_rows, alpha=o.gain_out_mv, y_lo=-o.drive_clip_mv,
             y_hi=o.drive_clip_mv)

    # ------------------------------------------------------------------ algorithmic bytes (roofline)
    def lif_bytes_per_step(self, group: int | None = None) -> int:
        """Bytes the LIF step must move per step for B flies: per neuron-fly v, g, refrac, rate read +
        written, adapt read (and written when adaptation is on), spike counts read + written when
        activity is recorded, drive / poisson_p (when the Poisson drive is on) / ring read, spikes
        written; per neuron active.
        Under pull delivery also its input tables once per delivery group of `group` steps
        (per input slot its packed entry, per chunk of 32 slots its base and, for wide count ranges,
        its 16 bit planes), the spike words written to and read back from the pull buffer, and the
        write slot read + written."""
        b = self.lif
        words = 4 * 2 + 1 + 1 + 1 + 1                       # v g refrac rate r+w, adapt / drive / ring r, spikes w
        words += (1 if b._adapt_on else 0) + (2 if b.record_activity else 0) + (1 if b._poisson_on else 0)
        total = self.cfg.n_spiking * (self.B * 4 * words + 4)
        if self.lif._pull_active() and getattr(self.lif, "_pull_t", None) is not None:
            # the input tables once per group of L steps, the write slot read + written every step
            ptr, pre, planes, meta = self.lif._pull_t
            L = self.lif.pull_group if group is None else group
            total += (pre.numel() * 4 + (0 if planes is None else planes.numel() * 4) + meta.numel() * 4) // L
            total += self.cfg.n_spiking * self.B * 4 * 2 + self.cfg.n_spiking * self.B // 8 * 2
        return total

    def optic_bytes_per_step(self) -> int:
        """CSR once (idx + w) + row pointers, per unit-fly v, adapt r+w, pr, spk, dr in / out."""
        o = self.cfg.optic
        nnz = int(o.W0.nnz)
        return nnz * 8 + (o.m + 1) * 4 + o.m * self.B * 4 * 8 + o.m * 8
