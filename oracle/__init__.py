"""flyb200 ORACLE -- test infrastructure, not product code.

Only tests/, __graft_entry__.smoke() and bench.py (its cpu_baseline leg and `--impl reference`
arm) import this package, always as the checker or as the timed CPU port, never as the thing
measured or shipped. It wraps:

  tracer.c      plain-C restatement of the eye's ray tracer (scenes, shadows, patterns, value
                noise, pose turn and column sums);
  flyoracle.c   plain-C restatement of the LIF step over an exact delay ring, Philox4x32-10, the
                optic substep (FP32 reference order, FP64) and the held-input products;
  optic64.py    FP64 numpy restatement of the optic dynamics parameterised by per-type-pair gains
                and per-type time constants, with central finite differences (the adjoint's pin).

Parity pins: the LIF restatement is checked against rasters and state that the reference's own
`flyverse.brain.Brain` produced on CPU (tests/golden/, made by tests/golden/make_golden.py); the
optic restatement against the reference's `OpticLobe` frames (same script). The adjoint has no
counterpart in the reference; its pin is FP64 central differences of optic64.py.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
BUILD = HERE / "_build"
LIB = BUILD / "libflyoracle.so"
_lib = None

sys.path.insert(0, str(ROOT / "flyverse-core_b200"))
from flyb200 import _abi  # noqa: E402  (struct layouts of include/flyb200.h only; no CUDA)


def build(force: bool = False) -> Path:
    """Compile flyoracle.c with gcc (no contraction of multiply-adds, OpenMP over flies)."""
    srcs = [HERE / "flyoracle.c", HERE / "tracer.c"]
    if LIB.exists() and not force and LIB.stat().st_mtime >= max([s.stat().st_mtime for s in srcs] +
                                                                 [(ROOT / "include" / "flyb200.h").stat().st_mtime]):
        return LIB
    BUILD.mkdir(exist_ok=True)
    tmp = BUILD / f"libflyoracle.{os.getpid()}.so"
    cmd = ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
           *map(str, srcs), "-o", str(tmp), "-lm"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    tmp.replace(LIB)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = ct.CDLL(str(LIB))
        L.oracle_lif_run.argtypes = [ct.POINTER(_abi.LifArgs), ct.c_int]
        L.oracle_optic_run.argtypes = [ct.POINTER(_abi.OpticArgs), ct.c_int]
        L.oracle_spmm.argtypes = [ct.POINTER(_abi.SpmmArgs)]
        L.oracle_uniform.argtypes = [ct.c_uint64, ct.c_uint64, ct.c_uint32, ct.c_uint32]
        L.oracle_uniform.restype = ct.c_float
        L.oracle_philox.argtypes = [ct.c_uint64] + [ct.c_uint32] * 4 + [ct.POINTER(ct.c_uint32)]
        L.oracle_optic_run_f64.argtypes = [ct.c_int] * 3 + [ct.c_void_p] * 9 + [ct.c_double] * 3
        L.oracle_trace.argtypes = [ct.POINTER(_abi.TraceArgs), ct.c_int]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def uniform(seed: int, step: int, neuron: int, fly: int) -> float:
    return float(lib().oracle_uniform(seed, step, neuron, fly))


def philox(seed: int, counter) -> np.ndarray:
    out = (ct.c_uint32 * 4)()
    lib().oracle_philox(seed, *[int(c) & 0xFFFFFFFF for c in counter], out)
    return np.array(out, dtype=np.uint32)


class LifState:
    """Host copy of one LIF run: every array fly-minor [n][batch], ring [R][n][batch]."""

    NAMES = ("v", "g", "refrac", "adapt", "res", "rate", "counts", "spikes", "drive", "poisson_p")

    def __init__(self, n, batch, ring_slots, ring_mode, v_rest):
        self.n, self.batch, self.ring_slots, self.ring_mode = n, batch, ring_slots, ring_mode
        for name in self.NAMES:
            setattr(self, name, np.zeros((n, batch), np.float32))
        self.v[:] = v_rest
        self.res[:] = 1.0
        self.active = np.ones(n, np.float32)
        self.std_u = np.zeros(n, np.float32)
        self.ring = np.zeros((ring_slots, n, batch), np.int32 if ring_mode == _abi.RING_COUNT else np.int64)
        self.ring_pos = 0
        self.step = 0

    def copy(self):
        c = LifState.__new__(LifState)
        c.__dict__ = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self.__dict__.items()}
        return c


def lif_run(state: LifState, out_ptr, out_edge, params, *, n_delay, flags, nsteps, seed=0,
            uniforms=None, fly_steps=None, raster=False, threads=0, fly0=0, adapt_jump=None, clocks=None,
            slow=None):
    """Advance `state` in place by `nsteps`; returns (raster bits [nsteps][words] or None, events).
    With `fly_steps` (EPISODES), fly b is live for its first fly_steps[b] steps; the array is then
    reduced by the steps taken, as the host layer does after a launch. `adapt_jump` (n,): per-neuron
    adaptation jumps (the reference's adapt_by_type, brain.py:497-506). `clocks` = (period (n,),
    coefficient table [max period + 1][CLOCK_NCOEF]): per-neuron clocks (brain.py:899-957); the
    pending input of slow neurons lives in `state.clock_acc` (and, with the slow tone, per class in
    `state.slow_clock_acc`). `slow` = {"mode", "norm", "clip",
    "th_max", "classes": [(out_ptr, out_edge, decay), ...]}: the slow receptor tone (brain.py:551-585);
    its rings, per-class tones and summed tone live in `state.slow_ring`, `state.slow_g`,
    `state.g_slow`."""
    n, B = state.n, state.batch
    words = (n * B + 31) // 32
    r = np.zeros((nsteps, words), np.uint32) if raster else None
    events = np.zeros(1, np.uint64)
    out_ptr = np.ascontiguousarray(out_ptr, np.int32)
    out_edge = np.ascontiguousarray(out_edge, np.int32)
    P = _f32(params)
    uni = None if uniforms is None else _f32(uniforms)
    fs = None if fly_steps is None else np.ascontiguousarray(fly_steps, np.int32)
    aj = None if adapt_jump is None else _f32(adapt_jump)
    ck = cc = None
    if clocks is not None:
        ck = np.ascontiguousarray(clocks[0], np.uint8)
        cc = _f32(clocks[1])
        if getattr(state, "clock_acc", None) is None:
            state.clock_acc = np.zeros((n, B), np.int64)
    keep = []
    if slow is not None:
        K = len(slow["classes"])
        if getattr(state, "slow_ring", None) is None:
            state.slow_ring = np.zeros((K, state.ring_slots, n, B), np.int64)
            state.slow_g = np.zeros((K, n, B), np.float32)
            state.g_slow = np.zeros((n, B), np.float32)
    a = _abi.LifArgs(n=n, batch=B, n_delay=n_delay, ring_slots=state.ring_slots, ring_mode=state.ring_mode,
                     ring_pos=state.ring_pos, flags=flags, nsteps=nsteps, step0=state.step, seed=seed, fly0=fly0,
                     out_ptr=_p(out_ptr), out_edge=_p(out_edge), v=_p(state.v), g=_p(state.g),
                     refrac=_p(state.refrac), adapt=_p(state.adapt), res=_p(state.res), rate=_p(state.rate),
                     counts=_p(state.counts), spikes=_p(state.spikes), drive=_p(state.drive),
                     poisson_p=_p(state.poisson_p), active=_p(state.active), std_u=_p(state.std_u),
                     params=_p(P), ring=_p(state.ring), uniforms=_p(uni), fly_steps=_p(fs),
                     raster=_p(r), events=_p(events), adapt_jump=_p(aj), clock_k=_p(ck), clock_coef=_p(cc),
                     clock_acc=_p(getattr(state, "clock_acc", None)) if clocks is not None else None)
    if slow is not None:
        a.slow_classes, a.slow_mode = len(slow["classes"]), _abi.SLOW_MODE_CODES[slow["mode"]]
        a.slow_norm, a.slow_th_max = slow["norm"], slow["th_max"]
        a.slow_clip_lo, a.slow_clip_hi = slow["clip"]
        for c, (sp_, se_, decay) in enumerate(slow["classes"]):
            sp_, se_ = np.ascontiguousarray(sp_, np.int32), np.ascontiguousarray(se_, np.int32)
            keep += [sp_, se_]
            a.slow_out_ptr[c], a.slow_out_edge[c] = _p(sp_), _p(se_)
            a.slow_ring[c], a.slow_g[c] = state.slow_ring[c].ctypes.data, state.slow_g[c].ctypes.data
            a.slow_decay[c] = decay
        a.g_slow = _p(state.g_slow)
        if clocks is not None:           # the slow input pending at clocked neurons, per class
            if getattr(state, "slow_clock_acc", None) is None:
                state.slow_clock_acc = np.zeros((K, n, B), np.int64)
            for c in range(K):
                a.slow_clock_acc[c] = state.slow_clock_acc[c].ctypes.data
    rc = lib().oracle_lif_run(ct.byref(a), threads)
    if rc:
        raise ValueError(f"oracle_lif_run: status {rc}")
    state.ring_pos = (state.ring_pos + nsteps) % state.ring_slots
    state.step += nsteps
    if fly_steps is not None:
        fly_steps[...] = fs
    return r, int(events[0])


def optic_run(v, adapt, ptr, col, w, pr, spk, a, b, gr, ga, aad, nsteps, history=False, threads=0):
    """FP32 optic substeps on [m][batch] arrays, in place; optional (v_hist, inp_hist)."""
    m, B = v.shape
    ptr, col, w = np.ascontiguousarray(ptr, np.int32), np.ascontiguousarray(col, np.int32), _f32(w)
    pr, spk, a, b = _f32(pr), _f32(spk), _f32(a), _f32(b)
    vh = np.zeros((nsteps, m, B), np.float32) if history else None
    ih = np.zeros((nsteps, m, B), np.float32) if history else None
    cw = np.ascontiguousarray(np.stack([col, w.view(np.int32)], axis=1))
    args = _abi.OpticArgs(m=m, batch=B, nsteps=nsteps, ptr=_p(ptr), cw=_p(cw), v=_p(v),
                          adapt=_p(adapt), pr=_p(pr), spk=_p(spk), a=_p(a), b=_p(b), gr=gr, ga=ga, aad=aad,
                          v_hist=_p(vh), inp_hist=_p(ih))
    assert v.dtype == np.float32 and v.flags.c_contiguous and adapt.dtype == np.float32 and adapt.flags.c_contiguous
    rc = lib().oracle_optic_run(ct.byref(args), threads)
    if rc:
        raise ValueError(f"oracle_optic_run: status {rc}")
    return (vh, ih) if history else None


def optic_run_f64(v, adapt, ptr, col, w, pr, spk, a, b, gr, ga, aad, nsteps):
    m, B = v.shape
    d = lambda x: np.ascontiguousarray(x, np.float64)  # noqa: E731
    ptr, col = np.ascontiguousarray(ptr, np.int32), np.ascontiguousarray(col, np.int32)
    w, pr, spk, a, b = d(w), d(pr), d(spk), d(a), d(b)
    assert v.dtype == np.float64 and adapt.dtype == np.float64
    rc = lib().oracle_optic_run_f64(m, B, nsteps, _p(ptr), _p(col), _p(w), _p(v), _p(adapt), _p(pr), _p(spk),
                                    _p(a), _p(b), gr, ga, aad)
    if rc:
        raise ValueError(f"oracle_optic_run_f64: status {rc}")


def spmm(ptr, col, w, x, batch, *, rows, x_index=None, x_div=1.0, x_lo=-np.inf, x_hi=np.inf,
         y=None, y_index=None, alpha=1.0, y_lo=-np.inf, y_hi=np.inf, accumulate=False):
    ptr, col, w = np.ascontiguousarray(ptr, np.int32), np.ascontiguousarray(col, np.int32), _f32(w)
    x = _f32(x)
    xi = None if x_index is None else np.ascontiguousarray(x_index, np.int32)
    yi = None if y_index is None else np.ascontiguousarray(y_index, np.int32)
    if y is None:
        y = np.zeros((rows if y_index is None else int(yi.max()) + 1, batch), np.float32)
    args = _abi.SpmmArgs(rows=rows, cols=0, batch=batch, accumulate=int(accumulate), ptr=_p(ptr), col=_p(col),
                         w=_p(w), x=_p(x), x_index=_p(xi), x_rows=x.shape[0], x_div=x_div, x_lo=x_lo, x_hi=x_hi,
                         y=_p(y), y_index=_p(yi), y_rows=y.shape[0], alpha=alpha, y_lo=y_lo, y_hi=y_hi)
    lib().oracle_spmm(ct.byref(args))
    return y


def trace(scene, shape, detail, *, origins, dirs=None, eye_dirs=None, pose=None, weights=None,
          shared_origin=False, batch=1, threads=0):
    """The tracer restatement on host arrays, arguments as flyb_trace_args: returns
    (batch, rays / samples, 4) float32."""
    scene, origins = _f32(scene), _f32(origins)
    dirs = None if dirs is None else _f32(dirs)
    eye_dirs = None if eye_dirs is None else np.ascontiguousarray(eye_dirs, dtype=np.float64)
    pose = None if pose is None else np.ascontiguousarray(pose, dtype=np.float64)
    weights = None if weights is None else _f32(weights)
    rays = (len(eye_dirs.reshape(-1, 3)) if eye_dirs is not None else dirs.reshape(batch, -1, 3).shape[1])
    samples = 1 if weights is None else weights.size
    out = np.zeros((batch, rays // samples, 4), np.float32)
    a = _abi.TraceArgs(batch=batch, rays=rays, n_sph=shape[0], n_box=shape[1], n_pln=shape[2],
                       shared_origin=int(shared_origin), samples=samples, detail=float(detail), scene=_p(scene),
                       origins=_p(origins), dirs=_p(dirs), eye_dirs=_p(eye_dirs), pose=_p(pose),
                       weights=_p(weights), out=_p(out))
    if lib().oracle_trace(ct.byref(a), threads or os.cpu_count() or 1):
        raise ValueError("oracle_trace: invalid arguments")
    return out
