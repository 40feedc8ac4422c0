"""ctypes mirror of include/flyb200.h and the loader of the in-tree CUDA library.

The library is a plain C ABI (`extern "C"`, raw device pointers, the caller's stream), bound the
same way the reference binds its kernels (flyverse/cuda.py:37-91): a ctypes CDLL whose functions
take pointers and return an int status. There is no fallback: if the library is missing or no
CUDA device is visible, every native call raises.
"""
from __future__ import annotations

import ctypes as ct
import os
import threading
from pathlib import Path

LIB_NAME = "libflyb200.so"
_HERE = Path(__file__).resolve().parent
_LOCK = threading.Lock()
_LIB = None

# ------------------------------------------------------------------ constants (flyb200.h)
OK, EINVAL, EBARRIER, ECOOP, ETOOBIG = 0, 1001, 1002, 1003, 1004
LIF_POISSON, LIF_STD, LIF_COUNTS, LIF_ADAPT = 1, 2, 4, 8
LIF_EXT_UNIFORM, LIF_SKIP_FROZEN, LIF_EPISODES, LIF_NO_ADVANCE, LIF_DEFER_DELIVERY = 16, 32, 64, 128, 256
LIF_PULL_DELIVERY = 512
RING_COUNT, RING_FIXED = 0, 1
LAUNCH_STEP, LAUNCH_PERSISTENT = 0, 1
LAUNCHES_BY_NAME = {"step": LAUNCH_STEP, "persistent": LAUNCH_PERSISTENT}
(P_V_REST, P_V_RESET, P_V_TH, P_A_M, P_A_S, P_DT, P_T_REF, P_ADAPT_JUMP, P_A_AD, P_A_STD, P_A_R,
 P_RATE_GAIN, P_W_SYN, LIF_NPARAM) = range(14)
LIF_SYNC_WORDS = 64
OPTIC_HISTORY, OPTIC_DR_VALID = 1, 2
SLOW_MAX_CLASSES = 2
SLOW_MODE_CODES = {"additive": 0, "gain": 1, "threshold": 2}
(CLOCK_A_M, CLOCK_A_S, CLOCK_DT, CLOCK_A_AD, CLOCK_A_STD, CLOCK_A_R, CLOCK_RATE_GAIN, CLOCK_U, CLOCK_POIS,
 CLOCK_A_SLOW0, CLOCK_A_SLOW1, CLOCK_NCOEF) = range(12)

_VP = ct.c_void_p
_I = ct.c_int


class LifArgs(ct.Structure):
    _fields_ = [("n", _I), ("batch", _I), ("n_delay", _I), ("ring_slots", _I), ("ring_mode", _I),
                ("ring_pos", _I), ("flags", _I), ("nsteps", _I), ("launch", _I), ("block", _I),
                ("grid", _I), ("raster_slots", _I), ("raster_pos", _I), ("fly0", _I),
                ("items_per_thread", _I), ("staged", _I), ("n_first", _I), ("n_count", _I),
                ("step0", ct.c_longlong), ("seed", ct.c_ulonglong),
                ("out_ptr", _VP), ("out_edge", _VP),
                ("v", _VP), ("g", _VP), ("refrac", _VP), ("adapt", _VP), ("res", _VP),
                ("rate", _VP), ("counts", _VP), ("spikes", _VP), ("drive", _VP), ("poisson_p", _VP),
                ("active", _VP), ("std_u", _VP), ("params", _VP), ("ring", _VP), ("uniforms", _VP),
                ("fly_steps", _VP), ("clock", _VP), ("raster", _VP), ("events", _VP), ("status", _VP),
                ("sync", _VP), ("spike_list", _VP), ("spike_n", _VP), ("spike_cap", ct.c_longlong),
                ("adapt_jump", _VP), ("clock_k", _VP), ("clock_coef", _VP), ("clock_acc", _VP),
                ("slow_clock_acc", _VP * 2),
                ("slow_classes", _I), ("slow_mode", _I), ("slow_norm", ct.c_float), ("slow_clip_lo", ct.c_float),
                ("slow_clip_hi", ct.c_float), ("slow_th_max", ct.c_float), ("slow_decay", ct.c_float * 2),
                ("slow_out_ptr", _VP * 2), ("slow_out_edge", _VP * 2), ("slow_ring", _VP * 2), ("slow_g", _VP * 2),
                ("g_slow", _VP), ("pull_ptr", _VP), ("pull_pre", _VP), ("pull_planes", _VP), ("pull_nplanes", _I),
                ("pull_meta", _VP), ("pull_group", _I), ("pull_steps", _I), ("pull_phase", _I),
                ("pull_bits", _VP), ("pull_state", _VP), ("pull_grid", _I)]


class OpticArgs(ct.Structure):
    _fields_ = [("m", _I), ("batch", _I), ("nsteps", _I), ("launch", _I), ("block", _I), ("grid", _I),
                ("variant", _I), ("flags", _I),
                ("ptr", _VP), ("cw", _VP), ("rows", _VP), ("v", _VP), ("adapt", _VP), ("dr", _VP),
                ("dr_tmp", _VP), ("pr", _VP), ("spk", _VP), ("a", _VP), ("b", _VP),
                ("gr", ct.c_float), ("ga", ct.c_float), ("aad", ct.c_float), ("n_long", _I),
                ("v_hist", _VP), ("inp_hist", _VP), ("status", _VP), ("sync", _VP)]


class SpmmArgs(ct.Structure):
    _fields_ = [("rows", _I), ("cols", _I), ("batch", _I), ("accumulate", _I),
                ("ptr", _VP), ("col", _VP), ("w", _VP),
                ("x", _VP), ("x_index", _VP), ("x_rows", _I),
                ("x_div", ct.c_float), ("x_lo", ct.c_float), ("x_hi", ct.c_float),
                ("y", _VP), ("y_index", _VP), ("y_rows", _I),
                ("alpha", ct.c_float), ("y_lo", ct.c_float), ("y_hi", ct.c_float),
                ("warps_per_row", _I)]


class AdjointArgs(ct.Structure):
    _fields_ = [("m", _I), ("batch", _I), ("nsteps", _I), ("launch", _I), ("block", _I), ("grid", _I),
                ("pad0", _I), ("pad1", _I),
                ("t_ptr", _VP), ("t_col", _VP), ("t_w", _VP), ("t_perm", _VP),
                ("v_hist", _VP), ("inp_hist", _VP), ("a", _VP), ("b", _VP),
                ("gr", ct.c_float), ("ga", ct.c_float), ("aad", ct.c_float), ("pad2", _I),
                ("lam_v", _VP), ("lam_a", _VP), ("lam_tmp", _VP), ("mu", _VP),
                ("g_edge", _VP), ("g_a", _VP), ("status", _VP), ("sync", _VP)]


class PhotoArgs(ct.Structure):
    _fields_ = [("n_pr", _I), ("n_col", _I), ("batch", _I), ("pad0", _I),
                ("rad", _VP), ("pr_column", _VP), ("sens", _VP),
                ("avg_ptr", _VP), ("avg_idx", _VP), ("avg_w", _VP), ("pr_cell", _VP), ("has", _VP),
                ("I_lp", _VP), ("I_mean", _VP), ("contrast", _VP), ("fresh", _VP),
                ("a_lp", ct.c_float), ("c_lp", ct.c_float), ("a_ad", ct.c_float), ("c_ad", ct.c_float),
                ("eps", ct.c_float), ("clip_hi", ct.c_float),
                ("a_pr", _VP)]


class TraceArgs(ct.Structure):
    _fields_ = [("batch", _I), ("rays", _I), ("n_sph", _I), ("n_box", _I), ("n_pln", _I), ("shared_origin", _I),
                ("samples", _I), ("detail", ct.c_float),
                ("scene", _VP), ("origins", _VP), ("dirs", _VP), ("eye_dirs", _VP), ("pose", _VP), ("weights", _VP),
                ("out", _VP)]


class OpticUnitArgs(ct.Structure):
    _fields_ = [("m", _I), ("batch", _I), ("classes", _I), ("mode", _I), ("adapt_gain", ct.c_float),
                ("a_ad", ct.c_float), ("norm", ct.c_float), ("clip_lo", ct.c_float), ("clip_hi", ct.c_float),
                ("scale", ct.c_float * 2), ("decay", ct.c_float * 2), ("v", _VP), ("adapt", _VP), ("g_slow", _VP),
                ("g_cls", _VP * 2), ("held", _VP * 2), ("rec_slow", _VP * 2), ("rec", _VP), ("pr", _VP), ("spk", _VP),
                ("dr", _VP), ("a", _VP)]


STRUCTS = (LifArgs, OpticArgs, SpmmArgs, AdjointArgs, PhotoArgs, TraceArgs, OpticUnitArgs)

# Every symbol include/flyb200.h declares, with its ctypes signature.
_P = ct.POINTER(ct.c_void_p)
SIGNATURES = {
    "launch_lif": [_P, _I, _I, _I, _VP],
    "launch_optic_dr": [_P, _I, _I, _VP],
    "launch_optic": [_P, _I, _I, ct.c_float, ct.c_float, ct.c_float, _VP],
    "launch_csr": [_P, _I, _I, _I, _I, _VP],
    "launch_events": [_P, _I, _I, _I, _I, _VP],
    "launch_means": [_P, _I, _I, _I, _I, _VP],
    "flyb_lif_run": [ct.POINTER(LifArgs), _VP],
    "flyb_lif_advance": [ct.POINTER(LifArgs), _VP],
    "flyb_lif_pull": [ct.POINTER(LifArgs), _VP],
    "flyb_lif_spike_capacity": [ct.POINTER(LifArgs)],
    "flyb_ring_deposit": [_I, _I, _I, _VP, _VP, _VP, _VP, _VP],
    "flyb_optic_run": [ct.POINTER(OpticArgs), _VP],
    "flyb_optic_run_noalloc": [ct.POINTER(OpticArgs), _VP],
    "flyb_spmm": [ct.POINTER(SpmmArgs), _VP],
    "flyb_optic_adjoint": [ct.POINTER(AdjointArgs), _VP],
    "flyb_segment_sum": [_VP, _VP, _VP, _VP, ct.c_float, _VP, _I, _VP],
    "flyb_photoreceptor": [ct.POINTER(PhotoArgs), _VP],
    "flyb_group_means": [_VP, _VP, _VP, _VP, _I, _I, _VP],
    "flyb_trace_scene_floats": [_I, _I, _I],
    "flyb_trace": [ct.POINTER(TraceArgs), _VP],
    "flyb_optic_unit_step": [ct.POINTER(OpticUnitArgs), _VP],
    "flyb_occupancy": [_I, _I, ct.POINTER(_I), ct.POINTER(_I)],
    "flyb_selftest_wait": [_VP, _VP, ct.c_longlong, _VP],
    "flyb_gather_probe": [_VP, _I, _VP, _I, _VP, _I, _VP],
    "flyb_version": [],
    "flyb_abi_sizes": [ct.POINTER(_I), _I],
}
RESTYPES = {"flyb_version": ct.c_char_p, "flyb_lif_spike_capacity": ct.c_longlong}


def library_path() -> Path:
    return Path(os.environ.get("FLYB200_LIB", _HERE / LIB_NAME))


def bind(lib: ct.CDLL) -> ct.CDLL:
    for name, argtypes in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = RESTYPES.get(name, _I)
    return lib


def lib() -> ct.CDLL:
    """The loaded native library; raises if it was not built (no fallback exists)."""
    global _LIB
    with _LOCK:
        if _LIB is None:
            path = library_path()
            if not path.exists():
                raise RuntimeError(f"flyb200 native library not found at {path}; run "
                                   "`python -m flyb200.build` (or __graft_entry__.build()) first")
            _LIB = bind(ct.CDLL(str(path)))
            check_abi(_LIB)
        return _LIB


def check_abi(library: ct.CDLL) -> None:
    sizes = (ct.c_int * len(STRUCTS))()
    n = library.flyb_abi_sizes(sizes, len(STRUCTS))
    for k, S in enumerate(STRUCTS[:n]):
        if sizes[k] != ct.sizeof(S):
            raise RuntimeError(f"ABI mismatch: {S.__name__} is {ct.sizeof(S)} bytes here, {sizes[k]} in the library")


def ptr(t) -> int | None:
    """Device (or host) address of a tensor / array, None for None."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data
