"""The C-ABI library builds, loads without a GPU, exports every symbol include/flyb200.h declares,
and agrees with the Python mirror of the argument structs. No compute calls."""
import re
from pathlib import Path

from flyb200 import _abi
from flyb200 import build as fbuild

HEADER = Path(__file__).resolve().parents[1] / "include" / "flyb200.h"


def declared_functions() -> set[str]:
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return set(re.findall(r"^\s*(?:const\s+)?(?:long\s+long|\w+)\s*\*?\s*(\w+)\s*\([^;{]*\)\s*;", text, flags=re.M))


def test_library_builds_and_exports_every_declared_symbol():
    fbuild.build()
    lib = _abi.lib()
    names = declared_functions()
    assert {"launch_lif", "launch_events", "flyb_lif_run", "flyb_optic_run", "flyb_optic_adjoint"} <= names
    assert names == set(_abi.SIGNATURES), "the Python binding and the header disagree"
    for name in names:
        assert getattr(lib, name) is not None


def test_struct_mirrors_match_the_library():
    _abi.check_abi(_abi.lib())
    assert b"sm_100a" in _abi.lib().flyb_version()


def test_library_is_built_for_sm100a_only():
    assert "arch=compute_100a,code=sm_100a" in " ".join(fbuild.ARCH)


def test_pull_delivery_arguments_are_validated_before_any_launch():
    """flyb_lif_pull / FLYB_LIF_PULL_DELIVERY reject what the pull cannot do (a batch that is not
    32, 64, 128 or 256 flies, the fixed-point ring, depression, persistent launches, missing tables,
    a lag without a history ring) with FLYB_EINVAL, before touching the device."""
    import ctypes as ct
    import numpy as np
    lib = _abi.lib()
    fake = 4096                # device pointers are never dereferenced: validation fails first
    params = np.zeros(64, np.float32)             # the one host array the validation reads

    def args(**kw):
        a = _abi.LifArgs(n=256, batch=64, n_delay=18, ring_slots=19, ring_mode=_abi.RING_COUNT, nsteps=1,
                         flags=_abi.LIF_PULL_DELIVERY, launch=_abi.LAUNCH_STEP, raster_slots=18)
        for f in ("out_ptr", "v", "g", "refrac", "adapt", "res", "rate", "counts", "spikes", "drive", "poisson_p",
                  "active", "ring", "raster", "pull_ptr", "pull_pre", "pull_planes", "pull_meta"):
            setattr(a, f, fake)
        a.params = params.ctypes.data
        a.pull_nplanes = 8
        for k, v in kw.items():
            setattr(a, k, v)
        return a

    einval = _abi.EINVAL
    bad = [dict(batch=48), dict(batch=512), dict(ring_mode=_abi.RING_FIXED),
           dict(flags=_abi.LIF_PULL_DELIVERY | _abi.LIF_STD, std_u=fake),
           dict(flags=_abi.LIF_PULL_DELIVERY | _abi.LIF_DEFER_DELIVERY), dict(launch=_abi.LAUNCH_PERSISTENT),
           dict(pull_ptr=None), dict(pull_meta=None), dict(pull_nplanes=12), dict(raster=fake + 4),
           dict(pull_lag=2), dict(pull_lag=1, raster_slots=0), dict(flags=0)]
    for kw in bad:
        assert lib.flyb_lif_pull(ct.byref(args(**kw)), None) == einval, kw
