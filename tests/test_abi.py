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


PULL_VALIDATION = r"""
import ctypes as ct, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from flyb200 import _abi
lib = _abi.lib()
fake = 4096                       # never dereferenced: validation rejects each case first
params = np.zeros(64, np.float32)  # the one host array the validation reads


def args(**kw):
    a = _abi.LifArgs(n=256, batch=64, n_delay=18, ring_slots=19, ring_mode=_abi.RING_COUNT, nsteps=1,
                     flags=_abi.LIF_PULL_DELIVERY, launch=_abi.LAUNCH_STEP, raster_slots=18, pull_group=4,
                     pull_steps=4)
    for f in ("out_ptr", "v", "g", "refrac", "adapt", "res", "rate", "counts", "spikes", "drive", "poisson_p",
              "active", "ring", "raster", "pull_ptr", "pull_pre", "pull_planes", "pull_meta", "pull_bits",
              "pull_state"):
        setattr(a, f, fake)
    a.params = params.ctypes.data
    a.pull_nplanes = 0
    for k, v in kw.items():
        setattr(a, k, v)
    return a


bad = [dict(batch=48), dict(batch=512), dict(ring_mode=_abi.RING_FIXED),
       dict(flags=_abi.LIF_PULL_DELIVERY | _abi.LIF_STD, std_u=fake),
       dict(flags=_abi.LIF_PULL_DELIVERY | _abi.LIF_DEFER_DELIVERY), dict(launch=_abi.LAUNCH_PERSISTENT),
       dict(pull_ptr=None), dict(pull_meta=None), dict(pull_nplanes=12), dict(pull_nplanes=8),
       dict(pull_nplanes=16, pull_planes=None), dict(pull_nplanes=16, pull_planes=fake + 4),
       dict(n=1 << 24), dict(pull_bits=None),
       dict(pull_state=None), dict(pull_bits=fake + 16), dict(pull_group=2), dict(pull_group=8),
       dict(pull_group=4, n_delay=7, ring_slots=8), dict(pull_steps=0), dict(pull_steps=5),
       dict(pull_phase=4), dict(pull_phase=-1), dict(pull_grid=-1), dict(flags=0)]
for kw in bad:
    rc = lib.flyb_lif_pull(ct.byref(args(**kw)), None)
    assert rc == _abi.EINVAL, (kw, rc)
print("rejected", len(bad))
"""


def test_pull_delivery_arguments_are_validated_before_any_launch():
    """flyb_lif_pull / FLYB_LIF_PULL_DELIVERY reject what the pull cannot do (a batch that is not
    32, 64, 128 or 256 flies, the fixed-point ring, depression, persistent launches, missing tables
    or buffers, an unknown table format, a plane table that is missing or misaligned, packed entries
    for more neurons than their 24-bit field holds, a misaligned pull buffer, a group size the batch
    or the delay does not allow, a step count outside 1..group, a bad phase, a negative block cap)
    with FLYB_EINVAL before touching the device. The
    cases run in a child process that sees no GPU, so that a check that ever weakens fails there
    instead of launching a kernel on the fake addresses."""
    import os
    import subprocess
    import sys
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    pkg = str(Path(__file__).resolve().parents[1] / "flyverse-core_b200")
    r = subprocess.run([sys.executable, "-c", PULL_VALIDATION, pkg], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "rejected 25" in r.stdout
