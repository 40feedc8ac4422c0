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
