"""libpbrt_b200.so loads on a CPU-only host and exports every symbol include/*.h declares."""
import ctypes
import glob
import os
import re

from conftest import ROOT
from pbrt_b200 import _capi


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(pbrt_[a-z0-9_]+)\s*\(", text))
    return names


def test_header_declares_entry_points():
    d = _declared()
    assert {"pbrt_ctx_create", "pbrt_scene_create", "pbrt_trace_closest", "pbrt_trace_any"} <= d


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_capi.LIB_PATH)
    missing = [n for n in sorted(_declared()) if not hasattr(lib, n)]
    assert not missing, f"declared in include/ but not exported: {missing}"


def test_python_signatures_cover_the_header():
    assert _declared() == set(_capi.SIGNATURES), "pbrt_b200/_capi.py must declare exactly the header's functions"
