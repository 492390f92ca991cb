"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: no GPU needed)."""
import ctypes
import glob
import os
import re

import rmt3d_b200
from rmt3d_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(rmt3d_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert declared_symbols(), "no declarations found"
    assert not missing, missing


def test_bindings_cover_declarations():
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_descriptor_layout_matches():
    L = rmt3d_b200.lib()
    assert L.rmt3d_desc_sizeof() == ctypes.sizeof(_lib.SceneDesc)


def test_null_arguments_are_rejected():
    L = rmt3d_b200.lib()
    assert L.rmt3d_desc_defaults(None) == _lib.ERR_INVALID
    assert L.rmt3d_step(None, 0, None) == _lib.ERR_INVALID
    assert L.rmt3d_scene_destroy(None) == _lib.OK
