"""The C ABI library: it loads and exports every entry point include/ggbtddft.h declares (CPU only)."""
import ctypes
import os
import re

from ggbtddft_b200 import build, engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(ggb_\w+)\s*\(", src))
    return names


def test_library_builds_and_exports_every_declared_symbol():
    path = build.build()
    lib = ctypes.CDLL(path)
    names = declared_symbols()
    assert "ggb_step" in names and "ggb_create" in names
    for n in sorted(names):
        assert hasattr(lib, n), f"{n} declared in include/ but not exported"


def test_wrapper_declares_every_export():
    assert declared_symbols() <= set(engine.EXPORTS) | {"ggb_set_orbitals"}
    lib = engine.load_library()
    assert lib.ggb_version().startswith(b"ggbtddft")
