"""The C-ABI library loads on a CPU-only machine and exports every function
that include/*.h declares (no compute call is made here)."""
import ctypes
import glob
import os
import re

from jxpamg_all_b200 import lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = "\n".join(l for l in text.splitlines() if not l.lstrip().startswith("#"))
        for m in re.finditer(r"JXCPR_API\s+[^;(]*?\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_something():
    assert len(declared_functions()) >= 5


def test_library_exports_every_declared_symbol():
    so = lib.load()
    missing = [n for n in declared_functions() if not hasattr(so, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_version_and_error_without_gpu():
    so = lib.load()
    assert so.jxcpr_version() >= 10000
    assert isinstance(so.jxcpr_last_error(), bytes)
