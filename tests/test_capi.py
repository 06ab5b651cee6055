"""The C-ABI library loads and exports every symbol include/gcl.h declares
(no GPU needed: nothing here launches work)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "gcl.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(gcl_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_header(pkg):
    api = pkg.api
    lib = api.load_library()
    names = declared_symbols()
    assert "gcl_canon_one" in names and "gcl_canon_batch" in names
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(api.EXPORTS) == names
    assert lib.gcl_version() >= 100
    assert lib.gcl_status_string(-4).decode().startswith("bad input")
