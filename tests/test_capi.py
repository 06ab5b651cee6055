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


def test_exceptions_stop_at_the_c_abi(tmp_path):
    # the entry points are function-try-blocks over gcl::exception_status()
    src = tmp_path / "guard.cpp"
    src.write_text(r'''
#include <cstdio>
#include <new>
#include <stdexcept>
#include <vector>
#include "gcl_guard.h"
extern "C" int f_alloc(int k) try {
  if (k == 0) throw std::bad_alloc();
  if (k == 1) { std::vector<int> v; v.reserve(v.max_size() + 1ull); }
  if (k == 2) throw std::runtime_error("x");
  return GCL_OK;
} GCL_CATCH_ALL
int main() {
  std::printf("%d %d %d %d\n", f_alloc(0), f_alloc(1), f_alloc(2), f_alloc(3));
  return 0;
}
''')
    exe = tmp_path / "guard"
    import subprocess
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-std=c++17", "-I", os.path.join(ROOT, "gpu-canonical-labeling_b200", "csrc"),
                    "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    assert out == ["-3", "-3", "-7", "0"]  # NOMEM, NOMEM, INTERNAL, OK


def test_create_rejects_a_missing_device(pkg):
    # device -1 never exists; without a GPU every device is missing
    lib = pkg.api.load_library()
    out = ctypes.c_void_p(1)
    rc = lib.gcl_create(-1, ctypes.byref(out))
    assert rc in (-1, -2) and not out.value


def test_ctypes_structs_match_the_header(pkg, tmp_path):
    # size and field offsets of every struct include/gcl.h passes by pointer,
    # as the C compiler lays them out, against the Python binding's ctypes
    api = pkg.api
    structs = {"gcl_tuning": api.Tuning, "gcl_serve_config": api.ServeConfig,
               "gcl_serve_result": api.ServeResult, "gcl_serve_stats": api.ServeStats}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "gcl.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    import subprocess
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)],
                   check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = {}
    for ln in out.splitlines():
        s, f, v = ln.split()
        got[(s, f)] = int(v)
    for cname, py in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_no_cpu_fallback_without_a_gpu(pkg, G):
    # the product path has no CPU fallback: without a device every call that
    # canonizes raises instead of answering from the host
    import torch
    if torch.cuda.is_available():
        import pytest
        pytest.skip("a GPU is present")
    g = G.torus(4)
    for call in (lambda: pkg.canon(g), lambda: pkg.canon_batch([g, g]),
                 lambda: pkg.is_isomorphic(g, g), lambda: pkg.group_order(g),
                 lambda: pkg.Nauty_Parallel(g)):
        try:
            call()
        except pkg.GclError as e:
            assert e.rc in (-1, -2)
        else:
            raise AssertionError("a canonization ran without a GPU")
