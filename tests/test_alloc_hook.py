"""The library's allocation helpers (csrc/gcl_alloc.h): every device and
pinned host allocation goes through them, and GCL_FAULT_ALLOC_AT=k fails
exactly the k-th one as out of memory without calling the allocator.  The
header is compiled with nvcc into a host program; without a GPU the real
allocations fail too, with another code, which the checks allow for."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "gpu-canonical-labeling_b200", "csrc")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SRC = r'''
#include <cstdio>
#include "gcl_alloc.h"
int main() {
  // device, device, pinned, device, pinned: code and whether the pointer is null
  for (int i = 0; i < 5; ++i) {
    void* p = (void*)&i;
    const cudaError_t e = (i == 2 || i == 4) ? gcl::pinned_alloc(&p, 4096)
                                             : gcl::device_alloc(&p, 1024, nullptr);
    std::printf("%d %d\n", (int)e, p == nullptr ? 1 : 0);
    if (e == cudaSuccess) {
      if (i == 2 || i == 4) cudaFreeHost(p); else cudaFreeAsync(p, nullptr);
    }
  }
  return 0;
}
'''


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    if not os.path.exists(NVCC):
        pytest.skip("nvcc not available")
    d = tmp_path_factory.mktemp("alloc")
    (d / "probe.cu").write_text(SRC)
    exe = d / "probe"
    subprocess.run([NVCC, "-std=c++17", "-Wno-deprecated-gpu-targets", "-I", CSRC, "-o",
                    str(exe), str(d / "probe.cu")], check=True, capture_output=True)
    return str(exe)


def _run(exe, value):
    env = dict(os.environ)
    env.pop("GCL_FAULT_ALLOC_AT", None)
    if value is not None:
        env["GCL_FAULT_ALLOC_AT"] = value
    out = subprocess.run([exe], check=True, capture_output=True, text=True, env=env).stdout
    return [tuple(map(int, ln.split())) for ln in out.split("\n") if ln.strip()]


OOM = 2  # cudaErrorMemoryAllocation


@pytest.mark.parametrize("k", [1, 2, 3, 5])
def test_kth_allocation_fails_once(probe, k):
    rows = _run(probe, str(k))
    assert len(rows) == 5
    for i, (code, null) in enumerate(rows, start=1):
        if i == k:
            assert (code, null) == (OOM, 1)
        else:
            assert code != OOM  # success with a GPU, an error code without one
            assert null == (code != 0)


@pytest.mark.parametrize("value", [None, "", "0", "-3", "abc", "2x", "99"])
def test_no_fault_unless_a_positive_count_is_reached(probe, value):
    for code, null in _run(probe, value):
        assert code != OOM
        assert null == (code != 0)


def test_every_allocation_goes_through_the_helpers():
    call = re.compile(r"\b(cudaMalloc\w*|cudaHostAlloc|cudaMallocHost)\s*\(")
    found = []
    for name in sorted(os.listdir(CSRC)):
        if name == "gcl_alloc.h" or not name.endswith((".cu", ".cuh", ".h", ".cpp")):
            continue
        for i, line in enumerate(open(os.path.join(CSRC, name)), start=1):
            code = line.split("//", 1)[0]
            if call.search(code):
                found.append(f"{name}:{i}: {line.strip()}")
    assert not found, found
