"""Byte layout of the wide search's device region (wide_layout in
csrc/canon_wide.cuh), checked on the host: every region 256-byte aligned,
in order and disjoint, the queue of handed-over subtrees appended after the
regions the search without work sharing uses (so their offsets do not move),
and a queue entry large enough for the deepest parent (L <= n + 1 levels).
The header is compiled with nvcc into a host program; no GPU is used."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "gpu-canonical-labeling_b200", "csrc")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SRC = r'''
#include <cstdio>
#include "canon_wide.cuh"
using namespace gcl;
static int bad = 0;
#define CHECK(c) do { if (!(c)) { std::printf("fail %s n=%u\n", #c, n); ++bad; } } while (0)
int main() {
  const uint32_t ns[] = {1, 2, 65, 100, 1024, 4097, 65536};
  for (uint32_t n : ns) {
    for (uint32_t cap : {1u, 256u, 10000u}) {
      const uint64_t m2 = 3ull * n;
      const WideLayout a = wide_layout(n, m2, cap), b = wide_layout(n, m2, cap, 4096);
      const uint64_t offs[] = {a.hdr, a.fcode, a.fseq, a.flabel, a.fcert, a.lelem, a.linlev,
                               a.lstb, a.tcfirst, a.tclen, a.cum, a.bcode, a.bseq, a.blabel,
                               a.bcert, a.auts, a.ready, a.fixlev, a.orb, a.gq, a.gready, a.bytes};
      for (size_t i = 0; i + 1 < sizeof offs / sizeof offs[0]; ++i) {
        CHECK(offs[i] % 256 == 0);
        CHECK(offs[i] <= offs[i + 1]);
      }
      CHECK(a.hdr + sizeof(WideHdr) <= a.fcode);
      CHECK(a.ready + 4ull * cap <= a.fixlev);
      CHECK(a.auts + 2ull * cap * a.stride <= a.ready);
      // the queue is appended: every other region keeps its offset
      CHECK(b.auts == a.auts && b.ready == a.ready && b.fixlev == a.fixlev && b.orb == a.orb);
      CHECK(a.qcap == 0 && a.gstride == 0 && a.gq == a.gready && a.gready == a.bytes);
      CHECK(b.gq >= a.orb + 4ull * (n + 2));
      CHECK(b.gready >= b.gq + 4ull * 4096 * b.gstride);
      CHECK(b.bytes >= b.gready + 4ull * 4096);
      // an entry: L, v, L - 1 <= n vertices at [2, 2 + n + 2), L <= n + 1 codes after
      CHECK(b.gstride >= 2 + (n + 2) + (n + 2));
      CHECK(b.gstride % 4 == 0);
    }
  }
  std::printf(bad ? "FAILED %d\n" : "ok\n", bad);
  return bad != 0;
}
'''


def test_wide_layout_regions(tmp_path):
    if not os.path.exists(NVCC):
        pytest.skip("nvcc not available")
    (tmp_path / "layout.cu").write_text(SRC)
    exe = tmp_path / "layout"
    subprocess.run([NVCC, "-std=c++17", "--expt-relaxed-constexpr", "-gencode",
                    "arch=compute_100a,code=sm_100a", "-I", CSRC, "-o", str(exe),
                    str(tmp_path / "layout.cu")], check=True, capture_output=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout
