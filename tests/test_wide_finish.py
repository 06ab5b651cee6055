"""The wide search's packed output (wide_row_word in csrc/canon_wide.cuh,
which the finish kernel's lanes call for each word of a canonical row): on
random graphs, labelings and certificates, every word equals the direct
packing of the relabelled adjacency matrix.  The header is compiled with nvcc
into a host program; no GPU is used."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "gpu-canonical-labeling_b200", "csrc")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SRC = r'''
#include <algorithm>
#include <cstdio>
#include <random>
#include <vector>
#include "canon_wide.cuh"
int main() {
  std::mt19937 rng(11);
  int bad = 0;
  for (int t = 0; t < 400; ++t) {
    const uint32_t n = 1 + rng() % 400;
    const uint32_t pct = rng() % 60;
    std::vector<std::vector<uint32_t>> adj(n);
    for (uint32_t a = 0; a < n; ++a)
      for (uint32_t b = a + 1; b < n; ++b)
        if (rng() % 1000 < pct) { adj[a].push_back(b); adj[b].push_back(a); }
    std::vector<int32_t> rp(n + 1, 0);
    for (uint32_t v = 0; v < n; ++v) rp[v + 1] = rp[v] + (int32_t)adj[v].size();
    std::vector<uint32_t> label(n), pos(n), cert(std::max<int32_t>(rp[n], 1));
    for (uint32_t i = 0; i < n; ++i) label[i] = i;
    std::shuffle(label.begin(), label.end(), rng);
    for (uint32_t i = 0; i < n; ++i) pos[label[i]] = i;
    for (uint32_t v = 0; v < n; ++v)
      for (size_t k = 0; k < adj[v].size(); ++k) cert[rp[v] + k] = pos[adj[v][k]];
    const uint32_t words = (n + 63) / 64;
    for (uint32_t i = 0; i < n; ++i) {
      std::vector<uint64_t> want(words, 0);
      for (uint32_t u : adj[label[i]]) want[pos[u] / 64] |= 1ull << (pos[u] % 64);
      for (uint32_t w = 0; w < words; ++w)
        if (gcl::wide_row_word(rp.data(), label.data(), cert.data(), i, w) != want[w]) ++bad;
    }
  }
  std::printf(bad ? "FAILED %d\n" : "ok\n", bad);
  return bad != 0;
}
'''


def test_packed_row_words(tmp_path):
    if not os.path.exists(NVCC):
        pytest.skip("nvcc not available")
    (tmp_path / "rows.cu").write_text(SRC)
    exe = tmp_path / "rows"
    subprocess.run([NVCC, "-std=c++17", "--expt-relaxed-constexpr", "-gencode",
                    "arch=compute_100a,code=sm_100a", "-I", CSRC, "-o", str(exe),
                    str(tmp_path / "rows.cu")], check=True, capture_output=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout
