"""CPU: the small-bucket sorting networks of the ESC kernel (csrc/cas_sortnet.cuh).

The header compiles as plain C++; a harness built here checks every network on
all 0/1 inputs (by the 0-1 principle a comparator network that sorts those sorts
everything) and on random packed (offset, slot) words with repeated offsets,
against std::sort, including the unpacking of offsets and slots."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "contention-aware-spgemm_b200", "csrc")

HARNESS = r"""
#include "cas_sortnet.cuh"
#include <algorithm>
#include <cstdio>
#include <random>
#include <vector>

template <int N>
int check(std::mt19937& rng) {
  int bad = 0;
  for (unsigned m = 0; m < (1u << N); ++m) {
    uint32_t w[N];
    for (int i = 0; i < N; ++i) w[i] = (m >> i) & 1u;
    cas::sort_net(w);
    for (int i = 1; i < N; ++i) bad += w[i - 1] > w[i];
  }
  for (int t = 0; t < 20000; ++t) {
    const int nb = 1 + (int)(rng() % N);
    const uint32_t span = 1u << (rng() % 24);   // offsets below 2^23, few distinct in narrow spans
    uint32_t w[N];
    std::vector<uint32_t> ref;
    for (int i = 0; i < N; ++i) {
      if (i < nb) {
        const uint32_t off = (uint32_t)(rng() % span) & ((1u << 23) - 1);
        w[i] = cas::sortnet_pack(off, i);
        ref.push_back(w[i]);
      } else {
        w[i] = 0xFFFFFFFFu;
      }
    }
    std::sort(ref.begin(), ref.end());
    cas::sort_net(w);
    for (int i = 0; i < nb; ++i) {
      bad += w[i] != ref[i];
      // stable: equal offsets keep slot order
      if (i > 0 && cas::sortnet_offset(w[i]) == cas::sortnet_offset(w[i - 1]))
        bad += cas::sortnet_slot(w[i]) < cas::sortnet_slot(w[i - 1]);
    }
    for (int i = nb; i < N; ++i) bad += w[i] != 0xFFFFFFFFu;
  }
  return bad;
}

int main() {
  std::mt19937 rng(7);
  const int b4 = check<4>(rng), b6 = check<6>(rng), b8 = check<8>(rng);
  std::printf("%d %d %d\n", b4, b6, b8);
  return b4 + b6 + b8 ? 1 : 0;
}
"""


def test_sorting_networks(tmp_path):
    src = tmp_path / "sortnet.cpp"
    src.write_text(HARNESS)
    exe = tmp_path / "sortnet"
    cc = subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, "-o", str(exe), str(src)],
                        capture_output=True, text=True)
    if cc.returncode != 0:
        pytest.fail(cc.stderr)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, f"network failures (4, 6, 8 inputs): {out.stdout}"
    assert out.stdout.split() == ["0", "0", "0"]
