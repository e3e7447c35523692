"""The host-side summed-volume index of flagged cells (GradedIndex in
rfnetwork_b200/csrc/fdtd_compile.cpp) against brute-force counts.

The split-storage plan and the streaming kernel's per-tile split masks are
read from it. A C++ program compiled with g++ against the compiler's source
fills a grid with random flags, then compares count() with a direct sum on
random boxes, boxes clipped at every face and empty boxes."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "rfnetwork_b200" / "csrc"

PROGRAM = r"""
#include "fdtd_compile.h"
#include <cstdio>
#include <random>
using namespace rfn;
int main() {
  std::mt19937 rng(7);
  const int shapes[][3] = {{1, 1, 1}, {2, 3, 4}, {17, 9, 5}, {40, 33, 29}, {64, 8, 70}};
  long checks = 0;
  for (const auto& sh : shapes) {
    CompiledGrid g;
    g.nx = sh[0]; g.ny = sh[1]; g.nz = sh[2];
    g.rows.resize(4);
    for (int r = 0; r < 4; ++r) for (int w = 0; w < kRowWords; ++w) g.rows[r].w[w] = 0;
    g.rows[1].w[R_FLAGS] = kFlagESplit;
    g.rows[2].w[R_FLAGS] = kFlagHSplit | kFlagGraded;
    g.rows[3].w[R_FLAGS] = kFlagGraded;
    const size_t n = size_t(g.nx) * g.ny * g.nz;
    g.ids.resize(n);
    for (auto& id : g.ids) id = uint16_t(rng() % 4);
    for (uint32_t mask : {kFlagESplit | kFlagHSplit, kFlagGraded}) {
      {  // leave non-zero bytes in memory the index may be given: its borders must be written
        int32_t* junk = new int32_t[1 << 16];
        for (int i = 0; i < (1 << 16); ++i) junk[i] = 12345;
        delete[] junk;
      }
      GradedIndex gi(g, mask);
      auto brute = [&](int x0, int x1, int y0, int y1, int z0, int z1) {
        long c = 0;
        for (int x = std::max(x0, 0); x < std::min(x1, g.nx); ++x)
          for (int y = std::max(y0, 0); y < std::min(y1, g.ny); ++y)
            for (int z = std::max(z0, 0); z < std::min(z1, g.nz); ++z)
              c += (g.rows[g.ids[(size_t(x) * g.ny + y) * g.nz + z]].w[R_FLAGS] & mask) ? 1 : 0;
        return c;
      };
      for (int t = 0; t < 400; ++t) {
        auto pick = [&](int len) { return int(rng() % unsigned(len + 4)) - 2; };
        int a[6];
        for (int k = 0; k < 3; ++k) {
          a[2 * k] = pick(sh[k]);
          a[2 * k + 1] = pick(sh[k]);
        }
        if (t % 4 == 0) { a[0] = 0; a[2] = 0; a[4] = 0; }                  // boxes at the low faces
        if (t % 4 == 1) { a[1] = g.nx; a[3] = g.ny; a[5] = g.nz; }        // and at the high faces
        const long want = brute(a[0], a[1], a[2], a[3], a[4], a[5]);
        const long got = gi.count(a[0], a[1], a[2], a[3], a[4], a[5]);
        if (want != got) {
          std::printf("MISMATCH %d %d %d box %d %d %d %d %d %d: %ld vs %ld\n", sh[0], sh[1], sh[2],
                      a[0], a[1], a[2], a[3], a[4], a[5], got, want);
          return 1;
        }
        ++checks;
      }
      if (gi.count(0, g.nx, 0, g.ny, 0, g.nz) != brute(0, g.nx, 0, g.ny, 0, g.nz)) return 1;
    }
  }
  std::printf("ok %ld\n", checks);
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_graded_index_counts_match_brute_force(tmp_path):
    src = tmp_path / "gi.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "gi"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", str(CSRC), str(src), str(CSRC / "fdtd_compile.cpp"),
                    "-o", str(exe), "-lpthread"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok ")
