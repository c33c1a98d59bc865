"""The Hilbert index used to order mesh primitives (csrc/scene_build.cu),
compiled for the host from its source: on the first 16^3 sub-cube it must be
a bijection onto 0..4095 whose consecutive cells are face-adjacent."""
from __future__ import annotations

import re
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_hilbert3_is_a_hilbert_curve(tmp_path):
    src = (ROOT / "diff-wos_b200" / "csrc" / "scene_build.cu").read_text()
    spread = re.search(r"__device__ __forceinline__ uint32_t spread3\(uint32_t x\) \{.*?\n\}", src, re.S).group(0)
    hil = re.search(r"__device__ __forceinline__ uint32_t hilbert3\(.*?\n\}", src, re.S).group(0)
    prog = "#include <cstdint>\n#include <cstdio>\n#include <cstdlib>\n#include <vector>\n"
    prog += "#define __device__\n#define __forceinline__ inline\n" + spread + "\n" + hil + "\n"
    prog += r"""
int main() {
    const int N = 16;
    std::vector<int> pos(N * N * N * 3, -1);
    for (int x = 0; x < N; ++x) for (int y = 0; y < N; ++y) for (int z = 0; z < N; ++z) {
        const uint32_t h = hilbert3(x, y, z);
        if (h >= (uint32_t)(N * N * N) || pos[3 * h] >= 0) return 1;
        pos[3 * h] = x; pos[3 * h + 1] = y; pos[3 * h + 2] = z;
    }
    for (int h = 1; h < N * N * N; ++h) {
        const int d = abs(pos[3*h] - pos[3*h-3]) + abs(pos[3*h+1] - pos[3*h-2]) + abs(pos[3*h+2] - pos[3*h-1]);
        if (d != 1) return 2;
    }
    return 0;
}
"""
    (tmp_path / "h.cpp").write_text(prog)
    subprocess.run(["g++", "-O1", "-o", str(tmp_path / "h"), str(tmp_path / "h.cpp")], check=True)
    assert subprocess.run([str(tmp_path / "h")]).returncode == 0
