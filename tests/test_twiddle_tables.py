"""The register FFTs' compile-time twiddle tables against NumPy (CPU, needs nvcc).

`kTwiddleTables` in csrc/cjx_fft.cuh is evaluated by the compiler (Taylor
series of cos and sin after an exact quadrant reduction, in double, rounded
once to float).  A host program built from the same header dumps the
constexpr tables; every entry must equal exp(-2 pi i brev5(l) k1 / n) rounded
to complex64 (to within 2e-16 where the exact value is zero and NumPy's
float64 cos / sin leave a residue of that size).
"""

import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "cryojax_b200", "csrc")
RADICES = [1, 2, 3, 4, 5, 6, 8, 10, 12, 16]

PROGRAM = r"""
#include <cstdio>
#include "cjx_fft.cuh"
int main(int argc, char** argv) {
  constexpr cjx::ct::TwiddleTables t = cjx::ct::make_twiddle_tables();
  FILE* f = fopen(argv[1], "wb");
  if (!f) return 1;
  fwrite(t.reg, sizeof(float2), cjx::ct::kRegTableSize, f);
  fwrite(t.w32, sizeof(float2), 32, f);
  fclose(f);
  for (int R : {1, 2, 3, 4, 5, 6, 8, 10, 12, 16}) printf("%d %d\n", R, cjx::ct::reg_table_offset(R));
  return 0;
}
"""


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    return None


def test_compile_time_twiddle_tables(tmp_path):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc not available")
    src = tmp_path / "dump.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "dump"
    subprocess.run([nvcc, "-std=c++17", "--expt-relaxed-constexpr", "-Wno-deprecated-gpu-targets", "-I", CSRC,
                    str(src), "-o", str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe), str(tmp_path / "tab.bin")], check=True, capture_output=True, text=True).stdout
    got = np.fromfile(tmp_path / "tab.bin", dtype=np.complex64)

    ref, offsets = [], {}
    for R in RADICES:
        n = 32 * R
        offsets[R] = len(ref)
        for k1 in range(R):
            for lane in range(32):
                b = int(f"{lane:05b}"[::-1], 2)
                ref.append(np.exp(-2j * np.pi * b * k1 / n))
    ref += [np.exp(-2j * np.pi * m / 32) for m in range(32)]
    ref = np.array(ref).astype(np.complex64)

    assert got.shape == ref.shape
    assert np.abs(got.astype(np.complex128) - ref.astype(np.complex128)).max() <= 2e-16
    assert {int(a): int(b) for a, b in (line.split() for line in out.strip().splitlines())} == offsets
