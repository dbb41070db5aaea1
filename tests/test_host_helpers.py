"""Host-side helpers of the library, compiled on the CPU with g++ against the library's
own header (no GPU): the NaN-propagating max that the refinement, exact-operator and
GMRES residual checks use (a NaN column residual must fail the check, where std::max
would drop it)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA_INC = "/usr/local/cuda/include"

PROGRAM = r"""
#include <cmath>
#include <cstdio>
#include <limits>
#include "hm_common.h"
int main() {
    const double nan = std::numeric_limits<double>::quiet_NaN();
    int bad = 0;
    bad += hm::max_nan(1.0, 2.0) != 2.0;
    bad += hm::max_nan(3.0, 2.0) != 3.0;
    bad += !std::isnan(hm::max_nan(1.0, nan));
    bad += !std::isnan(hm::max_nan(nan, 1.0));
    double w = 0.0;                          // the residual loops' pattern
    const double cols[4] = {1e-12, nan, 1e-13, 1e-11};
    for (double c : cols) w = hm::max_nan(w, c);
    bad += !std::isnan(w);
    bad += (w <= 1e-10);                     // the convergence test must fail
    std::printf("%d\n", bad);
    return bad;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None or not os.path.isdir(CUDA_INC), reason="g++ and CUDA headers")
def test_max_nan_propagates(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "t"
    r = subprocess.run(["g++", "-std=c++17", "-O2", f"-I{CUDA_INC}", f"-I{os.path.join(ROOT, 'hmat-omp_b200', 'csrc')}",
                        str(src), "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip() == "0", out.stdout + out.stderr
