"""The averaging's radmax threshold (AvgArgsK.rad2, computed on the host by
radmax_sq_threshold in i2g_launch.h) is the smallest double whose pow(., 0.5) in
the host's libm exceeds 0.95 xsize / 2 -- the reference's own comparison
(markmart.c:268, 335-340) -- for any box width.  Compiled here with nvcc as host
code only; no GPU needed."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "i2elvis_planet_b200", "csrc")

PROGRAM = r"""
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include "i2g_launch.h"
int main()
{
    srand(12345);
    int bad = 0, n = 0;
    for (int i = 0; i < 20000; i++) {
        const double xsize = (i < 4) ? (double[]){500000.0, 1.0, 3.0e6, 7.25}[i]
                                     : 1.0 + 1.0e7 * (double)rand() / RAND_MAX;
        const double R = xsize / 2.0 * 0.95, s = i2g::radmax_sq_threshold(xsize);
        const bool above = std::pow(s, 0.5) > R;
        const bool below = !(std::pow(std::nextafter(s, 0.0), 0.5) > R);
        n++;
        if (!above || !below) bad++;
    }
    std::printf("%d %d\n", n, bad);
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="needs nvcc")
def test_radmax_threshold_is_the_reference_comparison(tmp_path):
    src = tmp_path / "thr.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "thr"
    subprocess.run(["nvcc", "-std=c++17", "-I", CSRC, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    n, bad = (int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split())
    assert n == 20000 and bad == 0
