"""The kernels' shortened exp for the raster's arguments (sfm::exp_neg_ in
splatfield_b200/csrc/sf_math.cuh) gives the oracle's exp (sfo::expf_c in
oracle/sfo_math.h) bit for bit over every f32 in [-86, 0].

Both headers are compiled here for the host with the library's own flags for
floating point (-ffp-contract=off, no fast math), the same IEEE operations the
device runs under -fmad=false. The walk covers all 1.07e9 floats of the range
(OpenMP over the host's cores).
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <cstdio>
#include <cstdint>
#include "sf_math.cuh"
#include "sfo_math.h"
int main() {
    // -0.0 and the negative floats up to 86.0 in magnitude, by bit pattern.
    const uint32_t lo = 0x80000000u, hi = sfm::f2u(-86.0f);
    unsigned long long bad = 0, first = 0;
    #pragma omp parallel for reduction(+ : bad) schedule(static, 1 << 16)
    for (long long u = lo; u <= (long long)hi; ++u) {
        const float x = sfm::u2f((uint32_t)u);
        if (sfm::f2u(sfm::exp_neg_(x)) != sfm::f2u(sfo::expf_c(x))) {
            ++bad;
            #pragma omp critical
            if (!first) first = (unsigned long long)u;
        }
    }
    // +0.0 as well.
    if (sfm::f2u(sfm::exp_neg_(0.0f)) != sfm::f2u(sfo::expf_c(0.0f))) ++bad;
    std::printf("%llu %llu %llu\n", bad, first, (unsigned long long)(hi - lo + 2));
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_exp_neg_equals_oracle_exp(tmp_path):
    src = tmp_path / "exp_identity.cpp"
    exe = tmp_path / "exp_identity"
    src.write_text(PROGRAM)
    subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
                    "-I", os.path.join(ROOT, "splatfield_b200", "csrc"), "-I", os.path.join(ROOT, "oracle"),
                    str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=600).stdout.split()
    bad, first, total = (int(v) for v in out)
    assert total > 1_000_000_000
    assert bad == 0, f"{bad} mismatches, first at bits {first:#x}"
