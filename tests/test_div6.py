"""The tracer's RK4 average divides by 6 as a product with RN(1/6) plus one
FMA residual correction (csrc/psf_device.cuh, div6).  This checks, on the
host with the C library's correctly rounded fmaf, that the result equals the
IEEE quotient x / 6 for every float with |x| >= 2^-120 on a stride through
all bit patterns (every pattern of the full range is covered by running with
stride 1, which takes about a minute).
"""
import os
import shutil
import subprocess
import tempfile

import pytest

SRC = r"""
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
int main(int argc, char **argv) {
    const uint64_t stride = strtoull(argv[1], 0, 10);
    const float r = 1.0f / 6.0f;
    volatile float six = 6.0f;
    uint64_t checked = 0, bad = 0;
    for (uint64_t u = 0; u <= 0xffffffffull; u += stride) {
        uint32_t b = (uint32_t)u;
        float x;
        memcpy(&x, &b, 4);
        if (isnan(x) || isinf(x) || fabsf(x) < 0x1p-120f) continue;
        const float ref = x / six;
        const float q = x * r;
        const float q2 = fmaf(fmaf(-q, 6.0f, x), r, q);
        ++checked;
        if (memcmp(&ref, &q2, 4) != 0) ++bad;
    }
    printf("%llu %llu\n", (unsigned long long)checked, (unsigned long long)bad);
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_div6_equals_ieee_quotient():
    stride = int(os.environ.get("PSF_DIV6_STRIDE", "61"))
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "div6.c"), os.path.join(d, "div6")
        with open(src, "w") as f:
            f.write(SRC)
        # -ffp-contract=off: the product and the quotient stay separate roundings.
        subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", exe, src, "-lm"], check=True)
        out = subprocess.run([exe, str(stride)], check=True, capture_output=True, text=True).stdout.split()
    checked, bad = int(out[0]), int(out[1])
    assert checked > 4_000_000_000 // stride // 2
    assert bad == 0
