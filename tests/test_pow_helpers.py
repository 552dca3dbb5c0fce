"""The device power helpers (csrc/mgm_math.h) return correctly rounded results.

The header is compiled for the host with gcc (the same source the kernels
use) and compared with binary128 references on random arguments spanning the
ranges the weight solves see: coordinate differences 1e-6..1 and squared
distances 1e-12..1.
"""
import os
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROG = r"""
#include <stdio.h>
#include <stdint.h>
#include <math.h>
#include <quadmath.h>
#include "mgm_math.h"
static uint64_t s = 0x9E3779B97F4A7C15ULL;
static double rnd(void) { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return (s >> 11) * (1.0 / 9007199254740992.0); }
int main(void) {
    long bad = 0, n = 400000;
    for (long t = 0; t < n; t++) {
        double d = (rnd() - 0.5) * pow(10, -6 * rnd());
        double q = rnd() * pow(10, -12 * rnd()) + 1e-300;
        __float128 D = d, Q = q;
        if (mgm_pow_int(d, 2) != (double)(D * D)) bad++;
        if (mgm_pow_int(d, 3) != (double)(D * D * D)) bad++;
        if (mgm_pow_int(d, 4) != (double)(D * D * D * D)) bad++;
        if (mgm_pow_int(d, 5) != (double)(D * D * D * D * D)) bad++;
        if (mgm_pow_half(q, 1) != (double)sqrtq(Q)) bad++;
        if (mgm_pow_half(q, 3) != (double)(sqrtq(Q) * Q)) bad++;
        if (mgm_pow_half(q, 5) != (double)(sqrtq(Q) * Q * Q)) bad++;
    }
    printf("%ld\n", bad);
    return 0;
}
"""


def test_pow_helpers_correctly_rounded():
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(src, "w").write(PROG)
        subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-I", os.path.join(ROOT, "multigrid_meshless_b200", "csrc"),
                        "-o", exe, src, "-lquadmath", "-lm"], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.strip()
    assert int(out) == 0
