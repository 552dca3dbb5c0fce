"""The device power helpers (csrc/mgm_math.h) return correctly rounded results.

The header is compiled for the host with gcc (the same source the kernels
use) and compared with binary128 references on random arguments spanning the
ranges the weight solves see: coordinate differences 1e-6..1 and squared
distances 1e-12..1, and on arguments whose powers lie within ~2^-106 of a
rounding midpoint (squared distances a few ulps from a power of four or from
the square of a short dyadic number, as between nodes of a circle and its
concentric twin), where double-double evaluation alone can round the wrong way.
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
    /* near-midpoint arguments: 4^j (1 +- k 2^-53), t^2 4^j nudged by k ulps,
       2^j (1 +- k 2^-53) for the integer powers */
    long hard = 0;
    for (int j = -20; j <= 2; j++)
        for (int k = 1; k <= 64; k++)
            for (int t = 1; t <= 15; t += 2)
                for (int sg = -1; sg <= 1; sg += 2) {
                    double base = ldexp((double)(t * t), 2 * j - 8);
                    double q = base;
                    for (int u = 0; u < k; u++) q = nextafter(q, sg < 0 ? 0.0 : 1e300);
                    __float128 Q = q;
                    hard += mgm_pow_half(q, 3) != (double)(sqrtq(Q) * Q);
                    hard += mgm_pow_half(q, 5) != (double)(sqrtq(Q) * Q * Q);
                    double d = ldexp((double)t, j - 4);
                    for (int u = 0; u < k; u++) d = nextafter(d, sg < 0 ? 0.0 : 1e300);
                    for (int sd = -1; sd <= 1; sd += 2) {
                        double e = sd * d;
                        __float128 D = e;
                        hard += mgm_pow_int(e, 3) != (double)(D * D * D);
                        hard += mgm_pow_int(e, 4) != (double)(D * D * D * D);
                        hard += mgm_pow_int(e, 5) != (double)(D * D * D * D * D);
                        hard += mgm_pow_int(e, 7) != (double)(D * D * D * D * D * D * D);
                    }
                }
    /* the annulus case: s = 0.25 (1 - 2^-53) */
    hard += mgm_pow_half(0.24999999999999997, 3) != 0.12499999999999999;
    printf("%ld %ld\n", bad, hard);
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
    bad, hard = (int(v) for v in out.split())
    assert bad == 0
    assert hard == 0
