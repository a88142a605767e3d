"""The correctly rounded quotient the CT, prot and CFL kernels use in place of
the division subroutine (div_const in csrc/how_internal.cuh): with y = RN(1/d),
q0 = RN(x y), the remainder r = x - q0 d (exact in one FMA) and q = RN(q0 + r y)
(a second FMA) equal the IEEE quotient RN(x/d) (Markstein's correction step).  The device sequence
is one round-to-nearest multiply and two fused multiply-adds, so the same
sequence in C with fma() on the host is the same arithmetic; this runs it on
random and structured operands for the constant divisors the kernels use
(24, 18) and for random divisors with y from one IEEE division, and counts
mismatches against x / d."""
import shutil
import subprocess

import pytest

SRC = r"""
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
static uint64_t s = 0x9E3779B97F4A7C15ull;
static uint64_t rnd(void) { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return s; }
static double mk(uint64_t m, int e, int sign) {
    uint64_t b = ((uint64_t)sign << 63) | ((uint64_t)(e + 1023) << 52) | (m & 0xFFFFFFFFFFFFFull);
    double x; memcpy(&x, &b, 8); return x;
}
static uint64_t pat(uint64_t r, int k) {
    switch (k & 3) {
        case 0: return r;
        case 1: return r | 0xFFFFFFFFFFF00ull;
        case 2: return r & 0xFFFF0000000FFull;
        default: return ~(r & 0xFFFFFull);
    }
}
/* div_const of csrc/how_internal.cuh */
static double div_const(double x, double d, double y) {
    const double q0 = x * y;
    const double q = fma(fma(-q0, d, x), y, q0);
    const double ax = fabs(x), aq = fabs(q0);
    if (ax >= 0x1p-900 && ax <= 0x1p+900 && aq >= 0x1p-900 && aq <= 0x1p+900) return q;
    if (x == 0.0) return x;
    return x / d;
}
static int same(double a, double b) { return memcmp(&a, &b, 8) == 0; }
int main(int argc, char** argv) {
    long long n = atoll(argv[1]), bad = 0;
    const double cs[2] = {24.0, 18.0};
    for (long long it = 0; it < n; ++it) {
        const uint64_t r1 = rnd(), r2 = rnd();
        const double x = mk(pat(r1, (int)it), (int)(r2 % 1900) - 950, (int)(r1 >> 63));
        const double d0 = cs[it & 1];
        if (!same(div_const(x, d0, 1.0 / d0), x / d0)) ++bad;
        const double d = mk(pat(r2, (int)(it >> 2)), (int)((r1 >> 20) % 600) - 300, 0);
        if (!same(div_const(x, d, 1.0 / d), x / d)) ++bad;
    }
    /* zeros, infinities, NaN, tiny and huge operands */
    const double sp[8] = {0.0, -0.0, INFINITY, -INFINITY, 0x1p-1000, -0x1p-1070, 0x1p+1000, 1.0};
    for (int i = 0; i < 8; ++i)
        for (int k = 0; k < 2; ++k)
            if (!same(div_const(sp[i], cs[k], 1.0 / cs[k]), sp[i] / cs[k])) ++bad;
    if (!isnan(div_const(NAN, 24.0, 1.0 / 24.0))) ++bad;
    printf("%lld\n", bad);
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not found")
def test_div_const_is_the_ieee_quotient(tmp_path):
    c = tmp_path / "divc.c"
    c.write_text(SRC.replace("#include <math.h>", "#include <math.h>\n#include <stdlib.h>"))
    exe = tmp_path / "divc"
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", str(exe), str(c), "-lm"], check=True)
    out = subprocess.run([str(exe), "20000000"], check=True, capture_output=True, text=True).stdout
    assert int(out.strip()) == 0
