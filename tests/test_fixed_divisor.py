"""The division by a fixed divisor of the Darcy Jacobi loop (div_fixed in
sphere_b200/csrc/sph_darcy.cu): q0 = RN(a rb) with rb = RN(1 / b), one
FMA for the exact remainder r = a - b q0, and RN(q0 + r rb) -- Markstein's
correction (P. Markstein, IBM J. Res. Dev. 34(1), 1990) -- with a zero a
answered by q0 itself and tiny, huge, infinite or NaN q0 by the division.
The kernel's bit-for-bit parity with the oracle rests on this giving the
correctly rounded quotient; here the same steps, written in C and compiled
without contraction, are compared with IEEE division on random operands
over a wide exponent range, quotients next to the ends of a binade,
divisors with all-ones and near-power-of-two significands, and the
special values."""
import os
import shutil
import subprocess

import pytest

C_SOURCE = r"""
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
static uint64_t s = 88172645463325252ull;
static uint64_t rnd(void) { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return s; }
static double mkd(uint64_t mant, int e)
{
    uint64_t b = ((uint64_t)(e + 1023) << 52) | (mant & ((1ull << 52) - 1));
    double d;
    memcpy(&d, &b, 8);
    return d;
}
static double div_fixed(double a, double b, double rb)
{
    const double q0 = a * rb;
    const double aq = fabs(q0);
    if (aq > 0x1p-900 && aq < 0x1p+1000) return fma(fma(-q0, b, a), rb, q0);
    if (a == 0.0) return q0;
    return a / b;
}
static long bad = 0, n = 0;
static void check(double a, double b)
{
    const double x = a / b, y = div_fixed(a, b, 1.0 / b);
    ++n;
    if (memcmp(&x, &y, 8) != 0 && !(isnan(x) && isnan(y))) {
        if (bad < 5) printf("a=%a b=%a: %a vs %a\n", a, b, x, y);
        ++bad;
    }
}
int main(void)
{
    for (int t = 0; t < 4000; ++t) {
        double b = mkd(rnd(), (int)(rnd() % 40) - 20);
        if (t % 4 == 0) b = mkd((1ull << 52) - 1 - (rnd() % 8), (int)(rnd() % 10) - 8);
        if (t % 4 == 1) b = mkd(rnd() % 16, (int)(rnd() % 10) - 8);
        if (t & 8) b = -b;
        for (int k = 0; k < 5000; ++k) {
            const uint64_t m = rnd();
            double a;
            if (k % 4 == 0) {
                a = mkd(m, (int)(rnd() % 80) - 40);
            } else if (k % 4 == 1) {
                a = mkd((1ull << 52) - 1 - (m % 64), (int)(rnd() % 40) - 20) * b;
                a = nextafter(a, (m & 1) ? INFINITY : -INFINITY);
            } else if (k % 4 == 2) {
                a = mkd(m % 64, (int)(rnd() % 40) - 20) * b;
                a = nextafter(a, (m & 1) ? INFINITY : -INFINITY);
            } else {
                a = mkd(m, (int)(rnd() % 10));
            }
            if (m & 2) a = -a;
            check(a, b);
        }
    }
    const double sp[] = {0.0, -0.0, 1e-320, -1e-320, 1e-300, 1e300, INFINITY, -INFINITY, NAN, 1.0};
    const double bs[] = {0.1, -0.1, 0.0137, 3.0, 1e-3};
    for (int i = 0; i < 10; ++i)
        for (int j = 0; j < 5; ++j) check(sp[i], bs[j]);
    printf("%ld %ld\n", n, bad);
    return bad != 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_fixed_divisor_division_is_correctly_rounded(tmp_path):
    src = os.path.join(str(tmp_path), "div_fixed.c")
    exe = os.path.join(str(tmp_path), "div_fixed")
    with open(src, "w") as fh:
        fh.write(C_SOURCE)
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", exe, src, "-lm"], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    n, bad = (int(v) for v in out.stdout.split()[-2:])
    assert n == 4000 * 5000 + 50
    assert out.returncode == 0 and bad == 0, out.stdout
