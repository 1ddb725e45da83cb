"""Generates boys_tab.cuh: F_m(x) on a grid for the fast (exact) Boys mode.

Grid x_k = k / 16, k = 0..575 (x < 36), m = 0..15 (16 doubles per point, so the
seven Taylor coefficients F_{L..L+6}(x_k) a thread needs are contiguous and it
fetches them with 16-byte loads).  Values come from
F_m(x) = 1F1(m + 1/2; m + 3/2; -x) / (2m + 1) evaluated with mpmath at 40 digits.

Usage: python gen_boys_tab.py OUT.cuh
"""
import sys

import mpmath

NGRID = 576
NM = 16
STEP = 16  # points per unit of x


def main() -> None:
    mpmath.mp.dps = 40
    vals = []
    for k in range(NGRID):
        x = mpmath.mpf(k) / STEP
        for m in range(NM):
            v = mpmath.hyp1f1(m + mpmath.mpf(1) / 2, m + mpmath.mpf(3) / 2, -x) / (2 * m + 1)
            vals.append(float(v))
    with open(sys.argv[1], "w") as f:
        f.write("// Generated by gen_boys_tab.py -- do not edit.\n#pragma once\n")
        f.write(f"#define DSS_BOYS_NGRID {NGRID}\n#define DSS_BOYS_NM {NM}\n#define DSS_BOYS_STEP {STEP}\n")
        f.write("static __device__ const double g_boys_tab[%d] = {\n" % (NGRID * NM))
        for i in range(0, len(vals), 4):
            f.write("  " + ", ".join(repr(v) for v in vals[i:i + 4]) + ",\n")
        f.write("};\n")
        f.write("static __device__ const double g_odd_inv[256] = {\n")
        inv = [1.0 / (2 * k + 1) for k in range(256)]
        for i in range(0, 256, 4):
            f.write("  " + ", ".join(repr(v) for v in inv[i:i + 4]) + ",\n")
        f.write("};\n")


if __name__ == "__main__":
    main()
