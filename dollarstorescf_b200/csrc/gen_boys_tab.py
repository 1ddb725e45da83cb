"""Generates boys_tab.cuh: F_m(x) on a grid for the fast (exact) Boys mode.

Grid x_k = k / 16, k = 0..575 (x < 36), m = 0..23 (24 doubles per point, so the
seven Taylor coefficients F_{L..L+6}(x_k) a thread needs are contiguous and it
fetches them with 16-byte loads).  Values come from
F_m(x) = 1F1(m + 1/2; m + 3/2; -x) / (2m + 1) evaluated with mpmath at 40 digits.

Usage: python gen_boys_tab.py OUT.cuh
"""
import sys

import mpmath

NGRID = 576
NM = 24
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
        # Truncation breakpoints of the reference's series (boys.cuh, boys_ref):
        # for order L the m=L series stops at the first n >= 1 with
        # t_n = (2x)^n / prod_{j=1..n}(2L+2j+1) <= 1e-9, i.e. at n(x) = 1 + #{k >= 1 : B_L[k] < x}
        # with B_L[k] = 0.5 exp((ln 1e-9 + LP_L[k]) / k), LP_L[k] = sum_{j=1..k} ln(2L+2j+1).
        NLB, NB = 16, 160
        mpmath.mp.dps = 40
        LP = [[0.0] * (NB + 1) for _ in range(NLB)]
        BP = [[0.0] * (NB + 1) for _ in range(NLB)]
        for L in range(NLB):
            acc = mpmath.mpf(0)
            prev = mpmath.mpf(-1)
            for k in range(1, NB + 1):
                acc += mpmath.log(2 * L + 2 * k + 1)
                LP[L][k] = float(acc)
                b = mpmath.mpf("0.5") * mpmath.exp((mpmath.log(mpmath.mpf("1e-9")) + acc) / k)
                assert b > prev, (L, k)
                prev = b
                BP[L][k] = float(b)
        # Coarse index: for x in [g/4, (g+1)/4): the count of breakpoints below g/4.
        NG = 200
        IDX = [[sum(1 for k in range(1, NB + 1) if BP[L][k] < g / 4.0) for g in range(NG)] for L in range(NLB)]
        f.write(f"#define DSS_BOYS_NLB {NLB}\n#define DSS_BOYS_NB {NB}\n#define DSS_BOYS_NG {NG}\n")
        for name, tab in (("g_boys_bp", BP), ("g_boys_lp", LP)):
            f.write("static __device__ const double %s[%d] = {\n" % (name, NLB * (NB + 1)))
            for L in range(NLB):
                f.write("  " + ", ".join(repr(v) for v in tab[L]) + ",\n")
            f.write("};\n")
        f.write("static __device__ const unsigned char g_boys_idx[%d] = {\n" % (NLB * NG))
        for L in range(NLB):
            f.write("  " + ", ".join(str(v) for v in IDX[L]) + ",\n")
        f.write("};\n")
        # Reference-mode values without running the series.  Within one interval
        # I_n = (B_m[n-1], B_m[n]] of order m the reference returns the analytic
        # function G_{m,n}(x) = exp(-x) sum_{i=0..n} a_i x^i, a_i = 2^i / prod_{j=0..i}(2m+2j+1).
        # Taylor coefficients G^(j)(x0)/j!, j = 0..6 (8 doubles per node, the 8th 0),
        # at three kinds of nodes: the grid x0 = k/16 for the interval that holds it
        # (g_boys_rg, interval index in g_boys_rn), and both ends of every interval
        # (g_boys_rr: G_{m,n} at B_m[n]; g_boys_rl: G_{m,n} at B_m[n-1]).  A point x of I_n
        # takes the grid node k = round(16 x) when that node lies in I_n, else the
        # end of I_n on the node's side, so |x - x0| <= 1/32 always.
        NLR, NBR = 3, 86
        mpmath.mp.dps = 30
        def taylor(m, n, x0):
            x0 = mpmath.mpf(x0)
            a = []
            c = mpmath.mpf(1) / (2 * m + 1)
            a.append(c)
            for i in range(1, n + 1):
                c = c * 2 / (2 * m + 2 * i + 1)
                a.append(c)
            S = []
            for l in range(7):
                acc = mpmath.mpf(0)
                for i in range(l, n + 1):
                    acc += a[i] * mpmath.binomial(i, l) * x0 ** (i - l)
                S.append(acc)
            e = mpmath.exp(-x0)
            out = []
            for j in range(7):
                t = mpmath.mpf(0)
                for k in range(j + 1):
                    t += e * (-1) ** k / mpmath.factorial(k) * S[j - k]
                out.append(float(t))
            return out + [0.0]
        def nidx(m, x):
            return 1 + sum(1 for k in range(1, NB + 1) if BP[m][k] < x)
        RG, RN, RR, RL = [], [], [], []
        for m in range(NLR):
            lim = 1.1 * m + 25 + 1.0
            for k in range(NGRID):
                x0 = k / STEP
                n0 = nidx(m, x0)
                assert n0 < 256
                RN.append(n0)
                RG.extend(taylor(m, n0, x0) if x0 <= lim else [0.0] * 8)
            assert nidx(m, 1.1 * m + 25 + 1.0 / STEP) < NBR, m
            for n in range(NBR):
                if n == 0:
                    RR.extend([0.0] * 8)
                    RL.extend([0.0] * 8)
                    continue
                RR.extend(taylor(m, n, BP[m][n]))
                RL.extend(taylor(m, n, BP[m][n - 1] if n >= 2 else 0.0))
        f.write(f"#define DSS_BOYS_NLR {NLR}\n#define DSS_BOYS_NBR {NBR}\n")
        for name, tab in (("g_boys_rg", RG), ("g_boys_rr", RR), ("g_boys_rl", RL)):
            f.write("static __device__ __align__(16) const double %s[%d] = {\n" % (name, len(tab)))
            for i in range(0, len(tab), 8):
                f.write("  " + ", ".join(repr(v) for v in tab[i:i + 8]) + ",\n")
            f.write("};\n")
        f.write("static __device__ const unsigned char g_boys_rn[%d] = {\n" % len(RN))
        for i in range(0, len(RN), 32):
            f.write("  " + ", ".join(str(v) for v in RN[i:i + 32]) + ",\n")
        f.write("};\n")
        f.write("static __device__ const double g_odd_inv[256] = {\n")
        inv = [1.0 / (2 * k + 1) for k in range(256)]
        for i in range(0, 256, 4):
            f.write("  " + ", ".join(repr(v) for v in inv[i:i + 4]) + ",\n")
        f.write("};\n")


if __name__ == "__main__":
    main()
