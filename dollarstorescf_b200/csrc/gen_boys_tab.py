"""Generates the Boys function tables: boys_tab.cuh (sizes and the small
tables, defined per translation unit) and boys_cell_data.cu (the one definition
of the 627 KB cell-record table and the host function that returns its device
address; kernels receive that address in their argument structs, so the table
exists once per GPU whatever the number of kernel modules reading it).

Tables:
* g_boys_tab: F_m(x) for the fast (accurate) mode on the grid x_k = k / 16,
  k = 0..575 (x < 36), m = 0..23 (24 doubles per point, so the seven Taylor
  coefficients F_{L..L+6}(x_k) a thread needs are contiguous), from
  F_m(x) = 1F1(m + 1/2; m + 3/2; -x) / (2m + 1) with mpmath at 40 digits.
* g_boys_bp / g_boys_lp / g_boys_idx: truncation breakpoints of the
  reference's series (chem/GaussianIntegral.cpp:209-223) and their log
  products, for the accurate-minus-tail form (boys_ref_walk).
* g_boys_cell: per-cell Taylor records of the reference's own values
  (boys_ref_cells), orders 0..8.
* g_odd_inv: 1/(2k+1).

Usage: python gen_boys_tab.py OUT.cuh OUT_cells.cu
"""
import sys

import mpmath

NGRID = 576
NM = 24
STEP = 16  # points per unit of x


def fmt(v) -> str:
    return repr(v) if isinstance(v, float) else str(v)


def main() -> None:
    out_h, out_cu = sys.argv[1], sys.argv[2]
    tables = []  # (ctype, name, align, values)
    defines = []

    mpmath.mp.dps = 40
    vals = []
    for k in range(NGRID):
        x = mpmath.mpf(k) / STEP
        for m in range(NM):
            v = mpmath.hyp1f1(m + mpmath.mpf(1) / 2, m + mpmath.mpf(3) / 2, -x) / (2 * m + 1)
            vals.append(float(v))
    defines += [("DSS_BOYS_NGRID", NGRID), ("DSS_BOYS_NM", NM), ("DSS_BOYS_STEP", STEP)]
    tables.append(("double", "g_boys_tab", 16, vals))

    # Truncation breakpoints of the reference's series: for order L the m=L
    # series stops at the first n >= 1 with
    # t_n = (2x)^n / prod_{j=1..n}(2L+2j+1) <= 1e-9, i.e. at n(x) = 1 + #{k >= 1 : B_L[k] < x}
    # with B_L[k] = 0.5 exp((ln 1e-9 + LP_L[k]) / k), LP_L[k] = sum_{j=1..k} ln(2L+2j+1).
    NLB, NB = 16, 160
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
    defines += [("DSS_BOYS_NLB", NLB), ("DSS_BOYS_NB", NB), ("DSS_BOYS_NG", NG)]
    tables.append(("double", "g_boys_bp", 8, [v for row in BP for v in row]))
    tables.append(("double", "g_boys_lp", 8, [v for row in LP for v in row]))
    tables.append(("unsigned char", "g_boys_idx", 1, [v for row in IDX for v in row]))

    # Cell records of the reference's values.  Within one interval
    # I_n = (B_m[n-1], B_m[n]] of order m the reference returns the analytic
    # function G_{m,n}(x) = exp(-x) sum_{i=0..n} a_i x^i, a_i = 2^i / prod_{j=0..i}(2m+2j+1);
    # taylor() gives G_{m,n}^(j)(x0)/j!, j = 0..6.
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
        return out

    def nidx(m, x):
        return 1 + sum(1 for k in range(1, NB + 1) if BP[m][k] < x)

    # Two 64-byte records per order m and grid point k (cell
    # [k/16 - 1/32, k/16 + 1/32]).  Away from x = 0 a cell holds at most one
    # truncation breakpoint b (checked below, with a margin), so the
    # reference's value in the cell is G_{m,nA} for x <= b and G_{m,nA+1} for
    # x > b; both are entire functions, so both expand about the cell's own node
    # x0 = k/16 with |x - x0| <= 1/32.  Record layout (doubles): [0..6] Taylor
    # coefficients, [7] b.  Block A (the first NMC * NCELL records) holds the
    # x <= b piece, block B (the next NMC * NCELL) the x > b piece at the same
    # index; b = 1e300 when the cell has no breakpoint (its B record is never
    # read).  A lane reads one 64-byte A record and, only when x > b, the B record.
    # Cell 0 (x < 1/32) holds several breakpoints and is not tabulated; cells
    # above 16 (1.1 m + 25) + 1 are not used.
    NMC = 9
    NCELL = 544
    MARGIN = 1e-9
    CA, CB = [], []
    for m in range(NMC):
        kmax = int(round(STEP * (1.1 * m + 25))) + 1
        assert kmax < NCELL
        for k in range(NCELL):
            if k == 0 or k > kmax:
                CA.extend([0.0] * 7 + [1e300])
                CB.extend([0.0] * 7 + [1e300])
                continue
            lo, hi = k / STEP - 0.5 / STEP - MARGIN, k / STEP + 0.5 / STEP + MARGIN
            bs = [BP[m][j] for j in range(1, NB + 1) if lo <= BP[m][j] <= hi]
            assert len(bs) <= 1, (m, k, bs)
            x0 = k / STEP
            if not bs:
                pa = taylor(m, nidx(m, x0), x0)
                CA.extend(pa + [1e300])
                CB.extend(pa + [1e300])
            else:
                b = bs[0]
                na = nidx(m, b)  # interval (B[na-1], B[na] = b]
                CA.extend(taylor(m, na, x0) + [b])
                CB.extend(taylor(m, na + 1, x0) + [b])
    CELL = CA + CB
    defines += [("DSS_BOYS_NMC", NMC), ("DSS_BOYS_NCELL", NCELL)]
    tables.append(("double", "g_odd_inv", 8, [1.0 / (2 * k + 1) for k in range(256)]))

    with open(out_h, "w") as f:
        f.write("// Generated by gen_boys_tab.py -- do not edit.\n#pragma once\n#include <cuda_runtime.h>\n")
        for name, v in defines:
            f.write(f"#define {name} {v}\n")
        for ctype, name, align, vals in tables:
            f.write(f"static __device__ __align__({align}) const {ctype} {name}[{len(vals)}] = {{\n")
            for i in range(0, len(vals), 8):
                f.write("  " + ", ".join(fmt(v) for v in vals[i:i + 8]) + ",\n")
            f.write("};\n")
        f.write("// Device address of the cell-record table on the current device.\n")
        f.write("cudaError_t dss_boys_cell_table(const double** out);\n")
    with open(out_cu, "w") as f:
        f.write("// Generated by gen_boys_tab.py -- do not edit.\n#include <cuda_runtime.h>\n")
        f.write(f"static __device__ __align__(128) const double g_boys_cell[{len(CELL)}] = {{\n")
        for i in range(0, len(CELL), 8):
            f.write("  " + ", ".join(fmt(v) for v in CELL[i:i + 8]) + ",\n")
        f.write("};\n")
        f.write("cudaError_t dss_boys_cell_table(const double** out) {\n")
        f.write("  return cudaGetSymbolAddress((void**)out, g_boys_cell);\n}\n")


if __name__ == "__main__":
    main()
