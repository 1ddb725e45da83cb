"""Generates the per-angular-class ERI device code (eri_gen.cuh).

For a shell-quartet class (la lb|lc ld) the generated code evaluates, for one
contracted quartet per thread:

  1. per primitive quartet: Boys F_0..F_L (boys.cuh), then the Obara-Saika
     vertical recursion (VRR) to [e0|f0]^(0) for la <= |e| <= la+lb,
     lc <= |f| <= lc+ld, accumulated over the primitive loop;
  2. once per contracted quartet: the Head-Gordon-Pople horizontal transfer
     (HRR) to the Cartesian (ab|cd) on bra then ket;
  3. the Cartesian -> function transform: the reference's real solid harmonics
     (chem/GTO.cpp:15-94) in 5D mode, or one normalised monomial per function
     in 6D mode.

The integral values are the same linear functionals of F_m(T) that the
reference's separable 1-D chain evaluates (chem/GaussianIntegral.cpp:334-642),
so with the reference's Boys values they agree to rounding.

Recurrences (p = a+b exponents, q = c+d, rho = pq/(p+q), W the weighted centre):
  [e+1_i|0]^m  = PA_i [e|0]^m + WP_i [e|0]^(m+1)
                 + e_i/(2p) ([e-1_i|0]^m - rho/p [e-1_i|0]^(m+1))
  [e|f+1_i]^m  = QC_i [e|f]^m + WQ_i [e|f]^(m+1)
                 + f_i/(2q) ([e|f-1_i]^m - rho/q [e|f-1_i]^(m+1))
                 + e_i/(2(p+q)) [e-1_i|f]^(m+1)
  (a, b+1_i| = (a+1_i, b| + AB_i (a, b|      and likewise on the ket.

Usage: python gen_eri.py OUT.cuh [LMAX]
"""
from __future__ import annotations

import math
import os
import sys
from typing import Dict, List, Tuple

PI_REF = 3.14159265358979  # lalib/MathUtil.hpp:8

Cart = Tuple[int, int, int]


def cart_list(l: int) -> List[Cart]:
    return [(a, b, l - a - b) for a in range(l, -1, -1) for b in range(l - a, -1, -1)]


def ncart(l: int) -> int:
    return (l + 1) * (l + 2) // 2


def _fact(n: int) -> float:
    return float(math.factorial(n)) if n > 0 else 1.0


def _dfact(n: int) -> float:
    r = 1.0
    while n > 0:
        r *= n
        n -= 2
    return r


def sph_terms(l: int, m: int) -> Dict[Cart, float]:
    """Real solid harmonic (l, m) as {monomial: weight}: the recursion of the
    reference's ContractedGaussian constructor (chem/GTO.cpp:15-88): a sectoral
    seed in x, y; the associated-Legendre step in z; Y-normalisation
    sqrt((2l+1)(l-m)!/(4 pi (l+m)!)) * sqrt(2) for m != 0."""
    am = abs(m)
    cur: Dict[Cart, float] = {}
    x = am if m <= 0 else am - 1
    i = 0
    while x >= 0:
        k = (x, am - x, 0)
        cur[k] = cur.get(k, 0.0) + (-1.0 if i & 1 else 1.0) * math.comb(am, x)
        x -= 2
        i += 1
    leg = _dfact(2 * am - 1)
    if m < 0:
        leg *= _fact(l - am) / _fact(l + am)
    cur = {k: v * leg for k, v in cur.items()}
    ynorm = math.sqrt((2 * l + 1) * _fact(l - m) / (4.0 * PI_REF * _fact(l + m)))
    if m:
        ynorm *= math.sqrt(2.0)
    if l > am:
        prev = dict(cur)
        cur = {(a, b, c + 1): v * (2 * am + 1) for (a, b, c), v in cur.items()}
        for ii in range(am + 1, l):
            sf = float(ii - am + 1)
            nxt: Dict[Cart, float] = {}
            for (a, b, c), v in cur.items():
                k = (a, b, c + 1)
                nxt[k] = nxt.get(k, 0.0) + v * (2 * ii + 1) / sf
            for (a, b, c), v in prev.items():
                for k in ((a + 2, b, c), (a, b + 2, c), (a, b, c + 2)):
                    nxt[k] = nxt.get(k, 0.0) - v * (ii + am) / sf
            prev, cur = cur, nxt
    return {k: v * ynorm for k, v in cur.items() if v != 0.0}


def cart_weight(c: Cart) -> float:
    a, b, cc = c
    l = a + b + cc
    return math.sqrt(_dfact(2 * l + 1) / (4.0 * PI_REF * _dfact(2 * a - 1) * _dfact(2 * b - 1) * _dfact(2 * cc - 1)))


def transform_rows(l: int, pure: bool) -> List[List[Tuple[int, float]]]:
    """For each output function of a shell: [(cartesian index, weight)]."""
    cl = cart_list(l)
    if pure:
        return [[(cl.index(k), v) for k, v in sorted(sph_terms(l, m).items(), key=lambda kv: cl.index(kv[0]))]
                for m in range(-l, l + 1)]
    return [[(i, cart_weight(c))] for i, c in enumerate(cl)]


def nfunc(l: int, pure: bool) -> int:
    return 2 * l + 1 if pure else ncart(l)


def lit(v: float) -> str:
    return repr(float(v))


def sub1(c: Cart, i: int) -> Cart:
    t = list(c)
    t[i] -= 1
    return tuple(t)  # type: ignore


def add1(c: Cart, i: int) -> Cart:
    t = list(c)
    t[i] += 1
    return tuple(t)  # type: ignore


def cname(c: Cart) -> str:
    return f"{c[0]}{c[1]}{c[2]}"


def pick_dir(c: Cart) -> int:
    best = -1
    for i in range(3):
        if c[i] > 0 and (best < 0 or c[i] > c[best]):
            best = i
    return best


class ClassGen:
    def __init__(self, la: int, lb: int, lc: int, ld: int):
        self.la, self.lb, self.lc, self.ld = la, lb, lc, ld
        self.E = la + lb
        self.F = lc + ld
        self.L = self.E + self.F
        self.name = f"{la}{lb}{lc}{ld}"
        self.vrr_lines: List[str] = []
        self.vrr_done: Dict[Tuple[Cart, Cart, int], str] = {}
        self.flops_vrr = 0      # flops per primitive quartet in the VRR as generated
        self.flops_alg_vrr = 0  # algorithmic count (2 flops per recurrence term, e>=la, f>=lc)

    # ------------------------------------------------------------------ VRR
    def vrr(self, e: Cart, f: Cart, m: int) -> str:
        key = (e, f, m)
        if key in self.vrr_done:
            return self.vrr_done[key]
        ne, nf = sum(e), sum(f)
        name = f"v{cname(e)}_{cname(f)}_{m}"
        if ne == 0 and nf == 0:
            self.vrr_done[key] = f"F[{m}]"
            return f"F[{m}]"
        terms: List[str] = []
        if nf > 0:
            i = pick_dir(f)
            f1 = sub1(f, i)
            ax = "xyz"[i]
            terms.append(f"QC{ax} * {self.vrr(e, f1, m)}")
            terms.append(f"WQ{ax} * {self.vrr(e, f1, m + 1)}")
            if f1[i] > 0:
                f2 = sub1(f1, i)
                terms.append(f"(R){lit(f1[i])} * oo2q * ({self.vrr(e, f2, m)} - rho_q * {self.vrr(e, f2, m + 1)})")
            if e[i] > 0:
                terms.append(f"(R){lit(e[i])} * oo2pq * {self.vrr(sub1(e, i), f1, m + 1)}")
        else:
            i = pick_dir(e)
            e1 = sub1(e, i)
            ax = "xyz"[i]
            terms.append(f"PA{ax} * {self.vrr(e1, f, m)}")
            terms.append(f"WP{ax} * {self.vrr(e1, f, m + 1)}")
            if e1[i] > 0:
                e2 = sub1(e1, i)
                terms.append(f"(R){lit(e1[i])} * oo2p * ({self.vrr(e2, f, m)} - rho_p * {self.vrr(e2, f, m + 1)})")
        nterm = len(terms) + sum(1 for t in terms if "(" in t)  # bracketed terms carry two products
        self.flops_vrr += 2 * nterm
        if ne >= self.la and nf >= self.lc:
            self.flops_alg_vrr += 2 * nterm
        self.vrr_lines.append(f"const R {name} = " + " + ".join(terms) + ";")
        self.vrr_done[key] = name
        return name

    # ------------------------------------------------------------------ emit
    def emit(self, out: List[str]) -> None:
        la, lb, lc, ld, E, F, L = self.la, self.lb, self.lc, self.ld, self.E, self.F, self.L
        ecomps = [c for l in range(la, E + 1) for c in cart_list(l)]
        fcomps = [c for l in range(lc, F + 1) for c in cart_list(l)]
        eidx = {c: i for i, c in enumerate(ecomps)}
        fidx = {c: i for i, c in enumerate(fcomps)}
        nE, nF = len(ecomps), len(fcomps)
        for e in ecomps:
            for f in fcomps:
                self.vrr(e, f, 0)
        self.nacc = nE * nF
        o = out.append
        o(f"// ---- class ({la}{lb}|{lc}{ld}): L={L}, {nE}x{nF} contracted VRR outputs")
        o(f"template <int BOYS, bool PURE, typename R = double>")
        o(f"__device__ __forceinline__ void eri_{self.name}(const PrimPair* __restrict__ bra, int nbra,")
        o(f"    const PrimPair* __restrict__ ket, int nket, double ABx_, double ABy_, double ABz_,")
        o(f"    double CDx_, double CDy_, double CDz_, R* __restrict__ I, const double* __restrict__ cells) {{")
        o(f"  const R ABx = (R)ABx_, ABy = (R)ABy_, ABz = (R)ABz_;")
        o(f"  const R CDx = (R)CDx_, CDy = (R)CDy_, CDz = (R)CDz_;")
        o(f"  R acc[{nE * nF}];")
        o(f"#pragma unroll")
        o(f"  for (int t = 0; t < {nE * nF}; ++t) acc[t] = (R)0.0;")
        o(f"  for (int ik = 0; ik < nket; ++ik) {{")
        o(f"    const PrimPair kp = load_pp(ket + ik);")
        o(f"    for (int ib = 0; ib < nbra; ++ib) {{")
        o(f"      const PrimPair bp = load_pp(bra + ib);")
        o(f"      double Fd[{L + 1}];")
        o(f"      double PAx_, PAy_, PAz_, WPx_, WPy_, WPz_, QCx_, QCy_, QCz_, WQx_, WQy_, WQz_;")
        o(f"      double oo2p_, oo2q_, oo2pq_, rho_p_, rho_q_;")
        o(f"      prim_quartet<BOYS, {L}>(bp, kp, Fd, PAx_, PAy_, PAz_, WPx_, WPy_, WPz_, QCx_, QCy_, QCz_, WQx_,")
        o(f"                              WQy_, WQz_, oo2p_, oo2q_, oo2pq_, rho_p_, rho_q_, cells);")
        o(f"      R F[{L + 1}];")
        o(f"#pragma unroll")
        o(f"      for (int m = 0; m <= {L}; ++m) F[m] = (R)Fd[m];")
        o(f"      const R PAx = (R)PAx_, PAy = (R)PAy_, PAz = (R)PAz_, WPx = (R)WPx_, WPy = (R)WPy_, WPz = (R)WPz_;")
        o(f"      const R QCx = (R)QCx_, QCy = (R)QCy_, QCz = (R)QCz_, WQx = (R)WQx_, WQy = (R)WQy_, WQz = (R)WQz_;")
        o(f"      const R oo2p = (R)oo2p_, oo2q = (R)oo2q_, oo2pq = (R)oo2pq_, rho_p = (R)rho_p_, rho_q = (R)rho_q_;")
        o(f"      (void)PAx; (void)PAy; (void)PAz; (void)WPx; (void)WPy; (void)WPz; (void)QCx; (void)QCy; (void)QCz;")
        o(f"      (void)WQx; (void)WQy; (void)WQz; (void)oo2p; (void)oo2q; (void)oo2pq; (void)rho_p; (void)rho_q;")
        for line in self.vrr_lines:
            o("      " + line)
        for e in ecomps:
            for f in fcomps:
                o(f"      acc[{eidx[e] * nF + fidx[f]}] += {self.vrr_done[(e, f, 0)]};")
        o(f"    }}")
        o(f"  }}")
        # ---------------- HRR bra: h(a, b; f) for |a|=la, |b|=lb from acc
        hb: Dict[Tuple[Cart, Cart], str] = {}
        hlines: List[str] = []
        self.flops_hrr = 0

        def hbra(a: Cart, b: Cart, fi: int) -> str:
            key = (a, b, fi)
            if key in hb:
                return hb[key]
            if sum(b) == 0:
                s = f"acc[{eidx[a] * nF + fi}]"
                hb[key] = s
                return s
            i = pick_dir(b)
            b1 = sub1(b, i)
            x = hbra(add1(a, i), b1, fi)
            y = hbra(a, b1, fi)
            nm = f"hb{cname(a)}_{cname(b)}_{fi}"
            hlines.append(f"const R {nm} = {x} + AB{'xyz'[i]} * {y};")
            self.flops_hrr += 2
            hb[key] = nm
            return nm

        acomps, bcomps = cart_list(la), cart_list(lb)
        ccomps, dcomps = cart_list(lc), cart_list(ld)
        # ---------------- HRR ket: for each (a,b) and |c|=lc,|d|=ld
        hk: Dict = {}

        def hket(a: Cart, b: Cart, c: Cart, d: Cart) -> str:
            key = (a, b, c, d)
            if key in hk:
                return hk[key]
            if sum(d) == 0:
                s = hbra(a, b, fidx[c])
                hk[key] = s
                return s
            i = pick_dir(d)
            d1 = sub1(d, i)
            x = hket(a, b, add1(c, i), d1)
            y = hket(a, b, c, d1)
            nm = f"hk{cname(a)}_{cname(b)}_{cname(c)}_{cname(d)}"
            hlines.append(f"const R {nm} = {x} + CD{'xyz'[i]} * {y};")
            self.flops_hrr += 2
            hk[key] = nm
            return nm

        cart_names: Dict[Tuple[int, int, int, int], str] = {}
        for ia, a in enumerate(acomps):
            for ib, b in enumerate(bcomps):
                for ic, c in enumerate(ccomps):
                    for idd, d in enumerate(dcomps):
                        cart_names[(ia, ib, ic, idd)] = hket(a, b, c, d)
        for line in hlines:
            o("  " + line)
        # ---------------- transform to functions, one index at a time (d, c, b, a)
        na, nb_, nc, nd = len(acomps), len(bcomps), len(ccomps), len(dcomps)
        for pure in (True, False):
            o(f"  if constexpr ({'PURE' if pure else '!PURE'}) {{")
            ra, rb, rc, rd = (transform_rows(l, pure) for l in (la, lb, lc, ld))
            cur = dict(cart_names)
            dims = [na, nb_, nc, nd]
            tag = "s" if pure else "c"
            for axis, rows in ((3, rd), (2, rc), (1, rb), (0, ra)):
                new: Dict[Tuple[int, int, int, int], str] = {}
                newdims = list(dims)
                newdims[axis] = len(rows)
                for idx in _iter(newdims):
                    terms = []
                    for (ci, w) in rows[idx[axis]]:
                        src = list(idx)
                        src[axis] = ci
                        terms.append((w, cur[tuple(src)]))
                    nm = f"t{tag}{axis}_{idx[0]}_{idx[1]}_{idx[2]}_{idx[3]}"
                    if len(terms) == 1 and terms[0][0] == 1.0:
                        new[idx] = terms[0][1]
                        continue
                    o(f"    const R {nm} = " + " + ".join(f"(R){lit(w)} * {s}" for w, s in terms) + ";")
                    new[idx] = nm
                cur = new
                dims = newdims
            nfa, nfb, nfc, nfd = dims
            for idx in _iter(dims):
                flat = ((idx[0] * nfb + idx[1]) * nfc + idx[2]) * nfd + idx[3]
                o(f"    I[{flat}] = {cur[idx]};")
            o("  }")
        o("}")
        o("")


def _iter(dims):
    for a in range(dims[0]):
        for b in range(dims[1]):
            for c in range(dims[2]):
                for d in range(dims[3]):
                    yield (a, b, c, d)


def quartet_classes(lmax: int) -> List[Tuple[int, int, int, int]]:
    pcls = [(a, b) for a in range(lmax + 1) for b in range(a + 1)]
    out = []
    for i, (la, lb) in enumerate(pcls):
        for j in range(i + 1):
            lc, ld = pcls[j]
            out.append((la, lb, lc, ld))
    return out


def pair_classes(lmax: int) -> List[Tuple[int, int]]:
    return [(a, b) for a in range(lmax + 1) for b in range(a + 1)]


def flop_table(lmax: int) -> Dict[str, Dict[str, int]]:
    """Per class: VRR flops per primitive quartet (generated / algorithmic) and
    HRR flops per contracted quartet."""
    res = {}
    for (la, lb, lc, ld) in quartet_classes(lmax):
        g = ClassGen(la, lb, lc, ld)
        lines: List[str] = []
        g.emit(lines)
        res[g.name] = {"vrr": g.flops_vrr, "vrr_alg": g.flops_alg_vrr, "hrr": g.flops_hrr, "L": g.L}
    return res


def main() -> None:
    out_path = sys.argv[1]
    lmax = int(sys.argv[2]) if len(sys.argv) > 2 else 2
    lines: List[str] = ["// Generated by gen_eri.py -- do not edit.", "#pragma once", ""]
    classes = quartet_classes(lmax)
    for (la, lb, lc, ld) in classes:
        ClassGen(la, lb, lc, ld).emit(lines)
    pcls = pair_classes(lmax)
    lines.append(f"#define DSS_GEN_LMAX {lmax}")
    lines.append(f"#define DSS_N_PAIR_CLASSES {len(pcls)}")
    lines.append(f"#define DSS_N_QUARTET_CLASSES {len(classes)}")
    # X-macro listing every class: (la, lb, lc, ld, bra_class, ket_class)
    lines.append("#define DSS_FOR_EACH_CLASS(X) \\")
    items = []
    for (la, lb, lc, ld) in classes:
        items.append(f"  X({la}, {lb}, {lc}, {ld}, {pcls.index((la, lb))}, {pcls.index((lc, ld))})")
    lines.append(" \\\n".join(items))
    lines.append("")
    with open(out_path, "w") as f:
        f.write("\n".join(lines) + "\n")
    write_sph_table(os.path.join(os.path.dirname(os.path.abspath(out_path)), "sph_tab.h"), lmax)


def write_sph_table(path: str, lmax: int) -> None:
    """Host table of the function transforms: for each l <= lmax and each output
    function (5D: m = -l..l; 6D: monomials), the (Cartesian index, weight) terms."""
    out = ["// Generated by gen_eri.py -- do not edit.", "#pragma once", "",
           "struct DssSphTerm { int l; int func; int cart; double w; int pure; };",
           "static const DssSphTerm kDssSphTerms[] = {"]
    for pure in (1, 0):
        for l in range(lmax + 1):
            for fidx, row in enumerate(transform_rows(l, bool(pure))):
                for ci, w in row:
                    out.append(f"  {{{l}, {fidx}, {ci}, {lit(w)}, {pure}}},")
    out.append("};")
    out.append("static const int kDssSphTermCount = sizeof(kDssSphTerms) / sizeof(kDssSphTerms[0]);")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


if __name__ == "__main__":
    main()
