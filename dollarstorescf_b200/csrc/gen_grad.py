"""Generates the derivative-ERI programs of the analytic nuclear gradient
(grad_gen.cuh).

The two-electron part of the gradient (chem/scf/Gradient.cpp:14-133 with the
four-centre term of chem/scf/ExactCoulomb.cpp:125-195) is

  dE_2e/dX = 1/2 sum_{ijkl} Gamma_ijkl d(ij|kl)/dX,
  Gamma_ijkl = D_ij D_kl - sum_s (D^s_ik D^s_jl),

D the total and D^s the spin densities.  A primitive Cartesian Gaussian moves
with its centre A, so

  d/dA_x (a b|c d) = 2 alpha (a+1_x b|c d) - a_x (a-1_x b|c d)

and likewise for B (exponent beta) and C (gamma); translational invariance
gives D = -(A + B + C).  Per shell-quartet class (la lb|lc ld) one program
evaluates, for one primitive quartet, the Obara-Saika VRR to the [e0|f0]^(0)
the shifted classes need and accumulates four contracted sets over the
primitive loop: unweighted (for the a-1, b-1, c-1 terms) and weighted by
2 alpha, 2 beta, 2 gamma.  A second program, once per contracted quartet, runs
the Head-Gordon-Pople HRR of each set to the shifted Cartesian classes
(la+1 lb|, (la lb+1|, |lc+1 ld), (la-1 lb|, (la lb-1|, |lc-1 ld) and contracts
every derivative integral with the quartet's two-particle density in the
Cartesian basis (Gc, the function-basis Gamma carried through the solid-harmonic
or 6D-normalisation transform) into nine sums: d/dA, d/dB, d/dC in x, y, z.

The programs use gen_coop's representation (operations over a per-warp value
array, grouped in dependency levels, value slots reused by liveness).  Record
entries: F_m times the prefactor at 0..L+1, PA 12-14, WP 15-17, QC 18-20, WQ
21-23, 1/2p 24, 1/2q 25, 1/2(p+q) 26, rho/p 27, rho/q 28, 2 alpha 29, 2 beta 30,
2 gamma 31.

Operation encoding (uint4), beyond gen_coop's VRR (kinds 0, 1) and HRR (2):
  weighted accumulate (kind 5): x = dst | src << 16, y = record index of the
    weight (29, 30, 31) or 0xFFFF (weight 1);
  gradient term (kind 6): x = direction (0..8: A x y z, B x y z, C x y z) |
    src_plus << 16, y = src_minus (0xFFFF: none) | Gc index << 16, w = 6 | k << 8:
    g[direction] += Gc[index] * (src_plus - k * src_minus).

Usage: python gen_grad.py OUT.cuh [LMAX]
"""
from __future__ import annotations

import os
import sys
from typing import Dict, List, Optional, Tuple

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import gen_coop as C  # noqa: E402
import gen_eri as G  # noqa: E402

K_WACC, K_GRAD = 5, 6
W_ALPHA, W_BETA, W_GAMMA = 29, 30, 31
SETS = ("u", "a", "b", "c")
SET_WEIGHT = {"u": C.NONE, "a": W_ALPHA, "b": W_BETA, "c": W_GAMMA}


def carts(lo: int, hi: int) -> List[Tuple[int, int, int]]:
    return [c for l in range(max(lo, 0), hi + 1) for c in G.cart_list(l)] if hi >= lo else []


class GradClass:
    """Programs of one class (la >= lb, lc >= ld, bra class >= ket class)."""

    def __init__(self, la: int, lb: int, lc: int, ld: int):
        self.la, self.lb, self.lc, self.ld = la, lb, lc, ld
        E, F = la + lb, lc + ld
        self.L = E + F + 1  # highest Boys order
        # Contracted [e0|f0] each set needs, as (e range, f range) rectangles.
        need: Dict[str, List[Tuple[int, int, int, int]]] = {s: [] for s in SETS}
        need["a"].append((la + 1, E + 1, lc, F))
        need["b"].append((la, E + 1, lc, F))
        need["c"].append((la, E, lc + 1, F + 1))
        if la > 0:
            need["u"].append((la - 1, E - 1, lc, F))
        if lb > 0:
            need["u"].append((la, E - 1, lc, F))
        if lc > 0:
            need["u"].append((la, E, lc - 1, F - 1))
        self.acc_keys: List[Tuple[str, tuple, tuple]] = []
        self.acc_id: Dict[Tuple[str, tuple, tuple], int] = {}
        for s in SETS:
            for (e0, e1, f0, f1) in need[s]:
                for e in carts(e0, e1):
                    for f in carts(f0, f1):
                        k = (s, e, f)
                        if k not in self.acc_id:
                            self.acc_id[k] = len(self.acc_keys)
                            self.acc_keys.append(k)
        self.nacc = len(self.acc_keys)
        self._build_vrr()
        self._build_post()
        self._allocate()

    # ------------------------------------------------------------------ VRR
    def _build_vrr(self) -> None:
        P = C.Program()
        memo: Dict = {}

        def node(e, f, m):
            key = (e, f, m)
            if key in memo:
                return memo[key]
            if sum(e) == 0 and sum(f) == 0:
                memo[key] = C.rec(m)
                return memo[key]
            src: List[Optional[int]] = [None] * 5
            if sum(f) > 0:
                i = G.pick_dir(f)
                f1 = G.sub1(f, i)
                src[0] = node(e, f1, m)
                src[1] = node(e, f1, m + 1)
                k1 = k2 = 0
                if f1[i] > 0:
                    f2 = G.sub1(f1, i)
                    src[2] = node(e, f2, m)
                    src[3] = node(e, f2, m + 1)
                    k1 = f1[i]
                if e[i] > 0:
                    src[4] = node(G.sub1(e, i), f1, m + 1)
                    k2 = e[i]
                op = C.Op(C.K_KET, P.new(), src, axis=i, k1=k1, k2=k2)
            else:
                i = G.pick_dir(e)
                e1 = G.sub1(e, i)
                src[0] = node(e1, f, m)
                src[1] = node(e1, f, m + 1)
                k1 = 0
                if e1[i] > 0:
                    e2 = G.sub1(e1, i)
                    src[2] = node(e2, f, m)
                    src[3] = node(e2, f, m + 1)
                    k1 = e1[i]
                op = C.Op(C.K_BRA, P.new(), src, axis=i, k1=k1)
            P.ops.append(op)
            memo[key] = op.dst
            return op.dst

        self.vrr_out = [node(e, f, 0) for (_, e, f) in self.acc_keys]
        self.Pv = P

    # ------------------------------------------------------------------ HRR + contraction
    def _build_post(self) -> None:
        la, lb, lc, ld = self.la, self.lb, self.lc, self.ld
        P = C.Program()
        P.nodes = self.nacc  # nodes 0..nacc-1: the accumulators
        hb: Dict = {}
        hk: Dict = {}

        def hbra(s, a, b, f):
            key = (s, a, b, f)
            if key in hb:
                return hb[key]
            if sum(b) == 0:
                hb[key] = self.acc_id[(s, a, f)]
                return hb[key]
            i = G.pick_dir(b)
            b1 = G.sub1(b, i)
            x = hbra(s, G.add1(a, i), b1, f)
            y = hbra(s, a, b1, f)
            op = C.Op(C.K_HRR, P.new(), [x, y, None, None, None], axis=i, side=0)
            P.ops.append(op)
            hb[key] = op.dst
            return op.dst

        def hket(s, a, b, c, d):
            key = (s, a, b, c, d)
            if key in hk:
                return hk[key]
            if sum(d) == 0:
                hk[key] = hbra(s, a, b, c)
                return hk[key]
            i = G.pick_dir(d)
            d1 = G.sub1(d, i)
            x = hket(s, a, b, G.add1(c, i), d1)
            y = hket(s, a, b, c, d1)
            op = C.Op(C.K_HRR, P.new(), [x, y, None, None, None], axis=i, side=1)
            P.ops.append(op)
            hk[key] = op.dst
            return op.dst

        A, B, Cc, D = (G.cart_list(l) for l in (la, lb, lc, ld))
        self.grad_ops: List[C.Op] = []
        gi = 0
        for a in A:
            for b in B:
                for c in Cc:
                    for d in D:
                        for centre in range(3):
                            for i in range(3):
                                if centre == 0:
                                    plus = hket("a", G.add1(a, i), b, c, d)
                                    k = a[i]
                                    minus = hket("u", G.sub1(a, i), b, c, d) if k else None
                                elif centre == 1:
                                    plus = hket("b", a, G.add1(b, i), c, d)
                                    k = b[i]
                                    minus = hket("u", a, G.sub1(b, i), c, d) if k else None
                                else:
                                    plus = hket("c", a, b, G.add1(c, i), d)
                                    k = c[i]
                                    minus = hket("u", a, b, G.sub1(c, i), d) if k else None
                                op = C.Op(K_GRAD, -1, [plus, minus, None, None, None], k1=k)
                                op.w = [3 * centre + i, gi]
                                P.ops.append(op)
                        gi += 1
        self.ngc = gi
        self.Pp = P

    # ------------------------------------------------------------------ slots
    def _allocate(self) -> None:
        C.levelize(self.Pv, {})
        vslot, nwork_v = C.allocate(self.Pv, {}, set(self.vrr_out), 0)
        # Post program: accumulators are level-0 inputs; gradient terms write nothing.
        _levelize_post(self.Pp, self.nacc)
        pslot0, nwork_p = _allocate_post(self.Pp, {}, 0)
        work = max(nwork_v, nwork_p)
        acc_pin = {i: work + i for i in range(self.nacc)}
        pslot, nwork_p2 = _allocate_post(self.Pp, acc_pin, 0)
        used = [s for n, s in pslot.items() if n not in acc_pin]
        if used and max(used) >= work:
            work = max(used) + 1
            acc_pin = {i: work + i for i in range(self.nacc)}
            pslot, _ = _allocate_post(self.Pp, acc_pin, 0)
        self.acc_base = work
        self.nslots = work + self.nacc
        self.vrr_ops = [C.encode(op, vslot) for op in sorted(self.Pv.ops, key=lambda o: o.level)]
        self.vrr_levels = C.CoopClass._level_offsets(self.Pv)
        self.wacc_ops = []
        for t, nd in enumerate(self.vrr_out):
            src = (-1 - nd) if nd < 0 else 32 + vslot[nd]
            w = SET_WEIGHT[self.acc_keys[t][0]]
            self.wacc_ops.append((32 + self.acc_base + t | src << 16, w | C.NONE << 16, C.NONE | C.NONE << 16,
                                  K_WACC))
        ops = sorted(self.Pp.ops, key=lambda o: o.level)
        self.post_ops = [_encode_post(op, pslot) for op in ops]
        self.post_levels = C.CoopClass._level_offsets(self.Pp)


def _levelize_post(P: C.Program, nacc: int) -> None:
    lvl: Dict[int, int] = {i: 0 for i in range(nacc)}
    for op in P.ops:
        l = 0
        for s in op.src:
            if s is not None and s >= 0:
                l = max(l, lvl.get(s, 0))
        op.level = l + 1
        if op.kind != K_GRAD:
            lvl[op.dst] = op.level


def _allocate_post(P: C.Program, pinned: Dict[int, int], first_free: int):
    """Slots for the post program's HRR values (gradient terms write none);
    a value's slot is free once the level of its last reader has run."""
    last_use: Dict[int, int] = {}
    for op in P.ops:
        for s in op.src:
            if s is not None and s >= 0:
                last_use[s] = max(last_use.get(s, 0), op.level)
    slot: Dict[int, int] = dict(pinned)
    free: List[int] = []
    nslots = first_free
    by_level: Dict[int, List[C.Op]] = {}
    for op in P.ops:
        by_level.setdefault(op.level, []).append(op)
    release: Dict[int, List[int]] = {}
    for lvl in sorted(by_level):
        for node in release.pop(lvl - 1, []):
            free.append(slot[node])
        for op in by_level[lvl]:
            if op.kind == K_GRAD or op.dst in pinned:
                continue
            if free:
                s = free.pop()
            else:
                s = nslots
                nslots += 1
            slot[op.dst] = s
            release.setdefault(last_use.get(op.dst, lvl), []).append(op.dst)
    return slot, nslots


def _encode_post(op: C.Op, slot: Dict[int, int]) -> Tuple[int, int, int, int]:
    def sidx(n):
        return C.NONE if n is None else 32 + slot[n]

    if op.kind == K_GRAD:
        direction, gi = op.w
        return (direction | sidx(op.src[0]) << 16, sidx(op.src[1]) | gi << 16, C.NONE | C.NONE << 16,
                K_GRAD | op.k1 << 8)
    return C.encode(op, slot)


def cart_function_table(l: int, pure: bool) -> List[List[Tuple[int, float]]]:
    """For each Cartesian component of a shell: the (function, weight) pairs of
    the function transform (gen_eri.transform_rows) that use it."""
    rows = G.transform_rows(l, pure)
    out: List[List[Tuple[int, float]]] = [[] for _ in range(G.ncart(l))]
    for fidx, row in enumerate(rows):
        for ci, w in row:
            out[ci].append((fidx, w))
    return out


# ---------------------------------------------------------------- Python interpreter (tests)
def run_grad(gc: GradClass, prim_records: List[List[float]], AB, CD, Gc: List[float]) -> List[float]:
    """Evaluates the programs on the CPU: prim_records are 32-entry records,
    Gc the Cartesian two-particle density of the quartet.  Returns the nine sums."""
    vals = [0.0] * gc.nslots

    def get(r, idx):
        return r[idx] if idx < 32 else vals[idx - 32]

    for r in prim_records:
        for (x, y, z, w) in gc.vrr_ops:
            dst, s0, s1, s2, s3, s4 = x & 0xFFFF, x >> 16, y & 0xFFFF, y >> 16, z & 0xFFFF, z >> 16
            kind, ax, k1, k2 = w & 15, (w >> 4) & 3, (w >> 8) & 0xFF, (w >> 16) & 0xFF
            if kind == C.K_BRA:
                v = r[C.OFF_PA + ax] * get(r, s0) + r[C.OFF_WP + ax] * get(r, s1)
                if s2 != C.NONE:
                    v += k1 * r[C.OFF_OO2P] * (get(r, s2) - r[C.OFF_RHOP] * get(r, s3))
            else:
                v = r[C.OFF_QC + ax] * get(r, s0) + r[C.OFF_WQ + ax] * get(r, s1)
                if s2 != C.NONE:
                    v += k1 * r[C.OFF_OO2Q] * (get(r, s2) - r[C.OFF_RHOQ] * get(r, s3))
                if s4 != C.NONE:
                    v += k2 * r[C.OFF_OO2PQ] * get(r, s4)
            vals[dst - 32] = v
        for (x, y, z, w) in gc.wacc_ops:
            dst, src, widx = x & 0xFFFF, x >> 16, y & 0xFFFF
            vals[dst - 32] += (1.0 if widx == C.NONE else r[widx]) * get(r, src)
    hdr = list(AB) + list(CD)
    g = [0.0] * 9
    for (x, y, z, w) in gc.post_ops:
        kind = w & 15
        if kind == C.K_HRR:
            dst, s0, s1 = x & 0xFFFF, x >> 16, y & 0xFFFF
            ax, side = (w >> 4) & 3, (w >> 6) & 1
            vals[dst - 32] = vals[s0 - 32] + hdr[3 * side + ax] * vals[s1 - 32]
        else:
            direction, sp, sm, gi, k = x & 0xFFFF, x >> 16, y & 0xFFFF, y >> 16, (w >> 8) & 0xFF
            v = vals[sp - 32]
            if sm != C.NONE:
                v -= k * vals[sm - 32]
            g[direction] += Gc[gi] * v
    return g


def emit(path: str, lmax: int) -> None:
    lines = ["// Generated by gen_grad.py -- do not edit.", "#pragma once", "#include <cuda_runtime.h>", ""]
    classes = G.quartet_classes(lmax)
    for (la, lb, lc, ld) in classes:
        gc = GradClass(la, lb, lc, ld)
        tag = f"{la}{lb}{lc}{ld}"

        def arr(name, ops):
            lines.append(f"static __device__ const uint4 {name}[{max(1, len(ops))}] = {{")
            for o in ops:
                lines.append("  {%du, %du, %du, %du}," % o)
            if not ops:
                lines.append("  {0u, 0u, 0u, 0u},")
            lines.append("};")

        arr(f"kGradVrr_{tag}", gc.vrr_ops)
        arr(f"kGradAcc_{tag}", gc.wacc_ops)
        arr(f"kGradPost_{tag}", gc.post_ops)
        for nm, offs in (("VrrLv", gc.vrr_levels), ("PostLv", gc.post_levels)):
            lines.append(f"static __device__ const unsigned short kGrad{nm}_{tag}[{len(offs)}] = {{" +
                         ", ".join(str(v) for v in offs) + "};")
        lines.append(f"#define DSS_GRAD_{tag}_NSLOTS {gc.nslots}")
        lines.append(f"#define DSS_GRAD_{tag}_NACC {gc.nacc}")
        lines.append(f"#define DSS_GRAD_{tag}_ACC_BASE {gc.acc_base}")
        lines.append(f"#define DSS_GRAD_{tag}_NVLV {len(gc.vrr_levels) - 1}")
        lines.append(f"#define DSS_GRAD_{tag}_NPLV {len(gc.post_levels) - 1}")
        lines.append("")
    # Cartesian component -> (function, weight) pairs per (pure, l): at most 3 each.
    for pure in (1, 0):
        for l in range(lmax + 1):
            tab = cart_function_table(l, bool(pure))
            assert all(len(t) <= 3 for t in tab)
            ents = []
            for t in tab:
                t = t + [(-1, 0.0)] * (3 - len(t))
                ents.append("{" + ", ".join(f"{{{f}, {G.lit(w)}}}" for f, w in t) + "}")
            lines.append(f"static __device__ const DssCartFun kGradCF_{'s' if pure else 'c'}{l}[{len(tab)}][3] = {{" +
                         ", ".join(ents) + "};")
    lines.append("")
    lines.append("#define DSS_FOR_EACH_GRAD_CLASS(X) \\")
    lines.append(" \\\n".join(f"  X({la}, {lb}, {lc}, {ld})" for (la, lb, lc, ld) in classes))
    lines.append("")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    emit(sys.argv[1], int(sys.argv[2]) if len(sys.argv) > 2 else 2)
