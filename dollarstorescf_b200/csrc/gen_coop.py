"""Generates the warp-cooperative ERI programs (coop_gen.cuh).

For the high-angular-momentum classes one thread per quartet needs far more
live values than a thread has registers ((dd|dd): 961 contracted VRR outputs,
1296 Cartesian integrals).  Those classes run instead as one warp per quartet:
the same recurrences as gen_eri.py (Obara-Saika VRR per primitive quartet,
accumulation, Head-Gordon-Pople HRR, function transform) are written as two
straight "programs" of small operations on a per-warp shared-memory value
array.  Operations are grouped in dependency levels; the 32 lanes execute the
operations of one level in parallel and synchronise between levels.  Value
slots are reused once every reader of a value has run (liveness by level).

Value index space of an operation: indices < 32 address the primitive-quartet
record (F_m times the prefactor at 0..L, then PA, WP, QC, WQ, 1/2p, 1/2q,
1/2(p+q), rho/p, rho/q at 12..28); indices >= 32 address value slot (i - 32).

Operation encoding (uint4):
  x = dst | s0 << 16,  y = s1 | s2 << 16,  z = s3 | s4 << 16,
  w = kind | axis << 4 | side << 6 | k1 << 8 | k2 << 16 (VRR/HRR/acc),
  transform: z = w0 | w1 << 16 (weight-table indices), w = kind | w2 << 16.
kinds: 0 bra VRR, 1 ket VRR, 2 HRR (side 0: AB, 1: CD), 3 transform, 4 accumulate.

Usage: python gen_coop.py OUT.cuh [LMAX]
"""
from __future__ import annotations

import os
import sys
from typing import Dict, List, Optional, Tuple

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import gen_eri as G  # noqa: E402

NONE = 0xFFFF
REC = 32  # doubles per primitive-quartet record
OFF_PA, OFF_WP, OFF_QC, OFF_WQ = 12, 15, 18, 21
OFF_OO2P, OFF_OO2Q, OFF_OO2PQ, OFF_RHOP, OFF_RHOQ = 24, 25, 26, 27, 28

K_BRA, K_KET, K_HRR, K_TRF, K_ACC = 0, 1, 2, 3, 4


class Op:
    __slots__ = ("kind", "dst", "src", "axis", "side", "k1", "k2", "w", "level")

    def __init__(self, kind, dst, src, axis=0, side=0, k1=0, k2=0, w=None):
        self.kind = kind
        self.dst = dst  # node id
        self.src = src  # list of node ids or None (5 entries)
        self.axis = axis
        self.side = side
        self.k1 = k1
        self.k2 = k2
        self.w = w or []
        self.level = 0


class Program:
    """Ops over node ids; node ids < 0 are fixed record entries (-1 - index)."""

    def __init__(self):
        self.ops: List[Op] = []
        self.nodes = 0

    def new(self) -> int:
        self.nodes += 1
        return self.nodes - 1


def rec(i: int) -> int:
    return -1 - i


def build_vrr(la, lb, lc, ld):
    E, F = la + lb, lc + ld
    L = E + F
    ecomps = [c for l in range(la, E + 1) for c in G.cart_list(l)]
    fcomps = [c for l in range(lc, F + 1) for c in G.cart_list(l)]
    P = Program()
    memo: Dict = {}

    def node(e, f, m):
        key = (e, f, m)
        if key in memo:
            return memo[key]
        if sum(e) == 0 and sum(f) == 0:
            memo[key] = rec(m)
            return memo[key]
        src = [None] * 5
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
            op = Op(K_KET, P.new(), src, axis=i, k1=k1, k2=k2)
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
            op = Op(K_BRA, P.new(), src, axis=i, k1=k1)
        P.ops.append(op)
        memo[key] = op.dst
        return op.dst

    outs = []
    for e in ecomps:
        for f in fcomps:
            outs.append(node(e, f, 0))
    return P, outs, ecomps, fcomps, L


def build_hrr(la, lb, lc, ld, pure, ecomps, fcomps):
    """HRR + transform over the accumulator nodes acc[e][f] (node ids 0..nE*nF-1)."""
    P = Program()
    nE, nF = len(ecomps), len(fcomps)
    P.nodes = nE * nF
    eidx = {c: i for i, c in enumerate(ecomps)}
    fidx = {c: i for i, c in enumerate(fcomps)}
    hb: Dict = {}

    def hbra(a, b, fi):
        key = (a, b, fi)
        if key in hb:
            return hb[key]
        if sum(b) == 0:
            hb[key] = eidx[a] * nF + fi
            return hb[key]
        i = G.pick_dir(b)
        b1 = G.sub1(b, i)
        x = hbra(G.add1(a, i), b1, fi)
        y = hbra(a, b1, fi)
        op = Op(K_HRR, P.new(), [x, y, None, None, None], axis=i, side=0)
        P.ops.append(op)
        hb[key] = op.dst
        return op.dst

    hk: Dict = {}

    def hket(a, b, c, d):
        key = (a, b, c, d)
        if key in hk:
            return hk[key]
        if sum(d) == 0:
            hk[key] = hbra(a, b, fidx[c])
            return hk[key]
        i = G.pick_dir(d)
        d1 = G.sub1(d, i)
        x = hket(a, b, G.add1(c, i), d1)
        y = hket(a, b, c, d1)
        op = Op(K_HRR, P.new(), [x, y, None, None, None], axis=i, side=1)
        P.ops.append(op)
        hk[key] = op.dst
        return op.dst

    A, B, C, D = (G.cart_list(l) for l in (la, lb, lc, ld))
    cart = {}
    for ia, a in enumerate(A):
        for ib, b in enumerate(B):
            for ic, c in enumerate(C):
                for idd, d in enumerate(D):
                    cart[(ia, ib, ic, idd)] = hket(a, b, c, d)
    # transform one index at a time: d, c, b, a
    dims = [len(A), len(B), len(C), len(D)]
    cur = dict(cart)
    weights: List[float] = []
    widx: Dict[float, int] = {}

    def wi(v):
        if v not in widx:
            widx[v] = len(weights)
            weights.append(v)
        return widx[v]

    for axis, l in ((3, ld), (2, lc), (1, lb), (0, la)):
        rows = G.transform_rows(l, pure)
        new = {}
        nd = list(dims)
        nd[axis] = len(rows)
        for idx in G._iter(nd):
            terms = []
            for (ci, w) in rows[idx[axis]]:
                s = list(idx)
                s[axis] = ci
                terms.append((w, cur[tuple(s)]))
            if len(terms) == 1 and terms[0][0] == 1.0:
                new[idx] = terms[0][1]
                continue
            assert len(terms) <= 3
            src = [t[1] for t in terms] + [None] * (5 - len(terms))
            op = Op(K_TRF, P.new(), src, w=[wi(t[0]) for t in terms])
            P.ops.append(op)
            new[idx] = op.dst
        cur = new
        dims = nd
    finals = [cur[idx] for idx in G._iter(dims)]
    return P, finals, weights, dims


def levelize(P: Program, fixed_level: Dict[int, int]):
    lvl: Dict[int, int] = dict(fixed_level)
    for op in P.ops:  # ops are created in dependency order
        l = 0
        for s in op.src:
            if s is None or s < 0:
                continue
            l = max(l, lvl.get(s, 0))
        op.level = l + 1
        lvl[op.dst] = op.level
    return max((op.level for op in P.ops), default=0)


def allocate(P: Program, pinned_slots: Dict[int, int], keep: set, first_free: int):
    """Assign slots to op destinations.  pinned_slots: node -> slot (inputs /
    fixed outputs).  keep: nodes never freed.  Returns node -> slot, slot count."""
    last_use: Dict[int, int] = {}
    for op in P.ops:
        for s in op.src:
            if s is not None and s >= 0:
                last_use[s] = max(last_use.get(s, 0), op.level)
    slot: Dict[int, int] = dict(pinned_slots)
    free: List[int] = []
    nslots = first_free
    by_level: Dict[int, List[Op]] = {}
    for op in P.ops:
        by_level.setdefault(op.level, []).append(op)
    live_by_release: Dict[int, List[int]] = {}
    for lvl in sorted(by_level):
        # values whose last reader ran in an earlier level are free now
        for node in live_by_release.pop(lvl - 1, []):
            free.append(slot[node])
        for op in by_level[lvl]:
            if op.dst in pinned_slots:
                continue
            if free:
                s = free.pop()
            else:
                s = nslots
                nslots += 1
            slot[op.dst] = s
            if op.dst not in keep:
                lu = last_use.get(op.dst)
                if lu is None:
                    free_after = lvl  # never read: free after this level
                else:
                    free_after = lu
                live_by_release.setdefault(free_after, []).append(op.dst)
        # release earlier-level inputs (pinned, not kept) handled only for op outputs
    return slot, nslots


def encode(op: Op, slot: Dict[int, int], acc_base: Optional[int] = None) -> Tuple[int, int, int, int]:
    def sidx(n):
        if n is None:
            return NONE
        if n < 0:
            return -1 - n  # record entry
        return 32 + slot[n]

    s = [sidx(x) for x in op.src]
    dst = 32 + slot[op.dst]
    if op.kind == K_TRF:
        w = op.w + [0] * (3 - len(op.w))
        return (dst | s[0] << 16, s[1] | s[2] << 16, w[0] | w[1] << 16, K_TRF | w[2] << 16)
    return (dst | s[0] << 16, s[1] | s[2] << 16, s[3] | s[4] << 16,
            op.kind | op.axis << 4 | op.side << 6 | op.k1 << 8 | op.k2 << 16)


class CoopClass:
    def __init__(self, la, lb, lc, ld, pure):
        self.la, self.lb, self.lc, self.ld, self.pure = la, lb, lc, ld, pure
        Pv, outs, ecomps, fcomps, L = build_vrr(la, lb, lc, ld)
        self.L = L
        nacc = len(ecomps) * len(fcomps)
        nv_levels = levelize(Pv, {})
        # VRR program: working slots from 0; outputs are ordinary nodes.
        vslot, nwork_v = allocate(Pv, {}, set(outs), 0)
        # acc region follows the largest working area of both programs; decided below
        Ph, finals, weights, dims = build_hrr(la, lb, lc, ld, pure, ecomps, fcomps)
        nh_levels = levelize(Ph, {i: 0 for i in range(nacc)})
        # HRR inputs are the accumulators; they live in a region that the VRR
        # program never writes.  Working slots of the HRR program reuse slot 0..
        hslot_tmp, nwork_h = allocate(Ph, {}, set(finals), 0)
        self.nwork = max(nwork_v, nwork_h)
        self.acc_base = self.nwork
        acc_pin = {i: self.acc_base + i for i in range(nacc)}
        hslot, nwork_h2 = allocate(Ph, acc_pin, set(finals), 0)
        # the allocator never hands out pinned slots; make sure working slots stay below acc_base
        used = [s for n, s in hslot.items() if n not in acc_pin]
        if used and max(used) >= self.acc_base:
            # grow the working area and pin again
            self.nwork = max(used) + 1
            self.acc_base = self.nwork
            acc_pin = {i: self.acc_base + i for i in range(nacc)}
            hslot, _ = allocate(Ph, acc_pin, set(finals), 0)
        self.nslots = self.acc_base + nacc
        self.vrr_ops = [encode(op, vslot) for op in sorted(Pv.ops, key=lambda o: o.level)]
        self.vrr_levels = self._level_offsets(Pv)
        # accumulate ops: acc[t] += out_t
        self.acc_ops = []
        for t, nd in enumerate(outs):
            src = NONE if nd < 0 else 32 + vslot[nd]
            if nd < 0:
                src = -1 - nd
            self.acc_ops.append((32 + self.acc_base + t | src << 16, NONE | NONE << 16, NONE | NONE << 16, K_ACC))
        self.hrr_ops = [encode(op, hslot) for op in sorted(Ph.ops, key=lambda o: o.level)]
        self.hrr_levels = self._level_offsets(Ph)
        self.final_slots = [32 + hslot[n] if n >= 0 and n not in acc_pin else
                            (32 + acc_pin[n] if n in acc_pin else None) for n in finals]
        self.weights = weights
        self.dims = dims
        self.nacc = nacc

    @staticmethod
    def _level_offsets(P):
        ops = sorted(P.ops, key=lambda o: o.level)
        offs = [0]
        cur = ops[0].level if ops else 0
        for i, op in enumerate(ops):
            if op.level != cur:
                offs.append(i)
                cur = op.level
        offs.append(len(ops))
        return offs


# ---------------------------------------------------------------- Python interpreter (tests)
def run_coop(cc: CoopClass, prim_records: List[List[float]], AB, CD) -> List[float]:
    """Evaluates the programs on the CPU: prim_records are 32-entry records."""
    vals = [0.0] * cc.nslots
    hdr = list(AB) + list(CD)

    def get(rec_, idx):
        return rec_[idx] if idx < 32 else vals[idx - 32]

    for r in prim_records:
        for (x, y, z, w) in cc.vrr_ops:
            dst, s0, s1, s2, s3, s4 = x & 0xFFFF, x >> 16, y & 0xFFFF, y >> 16, z & 0xFFFF, z >> 16
            kind, ax, k1, k2 = w & 15, (w >> 4) & 3, (w >> 8) & 0xFF, (w >> 16) & 0xFF
            if kind == K_BRA:
                v = r[OFF_PA + ax] * get(r, s0) + r[OFF_WP + ax] * get(r, s1)
                if s2 != NONE:
                    v += k1 * r[OFF_OO2P] * (get(r, s2) - r[OFF_RHOP] * get(r, s3))
            else:
                v = r[OFF_QC + ax] * get(r, s0) + r[OFF_WQ + ax] * get(r, s1)
                if s2 != NONE:
                    v += k1 * r[OFF_OO2Q] * (get(r, s2) - r[OFF_RHOQ] * get(r, s3))
                if s4 != NONE:
                    v += k2 * r[OFF_OO2PQ] * get(r, s4)
            vals[dst - 32] = v
        for (x, y, z, w) in cc.acc_ops:
            dst, s0 = x & 0xFFFF, x >> 16
            vals[dst - 32] += get(r, s0)
    dummy = [0.0] * 32
    for (x, y, z, w) in cc.hrr_ops:
        dst, s0, s1, s2 = x & 0xFFFF, x >> 16, y & 0xFFFF, y >> 16
        kind = w & 15
        if kind == K_HRR:
            ax, side = (w >> 4) & 3, (w >> 6) & 1
            v = get(dummy, s0) + hdr[3 * side + ax] * get(dummy, s1)
        else:
            w0, w1, w2 = z & 0xFFFF, z >> 16, w >> 16
            v = cc.weights[w0] * get(dummy, s0)
            if s1 != NONE:
                v += cc.weights[w1] * get(dummy, s1)
            if s2 != NONE:
                v += cc.weights[w2] * get(dummy, s2)
        vals[dst - 32] = v
    return [vals[s - 32] for s in cc.final_slots]


def coop_classes(lmax: int, min_ops: int = 600):
    """Classes that run warp-cooperatively: those with at least min_ops VRR
    operations or 150 accumulated outputs."""
    out = []
    for (la, lb, lc, ld) in G.quartet_classes(lmax):
        Pv, outs, ecomps, fcomps, L = build_vrr(la, lb, lc, ld)
        if len(Pv.ops) >= min_ops or len(outs) >= 150:
            out.append((la, lb, lc, ld))
    return out


def emit(path: str, lmax: int) -> None:
    lines = ["// Generated by gen_coop.py -- do not edit.", "#pragma once", "#include <cuda_runtime.h>", ""]
    classes = coop_classes(lmax)
    for (la, lb, lc, ld) in classes:
        for pure in (1, 0):
            cc = CoopClass(la, lb, lc, ld, bool(pure))
            tag = f"{la}{lb}{lc}{ld}_{'s' if pure else 'c'}"
            def arr(name, ops):
                lines.append(f"static __device__ const uint4 {name}[{max(1, len(ops))}] = {{")
                for o in ops:
                    lines.append("  {%du, %du, %du, %du}," % o)
                if not ops:
                    lines.append("  {0u, 0u, 0u, 0u},")
                lines.append("};")
            arr(f"kCoopVrr_{tag}", cc.vrr_ops)
            arr(f"kCoopAcc_{tag}", cc.acc_ops)
            arr(f"kCoopHrr_{tag}", cc.hrr_ops)
            for nm, offs in (("VrrLv", cc.vrr_levels), ("HrrLv", cc.hrr_levels)):
                lines.append(f"static __device__ const unsigned short kCoop{nm}_{tag}[{len(offs)}] = {{" +
                             ", ".join(str(v) for v in offs) + "};")
            lines.append(f"static __device__ const double kCoopW_{tag}[{max(1, len(cc.weights))}] = {{" +
                         ", ".join(G.lit(v) for v in (cc.weights or [0.0])) + "};")
            lines.append(f"static __device__ const unsigned short kCoopOut_{tag}[{len(cc.final_slots)}] = {{" +
                         ", ".join(str(v) for v in cc.final_slots) + "};")
            lines.append(f"#define DSS_COOP_{tag}_NSLOTS {cc.nslots}")
            lines.append(f"#define DSS_COOP_{tag}_NACC {cc.nacc}")
            lines.append(f"#define DSS_COOP_{tag}_ACC_BASE {cc.acc_base}")
            lines.append(f"#define DSS_COOP_{tag}_NVRR {len(cc.vrr_ops)}")
            lines.append(f"#define DSS_COOP_{tag}_NVLV {len(cc.vrr_levels) - 1}")
            lines.append(f"#define DSS_COOP_{tag}_NHRR {len(cc.hrr_ops)}")
            lines.append(f"#define DSS_COOP_{tag}_NHLV {len(cc.hrr_levels) - 1}")
            lines.append("")
    lines.append("#define DSS_FOR_EACH_COOP_CLASS(X) \\")
    lines.append(" \\\n".join(f"  X({la}, {lb}, {lc}, {ld})" for (la, lb, lc, ld) in classes))
    lines.append("")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    emit(sys.argv[1], int(sys.argv[2]) if len(sys.argv) > 2 else 2)
