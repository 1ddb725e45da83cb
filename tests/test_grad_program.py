"""The derivative-ERI programs of the analytic gradient (csrc/gen_grad.py),
run by their Python interpreter on the CPU: for shell quartets of every kind
the nine sums (d/dA, d/dB, d/dC in x, y, z of the Cartesian integrals
contracted with a random two-particle density) must equal central differences
of the oracle's contracted Cartesian integrals with the shells displaced
(chem/GaussianIntegral.cpp:1052-1459 differentiates the same primitives).
Every shell sits on its own centre so each displacement moves one position;
D's derivative is -(A + B + C).  Tolerance 1e-7 relative to the largest term
(the difference quotient's O(h^2) error at h = 1e-4 bohr is ~1e-8)."""
import copy
import itertools
import math
import os
import sys

import numpy as np
import pytest
from scipy.special import gamma, gammainc

from dollarstorescf_b200 import basis, geometry, shells
from oracle import oracle

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "dollarstorescf_b200",
                                "csrc"))
import gen_grad  # noqa: E402

H = 1e-4


def boys(m, T):
    if T < 1e-12:
        return 1.0 / (2 * m + 1)
    return gamma(m + 0.5) * gammainc(m + 0.5, T) / (2 * T ** (m + 0.5))


def records(sh, quartet, L):
    off = np.concatenate([[0], np.cumsum(sh.shell_nprim)])

    def prims(s):
        l = int(sh.shell_l[s])
        return [(sh.exps[k], sh.coefs[k] * oracle.prim_norm(l, sh.exps[k])) for k in range(off[s], off[s + 1])]

    A, B, C, D = (np.array(sh.centers[s], float) for s in quartet)
    out = []
    for (al, wa), (be, wb), (ga, wc), (de, wd) in itertools.product(*(prims(s) for s in quartet)):
        p, q = al + be, ga + de
        P, Q = (al * A + be * B) / p, (ga * C + de * D) / q
        kab = wa * wb * math.exp(-al * be / p * np.dot(A - B, A - B))
        kcd = wc * wd * math.exp(-ga * de / q * np.dot(C - D, C - D))
        rho = p * q / (p + q)
        W = (p * P + q * Q) / (p + q)
        pref = 2 * math.pi ** 2.5 / (p * q * math.sqrt(p + q)) * kab * kcd
        T = rho * np.dot(P - Q, P - Q)
        r = [0.0] * 32
        for m in range(L + 1):
            r[m] = boys(m, T) * pref
        r[12:15], r[15:18], r[18:21], r[21:24] = list(P - A), list(W - P), list(Q - C), list(W - Q)
        r[24], r[25], r[26], r[27], r[28] = 0.5 / p, 0.5 / q, 0.5 / (p + q), rho / p, rho / q
        r[29], r[30], r[31] = 2 * al, 2 * be, 2 * ga
        out.append(r)
    return out


@pytest.fixture(scope="module")
def spread_water():
    sh = shells.build_shells(geometry.water(), basis.builtin_basis("6-31G*"), pure=False)
    sh.centers = sh.centers + np.random.default_rng(3).standard_normal(sh.centers.shape) * 0.7
    return sh


# water 6-31G*: shells 0-5 on O (s s p s p d), 6-9 on the hydrogens (s s, s s)
QUARTETS = [(0, 6, 1, 8), (2, 0, 6, 6), (4, 2, 8, 1), (5, 2, 4, 0), (5, 5, 2, 4), (5, 4, 5, 2), (2, 9, 4, 7),
            (5, 3, 5, 5), (5, 5, 5, 4), (2, 2, 2, 2)]


@pytest.mark.parametrize("quartet", QUARTETS)
def test_gradient_program_matches_difference_quotient(spread_water, quartet):
    sh = spread_water
    ls = [int(sh.shell_l[s]) for s in quartet]
    gc = gen_grad.GradClass(*ls)
    recs = records(sh, quartet, gc.L)
    rng = np.random.default_rng(sum(quartet))
    Gc = rng.standard_normal(int(np.prod([(l + 1) * (l + 2) // 2 for l in ls])))
    A, B, C, D = (np.array(sh.centers[s], float) for s in quartet)
    g = np.array(gen_grad.run_grad(gc, recs, A - B, C - D, list(Gc))).reshape(3, 3)
    per = {}
    for pos, s in enumerate(quartet):
        per.setdefault(s, np.zeros(3))
        per[s] += g[pos] if pos < 3 else -g.sum(axis=0)
    base = sh.centers.copy()
    err = scale = 0.0
    for s, v in per.items():
        for i in range(3):
            vals = []
            for sign in (1.0, -1.0):
                sh2 = copy.deepcopy(sh)
                sh2.centers = base.copy()
                sh2.centers[s, i] += sign * H
                vals.append(oracle.eri_shell_cart(sh2, *quartet).ravel())
            fd = float(np.dot(Gc, (vals[0] - vals[1]) / (2 * H)))
            err = max(err, abs(fd - v[i]))
            scale = max(scale, abs(fd))
    assert err <= 1e-7 * max(scale, 1.0), (err, scale)


def test_programs_fit_one_warp_of_shared_memory():
    # The heaviest class, (dd|dd): values + records + Gc + density blocks under 227 KB.
    gc = gen_grad.GradClass(2, 2, 2, 2)
    doubles = gc.nslots + 8 * 32 + 8 + 6 ** 4 + 2 * (36 + 36 + 2 * (4 * 36))
    assert doubles * 8 <= 227 * 1024
