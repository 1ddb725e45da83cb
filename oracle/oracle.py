"""Test infrastructure (oracle): CPU restatement of the reference's Fock-build
and SCF path, used only by tests/, the smoke check and bench.py's CPU-baseline
leg to check the CUDA path.  The product never imports this module.

Pinning: tests/test_oracle.py checks every function here against the compiled
reference (oracle/_ref/libdssref.so, built by oracle/build_ref.sh) and against
the golden fixtures under tests/golden/ that the same library produced.

Restated pieces (file:line in the reference):
  sph_terms        ContractedGaussian ctor, real solid harmonics
                   chem/GTO.cpp:15-88 (Y-normalisation :32-33)
  prim_norm        primitive normalisation chem/GTO.cpp:90-93
  cart_terms       the 6D convention: one monomial per function with the
                   angular weight sqrt((2l+1)!!/(4 pi (2a-1)!!(2b-1)!!(2c-1)!!))
  eri_tensor       electronRepulsionIntegral chem/GaussianIntegral.cpp:561-642
                   through the C restatement oracle.c
  jk               getExactCoulombMatrix / getExactExchangeMatrix
                   chem/scf/ExactCoulomb.cpp:103-123 (J from the total density,
                   K from the alpha density)
  scf_rhf          solveMOs / runSCFIteration / updateFockMatrix / DIIS
                   chem/scf/SCFSolver.cpp:45-237, chem/scf/SCFDIIS.cpp:19-52,
                   lalib/DIIS.ipp:6-100; calculateEnergies chem/scf/Energy.cpp:21-50
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from typing import Dict, List, Tuple

import numpy as np
from scipy.linalg import lapack

HERE = os.path.dirname(os.path.abspath(__file__))
SO_PATH = os.path.join(HERE, "liboracle.so")
PI_REF = 3.14159265358979  # lalib/MathUtil.hpp:8

_lib = None


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "oracle.c")
    if force or not os.path.isfile(SO_PATH) or os.path.getmtime(SO_PATH) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-o", SO_PATH, src, "-lm"])
    return SO_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(SO_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        L.orc_boys_ref.argtypes = [ctypes.c_double, ctypes.c_uint]
        L.orc_boys_ref.restype = ctypes.c_double
        L.orc_eri_shell.argtypes = [ctypes.c_int] * 4 + [dp] * 4 + [ctypes.c_int, dp, dp] * 4 + [dp]
        L.orc_eri_shell.restype = None
        _lib = L
    return _lib


def boys_ref(x: float, m: int) -> float:
    return lib().orc_boys_ref(float(x), int(m))


# ----------------------------------------------------------------- basis functions
def _fact(n: int) -> float:
    return float(math.factorial(n)) if n > 0 else 1.0


def _dfact(n: int) -> float:
    r = 1.0
    while n > 0:
        r *= n
        n -= 2
    return r


def sph_terms(l: int, m: int) -> Dict[Tuple[int, int, int], float]:
    """Cartesian expansion {(a,b,c): weight} of the reference's real solid
    harmonic (l, m), including its Y-normalisation."""
    am = abs(m)
    cur: Dict[Tuple[int, int, int], float] = {}
    x = am if m <= 0 else am - 1
    i = 0
    while x >= 0:
        cur[(x, am - x, 0)] = cur.get((x, am - x, 0), 0.0) + (-1.0 if i & 1 else 1.0) * math.comb(am, x)
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
            nxt: Dict[Tuple[int, int, int], float] = {}
            for (a, b, c), v in cur.items():
                k = (a, b, c + 1)
                nxt[k] = nxt.get(k, 0.0) + v * (2 * ii + 1) / sf
            for (a, b, c), v in prev.items():
                for k in ((a + 2, b, c), (a, b + 2, c), (a, b, c + 2)):
                    nxt[k] = nxt.get(k, 0.0) - v * (ii + am) / sf
            prev, cur = cur, nxt
    return {k: v * ynorm for k, v in cur.items()}


def cart_list(l: int) -> List[Tuple[int, int, int]]:
    return [(a, b, l - a - b) for a in range(l, -1, -1) for b in range(l - a, -1, -1)]


def cart_weight(a: int, b: int, c: int) -> float:
    l = a + b + c
    return math.sqrt(_dfact(2 * l + 1) / (4.0 * PI_REF * _dfact(2 * a - 1) * _dfact(2 * b - 1) * _dfact(2 * c - 1)))


def prim_norm(l: int, zeta: float) -> float:
    return math.sqrt((2.0 * zeta) ** (l + 1.5) * 2.0 ** (l + 2) / (math.sqrt(PI_REF) * _dfact(2 * l + 1)))


def shell_transform(l: int, pure: bool) -> np.ndarray:
    """Matrix T [nfunc, ncart]: function = sum_c T[f, c] * monomial c."""
    cl = cart_list(l)
    if pure:
        T = np.zeros((2 * l + 1, len(cl)))
        for i, m in enumerate(range(-l, l + 1)):
            for k, v in sph_terms(l, m).items():
                T[i, cl.index(k)] += v
        return T
    return np.diag([cart_weight(*c) for c in cl])


# ----------------------------------------------------------------- integrals
def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def eri_shell_cart(sh, a: int, b: int, c: int, d: int) -> np.ndarray:
    """Contracted Cartesian (ab|cd) with normalised primitive weights."""
    L = lib()
    off = np.concatenate([[0], np.cumsum(sh.shell_nprim)])
    args = []
    for s in (a, b, c, d):
        l = int(sh.shell_l[s])
        e = np.ascontiguousarray(sh.exps[off[s]:off[s + 1]])
        w = np.ascontiguousarray([sh.coefs[k] * prim_norm(l, sh.exps[k]) for k in range(off[s], off[s + 1])],
                                 dtype=np.float64)
        args.append((len(e), e, w))
    ls = [int(sh.shell_l[s]) for s in (a, b, c, d)]
    nc = [(x + 1) * (x + 2) // 2 for x in ls]
    out = np.zeros(int(np.prod(nc)))
    cen = [np.ascontiguousarray(sh.centers[s], dtype=np.float64) for s in (a, b, c, d)]
    flat = []
    for n, e, w in args:
        flat += [n, _dp(e), _dp(w)]
    L.orc_eri_shell(ls[0], ls[1], ls[2], ls[3], _dp(cen[0]), _dp(cen[1]), _dp(cen[2]), _dp(cen[3]), *flat,
                    _dp(out))
    return out.reshape(nc)


def function_offsets(sh) -> np.ndarray:
    nf = [(2 * l + 1) if sh.pure else (l + 1) * (l + 2) // 2 for l in sh.shell_l]
    return np.concatenate([[0], np.cumsum(nf)]).astype(int)


def eri_tensor(sh) -> np.ndarray:
    """Full (mu nu|sigma tau) tensor over basis functions (small systems only)."""
    ns = sh.nshell
    fo = function_offsets(sh)
    n = int(fo[-1])
    Ts = [shell_transform(int(l), sh.pure) for l in sh.shell_l]
    G = np.zeros((n, n, n, n))
    for a in range(ns):
        for b in range(a + 1):
            for c in range(ns):
                for d in range(c + 1):
                    if (a * (a + 1) // 2 + b) < (c * (c + 1) // 2 + d):
                        continue
                    cart = eri_shell_cart(sh, a, b, c, d)
                    v = np.einsum("ia,jb,kc,ld,abcd->ijkl", Ts[a], Ts[b], Ts[c], Ts[d], cart)
                    sa, sb, sc, sd = (slice(fo[x], fo[x + 1]) for x in (a, b, c, d))
                    for (p, q, r, s, t) in ((sa, sb, sc, sd, v), (sb, sa, sc, sd, v.transpose(1, 0, 2, 3)),
                                            (sa, sb, sd, sc, v.transpose(0, 1, 3, 2)),
                                            (sb, sa, sd, sc, v.transpose(1, 0, 3, 2))):
                        G[p, q, r, s] = t
                        G[r, s, p, q] = t.transpose(2, 3, 0, 1)
    return G


def jk(eri: np.ndarray, D_alpha: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """J[2 D_alpha] and K[D_alpha] (dense)."""
    J = np.einsum("mnst,st->mn", eri, 2.0 * D_alpha)
    K = np.einsum("mtsn,st->mn", eri, D_alpha)
    return J, K


# ----------------------------------------------------------------- one-electron (via the reference)
def scf_rhf(S: np.ndarray, H: np.ndarray, eri: np.ndarray, n_alpha: int, e_nuc: float,
            conv: float = 1e-10, diis_size: int = 8, max_iter: int = 500):
    """The reference's RHF loop restated.  Returns (E_total, D_alpha, iterations)."""
    n = S.shape[0]
    s, U = np.linalg.eigh(S)
    X = (U * (1.0 / np.sqrt(s))) @ U.T
    D = np.zeros((n, n))
    E = 0.0
    E_prev = 0.0
    it = 0
    errs: List[np.ndarray] = []
    focks: List[np.ndarray] = []
    B = np.zeros((diis_size + 1, diis_size + 1))
    while True:
        if it and abs(E - E_prev) < conv:
            break
        if it >= max_iter:
            raise RuntimeError("oracle SCF did not converge")
        it += 1
        J, K = jk(eri, D)
        G = J - K
        Fnew = H + G
        if it == 1:
            F = Fnew
        else:
            spf = S @ (D @ Fnew)
            e = spf - spf.T
            rms = float(np.sum(e * e))
            if len(errs) < diis_size:
                idx = len(errs)
                errs.append(e)
                focks.append(Fnew)
            else:
                idx = int(np.argmax([B[i, i] for i in range(diis_size)]))
                errs[idx] = e
                focks[idx] = Fnew
            cnt = len(errs)
            B[idx, idx] = rms
            for i in range(cnt):
                if i != idx:
                    B[i, idx] = B[idx, i] = float(np.sum(errs[i] * e))
            if cnt <= 1:
                F = focks[0]
            else:
                M = np.zeros((cnt + 1, cnt + 1))
                M[:cnt, :cnt] = B[:cnt, :cnt]
                M[:cnt, cnt] = M[cnt, :cnt] = 1.0
                rhs = np.zeros(cnt + 1)
                rhs[cnt] = 1.0
                # dspsv (lalib/Lapack.cpp:145-170): Bunch-Kaufman LDL^T.  When D is
                # exactly singular LAPACK reports info > 0, skips the solve and the
                # reference keeps the right-hand side as the coefficients.
                _, _, c, info = lapack.dsysv(M, rhs, lower=0)
                if info > 0:
                    c = rhs
                F = sum(c[i] * focks[i] for i in range(cnt))
        eps, Cp = np.linalg.eigh(X @ F @ X)
        C = X @ Cp
        D = C[:, :n_alpha] @ C[:, :n_alpha].T
        E_prev = E
        E = 2.0 * float(np.sum(eps[:n_alpha])) - float(np.sum(D * G))
    J, K = jk(eri, D)
    E_tot = 2.0 * float(np.sum(D * H)) + float(np.sum(D * J)) - float(np.sum(D * K)) + e_nuc
    return E_tot, D, it


def _diis_ring(B, errs, focks, e, Fnew, diis_size):
    """One Pulay DIIS step of lalib/DIIS.ipp:19-100 (ring, bordered B, dspsv);
    returns the extrapolated Fock matrix."""
    rms = float(np.sum(e * e))
    if len(errs) < diis_size:
        idx = len(errs)
        errs.append(e)
        focks.append(Fnew)
    else:
        idx = int(np.argmax([B[i, i] for i in range(diis_size)]))
        errs[idx] = e
        focks[idx] = Fnew
    cnt = len(errs)
    B[idx, idx] = rms
    for i in range(cnt):
        if i != idx:
            B[i, idx] = B[idx, i] = float(np.sum(errs[i] * e))
    if cnt <= 1:
        return focks[0]
    M = np.zeros((cnt + 1, cnt + 1))
    M[:cnt, :cnt] = B[:cnt, :cnt]
    M[:cnt, cnt] = M[cnt, :cnt] = 1.0
    rhs = np.zeros(cnt + 1)
    rhs[cnt] = 1.0
    _, _, c, info = lapack.dsysv(M, rhs, lower=0)
    if info > 0:
        c = rhs
    return sum(c[i] * focks[i] for i in range(cnt))


def scf_uhf(S: np.ndarray, H: np.ndarray, eri: np.ndarray, n_alpha: int, n_beta: int, e_nuc: float,
            conv: float = 1e-10, diis_size: int = 8, max_iter: int = 500, guess=None):
    """The reference's unrestricted loop restated (chem/scf/SCFSolver.cpp:120-172,
    196-237; one DIIS solver per spin, chem/scf/SCFDIIS.cpp:14-52; final energy
    chem/scf/Energy.cpp:21-50).  Returns (E_total, D_alpha, D_beta, iterations).
    guess: optional dense (D_alpha, D_beta) that replaces the core guess (zero
    densities) as the start of the same loop, the restart of a checkpoint."""
    n = S.shape[0]
    s, U = np.linalg.eigh(S)
    X = (U * (1.0 / np.sqrt(s))) @ U.T
    if guess is None:
        D = [np.zeros((n, n)), np.zeros((n, n))]
    else:
        D = [np.array(guess[0], dtype=float), np.array(guess[1], dtype=float)]
    nocc = (n_alpha, n_beta)
    E = 0.0
    E_prev = 0.0
    it = 0
    rings = [([], [], np.zeros((diis_size + 1, diis_size + 1))) for _ in range(2)]
    while True:
        if it and abs(E - E_prev) < conv:
            break
        if it >= max_iter:
            raise RuntimeError("oracle UHF did not converge")
        it += 1
        Dt = D[0] + D[1]
        J = np.einsum("mnst,st->mn", eri, Dt)
        G = [J - np.einsum("mtsn,st->mn", eri, D[sp]) for sp in range(2)]
        F = []
        for sp in range(2):
            Fnew = H + G[sp]
            if it == 1:
                F.append(Fnew)
            else:
                spf = S @ (D[sp] @ Fnew)
                errs, focks, B = rings[sp]
                F.append(_diis_ring(B, errs, focks, spf - spf.T, Fnew, diis_size))
        eps = []
        for sp in range(2):
            e_s, Cp = np.linalg.eigh(X @ F[sp] @ X)
            C = X @ Cp
            D[sp] = C[:, :nocc[sp]] @ C[:, :nocc[sp]].T
            eps.append(e_s)
        E_prev = E
        E = (float(np.sum(eps[0][:n_alpha])) + float(np.sum(eps[1][:n_beta]))
             - 0.5 * float(np.sum(D[0] * G[0])) - 0.5 * float(np.sum(D[1] * G[1])))
    Dt = D[0] + D[1]
    J = np.einsum("mnst,st->mn", eri, Dt)
    Ks = [np.einsum("mtsn,st->mn", eri, D[sp]) for sp in range(2)]
    E_tot = (float(np.sum(Dt * H)) + 0.5 * float(np.sum(Dt * J))
             - 0.5 * float(np.sum(D[0] * Ks[0])) - 0.5 * float(np.sum(D[1] * Ks[1])) + e_nuc)
    return E_tot, D[0], D[1], it
