"""Test infrastructure (oracle): ctypes wrapper of oracle/_ref/libdssref.so, the
unmodified DollarStoreSCF sources driven by oracle/ref_harness.cpp.

Only tests, the smoke check and bench.py's reference arm use this module.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", os.environ.get("DSS_REF_LIB", "libdssref.so"))

_lib = None


def available() -> bool:
    return os.path.isfile(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} not built (oracle/build_ref.sh)")
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.ref_setup.argtypes = [ctypes.c_int, ip, dp, ctypes.c_int, ip, ip, ip, dp, dp,
                                ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.ref_setup.restype = ctypes.c_int
        L.ref_nbf.restype = ctypes.c_int
        L.ref_get_overlap.argtypes = [dp]
        L.ref_get_core_hamiltonian.argtypes = [dp]
        L.ref_basis_terms.argtypes = [ctypes.c_int, dp, ip]
        L.ref_basis_terms.restype = ctypes.c_int
        L.ref_basis_prims.argtypes = [ctypes.c_int, dp, dp]
        L.ref_basis_prims.restype = ctypes.c_int
        L.ref_scf.argtypes = [ctypes.c_double, dp, dp, dp, ctypes.c_int]
        L.ref_scf.restype = ctypes.c_int
        L.ref_get_density.argtypes = [ctypes.c_int, dp]
        L.ref_write_molden.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
        L.ref_write_wfx.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
        L.ref_gradient.argtypes = [dp, ctypes.c_int]
        L.ref_gradient.restype = ctypes.c_int
        L.ref_electron_counts.argtypes = [ip, ip]
        L.ref_fock_2e.argtypes = [dp, dp]
        L.ref_fock_2e.restype = ctypes.c_int
        L.ref_jk.argtypes = [dp, dp, dp]
        L.ref_jk.restype = ctypes.c_int
        L.ref_eri.argtypes = [ctypes.c_int] * 4
        L.ref_eri.restype = ctypes.c_double
        L.ref_boys.argtypes = [ctypes.c_double, ctypes.c_uint]
        L.ref_boys.restype = ctypes.c_double
        L.ref_time_eri_rows.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp]
        L.ref_time_eri_rows.restype = ctypes.c_longlong
        L.ref_time_eri_random.argtypes = [ctypes.c_double, ctypes.c_ulonglong, dp, dp]
        L.ref_time_eri_random.restype = ctypes.c_longlong
        L.ref_time_jk.argtypes = [dp]
        L.ref_time_jk.restype = ctypes.c_double
        L.ref_set_workers.argtypes = [ctypes.c_int]
        L.ref_scf_capped.argtypes = [ctypes.c_double, ctypes.c_int, dp, dp, dp, dp, ctypes.c_int]
        L.ref_scf_capped.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a, t=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(t))


def setup(sh, charge: int = 0, multiplicity: int = 1, build_tensor: bool = True, quiet: bool = True) -> int:
    """Load a ShellArrays into the reference's global SCF state."""
    L = lib()
    Z = np.ascontiguousarray(sh.Z, dtype=np.int32)
    xyz = np.ascontiguousarray(sh.atom_xyz, dtype=np.float64).ravel()
    sa = np.ascontiguousarray(sh.shell_atom, dtype=np.int32)
    sl = np.ascontiguousarray(sh.shell_l, dtype=np.int32)
    sn = np.ascontiguousarray(sh.shell_nprim, dtype=np.int32)
    ex = np.ascontiguousarray(sh.exps, dtype=np.float64)
    co = np.ascontiguousarray(sh.coefs, dtype=np.float64)
    return L.ref_setup(sh.natom, _p(Z, ctypes.c_int), _p(xyz), sh.nshell, _p(sa, ctypes.c_int),
                       _p(sl, ctypes.c_int), _p(sn, ctypes.c_int), _p(ex), _p(co),
                       charge, multiplicity, 0 if sh.pure else 1, 1 if build_tensor else 0, 1 if quiet else 0)


def scf(conv: float = 1e-10) -> Tuple[float, np.ndarray, int, float]:
    L = lib()
    n = L.ref_nbf()
    E = ctypes.c_double()
    secs = ctypes.c_double()
    D = np.zeros(n * (n + 1) // 2)
    it = L.ref_scf(conv, ctypes.byref(E), _p(D), ctypes.byref(secs), 1)
    if it < 0:
        raise RuntimeError("reference state has no ERI tensor")
    return E.value, D, it, secs.value


def set_workers(n: int) -> None:
    """Worker processes for the closed-shell tensor fill, J/K and SCF drivers
    (1: the reference's own serial loops).  Results are bitwise the same."""
    lib().ref_set_workers(int(n))


def scf_capped(conv: float = 1e-10, max_iter: int = 0):
    """Closed-shell SCF through the reference's own iteration functions with an
    optional iteration cap (0: none, like the reference).  Returns
    (E_total, D_alpha packed, iterations, converged, seconds, per-iteration
    electronic energies)."""
    L = lib()
    n = L.ref_nbf()
    E = ctypes.c_double()
    secs = ctypes.c_double()
    D = np.zeros(n * (n + 1) // 2)
    trace = np.zeros(4096)
    it = L.ref_scf_capped(conv, int(max_iter), ctypes.byref(E), _p(D), ctypes.byref(secs), _p(trace), 1)
    if it <= -1000000:
        raise RuntimeError("reference state has no ERI tensor, is open-shell, or a worker failed")
    conv_ok = it > 0
    it = abs(it)
    return E.value, D, it, conv_ok, secs.value, trace[:min(it, 4096)].copy()


def spin_density(spin: int) -> np.ndarray:
    """Final alpha (0) or beta (1) density of the last scf() call, packed-U."""
    L = lib()
    n = L.ref_nbf()
    D = np.zeros(n * (n + 1) // 2)
    L.ref_get_density(int(spin), _p(D))
    return D


def gradient(natom: int) -> np.ndarray:
    """The reference's nuclear gradient [natom, 3] at the last scf() density."""
    g = np.zeros(3 * natom)
    n = lib().ref_gradient(_p(g), 1)
    if n < 0:
        raise RuntimeError("reference state has no ERI tensor")
    return g.reshape(natom, 3)


def write_molden(path: str, write_virtual: bool = True) -> None:
    """The reference's Molden file of the last scf() call."""
    lib().ref_write_molden(path.encode(), 1 if write_virtual else 0, 1)


def write_wfx(path: str, write_virtual: bool = True) -> None:
    """The reference's WFX file of the last scf() call."""
    lib().ref_write_wfx(path.encode(), 1 if write_virtual else 0, 1)


def electron_counts() -> Tuple[int, int]:
    a, b = ctypes.c_int(), ctypes.c_int()
    lib().ref_electron_counts(ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


def fock_2e(D_alpha_packed: np.ndarray) -> np.ndarray:
    L = lib()
    n = L.ref_nbf()
    D = np.ascontiguousarray(D_alpha_packed, dtype=np.float64)
    G = np.zeros(n * (n + 1) // 2)
    if L.ref_fock_2e(_p(D), _p(G)) != 0:
        raise RuntimeError("reference state has no ERI tensor")
    return G


def jk(D_alpha_packed: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    L = lib()
    n = L.ref_nbf()
    D = np.ascontiguousarray(D_alpha_packed, dtype=np.float64)
    J = np.zeros(n * (n + 1) // 2)
    K = np.zeros(n * (n + 1) // 2)
    if L.ref_jk(_p(D), _p(J), _p(K)) != 0:
        raise RuntimeError("reference state has no ERI tensor")
    return J, K


def overlap() -> np.ndarray:
    L = lib()
    n = L.ref_nbf()
    S = np.zeros(n * (n + 1) // 2)
    L.ref_get_overlap(_p(S))
    return S


def core_hamiltonian() -> np.ndarray:
    L = lib()
    n = L.ref_nbf()
    H = np.zeros(n * (n + 1) // 2)
    L.ref_get_core_hamiltonian(_p(H))
    return H


def eri(mu: int, nu: int, sigma: int, tau: int) -> float:
    return lib().ref_eri(mu, nu, sigma, tau)


def boys(x: float, m: int) -> float:
    return lib().ref_boys(x, m)


def basis_terms(f: int):
    w = np.zeros(64)
    xyz = np.zeros(192, dtype=np.int32)
    n = lib().ref_basis_terms(f, _p(w), _p(xyz, ctypes.c_int))
    return w[:n].copy(), xyz[:3 * n].reshape(n, 3).copy()


def basis_prims(f: int):
    z = np.zeros(128)
    w = np.zeros(128)
    n = lib().ref_basis_prims(f, _p(z), _p(w))
    return z[:n].copy(), w[:n].copy()


def time_eri_rows(i_begin: int, i_end: int) -> Tuple[int, float, float]:
    s = ctypes.c_double()
    c = ctypes.c_double()
    n = lib().ref_time_eri_rows(i_begin, i_end, ctypes.byref(s), ctypes.byref(c))
    return int(n), s.value, c.value


def time_eri_random(max_seconds: float, seed: int) -> Tuple[int, float, float]:
    s = ctypes.c_double()
    c = ctypes.c_double()
    n = lib().ref_time_eri_random(max_seconds, seed, ctypes.byref(s), ctypes.byref(c))
    return int(n), s.value, c.value
