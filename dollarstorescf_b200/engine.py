"""Python mirror of the C ABI: the two-electron part of the reference's SCF.

``FockBuilder`` plays the role of the reference's ExactCoulomb module
(chem/scf/ExactCoulomb.hpp:9-15): ``set_basis`` replaces
``assignExactRepulsionTensor`` (no stored tensor: integrals are recomputed on
the GPU per build, "direct SCF"), ``jk`` returns the whole Coulomb and exchange
matrices that ``getExactCoulombMatrix`` / ``getExactExchangeMatrix`` return
element by element.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import numpy as np

from . import _lib
from .shells import ShellArrays

BOYS_REF = 0
BOYS_FAST = 1


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class FockBuilder:
    def __init__(self, device: int = 0, schwarz_threshold: float = 1e-12, boys_mode: int = BOYS_REF,
                 primitive_threshold: float = 1e-18):
        self._L = _lib.load()
        opts = _lib.DssOpts(device, schwarz_threshold, boys_mode, primitive_threshold)
        h = ctypes.c_void_p()
        rc = self._L.dss_create(ctypes.byref(h), ctypes.byref(opts))
        if rc != 0:
            raise _lib.DssError(rc, self._L.dss_last_error(None).decode())
        self._h = h
        self.nbf = 0

    def _check(self, rc: int) -> None:
        if rc != 0:
            raise _lib.DssError(rc, self._L.dss_last_error(self._h).decode())

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.dss_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_basis(self, sh: ShellArrays) -> int:
        l = np.ascontiguousarray(sh.shell_l, dtype=np.int32)
        n = np.ascontiguousarray(sh.shell_nprim, dtype=np.int32)
        e = np.ascontiguousarray(sh.exps, dtype=np.float64)
        c = np.ascontiguousarray(sh.coefs, dtype=np.float64)
        x = np.ascontiguousarray(sh.centers, dtype=np.float64).ravel()
        self._check(self._L.dss_set_basis(self._h, sh.nshell, _ip(l), _ip(n), _dp(e), _dp(c), _dp(x),
                                          1 if sh.pure else 0))
        self.nbf = self._L.dss_nbf(self._h)
        return self.nbf

    def jk(self, D_packed: np.ndarray, want_j: bool = True, want_k: bool = True
           ) -> Tuple[Optional[np.ndarray], Optional[np.ndarray]]:
        n = self.nbf
        np_ = n * (n + 1) // 2
        D = np.ascontiguousarray(D_packed, dtype=np.float64)
        if D.shape != (np_,):
            raise ValueError(f"D must be packed-U with {np_} entries")
        J = np.empty(np_) if want_j else None
        K = np.empty(np_) if want_k else None
        self._check(self._L.dss_build_jk(self._h, _dp(D), _dp(J) if J is not None else None,
                                         _dp(K) if K is not None else None))
        return J, K

    def jk_device(self, D_ptr: int, J_ptr: int, K_ptr: int) -> None:
        """Build on device-resident dense n x n buffers (raw device pointers)."""
        self._check(self._L.dss_build_jk_device(self._h, ctypes.c_void_p(D_ptr), ctypes.c_void_p(J_ptr),
                                                ctypes.c_void_p(K_ptr)))

    def jk_device_noalloc(self, D_ptr: int, J_ptr: int, K_ptr: int) -> None:
        """Same build as jk_device with the accumulators in the library's fixed
        device array: no device allocation in the call (n <= 512)."""
        self._check(self._L.dss_build_jk_device_noalloc(self._h, ctypes.c_void_p(D_ptr), ctypes.c_void_p(J_ptr),
                                                        ctypes.c_void_p(K_ptr)))

    def jk_host_ptrs(self, D_ptr: int, J_ptr: int, K_ptr: int) -> None:
        """dss_build_jk on raw host pointers (e.g. pinned buffers)."""
        self._check(self._L.dss_build_jk(self._h, ctypes.cast(D_ptr, ctypes.POINTER(ctypes.c_double)),
                                         ctypes.cast(J_ptr, ctypes.POINTER(ctypes.c_double)),
                                         ctypes.cast(K_ptr, ctypes.POINTER(ctypes.c_double))))

    def jk_mixed_device(self, D_ptr: int, J_ptr: int, K_ptr: int, fp32_threshold: float = 1e-7,
                        skip_threshold: float = 1e-12) -> None:
        self._check(self._L.dss_build_jk_mixed_device(self._h, ctypes.c_void_p(D_ptr), ctypes.c_void_p(J_ptr),
                                                      ctypes.c_void_p(K_ptr), fp32_threshold, skip_threshold))

    def stream_ptr(self) -> int:
        return int(self._L.dss_get_stream(self._h) or 0)

    def set_stream(self, stream_ptr: int) -> None:
        self._check(self._L.dss_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def class_info(self, i: int):
        l4 = (ctypes.c_int * 4)()
        a, b, c = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self._L.dss_class_info(self._h, i, l4, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return list(l4), a.value, b.value, c.value

    def eval_boys(self, mode: int, L: int, x: np.ndarray) -> np.ndarray:
        xs = np.ascontiguousarray(x, dtype=np.float64)
        F = np.empty((xs.size, L + 1))
        self._check(self._L.dss_eval_boys(self._h, mode, L, _dp(xs), xs.size, _dp(F)))
        return F

    def num_classes(self) -> int:
        return int(self._L.dss_num_classes())

    def set_class_variant(self, i: int, variant: int) -> None:
        self._check(self._L.dss_set_class_variant(self._h, i, variant))

    def class_variant(self, i: int) -> int:
        return int(self._L.dss_get_class_variant(self._h, i))

    def kernels_per_build(self) -> int:
        return int(self._L.dss_kernels_per_build(self._h))

    def profile_build(self, D_ptr: int, J_ptr: int, K_ptr: int):
        nc = self._L.dss_num_classes()
        ms = (ctypes.c_float * nc)()
        self._check(self._L.dss_profile_build(self._h, ctypes.c_void_p(D_ptr), ctypes.c_void_p(J_ptr),
                                              ctypes.c_void_p(K_ptr), ms))
        return [float(v) for v in ms]

    def time_build(self, D_ptr: int, J_ptr: int, K_ptr: int) -> float:
        """Device milliseconds of one whole J/K build in the current launch shape."""
        ms = ctypes.c_float()
        self._check(self._L.dss_time_build(self._h, ctypes.c_void_p(D_ptr), ctypes.c_void_p(J_ptr),
                                           ctypes.c_void_p(K_ptr), ctypes.byref(ms)))
        return float(ms.value)

    def set_persistent(self, on: bool) -> None:
        self._check(self._L.dss_set_persistent(self._h, 1 if on else 0))

    def persistent(self) -> bool:
        return bool(self._L.dss_get_persistent(self._h))

    def fp64_peak_tflops(self) -> float:
        t = ctypes.c_double()
        self._check(self._L.dss_probe_fp64_peak(self._h, ctypes.byref(t)))
        return t.value

    def one_electron(self, sh: ShellArrays):
        """(S, T, V, E_nuc) packed-U for the molecule of ``sh`` (the current basis)."""
        n = self.nbf
        np_ = n * (n + 1) // 2
        S, T, V = np.empty(np_), np.empty(np_), np.empty(np_)
        en = ctypes.c_double()
        Z = np.ascontiguousarray(sh.Z, dtype=np.int32)
        xyz = np.ascontiguousarray(sh.atom_xyz, dtype=np.float64).ravel()
        self._check(self._L.dss_one_electron(self._h, sh.natom, _ip(Z), _dp(xyz), _dp(S), _dp(T), _dp(V),
                                             ctypes.byref(en)))
        return S, T, V, en.value

    def scf(self, H: np.ndarray, S: np.ndarray, n_alpha: int, e_nuc: float, conv: float = 1e-8,
            diis_size: int = 8, max_iter: int = 128, guess: Optional[np.ndarray] = None,
            raise_on_noconv: bool = True, mixed: bool = False, fp32_threshold: float = 1e-7,
            skip_threshold: float = 1e-12, rebuild_every: int = 16, final_switch: float = 1e-8):
        """Device RHF.  Returns (E_total, D_alpha packed-U, iterations, status).
        mixed=True selects the incremental mixed-precision form."""
        n = self.nbf
        o = _lib.DssScfOpts(conv, diis_size, max_iter, 1 if guess is not None else 0, 1 if mixed else 0,
                            fp32_threshold, skip_threshold, rebuild_every, final_switch)
        D = np.ascontiguousarray(guess, dtype=np.float64).copy() if guess is not None else np.zeros(n * (n + 1) // 2)
        E = ctypes.c_double()
        it = ctypes.c_int()
        Hc = np.ascontiguousarray(H, dtype=np.float64)
        Sc = np.ascontiguousarray(S, dtype=np.float64)
        rc = self._L.dss_scf_solve(self._h, _dp(Hc), _dp(Sc), int(n_alpha), float(e_nuc), ctypes.byref(o),
                                   ctypes.byref(E), _dp(D), ctypes.byref(it))
        if rc != 0 and (raise_on_noconv or rc != -4):
            self._check(rc)
        return E.value, D, it.value, rc

    def uhf(self, H: np.ndarray, S: np.ndarray, n_alpha: int, n_beta: int, e_nuc: float, conv: float = 1e-8,
            diis_size: int = 8, max_iter: int = 128, guess: Optional[Tuple[np.ndarray, np.ndarray]] = None,
            raise_on_noconv: bool = True):
        """Device UHF (the unrestricted branch of scf::solveMOs).  Returns
        (E_total, D_alpha, D_beta (packed-U), iterations, status)."""
        n = self.nbf
        np_ = n * (n + 1) // 2
        o = _lib.DssScfOpts(conv, diis_size, max_iter, 1 if guess is not None else 0, 0, 1e-7, 1e-12, 8, 1e-5)
        if guess is not None:
            Da = np.ascontiguousarray(guess[0], dtype=np.float64).copy()
            Db = np.ascontiguousarray(guess[1], dtype=np.float64).copy()
        else:
            Da, Db = np.zeros(np_), np.zeros(np_)
        E = ctypes.c_double()
        it = ctypes.c_int()
        Hc = np.ascontiguousarray(H, dtype=np.float64)
        Sc = np.ascontiguousarray(S, dtype=np.float64)
        rc = self._L.dss_uhf_solve(self._h, _dp(Hc), _dp(Sc), int(n_alpha), int(n_beta), float(e_nuc),
                                   ctypes.byref(o), ctypes.byref(E), _dp(Da), _dp(Db), ctypes.byref(it))
        if rc != 0 and (raise_on_noconv or rc != -4):
            self._check(rc)
        return E.value, Da, Db, it.value, rc

    def orbitals(self, spin: int = 0) -> Tuple[np.ndarray, np.ndarray]:
        """(C [AO, MO], orbital energies) of the last scf()/uhf() for one spin."""
        n = self.nbf
        C = np.empty((n, n))
        eps = np.empty(n)
        self._check(self._L.dss_scf_orbitals(self._h, int(spin), _dp(C), _dp(eps)))
        return C, eps

    def write_molden(self, path: str, sh: ShellArrays, write_virtual: bool = True) -> None:
        """Molden file of the last scf()/uhf() (scf::writeOrbitalsMolden)."""
        Z = np.ascontiguousarray(sh.Z, dtype=np.int32)
        xyz = np.ascontiguousarray(sh.atom_xyz, dtype=np.float64).ravel()
        self._check(self._L.dss_write_molden(self._h, path.encode(), sh.natom, _ip(Z), _dp(xyz),
                                             1 if write_virtual else 0))

    def write_wfx(self, path: str, sh: ShellArrays, write_virtual: bool = True) -> None:
        """WFX file of the last scf()/uhf() (scf::writeOrbitalsWFX)."""
        Z = np.ascontiguousarray(sh.Z, dtype=np.int32)
        xyz = np.ascontiguousarray(sh.atom_xyz, dtype=np.float64).ravel()
        self._check(self._L.dss_write_wfx(self._h, path.encode(), sh.natom, _ip(Z), _dp(xyz),
                                          1 if write_virtual else 0))

    def save_density(self, path: str) -> None:
        """Density checkpoint of the last scf()/uhf() (restart file)."""
        self._check(self._L.dss_save_density(self._h, path.encode()))

    def load_density(self, path: str) -> Tuple[np.ndarray, np.ndarray, int, int, int]:
        """(D_alpha, D_beta (packed-U), spins, n_alpha, n_beta) of a density
        checkpoint for the current basis; usable as scf()/uhf() guesses."""
        return load_density(path, self.nbf, self)

    def gradient(self, sh: ShellArrays, step: float = 0.0) -> np.ndarray:
        """Nuclear gradient [natom, 3] (hartree/bohr) of the last scf()/uhf():
        analytic (step 0), or with the one-electron terms as central differences
        of that step (bohr)."""
        Z = np.ascontiguousarray(sh.Z, dtype=np.int32)
        xyz = np.ascontiguousarray(sh.atom_xyz, dtype=np.float64).ravel()
        g = np.zeros(3 * sh.natom)
        self._check(self._L.dss_gradient(self._h, sh.natom, _ip(Z), _dp(xyz), float(step), _dp(g)))
        return g.reshape(sh.natom, 3)

    def eri_gradient(self, sh: ShellArrays, D: np.ndarray, Da: Optional[np.ndarray] = None,
                     Db: Optional[np.ndarray] = None) -> np.ndarray:
        """Analytic four-centre gradient term [natom, 3] of packed-U densities
        (D total; Da, Db spin densities of an unrestricted determinant)."""
        atom = np.ascontiguousarray(sh.shell_atom, dtype=np.int32)
        g = np.zeros(3 * sh.natom)
        D = np.ascontiguousarray(D, dtype=np.float64)
        pa = np.ascontiguousarray(Da, dtype=np.float64) if Da is not None else None
        pb = np.ascontiguousarray(Db, dtype=np.float64) if Db is not None else None
        self._check(self._L.dss_eri_gradient(self._h, _dp(D), _dp(pa) if pa is not None else None,
                                             _dp(pb) if pb is not None else None, sh.natom, _ip(atom), _dp(g)))
        return g.reshape(sh.natom, 3)

    def sync(self) -> None:
        self._check(self._L.dss_sync(self._h))

    def work_stats(self) -> Tuple[int, int, int]:
        a, b, c = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self._L.dss_work_stats(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value


def load_density(path: str, nbf: int, fb: Optional["FockBuilder"] = None):
    """Reads a density checkpoint written by FockBuilder.save_density (host
    only): (D_alpha, D_beta (packed-U), spins, n_alpha, n_beta)."""
    L = _lib.load()
    np_ = nbf * (nbf + 1) // 2
    Da = np.zeros(np_)
    Db = np.zeros(np_)
    sp, na, nb = (ctypes.c_int(0) for _ in range(3))
    rc = L.dss_load_density(fb._h if fb is not None else None, path.encode(), int(nbf), ctypes.byref(sp),
                            ctypes.byref(na), ctypes.byref(nb), _dp(Da), _dp(Db))
    if rc != 0:
        msg = L.dss_last_error(fb._h).decode() if fb is not None else "dss_load_density failed"
        raise _lib.DssError(rc, msg)
    return Da, Db, sp.value, na.value, nb.value
