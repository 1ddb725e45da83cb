"""Python mirror of the batch C ABI (dss_batch_*): many molecules solved
together, with molecules joining and leaving between SCF iterations."""
from __future__ import annotations

import ctypes
from typing import List, Optional, Tuple

import numpy as np

from . import _lib
from .engine import BOYS_REF, _dp, _ip
from .shells import ShellArrays


class Batch:
    def __init__(self, device: int = 0, schwarz_threshold: float = 1e-12, boys_mode: int = BOYS_REF,
                 arena_bytes: int = 0, diis_size: int = 8, primitive_threshold: float = 1e-18):
        self._L = _lib.load()
        opts = _lib.DssOpts(device, schwarz_threshold, boys_mode, primitive_threshold)
        h = ctypes.c_void_p()
        rc = self._L.dss_batch_create(ctypes.byref(h), ctypes.byref(opts), arena_bytes, diis_size)
        if rc != 0:
            raise _lib.DssError(rc, self._L.dss_last_error(None).decode())
        self._h = h

    def _check(self, rc: int) -> None:
        if rc != 0:
            raise _lib.DssError(rc, self._L.dss_batch_last_error(self._h).decode())

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.dss_batch_destroy(self._h)
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

    def add(self, sh: ShellArrays, charge: int = 0, guess: Optional[np.ndarray] = None) -> int:
        """Admits a molecule; raises DssError with code -2 when the arena is full."""
        l = np.ascontiguousarray(sh.shell_l, dtype=np.int32)
        n = np.ascontiguousarray(sh.shell_nprim, dtype=np.int32)
        e = np.ascontiguousarray(sh.exps, dtype=np.float64)
        c = np.ascontiguousarray(sh.coefs, dtype=np.float64)
        x = np.ascontiguousarray(sh.centers, dtype=np.float64).ravel()
        Z = np.ascontiguousarray(sh.Z, dtype=np.int32)
        ax = np.ascontiguousarray(sh.atom_xyz, dtype=np.float64).ravel()
        g = np.ascontiguousarray(guess, dtype=np.float64) if guess is not None else None
        h = ctypes.c_int()
        self._check(self._L.dss_batch_add(self._h, sh.nshell, _ip(l), _ip(n), _dp(e), _dp(c), _dp(x),
                                          1 if sh.pure else 0, sh.natom, _ip(Z), _dp(ax), charge,
                                          _dp(g) if g is not None else None, ctypes.byref(h)))
        return h.value

    @staticmethod
    def opts(conv: float = 1e-8, diis_size: int = 8, max_iter: int = 128, mixed: bool = False,
             fp32_threshold: float = 1e-7, skip_threshold: float = 1e-12, rebuild_every: int = 16,
             final_switch: float = 1e-8):
        """SCF options; mixed=True selects the mixed-precision incremental form."""
        return _lib.DssScfOpts(conv, diis_size, max_iter, 0, 1 if mixed else 0, fp32_threshold, skip_threshold,
                               rebuild_every, final_switch)

    def step(self, iterations: int = 1, conv: float = 1e-8, max_iter: int = 128, mixed: bool = False,
             fp32_threshold: float = 1e-7, **mixed_opts) -> int:
        """mixed_opts: skip_threshold, rebuild_every, final_switch of the incremental form."""
        o = self.opts(conv, max_iter=max_iter, mixed=mixed, fp32_threshold=fp32_threshold, **mixed_opts)
        act = ctypes.c_int()
        self._check(self._L.dss_batch_step(self._h, ctypes.byref(o), iterations, ctypes.byref(act)))
        return act.value

    def solve(self, conv: float = 1e-8, max_iter: int = 128, mixed: bool = False,
              fp32_threshold: float = 1e-7, **mixed_opts) -> None:
        o = self.opts(conv, max_iter=max_iter, mixed=mixed, fp32_threshold=fp32_threshold, **mixed_opts)
        self._check(self._L.dss_batch_solve(self._h, ctypes.byref(o)))

    def result(self, handle: int, nbf: int = 0, want_density: bool = False) -> Tuple[float, Optional[np.ndarray], int, int]:
        E = ctypes.c_double()
        it = ctypes.c_int()
        st = ctypes.c_int()
        D = np.empty(nbf * (nbf + 1) // 2) if want_density else None
        self._check(self._L.dss_batch_result(self._h, handle, ctypes.byref(E), _dp(D) if D is not None else None,
                                             ctypes.byref(it), ctypes.byref(st)))
        return E.value, D, it.value, st.value

    def finished_handles(self) -> List[int]:
        """Handles whose results the last step produced (one library call)."""
        cnt = ctypes.c_int()
        self._check(self._L.dss_batch_finished(self._h, None, 0, ctypes.byref(cnt)))
        if not cnt.value:
            return []
        arr = (ctypes.c_int * cnt.value)()
        self._check(self._L.dss_batch_finished(self._h, arr, cnt.value, ctypes.byref(cnt)))
        return list(arr)

    def finished(self, handle: int) -> bool:
        E = ctypes.c_double()
        return self._L.dss_batch_result(self._h, handle, ctypes.byref(E), None, None, None) == 0

    def remove(self, handle: int) -> None:
        self._check(self._L.dss_batch_remove(self._h, handle))

    def info(self, n_for_region: int = 0) -> Tuple[int, int, int]:
        nl = ctypes.c_int()
        fb = ctypes.c_longlong()
        rb = ctypes.c_longlong(n_for_region)
        self._check(self._L.dss_batch_info(self._h, ctypes.byref(nl), ctypes.byref(fb), ctypes.byref(rb)))
        return nl.value, fb.value, rb.value if n_for_region else 0

    def profile(self):
        """Per-class milliseconds of one J/K accumulation over all live molecules."""
        nc = self._L.dss_num_classes()
        ms = (ctypes.c_float * nc)()
        self._check(self._L.dss_batch_profile(self._h, ms))
        return [float(v) for v in ms]

    def time_build(self) -> float:
        """Device milliseconds of one whole FP64 J/K accumulation over all live molecules."""
        ms = ctypes.c_float()
        self._check(self._L.dss_batch_time_build(self._h, ctypes.byref(ms)))
        return float(ms.value)

    def set_persistent(self, on: bool) -> None:
        self._check(self._L.dss_batch_set_persistent(self._h, 1 if on else 0))

    def work_stats(self) -> Tuple[int, int, int]:
        """(shell quartets, primitive quartets, warp tasks) of the current composition."""
        sq, pq, wt = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        ctx = self._L.dss_batch_context(self._h)
        self._check(self._L.dss_work_stats(ctx, ctypes.byref(sq), ctypes.byref(pq), ctypes.byref(wt)))
        return sq.value, pq.value, wt.value

    def set_class_variant(self, i: int, variant: int) -> None:
        self._check(self._L.dss_batch_set_class_variant(self._h, i, variant))
