"""ctypes binding of libdss.so (include/dss.h).

The library is the product; this module only loads it and declares the C
signatures.  Loading fails loudly when the built library is missing: there is
no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import re

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libdss.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "dss.h")

_lib = None


class DssError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"dss error {code}: {msg}")
        self.code = code


class DssScfOpts(ctypes.Structure):
    _fields_ = [("conv", ctypes.c_double), ("diis_size", ctypes.c_int), ("max_iter", ctypes.c_int),
                ("use_guess", ctypes.c_int), ("incremental", ctypes.c_int), ("fp32_threshold", ctypes.c_double),
                ("skip_threshold", ctypes.c_double), ("rebuild_every", ctypes.c_int),
                ("final_switch", ctypes.c_double)]


class DssOpts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("schwarz_threshold", ctypes.c_double), ("boys_mode", ctypes.c_int),
                ("primitive_threshold", ctypes.c_double)]


def header_symbols():
    """Function names declared in include/dss.h."""
    with open(HEADER) as f:
        text = f.read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\*?(dss_\w+)\s*\(", text, flags=re.M)))


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.isfile(LIB_PATH):
        raise FileNotFoundError(
            f"{LIB_PATH} is not built; run `python -m dollarstorescf_b200.build` (there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    llp = ctypes.POINTER(ctypes.c_longlong)
    L.dss_default_opts.argtypes = [ctypes.POINTER(DssOpts)]
    L.dss_default_opts.restype = None
    L.dss_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(DssOpts)]
    L.dss_create.restype = ctypes.c_int
    L.dss_destroy.argtypes = [vp]
    L.dss_destroy.restype = None
    L.dss_last_error.argtypes = [vp]
    L.dss_last_error.restype = ctypes.c_char_p
    L.dss_set_basis.argtypes = [vp, ctypes.c_int, ip, ip, dp, dp, dp, ctypes.c_int]
    L.dss_set_basis.restype = ctypes.c_int
    L.dss_nbf.argtypes = [vp]
    L.dss_nbf.restype = ctypes.c_int
    L.dss_build_jk.argtypes = [vp, dp, dp, dp]
    L.dss_build_jk.restype = ctypes.c_int
    L.dss_build_jk_device.argtypes = [vp, vp, vp, vp]
    L.dss_build_jk_device.restype = ctypes.c_int
    L.dss_sync.argtypes = [vp]
    L.dss_sync.restype = ctypes.c_int
    L.dss_work_stats.argtypes = [vp, llp, llp, llp]
    L.dss_work_stats.restype = ctypes.c_int
    L.dss_set_stream.argtypes = [vp, vp]
    L.dss_set_stream.restype = ctypes.c_int
    L.dss_get_stream.argtypes = [vp]
    L.dss_get_stream.restype = vp
    L.dss_num_classes.argtypes = []
    L.dss_num_classes.restype = ctypes.c_int
    L.dss_list_schedule.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.c_int, ctypes.c_int, ip, ip]
    L.dss_list_schedule.restype = ctypes.c_int
    L.dss_class_info.argtypes = [vp, ctypes.c_int, ip, llp, llp, llp]
    L.dss_class_info.restype = ctypes.c_int
    L.dss_kernels_per_build.argtypes = [vp]
    L.dss_kernels_per_build.restype = ctypes.c_int
    L.dss_profile_build.argtypes = [vp, vp, vp, vp, ctypes.POINTER(ctypes.c_float)]
    L.dss_profile_build.restype = ctypes.c_int
    L.dss_time_build.argtypes = [vp, vp, vp, vp, ctypes.POINTER(ctypes.c_float)]
    L.dss_time_build.restype = ctypes.c_int
    L.dss_set_persistent.argtypes = [vp, ctypes.c_int]
    L.dss_set_persistent.restype = ctypes.c_int
    L.dss_get_persistent.argtypes = [vp]
    L.dss_get_persistent.restype = ctypes.c_int
    L.dss_probe_fp64_peak.argtypes = [vp, dp]
    L.dss_probe_fp64_peak.restype = ctypes.c_int
    L.dss_set_class_variant.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    L.dss_set_class_variant.restype = ctypes.c_int
    L.dss_get_class_variant.argtypes = [vp, ctypes.c_int]
    L.dss_get_class_variant.restype = ctypes.c_int
    L.dss_eval_boys.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int, dp]
    L.dss_eval_boys.restype = ctypes.c_int
    L.dss_build_jk_mixed_device.argtypes = [vp, vp, vp, vp, ctypes.c_double, ctypes.c_double]
    L.dss_build_jk_mixed_device.restype = ctypes.c_int
    L.dss_one_electron.argtypes = [vp, ctypes.c_int, ip, dp, dp, dp, dp, dp]
    L.dss_one_electron.restype = ctypes.c_int
    L.dss_default_scf_opts.argtypes = [ctypes.POINTER(DssScfOpts)]
    L.dss_default_scf_opts.restype = None
    L.dss_scf_solve.argtypes = [vp, dp, dp, ctypes.c_int, ctypes.c_double, ctypes.POINTER(DssScfOpts), dp, dp,
                                ip]
    L.dss_scf_solve.restype = ctypes.c_int
    L.dss_uhf_solve.argtypes = [vp, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.POINTER(DssScfOpts),
                                dp, dp, dp, ip]
    L.dss_uhf_solve.restype = ctypes.c_int
    L.dss_scf_orbitals.argtypes = [vp, ctypes.c_int, dp, dp]
    L.dss_scf_orbitals.restype = ctypes.c_int
    L.dss_write_molden.argtypes = [vp, ctypes.c_char_p, ctypes.c_int, ip, dp, ctypes.c_int]
    L.dss_write_molden.restype = ctypes.c_int
    L.dss_write_wfx.argtypes = [vp, ctypes.c_char_p, ctypes.c_int, ip, dp, ctypes.c_int]
    L.dss_write_wfx.restype = ctypes.c_int
    L.dss_save_density.argtypes = [vp, ctypes.c_char_p]
    L.dss_save_density.restype = ctypes.c_int
    L.dss_load_density.argtypes = [vp, ctypes.c_char_p, ctypes.c_int, ip, ip, ip, dp, dp]
    L.dss_load_density.restype = ctypes.c_int
    L.dss_gradient.argtypes = [vp, ctypes.c_int, ip, dp, ctypes.c_double, dp]
    L.dss_gradient.restype = ctypes.c_int
    L.dss_eri_gradient.argtypes = [vp, dp, dp, dp, ctypes.c_int, ip, dp]
    L.dss_eri_gradient.restype = ctypes.c_int
    L.dss_build_jk_device_noalloc.argtypes = [vp, vp, vp, vp]
    L.dss_build_jk_device_noalloc.restype = ctypes.c_int
    szt = ctypes.c_size_t
    L.dss_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(DssOpts), szt, ctypes.c_int]
    L.dss_batch_create.restype = ctypes.c_int
    L.dss_batch_destroy.argtypes = [vp]
    L.dss_batch_destroy.restype = None
    L.dss_batch_last_error.argtypes = [vp]
    L.dss_batch_last_error.restype = ctypes.c_char_p
    L.dss_batch_add.argtypes = [vp, ctypes.c_int, ip, ip, dp, dp, dp, ctypes.c_int, ctypes.c_int, ip, dp,
                                ctypes.c_int, dp, ip]
    L.dss_batch_add.restype = ctypes.c_int
    L.dss_batch_step.argtypes = [vp, ctypes.POINTER(DssScfOpts), ctypes.c_int, ip]
    L.dss_batch_step.restype = ctypes.c_int
    L.dss_batch_solve.argtypes = [vp, ctypes.POINTER(DssScfOpts)]
    L.dss_batch_solve.restype = ctypes.c_int
    L.dss_batch_result.argtypes = [vp, ctypes.c_int, dp, dp, ip, ip]
    L.dss_batch_result.restype = ctypes.c_int
    L.dss_batch_profile.argtypes = [vp, ctypes.POINTER(ctypes.c_float)]
    L.dss_batch_profile.restype = ctypes.c_int
    L.dss_batch_time_build.argtypes = [vp, ctypes.POINTER(ctypes.c_float)]
    L.dss_batch_time_build.restype = ctypes.c_int
    L.dss_batch_set_persistent.argtypes = [vp, ctypes.c_int]
    L.dss_batch_set_persistent.restype = ctypes.c_int
    L.dss_batch_finished.argtypes = [vp, ip, ctypes.c_int, ip]
    L.dss_batch_finished.restype = ctypes.c_int
    L.dss_batch_remove.argtypes = [vp, ctypes.c_int]
    L.dss_batch_remove.restype = ctypes.c_int
    L.dss_batch_info.argtypes = [vp, ip, llp, llp]
    L.dss_batch_info.restype = ctypes.c_int
    L.dss_batch_set_class_variant.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    L.dss_batch_set_class_variant.restype = ctypes.c_int
    L.dss_batch_context.argtypes = [vp]
    L.dss_batch_context.restype = vp
    _lib = L
    return L
