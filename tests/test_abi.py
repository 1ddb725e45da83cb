"""The C-ABI library loads and exports every function include/dss.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import subprocess

from dollarstorescf_b200 import _lib


def test_header_declares_the_boundary():
    syms = _lib.header_symbols()
    for s in ("dss_create", "dss_destroy", "dss_set_basis", "dss_build_jk", "dss_last_error"):
        assert s in syms


def test_library_exports_every_header_symbol(dss_lib):
    missing = [s for s in _lib.header_symbols() if not hasattr(dss_lib, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(_lib.header_symbols()) <= exported


def test_create_without_gpu_fails_cleanly(dss_lib):
    import torch

    if torch.cuda.is_available():
        return
    h = ctypes.c_void_p()
    rc = dss_lib.dss_create(ctypes.byref(h), None)
    assert rc == -3  # DSS_ERR_CUDA: no device, no abort
    assert b"no CUDA device" in dss_lib.dss_last_error(None)
