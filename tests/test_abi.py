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


def test_list_schedule_of_class_launches(dss_lib):
    # Host-only: the order and side stream of each class launch in a plain build
    # once the launch times are known (longest first, each onto the stream with
    # the least work so far), the same function the build calls.
    import numpy as np

    ms = np.array([0.3, 1.1, 0.9, 0.2, 0.9, 0.5, 0.6], dtype=np.float32)
    n = len(ms)
    order = np.empty(n, dtype=np.int32)
    stream = np.empty(n, dtype=np.int32)
    fp = ctypes.POINTER(ctypes.c_float)
    ip = ctypes.POINTER(ctypes.c_int)
    rc = dss_lib.dss_list_schedule(ms.ctypes.data_as(fp), n, 3, order.ctypes.data_as(ip), stream.ctypes.data_as(ip))
    assert rc == 0
    assert list(order) == [1, 2, 4, 6, 5, 0, 3]  # longest first, ties in index order
    # loads: s0 1.1, s1 0.9, s2 0.9; 0.6 -> s1 (tie, lowest index), 0.5 -> s2, 0.3 -> s0;
    # 0.2 -> s2 (0.9f + 0.5f lies just below 1.1f + 0.3f)
    assert list(stream) == [0, 1, 2, 1, 2, 0, 2]
    loads = np.zeros(3)
    for k in range(n):
        loads[stream[k]] += ms[order[k]]
    assert loads.max() - loads.min() < 0.2 + 1e-6
    assert dss_lib.dss_list_schedule(ms.ctypes.data_as(fp), n, 0, order.ctypes.data_as(ip),
                                     stream.ctypes.data_as(ip)) == -1
