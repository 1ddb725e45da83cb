"""The allocation-free J/K entry point (dss_build_jk_device_noalloc).

It serves callers that may not allocate device memory while they run (a memory
pool or budget that owns the device's memory, loops that cannot afford the
synchronisation cudaMalloc/cudaFree can cause); its accumulators sit in a fixed
array inside the library.  Through the C ABI, on a fresh context whose first
J/K call is the allocation-free one, two calls in a row must leave the device's
free memory unchanged and give the same J and K as dss_build_jk_device (the
regular entry point, which allocates its accumulators) within the 1e-10
tolerance of the other J/K tests; a basis above the array's limit must be
rejected.  This file is collected last, so a run that stops at the first
failure has already run every other test; it also passes on its own in a fresh
process."""
import numpy as np
import pytest
import torch

from conftest import load_case
from dollarstorescf_b200 import basis, geometry, shells
from dollarstorescf_b200._lib import DssError
from dollarstorescf_b200.engine import BOYS_REF, FockBuilder

pytestmark = pytest.mark.gpu


def test_noalloc_allocates_nothing_and_matches_regular_build_twice():
    d, mol, sh = load_case("w4_631gs")
    n = int(d["nbf"])
    rng = np.random.default_rng(21)
    dens = []
    for _ in range(2):
        A = rng.standard_normal((n, n)) * 0.1
        dens.append(torch.tensor(A + A.T, dtype=torch.float64, device="cuda:0"))
    out = [(torch.full_like(D, np.nan), torch.full_like(D, np.nan)) for D in dens]
    J0, K0 = torch.empty_like(dens[0]), torch.empty_like(dens[0])
    with FockBuilder(schwarz_threshold=1e-12, boys_mode=BOYS_REF) as fb:
        fb.set_basis(sh)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info(0)[0]
        for call, (D, (J1, K1)) in enumerate(zip(dens, out)):
            fb.jk_device_noalloc(D.data_ptr(), J1.data_ptr(), K1.data_ptr())
            fb.sync()
            assert torch.cuda.mem_get_info(0)[0] == free0, f"device memory changed in call {call}"
        # The regular entry point (it allocates its accumulators on first use).
        for call, (D, (J1, K1)) in enumerate(zip(dens, out)):
            fb.jk_device(D.data_ptr(), J0.data_ptr(), K0.data_ptr())
            fb.sync()
            assert torch.isfinite(J1).all() and torch.isfinite(K1).all()
            assert (J1 - J0).abs().max().item() < 1e-10, call
            assert (K1 - K0).abs().max().item() < 1e-10, call


def test_noalloc_rejects_basis_above_limit():
    mol = geometry.water_cluster(4, 4, 2, 32, seed=1)
    sh = shells.build_shells(mol, basis.builtin_basis("6-31G*"), pure=False)  # 608 functions
    with FockBuilder(schwarz_threshold=1e-12) as fb:
        assert fb.set_basis(sh) == 608
        D = torch.zeros((608, 608), dtype=torch.float64, device="cuda:0")
        J, K = torch.empty_like(D), torch.empty_like(D)
        with pytest.raises(DssError, match="exceed the maximum of 512"):
            fb.jk_device_noalloc(D.data_ptr(), J.data_ptr(), K.data_ptr())
