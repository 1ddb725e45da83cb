"""Mixed-precision incremental form: screened FP32/FP64 builds of a density
difference, and the incremental SCF's energy against the FP64 oracle value
(the reference's own energy); the stated bar is |dE| <= 1 uEh."""
import numpy as np
import pytest
import torch

from conftest import load_case
from dollarstorescf_b200 import shells
from dollarstorescf_b200.engine import BOYS_FAST, BOYS_REF, FockBuilder

pytestmark = pytest.mark.gpu


def test_mixed_build_of_small_difference():
    d, mol, sh = load_case("w4_631gs")
    n = int(d["nbf"])
    rng = np.random.default_rng(11)
    A = rng.standard_normal((n, n)) * 1e-6
    dD = A + A.T
    with FockBuilder(schwarz_threshold=1e-12, boys_mode=BOYS_FAST) as fb:
        fb.set_basis(sh)
        J64, K64 = fb.jk(shells.pack(dD))
        Dd = torch.tensor(dD, device="cuda:0")
        J = torch.empty_like(Dd)
        K = torch.empty_like(Dd)
        # bounds ~1e-6 * Q^2: most quartets run in FP32 at a 1e-4 threshold
        fb.jk_mixed_device(Dd.data_ptr(), J.data_ptr(), K.data_ptr(), fp32_threshold=1e-4, skip_threshold=1e-14)
        fb.sync()
        Jm = J.cpu().numpy()
        Km = K.cpu().numpy()
    J64 = shells.unpack(J64, n)
    K64 = shells.unpack(K64, n)
    # FP32 recurrences on 1e-6-sized contributions: absolute error far below 1e-10
    assert np.abs(Jm - J64).max() < 1e-10
    assert np.abs(Km - K64).max() < 1e-10
    assert np.abs(Jm - J64).max() > 0.0  # the FP32 path actually ran


@pytest.mark.parametrize("name", ["water_631gs", "dimer_631gs", "w4_631gs", "dimer_631gs_6d"])
def test_incremental_scf_within_one_microhartree(name):
    d, mol, sh = load_case(name)
    with FockBuilder(schwarz_threshold=1e-12, boys_mode=BOYS_REF) as fb:
        fb.set_basis(sh)
        E, D, it, rc = fb.scf(d["H"], d["S"], sh.n_electrons() // 2, float(d["e_nuc"]), conv=1e-10, mixed=True)
    assert rc == 0
    assert abs(E - float(d["E"])) < 1e-6, (E, float(d["E"]))
