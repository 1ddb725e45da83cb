import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_case(name):
    """A golden fixture and its ShellArrays (built from the package's basis data)."""
    from dollarstorescf_b200 import basis, shells
    from dollarstorescf_b200.basis import Molecule

    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    mol = Molecule([int(z) for z in d["Z"]], [tuple(p) for p in d["xyz"]])
    sh = shells.build_shells(mol, basis.builtin_basis(str(d["basis"])), pure=bool(d["pure"]))
    return d, mol, sh


GOLDEN_CASES = ["water_sto3g", "water_sto3g_6d", "water_631g", "water_631gs", "water_631gs_6d",
                "dimer_631gs", "dimer_631gs_6d", "ch4_631g", "c3h8_sto3g", "w4_631gs", "w8_631gs", "he_631g",
                "h2_631g", "testwater_631gs"]


@pytest.fixture(scope="session")
def dss_lib():
    """libdss.so, built in-tree on first use if it is missing."""
    from dollarstorescf_b200 import _lib

    if not os.path.isfile(_lib.LIB_PATH):
        from dollarstorescf_b200 import build

        build.build()
    return _lib.load()
