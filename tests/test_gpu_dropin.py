"""The reference's own SCF driver with the GPU engine dropped in.

oracle/_ref/libdssref_gpu.so is the unmodified reference with
chem/scf/ExactCoulomb.cpp replaced by dollarstorescf_b200/shim/ExactCoulomb_gpu.cpp
(linked against libdss.so).  Its scf::solveMOs / calculateEnergies must give the
reference CPU energy within 1e-9 Eh.  Each case runs in a fresh process (the
reference keeps global state)."""
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

GPU_LIB = os.path.join(ROOT, "oracle", "_ref", "libdssref_gpu.so")

SCRIPT = r"""
import sys, numpy as np
sys.path.insert(0, {root!r}); sys.path.insert(0, {root!r} + "/tests")
from conftest import load_case
from oracle import refpy
d, mol, sh = load_case({name!r})
refpy.setup(sh)
E, D, it, secs = refpy.scf(1e-10)
print(repr(E), repr(float(d["E"])))
"""


@pytest.mark.skipif(not os.path.isfile(GPU_LIB), reason="drop-in library not built")
@pytest.mark.parametrize("name", ["water_sto3g", "water_631gs", "dimer_631gs", "w4_631gs"])
def test_reference_driver_with_gpu_fock_build(name):
    env = dict(os.environ, DSS_REF_LIB="libdssref_gpu.so", DSS_SCHWARZ="0")
    out = subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT, name=name)], env=env,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    E, Eref = (float(v) for v in out.stdout.split())
    assert abs(E - Eref) < 1e-9, (name, E, Eref)
