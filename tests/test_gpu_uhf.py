"""GPU UHF parity: the unrestricted branch of the reference's SCF (multiplicity
> 1) through the C ABI against the reference's own converged energies (golden
fixtures, tests/golden/make_golden.py), plus invariants.

Tolerances: converged total energy 1e-9 Eh (the plain form's bar, both SCFs at
|dE| < 1e-10); S and H of the device one-electron kernels 1e-12 / 1e-11."""
import numpy as np
import pytest

from conftest import load_case
from dollarstorescf_b200 import _lib, shells
from dollarstorescf_b200.engine import BOYS_REF, FockBuilder

pytestmark = pytest.mark.gpu

UHF_CASES = ["ch2_631gs_uhf", "ch2_631g_uhf", "nh2_631g_uhf", "h2op_631g_uhf", "li_631g_uhf", "beh_631g_uhf",
             "hco_sto3g_uhf", "c2h3_sto3g_uhf"]


@pytest.fixture(scope="module")
def fb():
    f = FockBuilder(schwarz_threshold=0.0, boys_mode=BOYS_REF)
    yield f
    f.close()


@pytest.mark.parametrize("name", UHF_CASES)
def test_uhf_energy_matches_reference(fb, name):
    d, mol, sh = load_case(name)
    fb.set_basis(sh)
    S, T, V, en = fb.one_electron(sh)
    assert np.abs(S - d["S"]).max() < 1e-12
    assert np.abs((T + V) - d["H"]).max() < 1e-11
    na, nb = int(d["n_alpha"]), int(d["n_beta"])
    E, Da, Db, it, rc = fb.uhf(d["H"], d["S"], na, nb, float(d["e_nuc"]), conv=1e-10, max_iter=2000)
    assert rc == 0
    assert abs(E - float(d["E"])) < 1e-9, (name, E, float(d["E"]), it)
    n = int(d["nbf"])
    Sd = shells.unpack(d["S"], n)
    assert abs(np.sum(shells.unpack(Da, n) * Sd) - na) < 1e-8
    assert abs(np.sum(shells.unpack(Db, n) * Sd) - nb) < 1e-8


def test_uhf_closed_shell_equals_rhf(fb):
    # Equal spin occupations: the unrestricted loop lands on the RHF energy.
    d, mol, sh = load_case("water_631gs")
    fb.set_basis(sh)
    ne = sh.n_electrons() // 2
    E, Da, Db, it, rc = fb.uhf(d["H"], d["S"], ne, ne, float(d["e_nuc"]), conv=1e-10)
    assert rc == 0
    assert abs(E - float(d["E"])) < 1e-9
    assert np.abs(Da - Db).max() < 1e-8


def test_uhf_rejects_incremental_and_bad_counts(fb):
    d, mol, sh = load_case("li_631g_uhf")
    fb.set_basis(sh)
    n = int(d["nbf"])
    with pytest.raises(_lib.DssError):
        fb.uhf(d["H"], d["S"], n + 1, 1, float(d["e_nuc"]))
    rc = fb._L.dss_uhf_solve(fb._h, None, None, 1, 1, 0.0, None, None, None, None, None)
    assert rc != 0
