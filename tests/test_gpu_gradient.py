"""Nuclear gradient of device solves (dss_gradient) against the derivative of
the reference's own converged energy (golden: a 4-point central difference of
reference SCF energies, tests/golden/make_golden.py).  The reference's analytic
gradient routine is not the target: it does not reproduce that derivative.

Tolerance: 1e-6 Eh/bohr (SCF converged to 1e-10 here, the golden's stencil
error ~1e-9).  Open-shell gradients are checked through the closed-shell limit
of the unrestricted path and through invariances."""
import numpy as np
import pytest

from conftest import GOLDEN, load_case
from dollarstorescf_b200.engine import BOYS_REF, FockBuilder

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fb():
    f = FockBuilder(schwarz_threshold=1e-12, boys_mode=BOYS_REF)
    yield f
    f.close()


@pytest.mark.parametrize("name", ["water_631gs", "ch4_631g"])
def test_rhf_gradient_is_the_derivative_of_the_reference_energy(fb, name):
    d, mol, sh = load_case(name)
    fb.set_basis(sh)
    E, D, it, rc = fb.scf(d["H"], d["S"], sh.n_electrons() // 2, float(d["e_nuc"]), conv=1e-10)
    assert rc == 0
    g = fb.gradient(sh)
    ref = np.load(f"{GOLDEN}/{name}_grad.npz")["grad"]
    assert np.abs(g - ref).max() < 1e-6, np.abs(g - ref).max()
    # Translational invariance.
    assert np.abs(g.sum(axis=0)).max() < 1e-8


def test_uhf_gradient_of_a_closed_shell_equals_rhf(fb):
    # Equal spin occupations: the unrestricted path (one build digesting K for
    # both spins) must give the derivative of the reference's RHF energy.
    d, mol, sh = load_case("water_631gs")
    fb.set_basis(sh)
    ne = sh.n_electrons() // 2
    E, Da, Db, it, rc = fb.uhf(d["H"], d["S"], ne, ne, float(d["e_nuc"]), conv=1e-10)
    assert rc == 0
    g = fb.gradient(sh)
    ref = np.load(f"{GOLDEN}/water_631gs_grad.npz")["grad"]
    assert np.abs(g - ref).max() < 1e-6, np.abs(g - ref).max()


def test_uhf_gradient_is_translation_and_rotation_free(fb):
    # CH2 triplet: no net force and no net torque on the isolated molecule, and
    # the two hydrogens at (+-x, y, 0) are mirror images.  (Displaced open-shell
    # solves of the reference land on different states, so there is no
    # difference-quotient golden for it.)
    d, mol, sh = load_case("ch2_631gs_uhf")
    fb.set_basis(sh)
    E, Da, Db, it, rc = fb.uhf(d["H"], d["S"], int(d["n_alpha"]), int(d["n_beta"]), float(d["e_nuc"]), conv=1e-10)
    assert rc == 0
    g = fb.gradient(sh)
    r = np.asarray(mol.xyz)
    assert np.abs(g.sum(axis=0)).max() < 1e-8
    assert np.abs(np.cross(r, g).sum(axis=0)).max() < 1e-7
    assert abs(g[1, 0] + g[2, 0]) < 1e-7 and abs(g[1, 1] - g[2, 1]) < 1e-7


def test_gradient_of_symmetric_water_is_symmetric(fb):
    d, mol, sh = load_case("water_631gs")
    fb.set_basis(sh)
    fb.scf(d["H"], d["S"], sh.n_electrons() // 2, float(d["e_nuc"]), conv=1e-10)
    g = fb.gradient(sh)
    # H at (+-x, y, 0): mirror images.
    assert abs(g[1, 0] + g[2, 0]) < 1e-8 and abs(g[1, 1] - g[2, 1]) < 1e-8
    assert np.abs(g[:, 2]).max() < 1e-8


def test_gradient_needs_a_solve(fb):
    from dollarstorescf_b200 import _lib

    d, mol, sh = load_case("water_631gs")
    with FockBuilder() as fresh:
        fresh.set_basis(sh)
        with pytest.raises(_lib.DssError):
            fresh.gradient(sh)


@pytest.mark.parametrize("name", ["water_631gs", "water_631gs_6d", "ch4_631g"])
def test_analytic_one_electron_terms_equal_difference_quotients(fb, name):
    # step 0: overlap, kinetic and nuclear-attraction derivatives analytic
    # (Hellmann-Feynman term included); step 1e-4: the same terms as central
    # differences of the device one-electron integrals.  O(h^2) ~ 1e-9.
    d, mol, sh = load_case(name)
    fb.set_basis(sh)
    E, D, it, rc = fb.scf(d["H"], d["S"], sh.n_electrons() // 2, float(d["e_nuc"]), conv=1e-10)
    assert rc == 0
    ga = fb.gradient(sh, step=0.0)
    gf = fb.gradient(sh, step=1e-4)
    assert np.abs(ga - gf).max() < 1e-7, np.abs(ga - gf).max()
    assert np.abs(ga.sum(axis=0)).max() < 1e-9
