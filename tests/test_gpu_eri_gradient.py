"""Analytic four-centre gradient (dss_eri_gradient: derivative ERIs fused with
the two-particle-density digest) against central differences of the oracle's
two-electron energy

  E_2e(R) = 1/2 sum_{ijkl} (ij|kl)(R) [D_ij D_kl - sum_s D^s_ik D^s_jl]

at fixed densities, the shells moving with their nucleus (the four-centre term
of chem/scf/ExactCoulomb.cpp:125-195 differentiated as in
chem/GaussianIntegral.cpp:1052-1459).  Unscreened bases (Schwarz threshold 0)
so the device and the oracle sum the same quartets.  Tolerance 1e-7 Eh/bohr
(the difference quotient's O(h^2) error at h = 1e-4 bohr is ~1e-9)."""
import numpy as np
import pytest

from conftest import load_case
from dollarstorescf_b200 import shells
from dollarstorescf_b200.engine import BOYS_REF, FockBuilder
from oracle import oracle

pytestmark = pytest.mark.gpu

H = 1e-4


def e2e(sh, D, Da=None, Db=None):
    eri = oracle.eri_tensor(sh)
    J = np.einsum("ijkl,kl->ij", eri, D)
    if Da is None:
        K = np.einsum("ikjl,kl->ij", eri, D)
        return 0.5 * np.sum(D * J) - 0.25 * np.sum(D * K)
    Ka = np.einsum("ikjl,kl->ij", eri, Da)
    Kb = np.einsum("ikjl,kl->ij", eri, Db)
    return 0.5 * np.sum(D * J) - 0.5 * (np.sum(Da * Ka) + np.sum(Db * Kb))


def fd_gradient(sh, D, Da=None, Db=None):
    g = np.zeros((sh.natom, 3))
    base = sh.centers.copy()
    for a in range(sh.natom):
        for d in range(3):
            vals = []
            for s in (1.0, -1.0):
                sh.centers = base.copy()
                sh.centers[sh.shell_atom == a, d] += s * H
                vals.append(e2e(sh, D, Da, Db))
            g[a, d] = (vals[0] - vals[1]) / (2 * H)
    sh.centers = base
    return g


def random_density(n, rng, scale=0.3):
    A = rng.standard_normal((n, n)) * scale
    return A + A.T


@pytest.fixture(scope="module")
def fb():
    f = FockBuilder(schwarz_threshold=0.0, boys_mode=BOYS_REF, primitive_threshold=0.0)
    yield f
    f.close()


@pytest.mark.parametrize("name", ["water_631gs", "water_631gs_6d", "water_sto3g"])
def test_closed_shell_eri_gradient_matches_difference_quotient(fb, name):
    d, mol, sh = load_case(name)
    fb.set_basis(sh)
    n = sh.nbf()
    D = random_density(n, np.random.default_rng(5))
    g = fb.eri_gradient(sh, shells.pack(D))
    ref = fd_gradient(sh, D)
    assert np.abs(g - ref).max() < 1e-7, np.abs(g - ref).max()
    assert np.abs(g.sum(axis=0)).max() < 1e-9


def test_open_shell_eri_gradient_matches_difference_quotient(fb):
    d, mol, sh = load_case("ch2_631gs_uhf")
    fb.set_basis(sh)
    n = sh.nbf()
    rng = np.random.default_rng(8)
    Da, Db = random_density(n, rng), random_density(n, rng)
    g = fb.eri_gradient(sh, shells.pack(Da + Db), shells.pack(Da), shells.pack(Db))
    ref = fd_gradient(sh, Da + Db, Da, Db)
    assert np.abs(g - ref).max() < 1e-7, np.abs(g - ref).max()


def test_eri_gradient_adds_into_the_output(fb):
    d, mol, sh = load_case("water_sto3g")
    fb.set_basis(sh)
    D = random_density(sh.nbf(), np.random.default_rng(2))
    g1 = fb.eri_gradient(sh, shells.pack(D))
    from dollarstorescf_b200.engine import _dp, _ip

    atom = np.ascontiguousarray(sh.shell_atom, dtype=np.int32)
    out = np.ones(3 * sh.natom)
    Dp = np.ascontiguousarray(shells.pack(D))
    rc = fb._L.dss_eri_gradient(fb._h, _dp(Dp), None, None, sh.natom, _ip(atom), _dp(out))
    assert rc == 0
    assert np.abs(out.reshape(-1, 3) - 1.0 - g1).max() < 1e-12
    bad = atom.copy()
    bad[0] = sh.natom
    assert fb._L.dss_eri_gradient(fb._h, _dp(Dp), None, None, sh.natom, _ip(bad), _dp(out)) == -1  # DSS_ERR_INVALID
