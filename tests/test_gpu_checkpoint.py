"""Density checkpoint round trip after device solves: save the converged
densities, read them back, restart the solve from them.  The restarted solve
lands on the same energy (1e-9 Eh, the plain form's bar) within a few
iterations (at most 5: the last ones move with the rounding of the J/K
atomics) instead of the core guess's dozens, where the saved state is a fixed
point of the loop; where it is not (the reference's loop stops on |dE| alone),
the restart follows the reference's loop (the oracle) from the same densities."""
import numpy as np
import pytest

from conftest import load_case
from dollarstorescf_b200 import _lib, shells
from dollarstorescf_b200.engine import BOYS_REF, FockBuilder

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fb():
    f = FockBuilder(schwarz_threshold=0.0, boys_mode=BOYS_REF)
    yield f
    f.close()


def test_rhf_restart_from_checkpoint(fb, tmp_path):
    d, mol, sh = load_case("water_631gs")
    fb.set_basis(sh)
    ne = sh.n_electrons() // 2
    E0, D0, it0, rc = fb.scf(d["H"], d["S"], ne, float(d["e_nuc"]), conv=1e-10)
    assert rc == 0
    path = str(tmp_path / "water.dss")
    fb.save_density(path)
    Da, Db, spins, na, nb = fb.load_density(path)
    assert spins == 1 and na == ne and nb == ne
    assert np.abs(Da - D0).max() < 1e-12 and np.array_equal(Da, Db)
    E1, D1, it1, rc = fb.scf(d["H"], d["S"], ne, float(d["e_nuc"]), conv=1e-10, guess=Da)
    assert rc == 0
    assert abs(E1 - E0) < 1e-9 and abs(E1 - float(d["E"])) < 1e-9
    assert it1 <= 5 < it0, (it1, it0)


def test_uhf_restart_from_checkpoint(fb, tmp_path):
    # Li doublet: the converged state is a fixed point of the loop, so the
    # restart stops within a few iterations at the same energy.
    d, mol, sh = load_case("li_631g_uhf")
    fb.set_basis(sh)
    na0, nb0 = int(d["n_alpha"]), int(d["n_beta"])
    E0, Da0, Db0, it0, rc = fb.uhf(d["H"], d["S"], na0, nb0, float(d["e_nuc"]), conv=1e-10)
    assert rc == 0
    path = str(tmp_path / "li.dss")
    fb.save_density(path)
    Da, Db, spins, na, nb = fb.load_density(path)
    assert (spins, na, nb) == (2, na0, nb0)
    assert np.abs(Da - Da0).max() < 1e-12 and np.abs(Db - Db0).max() < 1e-12
    E1, Da1, Db1, it1, rc = fb.uhf(d["H"], d["S"], na, nb, float(d["e_nuc"]), conv=1e-10, guess=(Da, Db))
    assert rc == 0
    assert abs(E1 - E0) < 1e-9 and abs(E1 - float(d["E"])) < 1e-9
    assert it1 <= 5 < it0, (it1, it0)


def test_uhf_restart_follows_the_reference_loop(fb, tmp_path):
    # CH2 triplet: the reference's loop stops on |dE| < conv at a state that is
    # not a fixed point of the iteration; restarted from its densities, the same
    # loop (the oracle, started from the same densities) descends to a lower
    # state.  The device restart from the checkpoint must land where the
    # oracle's does.
    from oracle import oracle

    d, mol, sh = load_case("ch2_631gs_uhf")
    fb.set_basis(sh)
    n = int(d["nbf"])
    na0, nb0 = int(d["n_alpha"]), int(d["n_beta"])
    E0, Da0, Db0, it0, rc = fb.uhf(d["H"], d["S"], na0, nb0, float(d["e_nuc"]), conv=1e-10)
    assert rc == 0 and abs(E0 - float(d["E"])) < 1e-9
    path = str(tmp_path / "ch2.dss")
    fb.save_density(path)
    Da, Db, spins, na, nb = fb.load_density(path)
    E1, Da1, Db1, it1, rc = fb.uhf(d["H"], d["S"], na, nb, float(d["e_nuc"]), conv=1e-10, guess=(Da, Db),
                                   max_iter=2000)
    assert rc == 0
    S, H = shells.unpack(d["S"], n), shells.unpack(d["H"], n)
    Eo, _, _, _ = oracle.scf_uhf(S, H, oracle.eri_tensor(sh), na, nb, float(d["e_nuc"]), max_iter=2000,
                                 guess=(shells.unpack(Da, n), shells.unpack(Db, n)))
    assert abs(E1 - Eo) < 1e-9, (E1, Eo)
    assert E1 < E0


def test_checkpoint_needs_a_solve_and_the_same_basis(fb, tmp_path):
    d, mol, sh = load_case("water_631gs")
    with FockBuilder() as fresh:
        fresh.set_basis(sh)
        with pytest.raises(_lib.DssError):
            fresh.save_density(str(tmp_path / "none.dss"))
    fb.set_basis(sh)
    fb.scf(d["H"], d["S"], sh.n_electrons() // 2, float(d["e_nuc"]), conv=1e-8)
    path = str(tmp_path / "w.dss")
    fb.save_density(path)
    d2, mol2, sh2 = load_case("ch4_631g")
    fb.set_basis(sh2)
    with pytest.raises(_lib.DssError):
        fb.load_density(path)
