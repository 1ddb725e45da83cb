"""Molden output after device solves against the reference's own Molden files
(scf::writeOrbitalsMolden, tests/golden/*.molden from make_golden.py), compared
as parsed content: the reference prints 5 decimals for coordinates, 8
significant digits for exponents, coefficients and MO coefficients, and 6 for
orbital energies, so the tolerances follow those widths.  MO coefficients are
compared per orbital up to its sign (eigenvectors are defined up to sign).

The WFX files (scf::writeOrbitalsWFX, tests/golden/*.wfx) are compared the same
way: integer sections exactly, coordinates to the reference's 7 decimals,
exponents, energies and primitive coefficients to its 8 significant digits."""
import os
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, load_case
from dollarstorescf_b200.engine import BOYS_REF, FockBuilder

pytestmark = pytest.mark.gpu


def parse_molden(path):
    with open(path) as f:
        lines = [ln.rstrip("\n") for ln in f]
    assert lines[0] == "[Molden Format]" and lines[1] == "[5D]"
    i = lines.index("[Atoms] AU") + 1
    atoms = []
    while not lines[i].startswith("["):
        t = lines[i].split()
        atoms.append((t[0], int(t[1]), int(t[2]), [float(v) for v in t[3:6]]))
        i += 1
    assert lines[i] == "[GTO]"
    i += 1
    gto = []
    while lines[i] != "[MO]":
        if not lines[i].strip():
            i += 1
            continue
        t = lines[i].split()
        if len(t) == 2 and t[1] == "0":
            gto.append([])
            i += 1
            continue
        label, nprim = t[0], int(t[1])
        prims = [tuple(float(v) for v in lines[i + 1 + k].split()) for k in range(nprim)]
        gto[-1].append((label, prims))
        i += 1 + nprim
    i += 1
    mos = []
    while i < len(lines):
        if not lines[i].startswith("Sym="):
            i += 1
            continue
        sym = lines[i].split()[1]
        ene = float(lines[i + 1].split()[1])
        spin = lines[i + 2].split()[1]
        occ = int(lines[i + 3].split()[1])
        i += 4
        coefs = []
        while i < len(lines) and lines[i].strip() and not lines[i].startswith("Sym="):
            coefs.append(float(lines[i].split()[1]))
            i += 1
        mos.append((sym, ene, spin, occ, np.array(coefs)))
    return atoms, gto, mos


def compare(ours, ref):
    a1, g1, m1 = ours
    a2, g2, m2 = ref
    assert [(s, i, z) for s, i, z, _ in a1] == [(s, i, z) for s, i, z, _ in a2]
    for (_, _, _, x1), (_, _, _, x2) in zip(a1, a2):
        assert np.abs(np.array(x1) - np.array(x2)).max() < 1e-5
    assert len(g1) == len(g2)
    for sh1, sh2 in zip(g1, g2):
        assert [(lb, len(p)) for lb, p in sh1] == [(lb, len(p)) for lb, p in sh2]
        for (_, p1), (_, p2) in zip(sh1, sh2):
            assert np.allclose(np.array(p1), np.array(p2), rtol=2e-7, atol=0)
    assert [(s, sp, o) for s, _, sp, o, _ in m1] == [(s, sp, o) for s, _, sp, o, _ in m2]
    for (_, e1, _, _, c1), (_, e2, _, _, c2) in zip(m1, m2):
        assert abs(e1 - e2) <= 1e-5 * max(1.0, abs(e2))
        assert c1.shape == c2.shape
        sign = 1.0 if np.dot(c1, c2) >= 0 else -1.0
        assert np.abs(sign * c1 - c2).max() < 2e-6, (np.abs(sign * c1 - c2).max())


@pytest.fixture(scope="module")
def fb():
    f = FockBuilder(schwarz_threshold=0.0, boys_mode=BOYS_REF)
    yield f
    f.close()


def test_rhf_molden_matches_reference(fb, tmp_path):
    d, mol, sh = load_case("water_631gs")
    fb.set_basis(sh)
    E, D, it, rc = fb.scf(d["H"], d["S"], sh.n_electrons() // 2, float(d["e_nuc"]), conv=1e-10)
    assert rc == 0
    out = str(tmp_path / "water.molden")
    fb.write_molden(out, sh, write_virtual=True)
    compare(parse_molden(out), parse_molden(os.path.join(GOLDEN, "water_631gs.molden")))
    C, eps = fb.orbitals(0)
    n = sh.nbf()
    occ = sh.n_electrons() // 2
    Dm = C[:, :occ] @ C[:, :occ].T
    from dollarstorescf_b200 import shells

    assert np.abs(shells.pack(Dm) - D).max() < 1e-12


def test_uhf_molden_matches_reference(fb, tmp_path):
    d, mol, sh = load_case("ch2_631gs_uhf")
    fb.set_basis(sh)
    E, Da, Db, it, rc = fb.uhf(d["H"], d["S"], int(d["n_alpha"]), int(d["n_beta"]), float(d["e_nuc"]), conv=1e-10)
    assert rc == 0
    out = str(tmp_path / "ch2.molden")
    fb.write_molden(out, sh, write_virtual=True)
    compare(parse_molden(out), parse_molden(os.path.join(GOLDEN, "ch2_631gs_uhf.molden")))


def test_molden_rejects_cartesian_and_unsolved(fb, tmp_path):
    from dollarstorescf_b200 import _lib

    d, mol, sh = load_case("water_631gs_6d")
    fb.set_basis(sh)
    fb.scf(d["H"], d["S"], sh.n_electrons() // 2, float(d["e_nuc"]), conv=1e-8)
    with pytest.raises(_lib.DssError):
        fb.write_molden(str(tmp_path / "x.molden"), sh)
    with FockBuilder() as fresh:
        fresh.set_basis(sh)
        with pytest.raises(_lib.DssError):
            fresh.write_molden(str(tmp_path / "y.molden"), sh)


def parse_wfx(path):
    """{section: [lines]} of a WFX file (MO coefficients: one list per orbital)."""
    with open(path) as f:
        lines = [ln.strip() for ln in f]
    out, i = {}, 0
    while i < len(lines):
        ln = lines[i]
        if ln.startswith("<") and not ln.startswith("</"):
            tag = ln[1:-1]
            j = lines.index(f"</{tag}>", i + 1)
            if tag == "Molecular Orbital Primitive Coefficients":
                mos, k = [], i + 1
                while k < j:
                    assert lines[k] == "<MO Number>" and lines[k + 2] == "</MO Number>"
                    k += 3
                    vals = []
                    while k < j and lines[k] != "<MO Number>":
                        vals += [float(v) for v in lines[k].split()]
                        k += 1
                    mos.append(np.array(vals))
                out[tag] = mos
            else:
                out[tag] = [x for x in lines[i + 1:j] if x]
            i = j + 1
        else:
            i += 1
    return out


def compare_wfx(ours, ref, n_beta=None):
    exact = ["Keywords", "Number of Nuclei", "Net Charge", "Number of Electrons", "Number of Alpha Electrons",
             "Number of Beta Electrons", "Electronic Spin Multiplicity", "Nuclear Names", "Atomic Numbers",
             "Number of Primitives", "Molecular Orbital Spin Types"]
    for tag in exact:
        assert ours[tag] == ref[tag], tag
    for tag in ("Primitive Centers", "Primitive Types"):
        assert " ".join(ours[tag]).split() == " ".join(ref[tag]).split(), tag

    def nums(d, tag):
        return np.array([float(v) for v in " ".join(d[tag]).split()])

    # The reference prints coordinates with 7 decimals, exponents and energies
    # with 8 significant digits.
    assert np.abs(nums(ours, "Nuclear Cartesian Coordinates") - nums(ref, "Nuclear Cartesian Coordinates")).max() < 1e-6
    assert np.allclose(nums(ours, "Primitive Exponents"), nums(ref, "Primitive Exponents"), rtol=2e-7, atol=0)
    e1, e2 = nums(ours, "Molecular Orbital Energies"), nums(ref, "Molecular Orbital Energies")
    assert np.all(np.abs(e1 - e2) <= 1e-5 * np.maximum(1.0, np.abs(e2)))
    occ1, occ2 = nums(ours, "Molecular Orbital Occupation Numbers"), nums(ref, "Molecular Orbital Occupation Numbers")
    if n_beta is None:
        assert np.array_equal(occ1, occ2)
    else:
        # Beta occupations: the reference counts alpha electrons there
        # (WriteOrbitals.cpp:350); these count beta electrons.
        nmo = len(occ1) // 2
        assert np.array_equal(occ1[:nmo], occ2[:nmo])
        assert np.array_equal(occ1[nmo:], (np.arange(nmo) < n_beta).astype(float))
    m1, m2 = ours["Molecular Orbital Primitive Coefficients"], ref["Molecular Orbital Primitive Coefficients"]
    assert len(m1) == len(m2)
    for c1, c2 in zip(m1, m2):
        assert c1.shape == c2.shape
        sign = 1.0 if np.dot(c1, c2) >= 0 else -1.0
        assert np.abs(sign * c1 - c2).max() < 2e-6 * max(1.0, np.abs(c2).max()), np.abs(sign * c1 - c2).max()


def test_rhf_wfx_matches_reference(fb, tmp_path):
    d, mol, sh = load_case("water_631gs")
    fb.set_basis(sh)
    E, D, it, rc = fb.scf(d["H"], d["S"], sh.n_electrons() // 2, float(d["e_nuc"]), conv=1e-10)
    assert rc == 0
    out = str(tmp_path / "water.wfx")
    fb.write_wfx(out, sh, write_virtual=True)
    compare_wfx(parse_wfx(out), parse_wfx(os.path.join(GOLDEN, "water_631gs.wfx")))


def test_uhf_wfx_matches_reference(fb, tmp_path):
    d, mol, sh = load_case("ch2_631gs_uhf")
    fb.set_basis(sh)
    nb = int(d["n_beta"])
    E, Da, Db, it, rc = fb.uhf(d["H"], d["S"], int(d["n_alpha"]), nb, float(d["e_nuc"]), conv=1e-10)
    assert rc == 0
    out = str(tmp_path / "ch2.wfx")
    fb.write_wfx(out, sh, write_virtual=True)
    compare_wfx(parse_wfx(out), parse_wfx(os.path.join(GOLDEN, "ch2_631gs_uhf.wfx")), n_beta=nb)


def test_wfx_occupied_only_and_rejections(fb, tmp_path):
    from dollarstorescf_b200 import _lib

    d, mol, sh = load_case("water_631gs")
    fb.set_basis(sh)
    fb.scf(d["H"], d["S"], sh.n_electrons() // 2, float(d["e_nuc"]), conv=1e-10)
    out = str(tmp_path / "occ.wfx")
    fb.write_wfx(out, sh, write_virtual=False)
    w = parse_wfx(out)
    assert len(w["Molecular Orbital Primitive Coefficients"]) == sh.n_electrons() // 2
    assert w["Molecular Orbital Occupation Numbers"] == ["2"] * (sh.n_electrons() // 2)
    d6, mol6, sh6 = load_case("water_631gs_6d")
    fb.set_basis(sh6)
    fb.scf(d6["H"], d6["S"], sh6.n_electrons() // 2, float(d6["e_nuc"]), conv=1e-8)
    with pytest.raises(_lib.DssError):
        fb.write_wfx(str(tmp_path / "x.wfx"), sh6)
