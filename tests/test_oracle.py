"""The oracle (CPU restatement) pinned against the reference's own outputs.

The golden fixtures were produced by the unmodified reference sources
(tests/golden/make_golden.py).  When oracle/_ref/libdssref.so is present the
oracle is also compared against the live reference.
"""
import math

import numpy as np
import pytest

from conftest import GOLDEN, load_case
from dollarstorescf_b200 import shells
from oracle import oracle, refpy


def test_boys_ref_matches_reference_values():
    d = np.load(f"{GOLDEN}/boys_ref.npz")
    for i, x in enumerate(d["x"]):
        for j, m in enumerate(d["m"]):
            got = oracle.boys_ref(float(x), int(m))
            ref = d["F"][i, j]
            assert got == pytest.approx(ref, rel=1e-15, abs=0.0), (x, m)


def test_boys_ref_truncation_is_visible():
    # The reference's 1e-9 series cut differs from the exact F_0 by ~1e-11 near x = 5.
    import mpmath

    x = 5.0
    exact = float(mpmath.sqrt(mpmath.pi / x) / 2 * mpmath.erf(mpmath.sqrt(x)))
    assert 1e-13 < abs(oracle.boys_ref(x, 0) - exact) < 1e-10


# Cartesian expansions printed by the reference's ContractedGaussian ctor at zeta=1.
EXPANSION_TABLE = {
    (0, 0): {(0, 0, 0): 0.2820947918},
    (1, -1): {(1, 0, 0): 0.4886025119},
    (1, 0): {(0, 0, 1): 0.4886025119},
    (1, 1): {(0, 1, 0): 0.4886025119},
    (2, -2): {(2, 0, 0): 0.5462742153, (0, 2, 0): -0.5462742153},
    (2, -1): {(1, 0, 1): 1.0925484306},
    (2, 0): {(0, 0, 2): 0.6307831305, (2, 0, 0): -0.3153915653, (0, 2, 0): -0.3153915653},
    (2, 1): {(0, 1, 1): 1.0925484306},
    (2, 2): {(1, 1, 0): 1.0925484306},
}


@pytest.mark.parametrize("lm", sorted(EXPANSION_TABLE))
def test_solid_harmonic_expansion(lm):
    got = oracle.sph_terms(*lm)
    want = EXPANSION_TABLE[lm]
    assert set(got) == set(want)
    for k, v in want.items():
        assert got[k] == pytest.approx(v, abs=1e-9)


def test_primitive_norm_table():
    assert oracle.prim_norm(0, 1.0) == pytest.approx(2.5264751110, abs=1e-9)
    assert oracle.prim_norm(1, 1.0) == pytest.approx(2.9173221709, abs=1e-9)
    assert oracle.prim_norm(2, 1.0) == pytest.approx(2.6093322745, abs=1e-9)


def test_generator_uses_same_expansion():
    import sys
    import os

    sys.path.insert(0, os.path.join(os.path.dirname(GOLDEN), "..", "dollarstorescf_b200", "csrc"))
    import gen_eri

    for l in range(4):
        for m in range(-l, l + 1):
            a = gen_eri.sph_terms(l, m)
            b = oracle.sph_terms(l, m)
            assert set(a) == {k for k, v in b.items() if v != 0.0}
            for k in a:
                assert a[k] == b[k]


@pytest.mark.parametrize("name", ["water_sto3g", "water_631gs", "water_631gs_6d", "ch4_631g", "h2_631g"])
def test_oracle_jk_matches_reference(name):
    d, mol, sh = load_case(name)
    n = int(d["nbf"])
    eri = oracle.eri_tensor(sh)
    for Dk, Jk, Kk in (("D", "J", "K"), ("D_rand", "J_rand", "K_rand")):
        D = shells.unpack(d[Dk], n)
        J, K = oracle.jk(eri, D)
        assert np.abs(shells.pack(J) - d[Jk]).max() < 1e-12
        assert np.abs(shells.pack(K) - d[Kk]).max() < 1e-12


@pytest.mark.parametrize("name", ["water_sto3g", "water_631gs", "water_631gs_6d", "ch4_631g", "he_631g"])
def test_oracle_scf_matches_reference_energy(name):
    d, mol, sh = load_case(name)
    n = int(d["nbf"])
    eri = oracle.eri_tensor(sh)
    S = shells.unpack(d["S"], n)
    H = shells.unpack(d["H"], n)
    E, D, it = oracle.scf_rhf(S, H, eri, sh.n_electrons() // 2, float(d["e_nuc"]))
    assert abs(E - float(d["E"])) < 1e-9


UHF_CASES = ["ch2_631gs_uhf", "ch2_631g_uhf", "nh2_631g_uhf", "h2op_631g_uhf", "li_631g_uhf", "beh_631g_uhf",
             "hco_sto3g_uhf", "c2h3_sto3g_uhf"]


@pytest.mark.parametrize("name", UHF_CASES)
def test_oracle_uhf_matches_reference_energy(name):
    d, mol, sh = load_case(name)
    n = int(d["nbf"])
    eri = oracle.eri_tensor(sh)
    S = shells.unpack(d["S"], n)
    H = shells.unpack(d["H"], n)
    E, Da, Db, it = oracle.scf_uhf(S, H, eri, int(d["n_alpha"]), int(d["n_beta"]), float(d["e_nuc"]), max_iter=2000)
    assert abs(E - float(d["E"])) < 1e-9
    # Electron counts tr(D_s S).  The densities themselves are not compared: where
    # occupied orbitals are (near-)degenerate the converged spin densities differ by
    # a rotation of equal energy between any two eigensolvers.
    assert abs(np.sum(Da * S) - int(d["n_alpha"])) < 1e-8
    assert abs(np.sum(Db * S) - int(d["n_beta"])) < 1e-8
    assert abs(np.sum(shells.unpack(d["Da"], n) * S) - int(d["n_alpha"])) < 1e-8


@pytest.mark.skipif(not refpy.available(), reason="oracle/_ref not built")
def test_oracle_eri_matches_live_reference():
    d, mol, sh = load_case("water_631gs_6d")
    refpy.setup(sh, build_tensor=False)
    eri = oracle.eri_tensor(sh)
    rng = np.random.default_rng(7)
    n = eri.shape[0]
    for _ in range(200):
        i, j, k, l = (int(v) for v in rng.integers(0, n, 4))
        assert abs(refpy.eri(i, j, k, l) - eri[i, j, k, l]) < 1e-13


@pytest.mark.skipif(not refpy.available(), reason="oracle/_ref not built")
def test_reference_harness_reproduces_golden_energy():
    d, mol, sh = load_case("water_sto3g")
    refpy.setup(sh)
    E, D, it, _ = refpy.scf(1e-10)
    assert E == pytest.approx(float(d["E"]), abs=1e-12)
    # The reference CPU program's published energy for water / STO-3G.
    assert E == pytest.approx(-74.9629349034878, abs=1e-12)


def test_oracle_uhf_restart_from_its_fixed_point():
    # Started from its own converged Li densities, the unrestricted loop stays.
    d, mol, sh = load_case("li_631g_uhf")
    n = int(d["nbf"])
    eri = oracle.eri_tensor(sh)
    S, H = shells.unpack(d["S"], n), shells.unpack(d["H"], n)
    a = (S, H, eri, int(d["n_alpha"]), int(d["n_beta"]), float(d["e_nuc"]))
    E0, Da, Db, it0 = oracle.scf_uhf(*a, max_iter=2000)
    E1, Da1, Db1, it1 = oracle.scf_uhf(*a, max_iter=2000, guess=(Da, Db))
    assert abs(E1 - E0) < 1e-12 and it1 <= 3 < it0
