"""GPU parity: J and K from the CUDA kernels (through the C ABI) against the
reference's own J[D_total], K[D_alpha] (golden fixtures) and the oracle.

Tolerances: reference Boys mode 1e-10 max-abs on the Fock-matrix pieces (the
plain-form bar); the accurate Boys mode 1e-8 (it differs from the reference's
truncated series by up to ~1e-10 per integral)."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_case
from dollarstorescf_b200 import shells
from dollarstorescf_b200.engine import BOYS_FAST, BOYS_REF, FockBuilder

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def builders():
    fb = {BOYS_REF: FockBuilder(schwarz_threshold=0.0, boys_mode=BOYS_REF),
          BOYS_FAST: FockBuilder(schwarz_threshold=0.0, boys_mode=BOYS_FAST)}
    yield fb
    for f in fb.values():
        f.close()


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_jk_matches_reference(builders, name):
    d, mol, sh = load_case(name)
    fb = builders[BOYS_REF]
    assert fb.set_basis(sh) == int(d["nbf"])
    for Dk, Jk, Kk in (("D", "J", "K"), ("D_rand", "J_rand", "K_rand")):
        # The reference's J uses D_total = 2 D_alpha and K uses D_alpha.
        J, K = fb.jk(2.0 * d[Dk])
        assert np.abs(J - d[Jk]).max() < 1e-10, name
        assert np.abs(0.5 * K - d[Kk]).max() < 1e-10, name
    # Fock two-electron part G = J - K/2 against the reference's computeCoulombTerms/ExchangeTerms.
    J, K = fb.jk(2.0 * d["D"])
    assert np.abs((J - 0.5 * K) - d["G"]).max() < 1e-10


@pytest.mark.parametrize("name", ["water_631gs", "dimer_631gs_6d", "w4_631gs"])
def test_fast_boys_close_to_reference(builders, name):
    d, mol, sh = load_case(name)
    fb = builders[BOYS_FAST]
    fb.set_basis(sh)
    J, K = fb.jk(2.0 * d["D"])
    assert np.abs(J - d["J"]).max() < 1e-8
    assert np.abs(0.5 * K - d["K"]).max() < 1e-8


def test_schwarz_screening_error_is_small(builders):
    d, mol, sh = load_case("w4_631gs")
    with FockBuilder(schwarz_threshold=1e-12, boys_mode=BOYS_REF) as fb:
        fb.set_basis(sh)
        sq, pq, wt = fb.work_stats()
        assert sq > 0 and pq >= sq and wt > 0
        J, K = fb.jk(2.0 * d["D"])
    assert np.abs(J - d["J"]).max() < 1e-10
    assert np.abs(0.5 * K - d["K"]).max() < 1e-10


def test_jk_linearity_and_symmetry(builders):
    d, mol, sh = load_case("dimer_631gs")
    fb = builders[BOYS_REF]
    fb.set_basis(sh)
    n = int(d["nbf"])
    rng = np.random.default_rng(3)
    A = rng.standard_normal((n, n)); A = A + A.T
    B = rng.standard_normal((n, n)); B = B + B.T
    Ja, Ka = fb.jk(shells.pack(A))
    Jb, Kb = fb.jk(shells.pack(B))
    Jab, Kab = fb.jk(shells.pack(2.0 * A - 0.5 * B))
    assert np.abs(Jab - (2 * Ja - 0.5 * Jb)).max() < 1e-10
    assert np.abs(Kab - (2 * Ka - 0.5 * Kb)).max() < 1e-10
    # tr(D_B J[D_A]) == tr(D_A J[D_B]) (ERI pair symmetry)
    ta = np.sum(B * shells.unpack(Ja, n))
    tb = np.sum(A * shells.unpack(Jb, n))
    assert abs(ta - tb) < 1e-9 * max(1.0, abs(ta))


def test_errors_are_reported_not_fatal(builders):
    fb = FockBuilder(schwarz_threshold=0.0)
    from dollarstorescf_b200._lib import DssError
    with pytest.raises(DssError, match="no basis"):
        fb.jk(np.zeros(0))  # no basis yet: rejected by the library
    d, mol, sh = load_case("water_sto3g")
    sh.shell_l[0] = 7
    with pytest.raises(DssError, match="above the compiled maximum"):
        fb.set_basis(sh)
    fb.close()


@pytest.mark.parametrize("name", ["dimer_631gs", "dimer_631gs_6d"])
def test_kernel_variants_agree(builders, name):
    # Every class through each kernel shape it has (thread per quartet in the
    # three register tiers and, where compiled, the warp-cooperative kernel):
    # all must reproduce the reference.
    d, mol, sh = load_case(name)
    fb = builders[BOYS_REF]
    fb.set_basis(sh)
    n = fb.num_classes()
    results = []
    for variant in (0, 2, 3, 1, 4, 5, 6, 7, 8):
        for i in range(n):
            try:
                fb.set_class_variant(i, variant)
            except Exception:
                fb.set_class_variant(i, 0)
        J, K = fb.jk(2.0 * d["D_rand"])
        assert np.abs(J - d["J_rand"]).max() < 1e-10
        assert np.abs(0.5 * K - d["K_rand"]).max() < 1e-10
        results.append((J, K))
    for i in range(n):
        fb.set_class_variant(i, -1)


@pytest.mark.parametrize("name", ["dimer_631gs", "dimer_631gs_6d", "water_sto3g"])
def test_persistent_launch_matches_reference(builders, name):
    # The grouped persistent kernels (device work queue over the classes of a
    # register group) reproduce the reference's J and K like the per-class launches.
    d, mol, sh = load_case(name)
    fb = builders[BOYS_REF]
    fb.set_basis(sh)
    fb.set_persistent(True)
    try:
        for _ in range(2):  # the queue heads are re-zeroed before every launch
            J, K = fb.jk(2.0 * d["D_rand"])
            assert np.abs(J - d["J_rand"]).max() < 1e-10
            assert np.abs(0.5 * K - d["K_rand"]).max() < 1e-10
    finally:
        fb.set_persistent(False)


@pytest.mark.parametrize("name", ["dimer_631gs", "dimer_631gs_6d"])
def test_list_scheduled_launches_match_reference(builders, name):
    # After a profile the context knows every class's launch time, and plain
    # builds launch the classes longest first onto the least-loaded side stream
    # (two profiles: the times of more than one shape are kept).  J and K must
    # not change.
    import torch

    d, mol, sh = load_case(name)
    fb = builders[BOYS_REF]
    n = fb.set_basis(sh)
    D = torch.tensor(2.0 * shells.unpack(d["D_rand"], n), dtype=torch.float64, device="cuda:0")
    J0, K0 = torch.empty_like(D), torch.empty_like(D)
    fb.profile_build(D.data_ptr(), J0.data_ptr(), K0.data_ptr())
    fb.set_class_variant(0, 2)
    fb.profile_build(D.data_ptr(), J0.data_ptr(), K0.data_ptr())
    try:
        for _ in range(2):
            J, K = fb.jk(2.0 * d["D_rand"])
            assert np.abs(J - d["J_rand"]).max() < 1e-10
            assert np.abs(0.5 * K - d["K_rand"]).max() < 1e-10
    finally:
        fb.set_class_variant(0, -1)
