"""Device Boys function against the reference's own values (golden fixture of
flo::boysFunctionExact) and against the accurate function."""
import numpy as np
import pytest

from conftest import GOLDEN
from dollarstorescf_b200.engine import BOYS_FAST, BOYS_REF, FockBuilder

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fb():
    f = FockBuilder()
    yield f
    f.close()


@pytest.mark.parametrize("mode", [BOYS_REF, 2])
def test_ref_mode_matches_reference(fb, mode):
    d = np.load(f"{GOLDEN}/boys_ref.npz")
    x, ref = d["x"], d["F"]
    for L in (0, 3, 8, 12):
        F = fb.eval_boys(mode, L, x)
        # per m: relative 1e-13 (rounding of the partial sums; the stop rule is exact)
        for m in range(L + 1):
            rel = np.abs(F[:, m] - ref[:, m]) / np.maximum(np.abs(ref[:, m]), 1e-300)
            assert rel.max() < 1e-13, (L, m, rel.max(), x[rel.argmax()])


def test_ref_mode_dense_random_against_series(fb):
    rng = np.random.default_rng(5)
    x = np.concatenate([rng.uniform(0, 40, 200000), 10 ** rng.uniform(-12, 1, 20000)])
    for L in (0, 1, 4, 8):
        a = fb.eval_boys(BOYS_REF, L, x)
        b = fb.eval_boys(2, L, x)
        rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
        assert rel.max() < 1e-13, (L, rel.max())


def test_fast_mode_is_accurate(fb):
    import mpmath

    xs = np.array([0.0, 1e-6, 0.3, 2.0, 7.5, 19.0, 33.0, 36.0, 50.0, 120.0])
    F = fb.eval_boys(BOYS_FAST, 8, xs)
    for i, x in enumerate(xs):
        for m in range(9):
            exact = float(mpmath.hyp1f1(m + 0.5, m + 1.5, -x) / (2 * m + 1))
            assert F[i, m] == pytest.approx(exact, rel=5e-14, abs=1e-300)
