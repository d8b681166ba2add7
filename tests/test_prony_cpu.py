"""Host-side Prony decomposition of the package (capytaine_b200.prony and
Delhommeau.find_best_exponential_decomposition) against the reference's
known answers (pytest/test_green_functions_finite_depth.py:114-182) and
against the oracle's independent restatement of the same method."""
import numpy as np
import pytest

from capytaine_b200 import _lib, prony
from capytaine_b200.green_function import Delhommeau


def test_two_exponentials():
    """test_green_functions_finite_depth.py:130-135"""
    x = np.linspace(0.0, 1.0, 100)
    a, lam = prony.exponential_decomposition(x, 2 * np.exp(-x) - 4 * np.exp(-2 * x), 2)
    order = np.argsort(lam)
    np.testing.assert_allclose(a[order], [-4.0, 2.0])
    np.testing.assert_allclose(lam[order], [-2.0, -1.0])


def test_six_exponentials():
    """test_green_functions_finite_depth.py:138-148 (same seed and draws; the
    fastest rate is not determined by the samples, see the oracle's test)."""
    rng = np.random.default_rng(seed=987654321)
    a_ref = rng.uniform(-10.0, 10.0, size=6)
    lam_ref = -rng.chisquare(1.0, size=6)

    def f(x):
        return sum(a_ref[i] * np.exp(lam_ref[i] * x) for i in range(6))
    a, lam = prony.find_best_exponential_decomposition(f, 0.0, 100.0, range(2, 15), tol=1e-4,
                                                       noise_on_domain_points_std=0.0)
    assert np.allclose(np.sort(a), np.sort(a_ref))
    np.testing.assert_allclose(np.sort(lam)[1:], np.sort(lam_ref)[1:], rtol=1e-5)


def test_green_function_decomposition_methods_and_domain():
    """test_green_functions_finite_depth.py:114-119, 151-163, 175-182."""
    gf = Delhommeau(tabulation_cache_dir=None)
    for kh in (0.10, 0.01):
        with pytest.raises((NotImplementedError, _lib.GreenFunctionEvaluationError)):
            gf.find_best_exponential_decomposition(kh)
    with pytest.raises(NotImplementedError):
        gf.find_best_exponential_decomposition(1.0, method="fortran")
    with pytest.raises(ValueError):
        gf.find_best_exponential_decomposition(1.0, method="unknown")
    for kh in (20.0, np.inf, 1.0):
        d = gf.find_best_exponential_decomposition(kh)
        assert d.shape[0] == 2 and np.all(d[0] < 0) and np.all(d[0] > -20)
    np.testing.assert_array_equal(gf.find_best_exponential_decomposition(3.0),
                                  Delhommeau(tabulation_cache_dir=None).find_best_exponential_decomposition(3.0))


@pytest.mark.parametrize("kh", [0.5, 1.0, 4.0, 20.0, 300.0, 1e6])
def test_same_decomposition_as_the_oracle(oracle_mod, kh):
    """Two independent implementations of the method, the same seeded stretch:
    the same number of terms and the same rates and amplitudes."""
    mine = prony.green_function_decomposition(kh)
    ref = oracle_mod.prony_decomposition(kh)
    assert mine.shape == ref.shape
    np.testing.assert_allclose(mine, ref, rtol=1e-6, atol=1e-9)
