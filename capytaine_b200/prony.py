"""Exponential (Prony) decomposition of the finite-depth part of Delhommeau's
Green function, on the host.

Capytaine approximates, for a dimensionless wavenumber kh = k h, the function

    f(x) = (x + kh tanh kh) e^x / (x sinh x - kh tanh kh cosh x)
           - c / (x - kh) - 2,     c = (1 + tanh kh)^2 / (1 - tanh^2 kh + tanh kh / kh)

(or its large-kh limit 2 - 2 / (1 + e^(-2x))) on [-0.1, 20] by a sum of
exponentials sum_i a_i exp(lambda_i x), with Prony's method and the first
number of terms in 4, 6, ..., 30 whose mean square error is below 1e-4
(green_functions/delhommeau.py:269-334, tools/prony_decomposition.py).  Each
exponential becomes four Rankine images in the finite-depth Green function
(Green_wave.f90:427-508).  The sampling interval is stretched by a random
factor of up to 1% per attempt so that a sample does not land twice on the
removable singularity x = kh; capytaine draws it from an unseeded generator,
this module from a seeded one, so that the decomposition of a given kh is
the same on every call and every run.
"""
from __future__ import annotations

from typing import Callable, Iterable, Tuple

import numpy as np

__all__ = ["PronyDecompositionFailure", "exponential_decomposition", "find_best_exponential_decomposition",
           "green_function_decomposition"]


class PronyDecompositionFailure(RuntimeError):
    """No decomposition met the tolerance (capytaine's PronyDecompositionFailure)."""


def exponential_decomposition(x: np.ndarray, y: np.ndarray, m: int) -> Tuple[np.ndarray, np.ndarray]:
    """Prony's method on equispaced samples y = f(x): amplitudes a and rates
    lambda of at most m exponentials.  The samples obey the recurrence
    y[j + m] + sum_i c_i y[j + i] = 0 (least squares over j); the roots z of
    z^m + sum_i c_i z^i give lambda = Re log z / dx, keeping roots where the
    logarithm is defined, distinct rates, and rates in (-20, 0); the
    amplitudes are then the least-squares fit of y."""
    x = np.asarray(x, dtype=float)
    y = np.asarray(y, dtype=float)
    if x.shape != y.shape or x.ndim != 1 or len(x) <= 2 * m:
        raise ValueError("need equispaced samples, more than 2 m of them")
    if not np.all(np.isfinite(y)):
        raise ValueError("a sample is not finite")
    n = len(y) - m
    hankel = np.lib.stride_tricks.sliding_window_view(y, m)[:n]  # hankel[j, i] = y[j + i]
    c, *_ = np.linalg.lstsq(hankel, -y[m:], rcond=None)
    roots = np.polynomial.polynomial.polyroots(np.append(c, 1.0))
    roots = roots[(np.imag(roots) != 0.0) | (np.real(roots) >= 0.0)]
    rates = np.unique(np.real(np.log(roots.astype(complex))) / (x[1] - x[0]))
    rates = rates[(rates > -20.0) & (rates < 0.0)]
    amplitudes, *_ = np.linalg.lstsq(np.exp(np.outer(x, rates)), y, rcond=None)
    return amplitudes, rates


def _mean_square_error(x, y, amplitudes, rates) -> float:
    return float(np.mean((np.exp(np.outer(x, rates)) @ amplitudes - y) ** 2))


def find_best_exponential_decomposition(f: Callable[[np.ndarray], np.ndarray], x_min: float, x_max: float,
                                        n_exp_range: Iterable[int], *, tol: float = 1e-4,
                                        noise_on_domain_points_std: float = 0.01,
                                        rng: np.random.Generator = None) -> Tuple[np.ndarray, np.ndarray]:
    """The first m of n_exp_range whose decomposition, fitted on 4 m + 1
    points of [x_min, x_max'], has a mean square error below tol on 8 m + 1
    points, x_max' = x_max (1 + noise U[0, 1)) drawn per attempt."""
    rng = np.random.default_rng(0) if rng is None else rng
    for m in n_exp_range:
        upper = (1.0 + noise_on_domain_points_std * rng.uniform()) * x_max
        try:
            xs = np.linspace(x_min, upper, 4 * m + 1)
            amplitudes, rates = exponential_decomposition(xs, f(xs), m)
            xs = np.linspace(x_min, upper, 8 * m + 1)
            if _mean_square_error(xs, f(xs), amplitudes, rates) < tol:
                return amplitudes, rates
        except (np.linalg.LinAlgError, ValueError, FloatingPointError):
            continue  # a failed attempt (singular sample, bad conditioning): next size
    raise PronyDecompositionFailure(f"No suitable Prony decomposition has been found in [{x_min}, {x_max}] for "
                                    f"tol={tol} using a number of terms in {list(n_exp_range)}.")


def green_function_decomposition(kh: float, *, rng: np.random.Generator = None) -> np.ndarray:
    """(2, nexp) array [rates; amplitudes] for the finite-depth Green function
    at kh (capytaine's "python" method).  NotImplementedError for kh <= 0.1,
    as capytaine."""
    kh = float(kh)
    if kh <= 0.1:
        raise NotImplementedError(f"cannot evaluate the finite depth Green function for kh<0.1 (kh={kh})")
    if kh < 1e5:
        t = np.tanh(kh)
        c = (1 + t) ** 2 / (1 - t ** 2 + t / kh)

        def f(x):
            with np.errstate(all="ignore"):
                return (x + kh * t) * np.exp(x) / (x * np.sinh(x) - kh * t * np.cosh(x)) - c / (x - kh) - 2
    else:
        def f(x):
            return 2.0 - 2.0 / (1.0 + np.exp(-2.0 * x))
    amplitudes, rates = find_best_exponential_decomposition(f, -0.1, 20.0, range(4, 31, 2), tol=1e-4, rng=rng)
    return np.stack([rates, amplitudes])
