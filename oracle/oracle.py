"""ORACLE — test infrastructure only.

CPU restatement of capytaine's Delhommeau Green function and of the indirect
BEM solve for one frequency.  Only ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` import this module; the product package
never does.

* Green function: ctypes bindings to ``liboracle_delhommeau.so`` (C++
  restatement of libs/libDelhommeau/src, built by ``oracle/Makefile``), wrapped
  the way capytaine ``green_functions/delhommeau.py:116-261, 336-520`` and
  ``green_functions/abstract_green_function.py:30-72`` wrap the Fortran core.
  Infinite depth, and finite depth by Delhommeau's method
  (``matrices.f90:197-305``, ``Green_wave.f90:311-508``) with the Prony
  decomposition of ``delhommeau.py:269-319`` restated here (seeded).
* Symmetric meshes: the block-circulant algebra of
  ``tools/block_circulant_matrices.py`` applied to the first block column.
* Solver glue: ``bem/solver.py:145-215`` (indirect method), boundary conditions
  ``bem/problems_and_results.py:373-381, 440-449``, Airy waves
  ``bem/airy_waves.py:19-102`` (finite depth too), force integration ``bodies/bodies.py:238-250``,
  coefficients ``bem/problems_and_results.py:583-592``; the linear algebra is
  SciPy's ``lu_factor``/``lu_solve``, which is what the reference calls
  (``tools/block_circulant_matrices.py:361-385``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass
from typing import Dict, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_delhommeau.so")

LEGACY_GRID, SCALED_NEMOH3_GRID = 0, 1
HIGH_FREQ, LOW_FREQ, LOW_FREQ_WITH_RANKINE_PART = 0, 1, 2
GRID_ENUM = {"legacy": LEGACY_GRID, "scaled_nemoh3": SCALED_NEMOH3_GRID}
SING_ENUM = {"high_freq": HIGH_FREQ, "low_freq": LOW_FREQ, "low_freq_with_rankine_part": LOW_FREQ_WITH_RANKINE_PART}


def build_oracle():
    """Compile the C++ restatement with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _load():
    if not os.path.exists(_LIB_PATH):
        build_oracle()
    lib = ctypes.CDLL(_LIB_PATH)
    d, i, p = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
    lib.oracle_exp_e1.argtypes = [d, d, p]
    lib.oracle_numerical_integration.argtypes = [d, d, i, p]
    lib.oracle_asymptotic_approximations.argtypes = [d, d, p]
    lib.oracle_default_r_spacing.argtypes = [i, d, i, p]
    lib.oracle_default_z_spacing.argtypes = [i, d, i, p]
    lib.oracle_nearest_r_index.argtypes = [d, p, i, i]
    lib.oracle_nearest_r_index.restype = i
    lib.oracle_nearest_z_index.argtypes = [d, p, i, i]
    lib.oracle_nearest_z_index.restype = i
    lib.oracle_construct_tabulation.argtypes = [p, i, p, i, i, p, i]
    lib.oracle_pick_in_default_tabulation.argtypes = [d, d, i, p, i, p, i, p, p]
    lib.oracle_wave_part_infinite_depth.argtypes = [i, p, p, d, i, i, p, i, p, i, p, i, p, p]
    lib.oracle_integral_of_rankine.argtypes = [i, p, p, p, p, p, p, i, i, p, p]
    lib.oracle_build_matrices.argtypes = [i, p, p, i, p, p, p, p, p, p, i, p, p, d, d, i, i, p, i, p, i, p, i, i,
                                          i, p, p, i]
    lib.oracle_build_matrices.restype = i
    lib.oracle_add_diagonal_term.argtypes = [i, i, p, p, d, i, p]
    lib.oracle_add_rankine_term_only.argtypes = [i, p, p, i, p, p, p, p, p, p, i, i, p, p, i]
    lib.oracle_build_matrices_finite_depth.argtypes = [i, p, p, i, p, p, p, p, p, p, i, p, p, d, d, i, i, p, i, p, i,
                                                       p, i, i, p, i, i, i, p, p, i]
    lib.oracle_build_matrices_finite_depth.restype = i
    lib.oracle_wave_parts_finite_depth.argtypes = [p, p, d, i, p, p, d, d, i, i, p, i, p, i, p, i, i, p]
    lib.oracle_wave_part_integral_infinite_depth.argtypes = [p, p, d, i, p, p, d, i, i, p, i, p, i, p, i, i, p]
    lib.oracle_prony_decomp_finite_depth.argtypes = [p, p, p, p, d, d, d, i, p, i, p]
    lib.oracle_pi.restype = d
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


# ---------------------------------------------------------------------------
# Delhommeau_integrals.f90 entry points
def exp_e1(z: complex) -> complex:
    out = np.zeros(2)
    lib().oracle_exp_e1(float(np.real(z)), float(np.imag(z)), _ptr(out))
    return complex(out[0], out[1])


def numerical_integration(r, z, npts) -> np.ndarray:
    out = np.zeros(5)
    lib().oracle_numerical_integration(float(r), float(z), int(npts), _ptr(out))
    return out


def asymptotic_approximations(r, z) -> np.ndarray:
    out = np.zeros(5)
    lib().oracle_asymptotic_approximations(float(r), float(z), _ptr(out))
    return out


def default_r_spacing(nr, rmax, method) -> np.ndarray:
    out = np.zeros(max(nr, 0))
    lib().oracle_default_r_spacing(int(nr), float(rmax), int(method), _ptr(out))
    return out


def default_z_spacing(nz, zmin, method) -> np.ndarray:
    out = np.zeros(max(nz, 0))
    lib().oracle_default_z_spacing(int(nz), float(zmin), int(method), _ptr(out))
    return out


def nearest_r_index(r, r_range, method) -> int:
    r_range = _c(r_range)
    return lib().oracle_nearest_r_index(float(r), _ptr(r_range), len(r_range), int(method))


def nearest_z_index(z, z_range, method) -> int:
    z_range = _c(z_range)
    return lib().oracle_nearest_z_index(float(z), _ptr(z_range), len(z_range), int(method))


def construct_tabulation(r_range, z_range, npts, nthreads=0) -> np.ndarray:
    r_range, z_range = _c(r_range), _c(z_range)
    out = np.zeros((len(r_range), len(z_range), 5))
    lib().oracle_construct_tabulation(_ptr(r_range), len(r_range), _ptr(z_range), len(z_range), int(npts),
                                      _ptr(out), int(nthreads))
    return out


# ---------------------------------------------------------------------------
class OracleDelhommeau:
    """CPU Delhommeau Green function with the reference's constructor defaults
    (capytaine green_functions/delhommeau.py:30-41)."""

    def __init__(self, *, tabulation_nr=676, tabulation_rmax=100.0, tabulation_nz=372, tabulation_zmin=-251.0,
                 tabulation_nb_integration_points=1001, tabulation_grid_shape="scaled_nemoh3",
                 gf_singularities="low_freq", nthreads=0, tabulation=None, finite_depth_method="newer"):
        if finite_depth_method not in ("legacy", "newer"):
            raise ValueError(f"finite_depth_method {finite_depth_method!r} is outside the oracle")
        self.finite_depth_method = finite_depth_method
        self.tabulation_nb_integration_points = int(tabulation_nb_integration_points)
        self.tabulation_grid_shape = tabulation_grid_shape
        self.tabulation_grid_shape_index = GRID_ENUM[tabulation_grid_shape]
        self.gf_singularities = gf_singularities
        self.floating_point_precision = "float64"
        self.nthreads = nthreads
        if tabulation is not None:
            r, z, v = tabulation
            self.tabulated_r_range, self.tabulated_z_range = _c(r), _c(z)
            self.tabulated_integrals = _c(v)
        else:
            self.tabulated_r_range = default_r_spacing(tabulation_nr, tabulation_rmax, self.tabulation_grid_shape_index)
            self.tabulated_z_range = default_z_spacing(tabulation_nz, tabulation_zmin, self.tabulation_grid_shape_index)
            self.tabulated_integrals = construct_tabulation(self.tabulated_r_range, self.tabulated_z_range,
                                                            self.tabulation_nb_integration_points, nthreads)

    @property
    def tabulation(self):
        return self.tabulated_r_range, self.tabulated_z_range, self.tabulated_integrals

    def _tab_args(self):
        t = self.tabulated_integrals if self.tabulated_integrals.size else np.zeros(5)
        return (self.tabulation_nb_integration_points, self.tabulation_grid_shape_index,
                _ptr(self.tabulated_r_range), len(self.tabulated_r_range),
                _ptr(self.tabulated_z_range), len(self.tabulated_z_range), _ptr(t))

    def wave_part_infinite_depth(self, x0i, x0j, k, gf_singularities=None):
        sing = SING_ENUM[gf_singularities or self.gf_singularities]
        x0i = _c(np.atleast_2d(x0i))
        x0j = _c(np.atleast_2d(x0j))
        n = x0i.shape[0]
        G = np.zeros((n, 2))
        nG = np.zeros((n, 3, 2))
        lib().oracle_wave_part_infinite_depth(n, _ptr(x0i), _ptr(x0j), float(k), *self._tab_args(), sing,
                                              _ptr(G), _ptr(nG))
        return G[:, 0] + 1j * G[:, 1], nG[..., 0] + 1j * nG[..., 1]

    @staticmethod
    def _colloc_and_normals(mesh1, mesh2, adjoint):
        """abstract_green_function.py:30-57"""
        if hasattr(mesh1, "faces_centers"):
            pts = mesh1.faces_centers
            nrm = mesh1.faces_normals if adjoint else mesh2.faces_normals
            return _c(pts), _c(nrm)
        pts = np.asarray(mesh1, dtype=float)
        if pts.ndim == 2 and pts.shape[1] == 3:
            nrm = np.zeros((pts.shape[0], 3)) if adjoint else mesh2.faces_normals
            return _c(pts), _c(nrm)
        raise ValueError(f"Unrecognized first input: {mesh1}")

    @staticmethod
    def _mesh_args(mesh2):
        qp, qw = mesh2.quadrature_points
        return (_c(mesh2.vertices), _c(mesh2.faces, np.int32), _c(mesh2.faces_centers), _c(mesh2.faces_normals),
                _c(mesh2.faces_areas), _c(mesh2.faces_radiuses), qp.shape[1], _c(qp), _c(qw))

    def evaluate_rankine_only(self, mesh1, mesh2, *, adjoint_double_layer=True, early_dot_product=True,
                              diagonal_term_in_double_layer=True):
        """delhommeau.py:336-402"""
        pts, nrm = self._colloc_and_normals(mesh1, mesh2, adjoint_double_layer)
        n, N = pts.shape[0], mesh2.nb_faces
        kdim = 1 if early_dot_product else 3
        S = np.zeros((n, N), order="F")
        K = np.zeros((kdim, n, N), order="F")
        v, f, c, nn, a, r, nq, qp, qw = self._mesh_args(mesh2)
        lib().oracle_add_rankine_term_only(n, _ptr(pts), _ptr(nrm), N, _ptr(v), _ptr(f), _ptr(c), _ptr(nn), _ptr(a),
                                           _ptr(r), int(adjoint_double_layer), kdim, _ptr(S), _ptr(K),
                                           self.nthreads)
        if diagonal_term_in_double_layer:
            Kc = K.astype(np.complex128, order="F")
            centers = _c(mesh2.faces_centers[:min(n, N)])
            lib().oracle_add_diagonal_term(n, N, _ptr(centers), _ptr(nrm), np.inf, kdim, _ptr(Kc))
            K = np.real(Kc).copy(order="F")
        if np.any(np.isnan(S)) or np.any(np.isnan(K)):
            raise FloatingPointError("Green function returned a NaN in the interaction matrix.")
        if early_dot_product:
            K = K.reshape((n, N), order="F")
        return S, K

    def evaluate(self, mesh1, mesh2, *, free_surface=0.0, water_depth=np.inf, wavenumber=1.0,
                 adjoint_double_layer=True, early_dot_product=True, diagonal_term_in_double_layer=True, prony=None):
        """delhommeau.py:405-520.  Finite water_depth: Delhommeau's finite-depth
        Green function with the Prony decomposition of prony_decomposition(k h)
        unless `prony` (2 x nexp: growth rates, then amplitudes) is given."""
        if free_surface == np.inf:
            if water_depth != np.inf:
                raise ValueError("When setting free_surface=inf, the water depth should also be infinite")
            return self.evaluate_rankine_only(mesh1, mesh2, adjoint_double_layer=adjoint_double_layer,
                                              early_dot_product=early_dot_product)
        pts, nrm = self._colloc_and_normals(mesh1, mesh2, adjoint_double_layer)
        n, N = pts.shape[0], mesh2.nb_faces
        kdim = 1 if early_dot_product else 3
        S = np.zeros((n, N), order="F", dtype=np.complex128)
        K = np.zeros((kdim, n, N), order="F", dtype=np.complex128)
        wavenumber = float(wavenumber)
        if water_depth < np.inf and self.finite_depth_method == "legacy" and self.gf_singularities != "low_freq":
            sing = "low_freq"  # delhommeau.py:467-471
        elif wavenumber == 0.0 and self.gf_singularities != "low_freq":
            sing = "low_freq"
        elif wavenumber == np.inf and self.gf_singularities != "high_freq":
            sing = "high_freq"
        elif np.any(abs(mesh2.faces_centers[:, 2]) < 1e-6) and self.gf_singularities != "low_freq":
            sing = "low_freq"
        else:
            sing = self.gf_singularities
        v, f, c, nn, a, r, nq, qp, qw = self._mesh_args(mesh2)
        if water_depth < np.inf:
            # delhommeau.py:492-497 and matrices.f90:197-305 (Delhommeau's method)
            if prony is None:
                prony = prony_decomposition(wavenumber * water_depth)
            pr = _c(prony)
            status = lib().oracle_build_matrices_finite_depth(
                n, _ptr(pts), _ptr(nrm), N, _ptr(v), _ptr(f), _ptr(c), _ptr(nn), _ptr(a), _ptr(r), nq, _ptr(qp),
                _ptr(qw), wavenumber, float(water_depth), *self._tab_args(),
                0 if self.finite_depth_method == "legacy" else 1, pr.shape[1], _ptr(pr), SING_ENUM[sing],
                int(adjoint_double_layer), kdim, _ptr(S), _ptr(K), self.nthreads)
        else:
            status = lib().oracle_build_matrices(n, _ptr(pts), _ptr(nrm), N, _ptr(v), _ptr(f), _ptr(c), _ptr(nn),
                                                 _ptr(a), _ptr(r), nq, _ptr(qp), _ptr(qw), wavenumber,
                                                 float(water_depth), *self._tab_args(), SING_ENUM[sing],
                                                 int(adjoint_double_layer), kdim, _ptr(S), _ptr(K), self.nthreads)
        if status != 0:
            raise RuntimeError(f"oracle_build_matrices failed with status {status}")
        if diagonal_term_in_double_layer:
            centers = _c(mesh2.faces_centers[:min(n, N)])
            lib().oracle_add_diagonal_term(n, N, _ptr(centers), _ptr(nrm), float(free_surface), kdim, _ptr(K))
        if early_dot_product:
            K = K.reshape((n, N), order="F")
        return S, K


    def wave_parts_finite_depth(self, x, face, k, depth, *, gf_singularities=None, deriv_first=True):
        """Green_wave.f90:311-425 for a point and the first face of `face`:
        (integral of G, integral of its gradient)."""
        return self._pair_wave(x, face, k, depth, gf_singularities, deriv_first)

    def wave_part_integral_infinite_depth(self, x, face, k, *, gf_singularities=None, deriv_first=True):
        """Green_wave.f90:50-124 for a point and the first face of `face`."""
        return self._pair_wave(x, face, k, None, gf_singularities, deriv_first)

    def _pair_wave(self, x, face, k, depth, gf_singularities, deriv_first):
        sing = SING_ENUM[gf_singularities or self.gf_singularities]
        qp, qw = face.quadrature_points
        x = _c(x)
        c = _c(face.faces_centers[0])
        q, w = _c(qp[0]), _c(qw[0])
        out = np.zeros(8)
        if depth is None:
            lib().oracle_wave_part_integral_infinite_depth(_ptr(x), _ptr(c), float(face.faces_areas[0]), len(w),
                                                           _ptr(q), _ptr(w), float(k), *self._tab_args(), sing,
                                                           int(deriv_first), _ptr(out))
        else:
            lib().oracle_wave_parts_finite_depth(_ptr(x), _ptr(c), float(face.faces_areas[0]), len(w), _ptr(q),
                                                 _ptr(w), float(k), float(depth), *self._tab_args(), sing,
                                                 int(deriv_first), _ptr(out))
        return complex(out[0], out[1]), out[2::2] + 1j * out[3::2]


def prony_decomp_finite_depth(x, face, depth, prony, deriv_first=True):
    """Green_wave.f90:427-508 for a point and the first face of `face`:
    (integral of the Prony terms, its gradient), real."""
    x = _c(x)
    nodes = _c(face.vertices[face.faces[0]])
    pr = _c(prony)
    out = np.zeros(4)
    lib().oracle_prony_decomp_finite_depth(_ptr(x), _ptr(nodes), _ptr(_c(face.faces_centers[0])),
                                           _ptr(_c(face.faces_normals[0])), float(face.faces_areas[0]),
                                           float(face.faces_radiuses[0]), float(depth), pr.shape[1], _ptr(pr),
                                           int(deriv_first), _ptr(out))
    return out[0], out[1:]


# ---------------------------------------------------------------------------
# Prony decomposition of the finite-depth Green function (restated from the
# method that capytaine's tools/prony_decomposition.py implements and that
# green_functions/delhommeau.py:269-319 applies, its default "python" method).
class PronyFailure(RuntimeError):
    pass


def exponential_fit(X, F, m):
    """Prony's method: approximate samples F = f(X) on the equispaced X by
    sum_i a_i exp(lambda_i x) with at most m terms.  The linear prediction
    F[j + m] = sum_l p_l F[j + m - l] is fitted by least squares, the roots z
    of z^m - sum_l p_l z^(m - l) give lambda = Re log(z) / dx (roots where the
    logarithm is undefined dropped, repeated rates merged, rates outside
    (-20, 0) dropped), then the amplitudes are fitted by least squares."""
    X, F = np.asarray(X, float), np.asarray(F, float)
    n = len(F)
    rows = np.array([F[j:j + m][::-1] for j in range(n - m)])   # F[j + m - 1], ..., F[j]
    p, *_ = np.linalg.lstsq(rows, F[m:], rcond=None)
    # z^m - p_1 z^(m-1) - ... - p_m, lowest degree first for polyroots
    coeffs = np.concatenate([-p[::-1], [1.0]])
    z = np.polynomial.polynomial.polyroots(coeffs)
    z = z[(np.imag(z) != 0.0) | (np.real(z) >= 0.0)]
    lam = np.unique(np.real(np.log(z.astype(complex)) / (X[1] - X[0])))
    lam = lam[(lam > -20.0) & (lam < 0.0)]
    E = np.exp(np.outer(X, lam))
    a, *_ = np.linalg.lstsq(E, F, rcond=None)
    return a, lam


def exponential_fit_error(X, F, a, lam):
    """Mean square error of sum_i a_i exp(lambda_i x) against F."""
    return float(np.mean((np.exp(np.outer(X, lam)) @ a - F) ** 2))


def best_exponential_fit(f, x_min, x_max, n_range, *, tol=1e-4, noise_std=0.01, rng=None):
    """First number of terms in n_range whose fit on 4 m + 1 points has a mean
    square error below tol on 8 m + 1 points; x_max is stretched by a random
    factor 1 + noise_std U[0, 1) per attempt, so that a point where f is
    singular (x = kh for the Green function, which is x_max when kh = 20) is
    not hit twice.  The reference draws from an unseeded generator; here the
    default generator is seeded, so that the oracle is deterministic."""
    rng = np.random.default_rng(0) if rng is None else rng
    for m in n_range:
        xm = (1 + noise_std * rng.uniform()) * x_max
        try:
            X = np.linspace(x_min, xm, 4 * m + 1)
            a, lam = exponential_fit(X, f(X), m)
            X = np.linspace(x_min, xm, 8 * m + 1)
            if exponential_fit_error(X, f(X), a, lam) < tol:
                return a, lam
        except Exception:  # a failed attempt moves on to the next size, as in the reference
            continue
    raise PronyFailure(f"no exponential decomposition in [{x_min}, {x_max}] for tol={tol} with m in {list(n_range)}")


def prony_decomposition(kh, *, noise_std=0.01, rng=None):
    """(2, nexp) array [growth rates; amplitudes] of the part of Delhommeau's
    finite-depth Green function approximated by exponentials, at kh = k h
    (delhommeau.py:296-319): the function of delhommeau.py:303-306 (or its
    large-kh limit) on [-0.1, 20] with 4 to 30 terms and tol 1e-4."""
    kh = float(kh)
    if kh <= 0.1:
        raise NotImplementedError(f"the finite-depth Green function is not evaluated for kh<=0.1 (kh={kh})")
    if kh < 1e5:
        t = np.tanh(kh)
        sing = (1 + t) ** 2 / (1 - t ** 2 + t / kh)

        def f(x):
            with np.errstate(all="ignore"):  # x = kh is a removable singularity; an attempt hitting it fails
                return (x + kh * t) * np.exp(x) / (x * np.sinh(x) - kh * t * np.cosh(x)) - sing / (x - kh) - 2
    else:
        def f(x):
            return -2 / (1 + np.exp(-2 * x)) + 2
    a, lam = best_exponential_fit(f, -0.1, 20.0, range(4, 31, 2), tol=1e-4, noise_std=noise_std, rng=rng)
    return np.stack([lam, a])


def finite_depth_wavenumber(omega, depth, g=9.81):
    """Root k > 0 of omega^2 / g = k tanh(k h) (problems_and_results.py:159-163)."""
    import scipy.optimize as so
    w2g = omega ** 2 / g
    if depth == np.inf or w2g in (0.0, np.inf):
        return w2g
    hi = max(w2g, 1.0) * 2 + 1.0 / depth
    while hi * np.tanh(hi * depth) < w2g:
        hi *= 2
    return so.brentq(lambda k: k * np.tanh(k * depth) - w2g, 1e-12, hi, xtol=1e-15, rtol=1e-15)


# ---------------------------------------------------------------------------
# Solver glue
@dataclass
class Dof:
    """Rigid-body dof: translation along ``direction`` or rotation about
    ``direction`` through ``center`` (capytaine bodies/dofs.py:60-98)."""
    kind: str
    direction: Sequence[float]
    center: Sequence[float] = (0.0, 0.0, 0.0)

    def motion(self, points: np.ndarray) -> np.ndarray:
        d = np.asarray(self.direction, float)
        if self.kind == "translation":
            return np.tile(d, (points.shape[0], 1))
        return np.cross(d, points - np.asarray(self.center, float))


@dataclass(frozen=True, eq=False)
class SubmeshDof:
    """A dof acting on the faces of `mask` only (capytaine bodies/dofs.py:100-127),
    zero elsewhere: the dofs of one body of a joined multibody."""
    dof: object
    mask: np.ndarray

    def motion(self, points: np.ndarray) -> np.ndarray:
        m = np.zeros((points.shape[0], 3))
        m[self.mask] = self.dof.motion(points[self.mask])
        return m


def rigid_body_dofs(rotation_center=(0.0, 0.0, 0.0), only=None) -> Dict[str, Dof]:
    """capytaine bodies/dofs.py:139-172"""
    dofs = {
        "Surge": Dof("translation", (1, 0, 0)),
        "Sway": Dof("translation", (0, 1, 0)),
        "Heave": Dof("translation", (0, 0, 1)),
        "Roll": Dof("rotation", (1, 0, 0), rotation_center),
        "Pitch": Dof("rotation", (0, 1, 0), rotation_center),
        "Yaw": Dof("rotation", (0, 0, 1), rotation_center),
    }
    if only is not None:
        dofs = {k: v for k, v in dofs.items() if k in only}
    return dofs


def _depth_profiles(z, k, depth):
    """cosh / sinh profiles of airy_waves.py:39-46, 76-81 (exp(kz) when k h >= 20)."""
    if 0 <= k * depth < 20:
        return np.cosh(k * (z + depth)) / np.cosh(k * depth), np.sinh(k * (z + depth)) / np.cosh(k * depth)
    return np.exp(k * z), np.exp(k * z)


def airy_waves_velocity(points, omega, k, g, beta, depth=np.inf):
    """airy_waves.py:56-95."""
    x, y, z = points.T
    wbar = x * np.cos(beta) + y * np.sin(beta)
    cih, sih = _depth_profiles(z, k, depth)
    v = g * k / omega * np.exp(1j * k * wbar) * np.array([np.cos(beta) * cih, np.sin(beta) * cih, -1j * sih])
    return v.T


def airy_waves_pressure(points, omega, k, g, rho, beta, depth=np.inf):
    """airy_waves.py:19-53 and 98-99."""
    x, y, z = points.T
    wbar = x * np.cos(beta) + y * np.sin(beta)
    cih, _ = _depth_profiles(z, k, depth)
    phi = -1j * g / omega * cih * np.exp(1j * k * wbar)
    return 1j * omega * rho * phi


def integrate_pressure(mesh, dofs: Dict[str, Dof], pressure):
    """bodies/bodies.py:238-250"""
    forces = {}
    for name, dof in dofs.items():
        m = dof.motion(mesh.faces_centers)
        ndof = -np.sum(m * mesh.faces_normals, axis=1)
        forces[name] = np.sum(pressure * ndof * mesh.faces_areas)
    return forces


def solve_gmres(A, b):
    """capytaine bem/engines.py:74-89: SciPy GMRES with atol=1e-6 (rtol 1e-5,
    restart 20 by default); RuntimeError when it does not converge."""
    import scipy.sparse.linalg as ssl
    x, info = ssl.gmres(A, b, atol=1e-6)
    if info > 0:
        raise RuntimeError(f"No convergence of the GMRES after {info} iterations.")
    return x


def solve_frequency(gf: OracleDelhommeau, mesh, dofs: Dict[str, Dof], omega: float, *, rho=1000.0, g=9.81,
                    wave_directions=(0.0,), free_surface=0.0, linear_solver="lu", hull_mask=None,
                    method="indirect", water_depth=np.inf):
    """One frequency-solve, indirect method (solver.py:188-207): assemble S and K at
    k = omega^2/g, factor K once, solve every radiation and diffraction RHS, take
    S @ sigma, integrate pressures.  Returns added mass, damping (dict of dict) and
    excitation forces (dict heading -> dict dof -> complex).  With `hull_mask`
    (mesh = hull faces then lid faces, problems_and_results.py:373-381,
    440-449) the boundary conditions are zero on the lid and the pressures are
    integrated on the hull only; dofs are then evaluated at the hull faces.
    method="direct": the potential solves D phi = S bc (bem/solver.py:172-187)."""
    import scipy.linalg as sl

    if water_depth != np.inf and free_surface == np.inf:
        raise ValueError("When setting free_surface=inf, the water depth should also be infinite")
    if method == "direct":
        return _solve_frequency_direct(gf, mesh, dofs, omega, rho=rho, g=g, wave_directions=wave_directions,
                                       water_depth=water_depth)
    if hull_mask is not None:
        return _solve_frequency_with_lid(gf, mesh, dofs, omega, rho=rho, g=g, wave_directions=wave_directions,
                                         water_depth=water_depth,
                                         linear_solver=linear_solver, hull_mask=np.asarray(hull_mask, bool))

    k = finite_depth_wavenumber(omega, water_depth, g) if free_surface != np.inf else 0.0
    S, K = gf.evaluate(mesh, mesh, free_surface=free_surface, water_depth=water_depth, wavenumber=k,
                       adjoint_double_layer=True, early_dot_product=True, diagonal_term_in_double_layer=True)
    lu = sl.lu_factor(K) if linear_solver == "lu" else None
    normals = mesh.faces_normals
    results = {"added_mass": {}, "radiation_damping": {}, "excitation": {}, "diffraction": {}, "froude_krylov": {}}
    rhs_list = []
    for name, dof in dofs.items():
        disp = np.sum(dof.motion(mesh.faces_centers) * normals, axis=1)
        rhs_list.append(("rad", name, -1j * omega * disp))
    if free_surface != np.inf:
        for beta in wave_directions:
            bc = -(airy_waves_velocity(mesh.faces_centers, omega, k, g, beta, water_depth) * normals).sum(axis=1)
            rhs_list.append(("dif", beta, bc))
    for kind, key, bc in rhs_list:
        rhs = bc.astype(np.complex128)
        if lu is not None:
            sigma = sl.lu_solve(lu, rhs)
        elif linear_solver == "gmres":
            sigma = solve_gmres(K, rhs)
        else:
            sigma = np.linalg.solve(K, rhs)
        potential = S @ sigma
        pressure = 1j * omega * rho * potential
        forces = integrate_pressure(mesh, dofs, pressure)
        if kind == "rad":
            results["added_mass"][key] = {d: float(np.real(f) / omega ** 2) for d, f in forces.items()}
            results["radiation_damping"][key] = {d: float(np.imag(f) / omega) for d, f in forces.items()}
        else:
            fk = integrate_pressure(mesh, dofs, airy_waves_pressure(mesh.faces_centers, omega, k, g, rho, key,
                                                                    water_depth))
            results["diffraction"][key] = forces
            results["froude_krylov"][key] = fk
            results["excitation"][key] = {d: forces[d] + fk[d] for d in forces}
    return results


def _solve_frequency_with_lid(gf, mesh, dofs, omega, *, rho, g, wave_directions, linear_solver, hull_mask,
                              water_depth=np.inf):
    """solve_frequency for a mesh whose faces outside hull_mask are a lid."""
    import scipy.linalg as sl
    k = finite_depth_wavenumber(omega, water_depth, g)
    S, K = gf.evaluate(mesh, mesh, free_surface=0.0, water_depth=water_depth, wavenumber=k,
                       adjoint_double_layer=True, early_dot_product=True, diagonal_term_in_double_layer=True)
    lu = sl.lu_factor(K) if linear_solver == "lu" else None
    c, nrm, area = mesh.faces_centers[hull_mask], mesh.faces_normals[hull_mask], mesh.faces_areas[hull_mask]
    N = mesh.nb_faces

    def solve(bc_hull):
        bc = np.zeros(N, dtype=np.complex128)
        bc[hull_mask] = bc_hull
        sigma = sl.lu_solve(lu, bc) if lu is not None else (solve_gmres(K, bc) if linear_solver == "gmres"
                                                            else np.linalg.solve(K, bc))
        return (1j * omega * rho * (S @ sigma))[hull_mask]

    def forces(pressure):
        return {name: np.sum(pressure * -np.sum(d.motion(c) * nrm, axis=1) * area) for name, d in dofs.items()}

    results = {"added_mass": {}, "radiation_damping": {}, "excitation": {}, "diffraction": {}, "froude_krylov": {}}
    for name, dof in dofs.items():
        f = forces(solve(-1j * omega * np.sum(dof.motion(c) * nrm, axis=1)))
        results["added_mass"][name] = {d: float(np.real(v) / omega ** 2) for d, v in f.items()}
        results["radiation_damping"][name] = {d: float(np.imag(v) / omega) for d, v in f.items()}
    for beta in wave_directions:
        dif = forces(solve(-(airy_waves_velocity(c, omega, k, g, beta, water_depth) * nrm).sum(axis=1)))
        fk = forces(airy_waves_pressure(c, omega, k, g, rho, beta, water_depth))
        results["diffraction"][beta] = dif
        results["froude_krylov"][beta] = fk
        results["excitation"][beta] = {d: dif[d] + fk[d] for d in dif}
    return results


def _solve_frequency_direct(gf, mesh, dofs, omega, *, rho, g, wave_directions, water_depth=np.inf):
    """Direct method (bem/solver.py:172-187): S, D with adjoint_double_layer=False,
    potential = D^-1 (S bc), pressure i omega rho potential."""
    import scipy.linalg as sl
    k = finite_depth_wavenumber(omega, water_depth, g)
    S, D = gf.evaluate(mesh, mesh, free_surface=0.0, water_depth=water_depth, wavenumber=k,
                       adjoint_double_layer=False, early_dot_product=True, diagonal_term_in_double_layer=True)
    lu = sl.lu_factor(D)
    c, nrm = mesh.faces_centers, mesh.faces_normals
    results = {"added_mass": {}, "radiation_damping": {}, "excitation": {}, "diffraction": {}, "froude_krylov": {}}

    def pressure(bc):
        return 1j * omega * rho * sl.lu_solve(lu, S @ bc.astype(np.complex128))
    for name, dof in dofs.items():
        f = integrate_pressure(mesh, dofs, pressure(-1j * omega * np.sum(dof.motion(c) * nrm, axis=1)))
        results["added_mass"][name] = {d: float(np.real(v) / omega ** 2) for d, v in f.items()}
        results["radiation_damping"][name] = {d: float(np.imag(v) / omega) for d, v in f.items()}
    for beta in wave_directions:
        dif = integrate_pressure(mesh, dofs, pressure(-(airy_waves_velocity(c, omega, k, g, beta, water_depth)
                                                        * nrm).sum(axis=1)))
        fk = integrate_pressure(mesh, dofs, airy_waves_pressure(c, omega, k, g, rho, beta, water_depth))
        results["diffraction"][beta] = dif
        results["froude_krylov"][beta] = fk
        results["excitation"][beta] = {d: dif[d] + fk[d] for d in dif}
    return results


# ---------------------------------------------------------------------------
# Symmetric meshes (bem/engines.py:178-247, tools/block_circulant_matrices.py)
def circulant_macro_blocks(blocks, nested):
    """Blocks of the first block column of a block-circulant matrix, from the
    first column of blocks of capytaine's matrix classes: BlockCirculantMatrix
    (nested=False: the blocks themselves) or NestedBlockCirculantMatrix
    (nested=True, 2n blocks: n macro-blocks of 2 x 2 blocks,
    NestedBlockCirculantMatrix.to_BlockCirculantMatrix,
    tools/block_circulant_matrices.py:226-266)."""
    blocks = np.asarray(blocks)
    if not nested:
        return blocks
    n = len(blocks) // 2
    macro = []
    for i in range(n):
        if i == 0:
            tl, tr, bl, br = blocks[0], blocks[1], blocks[1], blocks[0]
        else:
            tl, tr, bl, br = blocks[2 * i], blocks[2 * n - 2 * i + 1], blocks[2 * i + 1], blocks[2 * n - 2 * i]
        macro.append(np.block([[tl, tr], [bl, br]]))
    return np.asarray(macro)


def circulant_matvec(macro, x):
    """y = M x for the block-circulant M of first block column `macro`
    (BlockCirculantMatrix.__matmul__, tools/block_circulant_matrices.py:97-131):
    y_I = sum_J macro[(I - J) mod n] x_J."""
    n = len(macro)
    xs = np.split(np.asarray(x), n)
    return np.concatenate([sum(macro[(I - J) % n] @ xs[J] for J in range(n)) for I in range(n)])


def circulant_lu(macro):
    """LUDecomposedBlockCirculantMatrix (tools/block_circulant_matrices.py:404-419):
    the FFT of the first block column along the block axis, one LU per block."""
    import scipy.linalg as sl
    return [sl.lu_factor(b) for b in np.fft.fft(np.asarray(macro), axis=0)]


def circulant_solve(lus, b):
    """LUDecomposedBlockCirculantMatrix.solve: FFT of the right-hand side's
    segments, the block solves, the inverse FFT."""
    import scipy.linalg as sl
    n = len(lus)
    b = np.asarray(b, dtype=np.complex128)
    b_fft = np.fft.fft(b.reshape((n, -1)), axis=0)
    res = np.stack([sl.lu_solve(lu, bi) for lu, bi in zip(lus, b_fft)])
    return np.fft.ifft(res, axis=0).reshape(b.shape)


def solve_frequency_symmetric(gf, mesh, submesh, nb_blocks, nested, dofs, omega, *, rho=1000.0, g=9.81,
                              wave_directions=(0.0,), hull_mask=None, water_depth=np.inf):
    """solve_frequency for a mesh with symmetries, through capytaine's algorithm:
    S and K of the whole mesh's collocation points against the panels of the
    reference sub-mesh (the half, quarter, wedge or half wedge), split into the
    nb_blocks blocks of the first block column (engines.py:178-247, row blocks
    of the (N, N/nb_blocks) matrices), the block-circulant LU and solve, and
    S @ sigma as the block-circulant product.  `mesh` holds the faces of the
    whole mesh in the reference's order; nested=True for two planes or a
    rotation of a reflection (NestedBlockCirculantMatrix).  With hull_mask the
    faces outside it are a lid (zero boundary condition, no pressure)."""
    k = finite_depth_wavenumber(omega, water_depth, g)
    S, K = gf.evaluate(mesh, submesh, free_surface=0.0, water_depth=water_depth, wavenumber=k,
                       adjoint_double_layer=True, early_dot_product=True, diagonal_term_in_double_layer=True)
    ns = submesh.nb_faces
    Sm = circulant_macro_blocks(np.ascontiguousarray(S).reshape((nb_blocks, ns, ns)), nested)
    Km = circulant_macro_blocks(np.ascontiguousarray(K).reshape((nb_blocks, ns, ns)), nested)
    lus = circulant_lu(Km)
    N = mesh.nb_faces
    mask = np.ones(N, dtype=bool) if hull_mask is None else np.asarray(hull_mask, bool)
    c, nrm, area = mesh.faces_centers[mask], mesh.faces_normals[mask], mesh.faces_areas[mask]

    def solve(bc_hull):
        bc = np.zeros(N, dtype=np.complex128)
        bc[mask] = bc_hull
        sigma = circulant_solve(lus, bc)
        return (1j * omega * rho * circulant_matvec(Sm, sigma))[mask]

    def forces(pressure):
        return {name: np.sum(pressure * -np.sum(d.motion(c) * nrm, axis=1) * area) for name, d in dofs.items()}

    results = {"added_mass": {}, "radiation_damping": {}, "excitation": {}, "diffraction": {}, "froude_krylov": {}}
    for name, dof in dofs.items():
        f = forces(solve(-1j * omega * np.sum(dof.motion(c) * nrm, axis=1)))
        results["added_mass"][name] = {d: float(np.real(v) / omega ** 2) for d, v in f.items()}
        results["radiation_damping"][name] = {d: float(np.imag(v) / omega) for d, v in f.items()}
    for beta in wave_directions:
        dif = forces(solve(-(airy_waves_velocity(c, omega, k, g, beta, water_depth) * nrm).sum(axis=1)))
        fk = forces(airy_waves_pressure(c, omega, k, g, rho, beta, water_depth))
        results["diffraction"][beta] = dif
        results["froude_krylov"][beta] = fk
        results["excitation"][beta] = {d: dif[d] + fk[d] for d in dif}
    return results


def solve_radiation_limit_frequency(gf, mesh, dofs, omega, *, rho=1000.0, method="indirect", hull_mask=None,
                                    water_depth=np.inf):
    """Radiation problems at omega = 0 or infinity (bem/problems_and_results.py:
    440-449, 583-592 with the symbolic frequency of tools/symbolic_multiplication.py):
    the boundary condition -i omega (dof . n) and the pressure i omega rho phi
    carry omega as a symbolic factor that the added mass Re(F) / omega^2 cancels,
    so A = Re(F') with F' the force of the problem with boundary condition
    -i (dof . n) and pressure i rho phi, solved with the Green function at
    k = 0 (omega = 0, low_freq variant) or k = infinity (high_freq variant);
    the damping is zero.  Returns {"added_mass": {i: {j}}, "radiation_damping": ...}.
    Finite depth at omega = 0 raises NotImplementedError (no Prony
    decomposition at kh = 0), as the reference does."""
    import scipy.linalg as sl
    if omega not in (0.0, np.inf):
        raise ValueError("omega must be 0 or infinity")
    k = 0.0 if omega == 0.0 else np.inf
    mask = np.ones(mesh.nb_faces, dtype=bool) if hull_mask is None else np.asarray(hull_mask, bool)
    c, nrm, area = mesh.faces_centers[mask], mesh.faces_normals[mask], mesh.faces_areas[mask]
    adjoint = method == "indirect"
    S, K = gf.evaluate(mesh, mesh, free_surface=0.0, water_depth=water_depth, wavenumber=k,
                       adjoint_double_layer=adjoint, early_dot_product=True, diagonal_term_in_double_layer=True)
    lu = sl.lu_factor(K)
    out = {"added_mass": {}, "radiation_damping": {}}
    for name, dof in dofs.items():
        bc = np.zeros(mesh.nb_faces, dtype=np.complex128)
        bc[mask] = -1j * np.sum(dof.motion(c) * nrm, axis=1)
        phi = sl.lu_solve(lu, S @ bc) if not adjoint else S @ sl.lu_solve(lu, bc)
        p = (1j * rho * phi)[mask]
        forces = {d: np.sum(p * -np.sum(dd.motion(c) * nrm, axis=1) * area) for d, dd in dofs.items()}
        out["added_mass"][name] = {d: float(np.real(v)) for d, v in forces.items()}
        out["radiation_damping"][name] = {d: 0.0 for d in forces}
    return out
