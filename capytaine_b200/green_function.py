"""Drop-in Delhommeau Green function evaluated by the sm_100a kernels.

Mirrors capytaine ``green_functions/delhommeau.py`` (constructor keywords and
defaults ``:30-41, 116-183``, tabulation cache file name ``:208-247``,
``evaluate`` ``:405-520``, ``evaluate_rankine_only`` ``:336-402``) and
``green_functions/abstract_green_function.py:30-72`` (collocation points,
normals, output shapes and dtypes).  ``evaluate`` returns NumPy arrays like the
reference; ``evaluate_device`` returns device tensors for the GPU engine.
"""
from __future__ import annotations

import logging
import os
import threading
from collections import OrderedDict
from typing import Optional

import numpy as np

from . import _lib

LOG = logging.getLogger(__name__)

_default_parameters = dict(
    tabulation_nr=676,
    tabulation_rmax=100.0,
    tabulation_nz=372,
    tabulation_zmin=-251.0,
    tabulation_nb_integration_points=1001,
    tabulation_grid_shape="scaled_nemoh3",
    finite_depth_method="newer",
    finite_depth_prony_decomposition_method="python",
    floating_point_precision="float64",
    gf_singularities="low_freq",
)

_GRID = {"legacy": _lib.BEM_GRID_LEGACY, "scaled_nemoh3": _lib.BEM_GRID_SCALED_NEMOH3}
_SING = {"high_freq": _lib.BEM_GF_HIGH_FREQ, "low_freq": _lib.BEM_GF_LOW_FREQ,
         "low_freq_with_rankine_part": _lib.BEM_GF_LOW_FREQ_WITH_RANKINE_PART}


def default_cache_directory() -> Optional[str]:
    """``$CAPYTAINE_CACHE_DIR`` when set (shares the reference's tabulation
    files), else a per-user directory."""
    d = os.environ.get("CAPYTAINE_CACHE_DIR")
    if d:
        return d
    return os.path.join(os.path.expanduser("~"), ".cache", "capytaine_b200")


class DeviceMesh:
    """Device copies of the per-face arrays the assembly kernel reads."""

    def __init__(self, mesh, device):
        import torch
        qp, qw = mesh.quadrature_points
        f64 = torch.float64
        self.nb_faces = mesh.nb_faces
        self.nb_vertices = mesh.nb_vertices
        # one transfer, no wait for the stream's earlier work
        (self.vertices, self.faces, self.centers, self.normals, self.areas, self.radii, self.quad_points,
         self.quad_weights) = _lib.upload_many(
            [(mesh.vertices, f64), (np.asarray(mesh.faces, dtype=np.int32), torch.int32), (mesh.faces_centers, f64),
             (mesh.faces_normals, f64), (mesh.faces_areas, f64), (mesh.faces_radiuses, f64), (qp, f64), (qw, f64)],
            device)
        self.nb_quad_points = qp.shape[1]
        self.centers_z = np.asarray(mesh.faces_centers[:, 2])
        # one quadrature point per face, at the face centre (collocation point)
        self.collocation_at_quadrature = bool(qp.shape[1] == 1 and np.array_equal(qp[:, 0, :], mesh.faces_centers))
        self.nbytes = sum(t.numel() * t.element_size() for t in
                          (self.vertices, self.faces, self.centers, self.normals, self.areas, self.radii,
                           self.quad_points, self.quad_weights))
        self.shared = _lib.StreamShared(self.vertices, self.faces, self.centers, self.normals, self.areas,
                                        self.radii, self.quad_points, self.quad_weights)


class Delhommeau:
    """Delhommeau's infinite-depth Green function on a B200.

    Same keywords and defaults as capytaine's ``Delhommeau``, plus
    ``precision`` ("fp64": every term in float64; "mixed": float32 far field and
    wave term, float64 near field) and ``device``.
    """

    dispersion_relation_roots = np.empty(1)

    def __init__(self, *, tabulation_nr=_default_parameters["tabulation_nr"],
                 tabulation_rmax=_default_parameters["tabulation_rmax"],
                 tabulation_nz=_default_parameters["tabulation_nz"],
                 tabulation_zmin=_default_parameters["tabulation_zmin"],
                 tabulation_nb_integration_points=_default_parameters["tabulation_nb_integration_points"],
                 tabulation_grid_shape=_default_parameters["tabulation_grid_shape"],
                 tabulation_cache_dir="default",
                 finite_depth_method=_default_parameters["finite_depth_method"],
                 finite_depth_prony_decomposition_method=_default_parameters["finite_depth_prony_decomposition_method"],
                 floating_point_precision=_default_parameters["floating_point_precision"],
                 gf_singularities=_default_parameters["gf_singularities"],
                 precision="fp64", device=None):
        if tabulation_grid_shape not in _GRID:
            raise KeyError(tabulation_grid_shape)
        if gf_singularities not in _SING:
            raise KeyError(gf_singularities)
        if floating_point_precision not in ("float32", "float64"):
            raise NotImplementedError(f"Unsupported floating point precision: {floating_point_precision}")
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.tabulation_grid_shape = tabulation_grid_shape
        self.tabulation_grid_shape_index = _GRID[tabulation_grid_shape]
        self.gf_singularities = gf_singularities
        self.gf_singularities_fortran_enum = dict(_SING)
        self.finite_depth_method = finite_depth_method
        self.finite_depth_prony_decomposition_method = finite_depth_prony_decomposition_method
        self.floating_point_precision = floating_point_precision
        self.tabulation_nb_integration_points = int(tabulation_nb_integration_points)
        self.precision = precision
        self._device = device
        self.tabulation_cache_dir = default_cache_directory() if tabulation_cache_dir == "default" \
            else tabulation_cache_dir
        self._tab_params = (int(tabulation_nr), float(tabulation_rmax), int(tabulation_nz), float(tabulation_zmin))
        self.tabulated_r_range = self._spacing("r")
        self.tabulated_z_range = self._spacing("z")
        self._tab_host = None
        self._dev_tab = None
        self._dev_tab_inv = (0, 0)
        self._mesh_cache: "OrderedDict[str, DeviceMesh]" = OrderedDict()
        # The caches are shared by the threads (and CUDA streams) of a request
        # server: dictionary updates under this lock, device readiness through
        # StreamShared events.
        self._lock = threading.RLock()
        # Rankine parts of mesh-with-itself assemblies, reused across wavenumbers
        # (device memory budget in bytes; 0 disables the reuse).
        self.rankine_cache_bytes = 4 << 30
        # A mesh with itself without a reusable Rankine part: Rankine part into K,
        # then the wave term once per pair of faces (False: the general kernel).
        self.symmetric_assembly = True
        self._rankine_cache: "OrderedDict[tuple, object]" = OrderedDict()
        # Prony decompositions by k h (the 128 most recently used)
        self._prony_cache: "OrderedDict[float, np.ndarray]" = OrderedDict()
        self.exportable_settings = {
            "green_function": self.__class__.__name__,
            "tabulation_nr": tabulation_nr,
            "tabulation_rmax": tabulation_rmax,
            "tabulation_nz": tabulation_nz,
            "tabulation_zmin": tabulation_zmin,
            "tabulation_nb_integration_points": tabulation_nb_integration_points,
            "tabulation_grid_shape": tabulation_grid_shape,
            "finite_depth_method": finite_depth_method,
            "finite_depth_prony_decomposition_method": finite_depth_prony_decomposition_method,
            "floating_point_precision": floating_point_precision,
            "gf_singularities": gf_singularities,
            "precision": precision,
        }
        self._hash = hash(tuple(self.exportable_settings.values()))

    def __hash__(self):
        return self._hash

    def find_best_exponential_decomposition(self, dimensionless_wavenumber, *, method=None):
        """Exponential decomposition [rates; amplitudes] (2 x nexp) of the part of
        the finite-depth Green function at kh = dimensionless_wavenumber, as
        capytaine's Delhommeau.find_best_exponential_decomposition
        (delhommeau.py:269-334): method "python" (the default here and there)
        is capytaine_b200.prony.green_function_decomposition, deterministic for
        a given kh and cached (128 values); the legacy "fortran" method of Nemoh
        is not part of this library."""
        from . import prony
        method = (method or self.finite_depth_prony_decomposition_method).lower()
        if method == "fortran":
            raise NotImplementedError("the legacy Fortran Prony decomposition is not part of capytaine_b200; "
                                      "use method='python'")
        if method != "python":
            raise ValueError(f"Unrecognized name for the Prony decomposition method: {method!r}. "
                             "Expected 'python' or 'fortran'.")
        kh = float(dimensionless_wavenumber)
        cache = self._prony_cache
        with self._lock:
            hit = cache.get(kh)
            if hit is not None:
                cache.move_to_end(kh)  # least recently used first out
        if hit is None:
            try:
                hit = prony.green_function_decomposition(kh)
            except prony.PronyDecompositionFailure as e:
                raise _lib.GreenFunctionEvaluationError(
                    _lib.BEM_ERR_NOT_CONVERGED, f"{self} cannot evaluate finite depth Green function for kh={kh}") from e
            with self._lock:
                cache[kh] = hit
                while len(cache) > 128:
                    cache.popitem(last=False)
        return hit.copy()

    def __str__(self):
        items = [f"{k}={v!r}" for k, v in self.exportable_settings.items()
                 if k in _default_parameters and v != _default_parameters[k]]
        if self.precision != "fp64":
            items.append(f"precision={self.precision!r}")
        return f"{self.__class__.__name__}({', '.join(items)})"

    __repr__ = __str__

    # ---- tabulation -------------------------------------------------------
    def _spacing(self, axis):
        nr, rmax, nz, zmin = self._tab_params
        lib = _lib.load()
        if axis == "r":
            out = np.zeros(max(nr, 0))
            _lib.check(lib.bem_default_r_spacing(nr, rmax, self.tabulation_grid_shape_index,
                                                 out.ctypes.data_as(_lib.c_void_p)))
        else:
            out = np.zeros(max(nz, 0))
            _lib.check(lib.bem_default_z_spacing(nz, zmin, self.tabulation_grid_shape_index,
                                                 out.ctypes.data_as(_lib.c_void_p)))
        return out

    @property
    def _cache_filename(self):
        nr, rmax, nz, zmin = self._tab_params
        return "tabulation_{}_{}_{}_{}_{}_{}_{}.npz".format(
            self.floating_point_precision, self.tabulation_grid_shape, nr, rmax, nz, zmin,
            self.tabulation_nb_integration_points)

    @property
    def device(self):
        return _lib.require_cuda(self._device)

    def _device_tabulation(self):
        """Device table (float64 and float32 copies), built on the GPU or loaded
        from the tabulation cache (capytaine delhommeau.py:208-261)."""
        with self._lock:
            if self._dev_tab is None:
                self._build_device_tabulation()
            self._dev_tab_shared.acquire()
            return self._dev_tab

    def _build_device_tabulation(self):
        import torch
        dev = self.device
        r = torch.as_tensor(self.tabulated_r_range, dtype=torch.float64, device=dev)
        z = torch.as_tensor(self.tabulated_z_range, dtype=torch.float64, device=dev)
        nr, nz = r.numel(), z.numel()
        table = None
        path = None
        if self.tabulation_cache_dir is not None and nr > 1 and nz > 1:
            path = os.path.join(self.tabulation_cache_dir, self._cache_filename)
            if os.path.exists(path):
                try:
                    arrs = np.load(path)
                    if arrs["values"].shape == (nr, nz, 5):
                        table = torch.as_tensor(np.ascontiguousarray(arrs["values"], dtype=np.float64), device=dev)
                        r = torch.as_tensor(arrs["r_range"], dtype=torch.float64, device=dev)
                        z = torch.as_tensor(arrs["z_range"], dtype=torch.float64, device=dev)
                        self.tabulated_r_range = np.asarray(arrs["r_range"], dtype=np.float64)
                        self.tabulated_z_range = np.asarray(arrs["z_range"], dtype=np.float64)
                except (EOFError, FileNotFoundError, KeyError, ValueError, OSError):
                    LOG.warning("Error loading tabulation from %s", path)
                    table = None
        if table is None:
            table = torch.empty((max(nr, 1), max(nz, 1), 5), dtype=torch.float64, device=dev)
            if nr > 1 and nz > 1:
                _lib.call("bem_construct_tabulation", _lib.ptr(r), nr, _lib.ptr(z), nz,
                          self.tabulation_nb_integration_points, _lib.ptr(table), _lib.stream_ptr())
                if path is not None:
                    try:
                        os.makedirs(self.tabulation_cache_dir, exist_ok=True)
                        np.savez_compressed(path, r_range=self.tabulated_r_range, z_range=self.tabulated_z_range,
                                            values=table.cpu().numpy())
                    except OSError:
                        LOG.warning("Could not save tabulation to %s", path)
        self._dev_tab = (r, z, table, table.to(torch.float32))
        # reciprocal denominators of the Lagrange weights of both grids: the
        # lookup multiplies instead of dividing (bem_tabulation_inverse_denominators)
        self._dev_tab_inv = (0, 0)
        if nr > 2 and nz > 2:
            inv = []
            for rng in (np.ascontiguousarray(self.tabulated_r_range, dtype=np.float64),
                        np.ascontiguousarray(self.tabulated_z_range, dtype=np.float64)):
                out = np.zeros(3 * len(rng))
                _lib.check(_lib.load().bem_tabulation_inverse_denominators(rng.ctypes.data_as(_lib.c_void_p),
                                                                           len(rng),
                                                                           out.ctypes.data_as(_lib.c_void_p)))
                inv.append(torch.as_tensor(out, device=dev))
            self._dev_tab_inv_tensors = tuple(inv)
            self._dev_tab_inv = tuple(t.data_ptr() for t in inv)
        self._dev_tab_shared = _lib.StreamShared(*self._dev_tab)

    @property
    def tabulated_integrals(self) -> np.ndarray:
        r, z, table, _ = self._device_tabulation()
        return table.cpu().numpy()

    @property
    def all_tabulation_parameters(self):
        return (self.tabulation_nb_integration_points, self.tabulation_grid_shape_index,
                self.tabulated_r_range, self.tabulated_z_range, self.tabulated_integrals)

    # ---- meshes -------------------------------------------------------------
    def device_mesh(self, mesh) -> DeviceMesh:
        key = mesh.content_hash
        with self._lock:
            dm = self._mesh_cache.get(key)
            if dm is not None:
                self._mesh_cache.move_to_end(key)
                dm.shared.acquire()
                return dm
        # built outside the lock (host geometry and uploads on this thread's
        # stream), so that threads with cached meshes do not wait for it
        fresh = DeviceMesh(mesh, self.device)
        with self._lock:
            dm = self._mesh_cache.get(key)
            if dm is None:  # another thread may have built the same mesh meanwhile
                dm = fresh
                self._mesh_cache[key] = dm
                while len(self._mesh_cache) > 8:
                    self._mesh_cache.popitem(last=False)
            else:
                self._mesh_cache.move_to_end(key)
            dm.shared.acquire()
        return dm

    def _collocation(self, mesh1, mesh2, adjoint):
        """abstract_green_function.py:30-57 on the device."""
        import torch
        dev = self.device
        if hasattr(mesh1, "faces_centers"):
            dm1 = self.device_mesh(mesh1)
            pts = dm1.centers
            nrm = dm1.normals if adjoint else self.device_mesh(mesh2).normals
            return pts, nrm
        pts = np.asarray(mesh1, dtype=float)
        if pts.ndim == 2 and pts.shape[1] == 3:
            pts_t = torch.as_tensor(np.ascontiguousarray(pts), dtype=torch.float64, device=dev)
            nrm = torch.zeros_like(pts_t) if adjoint else self.device_mesh(mesh2).normals
            return pts_t, nrm
        raise ValueError(f"Unrecognized first input for {self.__class__.__name__}.evaluate:\n{mesh1}")

    # ---- evaluation ---------------------------------------------------------
    def _variant(self, mesh2_centers_z, wavenumber):
        """Singularity variant overrides of delhommeau.py:466-490."""
        if wavenumber == 0.0 and self.gf_singularities != "low_freq":
            return "low_freq"
        if wavenumber == np.inf and self.gf_singularities != "high_freq":
            return "high_freq"
        if np.any(abs(mesh2_centers_z) < 1e-6) and self.gf_singularities != "low_freq":
            LOG.warning("Overriding gf_singularities=%r because of free surface panels", self.gf_singularities)
            return "low_freq"
        return self.gf_singularities

    def assemble_into(self, mesh1, mesh2, S, K, *, free_surface=0.0, water_depth=np.inf, wavenumber=1.0,
                      adjoint_double_layer=True, early_dot_product=True, diagonal_term_in_double_layer=True,
                      lds=None, ldk=None, k_plane_stride=None, precision=None, stream=None, nan_flag=None,
                      reuse_rankine=True, sweep=None, lu_planes=None):
        """Write S and K into caller-owned device buffers (column-major with
        leading dimensions lds/ldk) through ``bem_assemble``.  For a mesh with
        itself the wavenumber-independent Rankine part is kept and reused
        across calls unless reuse_rankine is False.  sweep = (wavenumbers,
        s_stride, k_stride): S and K of every wavenumber (finite, > 0; the
        variant is chosen with the first), the outputs of wavenumber i at
        S + i * s_stride and K + i * k_stride elements, in one launch per 64
        wavenumbers on the Rankine-reuse path.  lu_planes = (workspace pointer,
        npad, first matrix): on that path K is also written rounded to float32
        into the planes of a mixed-LU workspace; returns True when it was."""
        import torch
        if free_surface == np.inf and water_depth != np.inf:
            raise ValueError("When setting free_surface=inf, the water depth should also be infinite")
        if water_depth != np.inf:
            return self._assemble_finite_depth(mesh1, mesh2, S, K, free_surface=free_surface, water_depth=water_depth,
                                               wavenumber=wavenumber, adjoint_double_layer=adjoint_double_layer,
                                               early_dot_product=early_dot_product,
                                               diagonal_term_in_double_layer=diagonal_term_in_double_layer,
                                               lds=lds, ldk=ldk, k_plane_stride=k_plane_stride,
                                               precision=precision, stream=stream, nan_flag=nan_flag, sweep=sweep)
        pts, nrm = self._collocation(mesh1, mesh2, adjoint_double_layer)
        dm2 = self.device_mesh(mesh2)
        n = pts.shape[0]
        wavenumber = float(wavenumber)
        sing = self._variant(dm2.centers_z, wavenumber) if free_surface != np.inf else self.gf_singularities
        # the table is loaded when any wavenumber of the call is finite and > 0;
        # the paths that share work across a sweep need every one of them to be
        ks_all = [wavenumber] if sweep is None else [float(k) for k in sweep[0]]
        finite_ks = [0.0 < k < np.inf for k in ks_all]
        need_wave = free_surface != np.inf and any(finite_ks)
        all_wave = free_surface != np.inf and all(finite_ks)
        prec = self.precision if precision is None else precision
        if need_wave:
            r, z, table, table32 = self._device_tabulation()
        else:
            r = z = table = table32 = None
        nr = r.numel() if r is not None else 0
        nz = z.numel() if z is not None else 0
        if S.dtype == torch.complex128:
            dtype = _lib.BEM_DTYPE_C128
        elif S.dtype == torch.complex64:
            dtype = _lib.BEM_DTYPE_C64
        else:
            raise TypeError(f"unsupported output dtype {S.dtype}")
        if K.dtype != S.dtype:
            raise TypeError("S and K must share a dtype")
        a = _lib.AssemblyArgs(
            n=n, points_dev=pts.data_ptr(), dot_normals_dev=nrm.data_ptr(),
            nb_faces=dm2.nb_faces, nb_vertices=dm2.nb_vertices, vertices_dev=dm2.vertices.data_ptr(),
            faces_dev=dm2.faces.data_ptr(), centers_dev=dm2.centers.data_ptr(), normals_dev=dm2.normals.data_ptr(),
            areas_dev=dm2.areas.data_ptr(), radii_dev=dm2.radii.data_ptr(), nb_quad_points=dm2.nb_quad_points,
            quad_points_dev=dm2.quad_points.data_ptr(), quad_weights_dev=dm2.quad_weights.data_ptr(),
            tabulation_nb_integration_points=self.tabulation_nb_integration_points,
            tabulation_grid_shape=self.tabulation_grid_shape_index, nr=nr if nr > 1 and nz > 1 else 0,
            nz=nz if nr > 1 and nz > 1 else 0,
            r_range_dev=r.data_ptr() if r is not None else 0, z_range_dev=z.data_ptr() if z is not None else 0,
            table_dev=table.data_ptr() if table is not None else 0,
            table32_dev=table32.data_ptr() if table32 is not None else 0,
            r_inv_den_dev=self._dev_tab_inv[0] if table is not None else 0,
            z_inv_den_dev=self._dev_tab_inv[1] if table is not None else 0,
            wavenumber=wavenumber, free_surface=float(free_surface), gf_singularities=_SING[sing],
            adjoint_double_layer=int(bool(adjoint_double_layer)), early_dot_product=int(bool(early_dot_product)),
            diagonal_term=int(bool(diagonal_term_in_double_layer)),
            precision=_lib.BEM_PREC_MIXED if prec == "mixed" else _lib.BEM_PREC_FP64,
            out_dtype=dtype, S_dev=S.data_ptr(), K_dev=K.data_ptr(),
            lds=lds if lds is not None else n, ldk=ldk if ldk is not None else n,
            k_plane_stride=k_plane_stride if k_plane_stride is not None else 0,
            nan_flag_dev=nan_flag.data_ptr() if nan_flag is not None else 0,
        )
        lib = _lib.load()
        same_mesh = hasattr(mesh1, "faces_centers") and mesh1.content_hash == mesh2.content_hash
        if (reuse_rankine and same_mesh and dm2.collocation_at_quadrature and all_wave
                and sing in ("low_freq", "high_freq")
                and (prec == "fp64" or (prec == "mixed" and nr > 1 and nz > 1)) and dtype == _lib.BEM_DTYPE_C128
                and early_dot_product and 16 * n * n <= self.rankine_cache_bytes):
            # Rankine part reused across wavenumbers (float64 always); wave term
            # once per pair of faces (float32 interpolation with "mixed").
            q = dm2.quad_points.data_ptr()
            a.points_dev = a.centers_dev = a.quad_points_dev = q
            a.precision = _lib.BEM_PREC_FP64
            rank = self._rankine_part(mesh2.content_hash, dm2, a, bool(adjoint_double_layer), sing,
                                      float(free_surface), stream)
            a.precision = _lib.BEM_PREC_MIXED if prec == "mixed" else _lib.BEM_PREC_FP64
            if sweep is not None:
                ks, s_stride, k_stride = sweep
                kh = np.ascontiguousarray(np.asarray(ks, dtype=np.float64))
                if lu_planes is not None:
                    work, npad, first = lu_planes
                    _lib.check(lib.bem_assemble_wave_symmetric_batched_lu(
                        a, rank.data_ptr(), n, kh.ctypes.data_as(_lib.c_void_p), len(kh), int(s_stride),
                        int(k_stride), _lib.c_void_p(int(work)), int(npad), int(first), _lib.stream_ptr(stream)))
                    return True
                _lib.check(lib.bem_assemble_wave_symmetric_batched(a, rank.data_ptr(), n,
                                                                   kh.ctypes.data_as(_lib.c_void_p), len(kh),
                                                                   int(s_stride), int(k_stride),
                                                                   _lib.stream_ptr(stream)))
                return False
            _lib.check(lib.bem_assemble_wave_symmetric(a, rank.data_ptr(), n, _lib.stream_ptr(stream)))
            return False
        if (self.symmetric_assembly and same_mesh and dm2.collocation_at_quadrature and all_wave
                and sing in ("low_freq", "high_freq") and prec == "fp64" and dtype == _lib.BEM_DTYPE_C128
                and early_dot_product and (ldk if ldk is not None else n) >= n):
            # One wavenumber at a time, nothing reused: Rankine part into K, then the
            # wave term once per pair of faces, in place.
            q = dm2.quad_points.data_ptr()
            a.points_dev = a.centers_dev = a.quad_points_dev = q
            todo = [(float(wavenumber), 0, 0)]
            if sweep is not None:
                ks, s_stride, k_stride = sweep
                todo = [(float(k), i * int(s_stride), i * int(k_stride)) for i, k in enumerate(ks)]
            esize = S.element_size()
            for k, so, ko in todo:
                a.wavenumber = k
                a.S_dev = S.data_ptr() + so * esize
                a.K_dev = K.data_ptr() + ko * esize
                _lib.check(lib.bem_assemble_symmetric(a, _lib.stream_ptr(stream)))
            return
        if (reuse_rankine and sweep is not None and not same_mesh and hasattr(mesh1, "faces_centers")
                and dm2.collocation_at_quadrature and all_wave and sing in ("low_freq", "high_freq")
                and prec == "fp64" and dtype == _lib.BEM_DTYPE_C128 and early_dot_product
                and 16 * n * dm2.nb_faces <= self.rankine_cache_bytes):
            # Any points against a mesh over a sweep (the first block column of a
            # mesh with symmetries): Rankine part once, wave term per wavenumber.
            a.centers_dev = a.quad_points_dev = dm2.quad_points.data_ptr()
            rank = self._rankine_part((mesh1.content_hash, mesh2.content_hash), dm2, a, bool(adjoint_double_layer),
                                      sing, float(free_surface), stream, rows=n)
            ks, s_stride, k_stride = sweep
            kh = np.ascontiguousarray(np.asarray(ks, dtype=np.float64))
            _lib.check(lib.bem_assemble_wave_cached(a, rank.data_ptr(), n, kh.ctypes.data_as(_lib.c_void_p), len(kh),
                                                    int(s_stride), int(k_stride), _lib.stream_ptr(stream)))
            return
        if sweep is not None:
            ks, s_stride, k_stride = sweep
            esize = S.element_size()
            variants = {}  # the variant of each wavenumber (delhommeau.py:466-490): finite, 0 or infinity
            for i, k in enumerate(ks):
                a.wavenumber = float(k)
                if free_surface != np.inf:
                    key = a.wavenumber if a.wavenumber in (0.0, np.inf) else 1.0
                    if key not in variants:
                        variants[key] = _SING[self._variant(dm2.centers_z, key)]
                    a.gf_singularities = variants[key]
                a.S_dev = S.data_ptr() + i * int(s_stride) * esize
                a.K_dev = K.data_ptr() + i * int(k_stride) * esize
                _lib.check(lib.bem_assemble(a, _lib.stream_ptr(stream)))
            return
        _lib.check(lib.bem_assemble(a, _lib.stream_ptr(stream)))

    def _assemble_finite_depth(self, mesh1, mesh2, S, K, *, free_surface, water_depth, wavenumber,
                               adjoint_double_layer, early_dot_product, diagonal_term_in_double_layer, lds, ldk,
                               k_plane_stride=None, precision=None, stream=None, nan_flag=None, sweep=None):
        """S and K in water of finite depth by Delhommeau's method
        (matrices.f90:197-305) through bem_assemble_finite_depth, with the Prony
        decomposition of find_best_exponential_decomposition(k h) and the
        variant rules of delhommeau.py:467-487 (the legacy method uses low_freq).
        Every term in float64; complex128 or complex64 outputs; K with the dot
        product taken or the three gradient planes; a sweep is one launch per
        wavenumber (each has its own decomposition)."""
        todo = [(float(wavenumber), 0, 0)]
        if sweep is not None:
            ks, s_stride, k_stride = sweep
            todo = [(float(k), i * int(s_stride), i * int(k_stride)) for i, k in enumerate(ks)]
        for k, so, ko in todo:
            self._assemble_finite_depth_one(mesh1, mesh2, S, K, so, ko, free_surface=free_surface,
                                            water_depth=water_depth, wavenumber=k,
                                            adjoint_double_layer=adjoint_double_layer,
                                            early_dot_product=early_dot_product,
                                            diagonal_term_in_double_layer=diagonal_term_in_double_layer, lds=lds,
                                            ldk=ldk, k_plane_stride=k_plane_stride, stream=stream,
                                            nan_flag=nan_flag)

    def _assemble_finite_depth_one(self, mesh1, mesh2, S, K, s_offset, k_offset, *, free_surface, water_depth,
                                   wavenumber, adjoint_double_layer, early_dot_product,
                                   diagonal_term_in_double_layer, lds, ldk, k_plane_stride, stream, nan_flag):
        """One wavenumber of _assemble_finite_depth, S and K written s_offset and
        k_offset elements after the start of their buffers.  Every term in
        float64, whatever precision was asked (there is no mixed-precision
        finite-depth kernel)."""
        import torch
        dtypes = {torch.complex128: _lib.BEM_DTYPE_C128, torch.complex64: _lib.BEM_DTYPE_C64}
        if S.dtype not in dtypes or K.dtype != S.dtype:
            raise TypeError(f"unsupported output dtypes {S.dtype}, {K.dtype}")
        pts, nrm = self._collocation(mesh1, mesh2, adjoint_double_layer)
        dm2 = self.device_mesh(mesh2)
        n = pts.shape[0]
        k = float(wavenumber)
        if self.finite_depth_method not in ("legacy", "newer"):
            raise NotImplementedError(f"finite_depth_method={self.finite_depth_method!r} is not part of this library")
        if self.finite_depth_method == "legacy" and self.gf_singularities != "low_freq":
            sing = "low_freq"
        else:
            sing = self._variant(dm2.centers_z, k)
        decomposition = self.find_best_exponential_decomposition(k * float(water_depth))
        prony = torch.as_tensor(np.ascontiguousarray(decomposition, dtype=np.float64), device=self.device)
        if stream is not None:
            stream.wait_stream(torch.cuda.current_stream())
        finite_k = 0.0 < k < np.inf
        if finite_k:
            r, z, table, table32 = self._device_tabulation()
        else:
            r = z = table = table32 = None
        nr = r.numel() if r is not None else 0
        nz = z.numel() if z is not None else 0
        a = _lib.AssemblyArgs(
            n=n, points_dev=pts.data_ptr(), dot_normals_dev=nrm.data_ptr(),
            nb_faces=dm2.nb_faces, nb_vertices=dm2.nb_vertices, vertices_dev=dm2.vertices.data_ptr(),
            faces_dev=dm2.faces.data_ptr(), centers_dev=dm2.centers.data_ptr(), normals_dev=dm2.normals.data_ptr(),
            areas_dev=dm2.areas.data_ptr(), radii_dev=dm2.radii.data_ptr(), nb_quad_points=dm2.nb_quad_points,
            quad_points_dev=dm2.quad_points.data_ptr(), quad_weights_dev=dm2.quad_weights.data_ptr(),
            tabulation_nb_integration_points=self.tabulation_nb_integration_points,
            tabulation_grid_shape=self.tabulation_grid_shape_index, nr=nr if nr > 1 and nz > 1 else 0,
            nz=nz if nr > 1 and nz > 1 else 0,
            r_range_dev=r.data_ptr() if r is not None else 0, z_range_dev=z.data_ptr() if z is not None else 0,
            table_dev=table.data_ptr() if table is not None else 0,
            table32_dev=table32.data_ptr() if table32 is not None else 0,
            r_inv_den_dev=self._dev_tab_inv[0] if table is not None else 0,
            z_inv_den_dev=self._dev_tab_inv[1] if table is not None else 0,
            wavenumber=k, free_surface=float(free_surface), gf_singularities=_SING[sing],
            adjoint_double_layer=int(bool(adjoint_double_layer)), early_dot_product=int(bool(early_dot_product)),
            diagonal_term=int(bool(diagonal_term_in_double_layer)), precision=_lib.BEM_PREC_FP64,
            out_dtype=dtypes[S.dtype], S_dev=S.data_ptr() + s_offset * S.element_size(),
            K_dev=K.data_ptr() + k_offset * K.element_size(),
            lds=lds if lds is not None else n, ldk=ldk if ldk is not None else n,
            k_plane_stride=k_plane_stride if k_plane_stride is not None else 0,
            nan_flag_dev=nan_flag.data_ptr() if nan_flag is not None else 0,
        )
        _lib.check(_lib.load().bem_assemble_finite_depth(a, float(water_depth),
                                                         0 if self.finite_depth_method == "legacy" else 1,
                                                         _lib.c_void_p(prony.data_ptr()), decomposition.shape[1],
                                                         _lib.stream_ptr(stream)))
        if stream is not None:
            # the decomposition was copied on the current stream and is freed on return
            prony.record_stream(stream)

    def _rankine_part(self, mesh_key, dm, args, adjoint, sing, free_surface, stream, rows=None):
        """Device array of the wavenumber-independent Rankine part of the rows
        (collocation points, default: the mesh's own) against the faces of dm
        (bem_assemble_rankine_part), cached per meshes and variant."""
        import torch
        key = (mesh_key, adjoint, sing == "high_freq", free_surface)
        with self._lock:
            hit = self._rankine_cache.get(key)
            if hit is not None:
                self._rankine_cache.move_to_end(key)
                hit.acquire()
                return hit.tensors[0]
            N = dm.nb_faces
            n = N if rows is None else rows
            while self._rankine_cache and (sum(e.tensors[0].numel() * 16 for e in self._rankine_cache.values())
                                           + 16 * n * N > self.rankine_cache_bytes):
                self._rankine_cache.popitem(last=False)
            rank = torch.empty((N, n), dtype=torch.complex128, device=self.device)  # column-major n x N
            _lib.check(_lib.load().bem_assemble_rankine_part(args, rank.data_ptr(), n, _lib.stream_ptr(stream)))
            self._rankine_cache[key] = _lib.StreamShared(rank)
            return rank

    def clear_rankine_cache(self):
        """Release the cached Rankine parts."""
        with self._lock:
            self._rankine_cache.clear()

    def evaluate_device(self, mesh1, mesh2, *, free_surface=0.0, water_depth=np.inf, wavenumber=1.0,
                        adjoint_double_layer=True, early_dot_product=True, diagonal_term_in_double_layer=True,
                        dtype=None):
        """Like ``evaluate`` but returns device tensors (S (n, N), K (n, N) or
        (3, n, N)), column-major, and raises on NaN."""
        import torch
        dev = self.device
        if dtype is None:
            dtype = torch.complex64 if self.floating_point_precision == "float32" else torch.complex128
        n = mesh1.nb_faces if hasattr(mesh1, "faces_centers") else np.asarray(mesh1).shape[0]
        N = mesh2.nb_faces
        S_buf = torch.empty((N, n), dtype=dtype, device=dev)
        kdim = 1 if early_dot_product else 3
        K_buf = torch.empty((kdim, N, n), dtype=dtype, device=dev)
        flag = torch.zeros(1, dtype=torch.int32, device=dev)
        self.assemble_into(mesh1, mesh2, S_buf, K_buf, free_surface=free_surface, water_depth=water_depth,
                           wavenumber=wavenumber, adjoint_double_layer=adjoint_double_layer,
                           early_dot_product=early_dot_product,
                           diagonal_term_in_double_layer=diagonal_term_in_double_layer,
                           lds=n, ldk=n, k_plane_stride=n * N, nan_flag=flag)
        if int(flag.item()) != 0:
            raise _lib.GreenFunctionEvaluationError(
                _lib.BEM_ERR_NAN, "Green function returned a NaN in the interaction matrix.\n"
                                  "It could be due to overlapping panels.")
        S = S_buf.T
        K = K_buf.transpose(1, 2)
        if early_dot_product:
            K = K[0]
        return S, K

    def evaluate(self, mesh1, mesh2, *, free_surface=0.0, water_depth=np.inf, wavenumber=1.0,
                 adjoint_double_layer=True, early_dot_product=True, diagonal_term_in_double_layer=True):
        """Same contract as capytaine ``Delhommeau.evaluate`` (delhommeau.py:405-520):
        NumPy arrays S (n, N) and K (n, N) or (3, n, N); real-valued when
        free_surface is infinite (Rankine kernel only)."""
        if free_surface == np.inf:
            return self.evaluate_rankine_only(mesh1, mesh2, adjoint_double_layer=adjoint_double_layer,
                                              early_dot_product=early_dot_product,
                                              _water_depth=water_depth)
        S, K = self.evaluate_device(mesh1, mesh2, free_surface=free_surface, water_depth=water_depth,
                                    wavenumber=wavenumber, adjoint_double_layer=adjoint_double_layer,
                                    early_dot_product=early_dot_product,
                                    diagonal_term_in_double_layer=diagonal_term_in_double_layer)
        return S.cpu().numpy(), K.cpu().numpy()

    def evaluate_rankine_only(self, mesh1, mesh2, *, adjoint_double_layer=True, early_dot_product=True,
                              diagonal_term_in_double_layer=True, _water_depth=np.inf):
        """capytaine delhommeau.py:336-402: real-valued Rankine matrices."""
        if _water_depth != np.inf:
            raise ValueError("When setting free_surface=inf, the water depth should also be infinite "
                             f"(got water_depth={_water_depth})")
        S, K = self.evaluate_device(mesh1, mesh2, free_surface=np.inf, wavenumber=0.0,
                                    adjoint_double_layer=adjoint_double_layer, early_dot_product=early_dot_product,
                                    diagonal_term_in_double_layer=diagonal_term_in_double_layer)
        return S.real.cpu().numpy(), K.real.cpu().numpy()


class XieDelhommeau(Delhommeau):
    """Legacy alias of the gf_singularities="low_freq" variant (delhommeau.py:524-528)."""

    def __init__(self, **kwargs):
        super().__init__(gf_singularities="low_freq", **kwargs)
