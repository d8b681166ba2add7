"""Matrix engine on the B200: device-resident S/K, batched LU, frequency solves.

Two entry points:

* ``B200Engine.solve_frequencies(body, omegas, ...)``: the whole indirect
  solve of many frequencies of one body, batched on the device (assembly of S
  and K at the wavenumber of each omega, k = omega^2/g in infinite depth, LU of
  K, every radiation and diffraction RHS, S @ sigma, pressure integration) with
  only the coefficients coming back to the host.
  One frequency-solve is what capytaine does for one (body, omega) group in
  ``BEMSolver.solve_all`` (bem/solver.py:268-372, problems grouped by
  bem/problems_and_results.py:267-275).
* the ``MatrixEngine`` interface of capytaine (bem/engines.py:46-59, 142-176,
  273-346, 348-398): ``build_matrices`` returns device-backed matrices whose
  ``@`` and whose LU (``linear_solver``) run on the GPU, so capytaine's own
  ``BEMSolver`` can use this engine unchanged.
"""
from __future__ import annotations

import ctypes
import logging
import math
import threading
import weakref
from collections import OrderedDict
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _lib
from .arena import DeviceArena
from .green_function import Delhommeau
from .symmetry import block_structure

LOG = logging.getLogger(__name__)

NB = 64  # LU block size; matrices are padded to a multiple of it
RHS_CHUNK = 16  # right-hand sides per refinement / GMRES / tall-GEMM call
# Relative residual |b - K x| / |b| that a float64 LU solve is refined to; a
# solve whose residual stops decreasing above it (the float64 floor of an
# ill-conditioned K) is accepted up to the engine's refine_tol.
FP64_RESIDUAL_TOL = 1e-13


def padded_size(n: int) -> int:
    return int(math.ceil(n / NB) * NB)


def _vp(x):
    return ctypes.c_void_p(x.data_ptr() if hasattr(x, "data_ptr") else int(x))


def wavenumbers(omegas, water_depth: float = np.inf, g: float = 9.81) -> np.ndarray:
    """Wavenumbers of the angular frequencies omegas: omega^2 / g in infinite
    depth, else the root k > 0 of the dispersion relation k tanh(k h) = omega^2 / g
    (bem/problems_and_results.py:159-163), by Newton's method kept inside a
    bracket [lo, hi] that halves whenever a step leaves it.  0 and +inf map to
    themselves."""
    omegas = np.asarray(omegas, dtype=float)
    w2g = omegas ** 2 / g
    if water_depth == np.inf:
        return w2g
    if not water_depth > 0:
        raise ValueError(f"water_depth must be > 0 (got {water_depth})")
    h = float(water_depth)
    out = np.empty_like(w2g)
    for i, c in enumerate(w2g.ravel()):
        if c == 0.0 or c == np.inf:
            out.flat[i] = c
            continue
        # k tanh(k h) is increasing, below k, and above c at k = hi
        lo, hi = c, c + np.sqrt(c / h)
        while hi * np.tanh(hi * h) <= c:
            hi *= 2.0
        k = 0.5 * (lo + hi)
        for _ in range(200):
            t = np.tanh(k * h)
            f = k * t - c
            if f > 0:
                hi = k
            else:
                lo = k
            step = f / (t + k * h * (1.0 - t * t))
            k_new = k - step
            if not lo < k_new < hi:
                k_new = 0.5 * (lo + hi)
            if abs(k_new - k) <= 4e-16 * k_new:
                k = k_new
                break
            k = k_new
        out.flat[i] = k
    return out


def band_batches(sizes, nq, band, capacity):
    """Batches of (body, omega index) pairs for the grouped factorisation:
    bodies in decreasing padded size (sizes[i]), the nq frequencies of each
    together, a new batch when a body is smaller than the batch's largest
    divided by band or when the batch holds capacity(largest) pairs.
    Returns [(padded size of the batch, [(i, q), ...]), ...]."""
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i], i))
    out, cur, top, cap = [], [], 0, 0
    for i in order:
        for q in range(nq):
            if cur and (sizes[i] * band < top or len(cur) >= cap):
                out.append((top, cur))
                cur = []
            if not cur:
                top = sizes[i]
                cap = max(1, int(capacity(top)))
            cur.append((i, q))
    if cur:
        out.append((top, cur))
    return out


@dataclass
class FrequencyResults:
    """Coefficients of a frequency sweep.  Arrays are indexed [omega, ...]:
    added_mass / radiation_damping [omega, radiating_dof, influenced_dof],
    diffraction / froude_krylov / excitation [omega, heading, influenced_dof]."""
    omegas: np.ndarray
    dofs: List[str]
    wave_directions: np.ndarray
    added_mass: np.ndarray
    radiation_damping: np.ndarray
    diffraction: np.ndarray
    froude_krylov: np.ndarray
    excitation: np.ndarray
    stats: Dict[str, float] = field(default_factory=dict)

    def coefficients(self) -> Dict[str, np.ndarray]:
        return dict(added_mass=self.added_mass, radiation_damping=self.radiation_damping,
                    excitation=self.excitation)


def _allocator(device, alloc):
    """(shape, dtype, zero) -> tensor: torch's allocator, or the caller's
    (views of a preallocated arena, see serving.DeviceArena)."""
    if alloc is not None:
        return alloc
    import torch

    def torch_alloc(shape, dtype, zero=False):
        return (torch.zeros if zero else torch.empty)(shape, dtype=dtype, device=device)
    return torch_alloc


class _Factors:
    """Device storage of the matrices of `batch` frequency-solves of one mesh
    (n panels): S, K and the factorisation of K.

    fp64:  K with leading dimension npad (a multiple of 64) and, unless lu is
           False (plain GMRES), its float64 LU in a second buffer of the same
           layout (identity padding), so that every solve checks its residual
           against K.
    mixed: K unpadded (float64 residuals) and the float32 LU workspace padded
           to a multiple of 128."""

    def __init__(self, n, batch, device, precision, alloc=None, lu=True):
        import torch
        self.n, self.batch, self.precision = n, batch, precision
        self.planes_ready = False  # K already in the mixed LU's float32 planes (assemble_stage)
        lib = _lib.load()
        mk = _allocator(device, alloc)
        self.S = mk((batch, n * n), torch.complex128)
        self.info = mk((batch,), torch.int32, True)
        self.LU = None
        if precision == "fp64":
            self.npad = padded_size(n)
            self.K = mk((batch, self.npad * self.npad), torch.complex128)
            self.ldk = self.npad
            self.strideK = self.npad * self.npad
            if lu:
                self.LU = mk((batch, self.npad * self.npad), torch.complex128)
            self.lu_work = mk((int(lib.bem_zlu_workspace_bytes(self.npad, batch)),), torch.uint8)
            self.lu_work_ptr = self.lu_work.data_ptr()
        else:
            self.npad = int(math.ceil(n / 128) * 128)
            self.K = mk((batch, n * n), torch.complex128)
            self.ldk = n
            self.strideK = n * n
            nbytes = int(lib.bem_clu_workspace_bytes(self.npad, batch))
            self.lu_work = mk((nbytes + 1024,), torch.uint8)
            self.lu_work_ptr = (self.lu_work.data_ptr() + 1023) // 1024 * 1024  # 1024-byte aligned start
        self.piv = mk((batch, self.npad), torch.int32)

    @staticmethod
    def estimate_bytes(n, batch, precision, lu=True):
        """Device bytes of a _Factors of this shape (admission by footprint)."""
        lib = _lib.load()
        if precision == "fp64":
            npad = padded_size(n)
            return (batch * (16 * n * n + (32 if lu else 16) * npad * npad)
                    + int(lib.bem_zlu_workspace_bytes(npad, batch)))
        npad = int(math.ceil(n / 128) * 128)
        return batch * 32 * n * n + int(lib.bem_clu_workspace_bytes(npad, batch)) + 1024

    @property
    def nbytes(self):
        ts = [self.S, self.K, self.lu_work, self.piv, self.info] + ([self.LU] if self.LU is not None else [])
        return sum(t.numel() * t.element_size() for t in ts)


class _Rhs:
    """Right-hand sides, solutions, potentials and the small work buffers of
    `batch` frequency-solves with nrhs columns each (padded rows zero)."""

    def __init__(self, n, npad, batch, nrhs, device, precision, alloc=None):
        import torch
        self.n, self.npad, self.batch, self.nrhs, self.precision = n, npad, batch, nrhs, precision
        lib = _lib.load()
        mk = _allocator(device, alloc)
        self._mk = mk
        self.chunk = min(nrhs, RHS_CHUNK)  # columns per solve call
        self.B = mk((batch, npad * nrhs), torch.complex128, True)
        self.X = mk((batch, npad * nrhs), torch.complex128, True)
        self.R = mk((batch, npad * nrhs), torch.complex128, True)
        self.phi = mk((batch, n * nrhs), torch.complex128)
        self.norms = mk((2 * batch * self.chunk + 2,), torch.float64, True)
        self.ts_work = mk((int(lib.bem_zgemm_ts_workspace_bytes(n, n, self.chunk, batch)),), torch.uint8)
        self.flags = mk((2,), torch.int32, True)  # [err, nan]
        self._gmres = None

    @property
    def err(self):
        return self.flags[0:1]

    @property
    def nan(self):
        return self.flags[1:2]

    def gmres_work(self, restart):
        """256-byte aligned workspace of bem_gmres_solve for this shape."""
        import torch
        if self._gmres is None or self._gmres[0] != restart:
            nbytes = int(_lib.load().bem_gmres_workspace_bytes(self.n, self.npad, self.chunk, self.batch, restart))
            if nbytes < 0:
                raise ValueError("bad GMRES workspace shape")
            buf = self._mk((nbytes + 256,), torch.uint8)
            self._gmres = (restart, buf, (buf.data_ptr() + 255) // 256 * 256)
        return self._gmres[2]

    @staticmethod
    def estimate_bytes(n, npad, batch, nrhs):
        lib = _lib.load()
        chunk = min(nrhs, RHS_CHUNK)
        return 16 * batch * nrhs * (3 * npad + n) + int(lib.bem_zgemm_ts_workspace_bytes(n, n, chunk, batch)) + 4096

    @property
    def nbytes(self):
        ts = [self.B, self.X, self.R, self.phi, self.norms, self.ts_work, self.flags]
        if self._gmres is not None:
            ts.append(self._gmres[1])
        return sum(t.numel() * t.element_size() for t in ts)


class _Workspace:
    """Factor storage and RHS buffers of one (n, batch, nrhs, precision) shape,
    reused across the batches of a sweep."""

    def __init__(self, n, batch, nrhs, device, precision, lu=True):
        self.n, self.batch, self.nrhs, self.precision = n, batch, nrhs, precision
        self.f = _Factors(n, batch, device, precision, lu=lu)
        self.r = _Rhs(n, self.f.npad, batch, nrhs, device, precision)

    @property
    def nbytes(self):
        return self.f.nbytes + self.r.nbytes


def _combine_first_column(st, W, src, cols_ptr, n_full, nb, out_ptr, ld_out, stride_out, stream):
    """Systems k of nb first block columns (column-major n_full x n_sub at
    cols_ptr + f * n_full * n_sub elements, image j at rows j n_sub) into out
    (system f * nsys + k at out_ptr + that index * stride_out elements, leading
    dimension ld_out): one bem_block_combine per (row part, column part) of
    the macro-blocks."""
    lib = _lib.load()
    ns = st.n_sub
    for a in range(st.q):
        for b in range(st.q):
            s = src[a][b]
            _lib.check(lib.bem_block_combine(_vp(cols_ptr), n_full * ns, ns, n_full,
                                             _vp(int(out_ptr) + 16 * (a * ns + b * ns * ld_out)), st.nsys * stride_out,
                                             stride_out, ld_out, _vp(W), _vp(s) if s is not None else None, st.nsys,
                                             st.nsys, ns, ns, nb, stream))


def _transform_tensors(st, device):
    """W, Winv and the per-(row part, column part) image maps on the device."""
    import torch
    W = torch.as_tensor(np.ascontiguousarray(st.W), dtype=torch.complex128, device=device)
    Winv = torch.as_tensor(np.ascontiguousarray(st.Winv), dtype=torch.complex128, device=device)
    src = [[None if st.q == 1 else
            torch.as_tensor(np.ascontiguousarray(st.source[:, a, b]), dtype=torch.int32, device=device)
            for b in range(st.q)] for a in range(st.q)]
    return W, Winv, src


class _SymWorkspace:
    """Buffers of the frequency-solves of a mesh with symmetries: the reduced
    systems (factors and right-hand sides of batch x nsys systems of size
    n_sys), the first block columns of S and K (N x n_sub per frequency), the
    right-hand sides and potentials of the whole mesh, and the transform."""

    def __init__(self, st, n_full, batch, nrhs, device, precision):
        import torch
        self.st, self.n_full, self.batch, self.nrhs = st, n_full, batch, nrhs
        self.f = _Factors(st.n_sys, batch * st.nsys, device, precision)
        self.r = _Rhs(st.n_sys, self.f.npad, batch * st.nsys, nrhs, device, precision)
        self.cols = torch.empty((2, batch, n_full * st.n_sub), dtype=torch.complex128, device=device)
        self.full = torch.zeros((batch, n_full * nrhs), dtype=torch.complex128, device=device)
        self.W, self.Winv, self.src = _transform_tensors(st, device)

    @property
    def nbytes(self):
        return self.f.nbytes + self.r.nbytes + 16 * (self.cols.numel() + self.full.numel())

    def combine_matrices(self, cols, nb, out, ld_out, stride_out, stream):
        """Systems k of frequencies 0..nb-1 from their first block columns
        (`cols`: nb x (N x n_sub) column-major, image j at rows j n_sub) into
        `out` (system f * nsys + k at out + that index * stride_out, leading
        dimension ld_out)."""
        _combine_first_column(self.st, self.W, self.src, cols.data_ptr(), self.n_full, nb, out.data_ptr(), ld_out,
                              stride_out, stream)

    def to_systems(self, nb, out, ld_out, stride_out, stream):
        """Right-hand sides of the whole mesh (self.full) to those of the systems."""
        st, N, nrhs = self.st, self.n_full, self.nrhs
        _lib.check(_lib.load().bem_block_combine(_vp(self.full), N * nrhs, st.n_sys, N, _vp(out),
                                                 st.nsys * stride_out, stride_out, ld_out, _vp(self.W), None,
                                                 st.nsys, st.nsys, st.n_sys, nrhs, nb, stream))

    def from_systems(self, nb, src_ptr, ld_in, stride_in, stream):
        """Potentials of the systems back to the whole mesh (into self.full)."""
        st, N, nrhs = self.st, self.n_full, self.nrhs
        _lib.check(_lib.load().bem_block_combine(_vp(src_ptr), st.nsys * stride_in, stride_in, ld_in,
                                                 _vp(self.full), N * nrhs, st.n_sys, N, _vp(self.Winv), None,
                                                 st.nsys, st.nsys, st.n_sys, nrhs, nb, stream))


class B200Engine:
    """capytaine-compatible matrix engine running the Delhommeau assembly and the
    dense solves on one B200.

    precision: "fp64" (float64 LU) or "mixed" (float32 LU with TF32
    tensor-core trailing updates, float64-residual iterative refinement to
    refine_tol).  assembly_precision: "fp64" (default) or "mixed" (float32
    tabulated wave term, float64 Rankine terms).

    linear_solver (as capytaine's DefaultMatrixEngine, bem/engines.py:300-346):
    "lu_decomposition" (default), "lu_decomposition_with_overwrite" (the same
    here: K is always factored in place on the device), "gmres" (restarted
    GMRES on the float64 K with SciPy's settings as capytaine's solve_gmres,
    bem/engines.py:74-89: atol 1e-6, rtol 1e-5, restart 20; with precision
    "fp64" only), or a callable ``(A, b) -> x`` used by ``linear_solver``.

    method: "indirect" (sources sigma = K^-1 bc, potential S sigma) or "direct"
    (potential = D^-1 S bc with the double-layer matrix D), as capytaine's
    BEMSolver(method=...) (bem/solver.py:172-207), for the device sweeps.

    refinement (precision "mixed"): "classical" (x += (LU)^-1 r) or "gmres"
    (flexible GMRES on the float64 K right-preconditioned by the float32 LU), both to
    refine_tol relative residual.  When the classical iteration stops
    contracting (K nearly singular, e.g. near an irregular frequency) the
    solve continues with the preconditioned GMRES (stats["escalated_to_gmres"]).
    """

    def __init__(self, *, green_function: Optional[Delhommeau] = None, precision: str = "fp64",
                 linear_solver="lu_decomposition", max_batch: int = 8, device=None,
                 refine_tol: float = 1e-10, refine_max_iter: int = 30, assembly_precision: str = "fp64",
                 refinement: str = "classical", gmres_restart: int = 20, gmres_maxiter: Optional[int] = None,
                 method: str = "indirect", batch_tuner=None):
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        if assembly_precision not in ("fp64", "mixed"):
            raise ValueError("assembly_precision must be 'fp64' or 'mixed'")
        if not callable(linear_solver) and linear_solver not in ("lu_decomposition",
                                                                 "lu_decomposition_with_overwrite", "gmres"):
            raise NotImplementedError(f"Unknown `linear_solver` in B200Engine: {linear_solver}")
        if linear_solver == "gmres" and precision != "fp64":
            raise ValueError("linear_solver='gmres' is the float64 solver; use refinement='gmres' with 'mixed'")
        if refinement not in ("classical", "gmres"):
            raise ValueError("refinement must be 'classical' or 'gmres'")
        if method.lower() not in ("direct", "indirect"):
            raise ValueError(f"Unrecognized method: {method!r}. Expected \"direct\" or \"indirect\".")
        # solve_frequencies / solve_bodies / the server: indirect (sources, K) or
        # direct (potential, D with rhs = S bc), as BEMSolver(method=...) in
        # capytaine bem/solver.py:172-207
        self.method = method.lower()
        self.precision = precision
        self.refinement = refinement
        self.gmres_restart = int(gmres_restart)
        self.gmres_maxiter = gmres_maxiter
        self.gmres_escalation_cycles = 10
        # float32 wave terms perturb the O(k)-small imaginary parts that carry the
        # radiation damping at low frequency beyond 1e-5: float64 assembly by default.
        self.assembly_precision = assembly_precision
        self.refine_tol = float(refine_tol)
        self.refine_max_iter = int(refine_max_iter)
        self.green_function = green_function if green_function is not None else Delhommeau()
        self._linear_solver = linear_solver
        self.max_batch = int(max_batch)
        # matrices per grouped factorisation of solve_bodies, per size class
        from .tuning import DEFAULT_TUNER
        self.batch_tuner = batch_tuner if batch_tuner is not None else DEFAULT_TUNER
        self._device = device
        self._ws: Dict[tuple, _Workspace] = {}
        self._body_cache: "OrderedDict[tuple, tuple]" = OrderedDict()
        self._lock = threading.RLock()
        self.last_computed_inputs = None
        self.last_computed_matrices = None
        self.exportable_settings = {
            "engine": "B200Engine",
            "linear_solver": str(linear_solver),
            "precision": precision,
            "assembly_precision": assembly_precision,
            **({"refinement": refinement} if precision == "mixed" else {}),
            "method": method.lower(),
            **self.green_function.exportable_settings,
        }

    def __str__(self):
        return f"B200Engine(green_function={self.green_function}, precision={self.precision!r})"

    __repr__ = __str__

    @property
    def device(self):
        return _lib.require_cuda(self._device)

    def workspace(self, n, batch, nrhs) -> _Workspace:
        key = (n, batch, nrhs, self.precision)
        ws = self._ws.get(key)
        if ws is None:
            self._ws.clear()  # one resident shape at a time (memory)
            ws = _Workspace(n, batch, nrhs, self.device, self.precision, lu=not self._plain_gmres)
            self._ws[key] = ws
        return ws

    def release(self):
        """Drop the engine's device workspaces (they are re-created on demand)."""
        self._ws.clear()

    # ------------------------------------------------------------------------
    # Batched frequency solves
    def _body_arrays(self, body, mesh):
        """Device copies of the dof normal components, pressure weights and
        hull mask of a body, kept for the body's next call."""
        import torch
        key = (id(body), mesh.content_hash, tuple(body.dofs))
        with self._lock:
            hit = self._body_cache.get(key)
            if hit is not None and hit[0]() is body:
                hit[1].acquire()
                return hit[1].tensors
        # host arrays and uploads outside the lock (other threads' bodies go on)
        dev = self.device
        dnc = body.dof_normal_components()
        mask = body.hull_mask
        pw = -dnc  # pressure weights -(dof . n) area on the hull (FloatingBody.pressure_weights)
        pw[:, mask] *= body.mesh.faces_areas[None, :]
        arrays = tuple(_lib.upload_many([(dnc, torch.float64), (pw, torch.float64),
                                         (mask.astype(np.int32), torch.int32)], dev))
        with self._lock:
            self._body_cache[key] = (weakref.ref(body), _lib.StreamShared(*arrays))
            while len(self._body_cache) > 32:
                self._body_cache.popitem(last=False)
        return arrays

    def solve_frequencies(self, body, omegas: Sequence[float], *, wave_directions: Sequence[float] = (0.0,),
                          rho: float = 1000.0, g: float = 9.81, water_depth: float = np.inf,
                          batch: Optional[int] = None, sync_stats: bool = False) -> FrequencyResults:
        """Added mass, damping and excitation of `body` at every omega and wave
        direction, in water of depth water_depth (+inf: infinite depth; finite:
        Delhommeau's finite-depth Green function with its Prony decomposition,
        the assembly then in float64 whatever assembly_precision, and
        finite-depth Airy waves).  omega = 0 and omega = infinity give the
        limit-frequency radiation coefficients (zero damping) and NaN wave
        forces, as capytaine's symbolic-frequency problems do; omega = 0 in
        finite depth raises NotImplementedError (no Prony decomposition at
        k h = 0), as capytaine does."""
        import torch
        if not water_depth > 0:
            raise ValueError(f"water_depth must be > 0 (got {water_depth})")
        mesh = body.mesh_including_lid
        n = mesh.nb_faces
        omegas = np.asarray(omegas, dtype=float)
        if np.any(np.isnan(omegas)) or np.any(omegas < 0):
            raise ValueError("angular frequencies must be >= 0 (or infinity)")
        heads = np.asarray(wave_directions, dtype=float)
        ndof, nhead = len(body.dofs), len(heads)
        nrhs = ndof + nhead
        B = min(self.max_batch if batch is None else batch, len(omegas))
        st = block_structure(mesh)
        if st is not None:
            return self._solve_frequencies_symmetric(body, st, omegas, heads, rho, g, B, sync_stats, water_depth)
        ws = self.workspace(n, B, nrhs)
        F_all = np.zeros((len(omegas), nrhs, ndof), dtype=np.complex128)
        FK_all = np.zeros((len(omegas), max(nhead, 1), ndof), dtype=np.complex128)
        stats = {"assembly_ms": 0.0, "lu_ms": 0.0, "solve_ms": 0.0, "post_ms": 0.0}
        for start in range(0, len(omegas), B):
            om = omegas[start:start + B]
            nb = len(om)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)] if sync_stats else None
            if ev:
                ev[0].record()
            ws.r.flags.zero_()
            self.assemble_stage(ws.f, mesh, wavenumbers(om, water_depth, g), nan_flag=ws.r.nan,
                                water_depth=water_depth, planes=True)
            if ev:
                ev[1].record()
            self.factor_stage(ws.f, nb, ws.r.err)
            if ev:
                ev[2].record()
            F, FK = self.solve_stage(ws.f, ws.r, body, om, heads, rho=rho, g=g, stats=stats, events=ev,
                                     water_depth=water_depth)
            F_all[start:start + nb] = F
            FK_all[start:start + nb, :nhead] = FK
            if ev:
                torch.cuda.synchronize()
                stats["assembly_ms"] += ev[0].elapsed_time(ev[1])
                stats["lu_ms"] += ev[1].elapsed_time(ev[2])
                stats["solve_ms"] += ev[2].elapsed_time(ev[3])
                stats["post_ms"] += ev[3].elapsed_time(ev[4])
        return self._coefficients(body, omegas, heads, F_all, FK_all, stats)

    def _solve_frequencies_symmetric(self, body, st, omegas, heads, rho, g, B, sync_stats, water_depth=np.inf):
        """solve_frequencies for a mesh with symmetries (bem/engines.py:178-247,
        tools/block_circulant_matrices.py): per frequency, S and K of the whole
        mesh's collocation points against the panels of the reference sub-mesh
        (the first block column), the nsys independent systems of the
        block-diagonalised matrices (bem_block_combine), one batched LU of all
        systems of the batch, right-hand sides taken to the systems, solved,
        S sigma per system, the potentials taken back to the whole mesh, then
        the force integrals of the whole mesh."""
        import torch
        mesh = body.mesh_including_lid
        full = mesh.merged()
        N = full.nb_faces
        nhead = len(heads)
        nrhs = len(body.dofs) + nhead
        key = ("symmetric", st.kind, st.n_sub, st.nsys, N, B, nrhs, self.precision)
        ws = self._ws.get(key)
        if ws is None:
            self._ws.clear()
            ws = _SymWorkspace(st, N, B, nrhs, self.device, self.precision)
            self._ws[key] = ws
        F_all = np.zeros((len(omegas), nrhs, len(body.dofs)), dtype=np.complex128)
        FK_all = np.zeros((len(omegas), max(nhead, 1), len(body.dofs)), dtype=np.complex128)
        stats = {"assembly_ms": 0.0, "lu_ms": 0.0, "solve_ms": 0.0, "post_ms": 0.0, "symmetry": st.kind,
                 "systems_per_frequency": st.nsys, "system_size": st.n_sys}
        gf = self.green_function
        adjoint = self.method == "indirect"
        stream = _lib.stream_ptr()
        f = ws.f
        for start in range(0, len(omegas), B):
            om = omegas[start:start + B]
            nb = len(om)
            ks = [float(k) for k in wavenumbers(om, water_depth, g)]
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)] if sync_stats else None
            if ev:
                ev[0].record()
            ws.r.flags.zero_()
            cstride = N * st.n_sub
            gf.assemble_into(full, st.submesh, ws.cols[0, 0], ws.cols[1, 0], wavenumber=ks[0], lds=N, ldk=N,
                             nan_flag=ws.r.nan,
                             precision=self.assembly_precision,
                             adjoint_double_layer=adjoint, sweep=(ks, cstride, cstride), water_depth=water_depth)
            ws.combine_matrices(ws.cols[0], nb, f.S, st.n_sys, st.n_sys * st.n_sys, stream)
            ws.combine_matrices(ws.cols[1], nb, f.K, f.ldk, f.strideK, stream)
            if ev:
                ev[1].record()
            self.factor_stage(f, nb * st.nsys, ws.r.err)
            if ev:
                ev[2].record()
            (F, FK), = self._solve_segments(f, ws.r, [(body, 0, nb)], om, heads, rho=rho, g=g, stats=stats,
                                            events=ev, sym=ws, water_depth=water_depth)
            F_all[start:start + nb] = F
            FK_all[start:start + nb, :nhead] = FK
            if ev:
                torch.cuda.synchronize()
                stats["assembly_ms"] += ev[0].elapsed_time(ev[1])
                stats["lu_ms"] += ev[1].elapsed_time(ev[2])
                stats["solve_ms"] += ev[2].elapsed_time(ev[3])
                stats["post_ms"] += ev[3].elapsed_time(ev[4])
        return self._coefficients(body, omegas, heads, F_all, FK_all, stats)

    # ---- stages of a frequency-solve, on the caller's current stream -------
    # (solve_frequencies chains them; the request server of serving.py runs
    # them on one stream per slot and keeps factors resident between requests)
    @property
    def _plain_gmres(self):
        return self.precision == "fp64" and self._linear_solver == "gmres"

    def assemble_stage(self, f: "_Factors", mesh, ks, *, nan_flag=None, reuse_rankine=True, first=0, lds=None,
                       water_depth=np.inf, planes=False):
        """S and K of the mesh with itself at the wavenumbers ks into
        f[first:first+len(ks)] (one launch for all of them on the Rankine-reuse
        path when every wavenumber is finite and > 0; one per wavenumber in
        finite depth).  planes (mixed engine, f's matrices are the mesh's own,
        nothing padded afterwards): K also goes rounded to float32 into the LU
        workspace where the sweep kernel can write it, and f.planes_ready says
        whether every matrix of the batch got there (factor_stage then skips
        the conversion pass)."""
        gf = self.green_function
        n = mesh.nb_faces
        lds = n if lds is None else lds
        ks = [float(k) for k in ks]
        adjoint = self.method == "indirect"  # K (adjoint double layer) or D
        precs = [self._wave_precision(mesh, k, water_depth) for k in ks]
        planes = planes and self.precision == "mixed" and first == 0 and f.n == n
        f.planes_ready = False
        if len(ks) > 1 and all(0.0 < k < np.inf for k in ks):
            # one sweep call per run of consecutive wavenumbers of the same precision
            i = 0
            written = True
            while i < len(ks):
                j = i
                while j < len(ks) and precs[j] == precs[i]:
                    j += 1
                lu_planes = (f.lu_work_ptr, f.npad, first + i) if planes else None
                done = gf.assemble_into(mesh, mesh, f.S[first + i], f.K[first + i], wavenumber=ks[i], lds=lds,
                                        ldk=f.ldk, nan_flag=nan_flag, precision=precs[i],
                                        reuse_rankine=reuse_rankine, sweep=(ks[i:j], f.S.shape[1], f.K.shape[1]),
                                        adjoint_double_layer=adjoint, water_depth=water_depth, lu_planes=lu_planes)
                written = written and bool(done)
                i = j
            f.planes_ready = planes and written
            return
        for b, k in enumerate(ks):
            gf.assemble_into(mesh, mesh, f.S[first + b], f.K[first + b], wavenumber=k, lds=lds, ldk=f.ldk,
                             nan_flag=nan_flag, precision=precs[b], reuse_rankine=reuse_rankine,
                             adjoint_double_layer=adjoint, water_depth=water_depth)

    def _wave_precision(self, mesh, k, water_depth=np.inf):
        """Precision of the wave term at wavenumber k (one per engine: a
        per-frequency choice was measured and rejected, the float32 wave term
        loses accuracy at low and at high k alike)."""
        return self.assembly_precision

    def pad_stage(self, f: "_Factors", first, m, n_body):
        """Matrices first .. first+m-1 of f hold a body of n_body < f.n panels:
        zero rows and columns and a unit diagonal beyond its panels in S and K
        (the padded unknowns are zero and change nothing)."""
        if n_body >= f.n:
            return
        lib = _lib.load()
        n = f.n
        for M in (f.S, f.K):
            _lib.check(lib.bem_zpad_identity(_vp(M.data_ptr() + 16 * first * n * n), n, n * n, m, n_body, n,
                                             _lib.stream_ptr()))

    def factor_stage(self, f: "_Factors", nb, err, active=None):
        """LU of K (float64 DMMA, or float32 tcgen05 for the mixed engine); none
        for plain GMRES.  active (mixed engine): each matrix's own padded size,
        the rest of it identity padding, for the grouped LU."""
        lib = _lib.load()
        stream = _lib.stream_ptr()
        n, npad = f.n, f.npad
        if self.precision == "mixed" and active is not None:
            act = (ctypes.c_int32 * nb)(*[int(min(a, npad)) for a in active])
            _lib.check(lib.bem_clu_factor_grouped(_vp(f.K), n, n * n, n, npad, nb, act, _vp(f.piv), _vp(f.info),
                                                  _vp(f.lu_work_ptr), _vp(err), stream))
        elif self.precision == "mixed" and getattr(f, "planes_ready", False):
            # the assembly wrote K into the workspace's float32 planes
            _lib.check(lib.bem_clu_factor_planes(n, npad, nb, _vp(f.piv), _vp(f.info), _vp(f.lu_work_ptr),
                                                 _vp(err), stream))
        elif self.precision == "mixed":
            _lib.check(lib.bem_clu_factor(_vp(f.K), n, n * n, n, npad, nb, _vp(f.piv), _vp(f.info),
                                          _vp(f.lu_work_ptr), _vp(err), stream))
        elif not self._plain_gmres:
            # K stays as assembled (the residual of every solve is taken against
            # it); the LU is computed in place in a copy
            f.LU[:nb].copy_(f.K[:nb])
            _lib.check(lib.bem_zpad_identity(_vp(f.LU), npad, npad * npad, nb, n, npad, stream))
            _lib.check(lib.bem_zlu_factor(_vp(f.LU), npad, npad, npad * npad, nb, _vp(f.piv), _vp(f.info),
                                          _vp(f.lu_work), stream))
        f.planes_ready = False  # consumed

    def solve_stage(self, f: "_Factors", r: "_Rhs", body, om, heads, *, rho=1000.0, g=9.81, stats=None,
                    events=None, water_depth=np.inf):
        """Right-hand sides, solve with the factors, S @ sigma and the force
        integrals for the frequencies om (f[0:len(om)]); returns host arrays
        F (nb, nrhs, ndof) and FK (nb, nhead, ndof).  Raises the reference's
        exceptions on NaN, zero pivot or non-convergence."""
        ndof = len(body.dofs)
        if r.nrhs != ndof + len(heads) or r.batch < len(om):
            raise ValueError("right-hand side buffers of the wrong shape")
        (F, FK), = self._solve_segments(f, r, [(body, 0, len(om))], om, heads, rho=rho, g=g, stats=stats,
                                        events=events, water_depth=water_depth)
        return F, FK

    def _solve_segments(self, f: "_Factors", r: "_Rhs", segments, om, heads, *, rho=1000.0, g=9.81, stats=None,
                        events=None, sym: Optional[_SymWorkspace] = None, water_depth=np.inf):
        """solve_stage for batch entries holding several bodies: segments
        [(body, j0, m)] give the body of entries j0 .. j0+m-1.  A body smaller
        than the system (f.n, identity-padded) has zero right-hand-side rows
        beyond its panels; bodies with fewer dofs than r.nrhs - nhead have zero
        columns.  With `sym` (one body, a mesh with symmetries) the factors hold
        sym.st.nsys systems per frequency: right-hand sides go to the systems
        and potentials come back to the whole mesh through sym's transforms.
        Returns [(F (m, nrhs, ndof), FK (m, nhead, ndof))] per segment."""
        import torch
        lib = _lib.load()
        stream = _lib.stream_ptr()
        dev = f.K.device
        stats = {} if stats is None else stats
        n, npad = f.n, f.npad
        om = np.asarray(om, dtype=float)
        nb = len(om)
        nbs = nb * (sym.st.nsys if sym is not None else 1)  # systems of this batch
        ks = wavenumbers(om, water_depth, g)
        # omega = 0 or infinity: the frequency of the radiation problems is a
        # symbolic factor that the added mass cancels (problems_and_results.py:
        # 440-449, 583-592), so their right-hand sides and pressures take
        # omega = 1 (the matrices keep k = 0 or infinity); their diffraction
        # columns are left at zero (k = 0) and reported as NaN.
        limit = (om == 0.0) | np.isinf(om)
        om = np.where(limit, 1.0, om)
        ks = np.where(limit, 0.0, ks)
        heads = np.asarray(heads, dtype=float)
        nhead = len(heads)
        nrhs = r.nrhs
        ld = npad * nrhs  # batch stride of B, X, R
        small = _lib.upload(np.concatenate([om, ks, heads]), torch.float64, dev)
        om_t, k_t, heads_t = small[:nb], small[nb:2 * nb], small[2 * nb:]
        r.B.zero_()
        if sym is not None:  # right-hand sides of the whole mesh first
            rhs, rhs_ld, rhs_stride, n_max = sym.full, sym.n_full, sym.n_full * nrhs, sym.n_full
            rhs.zero_()
        else:
            rhs, rhs_ld, rhs_stride, n_max = r.B, npad, ld, n
        seg_arrays = []
        for body, j0, m in segments:
            mesh = body.mesh_including_lid
            ndof = len(body.dofs)
            if ndof + nhead > nrhs or mesh.nb_faces > n_max:
                raise ValueError("right-hand side buffers of the wrong shape")
            dm = self.green_function.device_mesh(mesh)
            dofn, wdof, hull = self._body_arrays(body, mesh)
            seg_arrays.append((mesh.nb_faces, ndof, dm, wdof))
            _lib.check(lib.bem_build_rhs(mesh.nb_faces, m, _vp(om_t.data_ptr() + 8 * j0),
                                         _vp(k_t.data_ptr() + 8 * j0), g, float(water_depth), ndof, _vp(dofn),
                                         nhead, _vp(heads_t), _vp(dm.centers), _vp(dm.normals), _vp(hull),
                                         _vp(rhs.data_ptr() + 16 * j0 * rhs_stride), rhs_ld, rhs_stride, stream))
        if sym is not None:
            sym.to_systems(nb, r.B, npad, ld, stream)
        direct = self.method == "direct"
        if direct:
            # rhs = S bc (bem/solver.py:182-183), through phi into the padded B
            for c0 in range(0, nrhs, RHS_CHUNK):
                nc = min(RHS_CHUNK, nrhs - c0)
                _lib.check(lib.bem_zgemm_ts(n, n, nc, 1.0, 0.0, _vp(f.S), n, n * n,
                                            _vp(r.B.data_ptr() + 16 * npad * c0), npad, ld, 0.0, 0.0,
                                            _vp(r.phi.data_ptr() + 16 * n * c0), n, n * nrhs, nbs, _vp(r.ts_work),
                                            stream))
            r.B.view(r.batch, nrhs, npad)[:nbs, :, :n].copy_(r.phi.view(r.batch, nrhs, n)[:nbs])
        sol = r.X
        for c0 in range(0, nrhs, RHS_CHUNK):
            nc = min(RHS_CHUNK, nrhs - c0)
            off = 16 * npad * c0  # byte offset of column c0
            Bc, Xc, Rc = (_vp(t.data_ptr() + off) for t in (r.B, r.X, r.R))
            if self._plain_gmres:
                self._gmres_solve(f, r, nbs, 1e-6, 1e-5, None, stats, stream, Bc, Xc, nc)
            elif self.precision == "mixed":
                self._refine(f, r, nbs, Bc, Xc, Rc, nc, stats, stream)
            else:
                self._solve_fp64(f, r, nbs, Bc, Xc, Rc, nc, stats, stream)
        if events:
            events[3].record()
        if direct:  # the solution is the potential
            phi_ptr, ldp, stp = sol.data_ptr(), npad, ld
        else:       # potential = S sigma
            for c0 in range(0, nrhs, RHS_CHUNK):
                nc = min(RHS_CHUNK, nrhs - c0)
                _lib.check(lib.bem_zgemm_ts(n, n, nc, 1.0, 0.0, _vp(f.S), n, n * n,
                                            _vp(sol.data_ptr() + 16 * npad * c0), npad, ld, 0.0, 0.0,
                                            _vp(r.phi.data_ptr() + 16 * n * c0), n, n * nrhs, nbs, _vp(r.ts_work),
                                            stream))
            phi_ptr, ldp, stp = r.phi.data_ptr(), n, n * nrhs
        if sym is not None:  # potentials of the systems back to the whole mesh
            sym.from_systems(nb, phi_ptr, ldp, stp, stream)
            phi_ptr, ldp, stp = sym.full.data_ptr(), sym.n_full, sym.n_full * nrhs
        sizes = [(m * nrhs * na[1], m * max(nhead, 1) * na[1]) for (_, _, m), na in zip(segments, seg_arrays)]
        out = torch.empty((sum(a + b for a, b in sizes),), dtype=torch.complex128, device=dev)
        views, pos = [], 0
        for (body, j0, m), (nf, ndof, dm, wdof), (sf, sk) in zip(segments, seg_arrays, sizes):
            F, FK = out[pos:pos + sf], out[pos + sf:pos + sf + sk]
            pos += sf + sk
            views.append((m, ndof, sf))
            _lib.check(lib.bem_integrate_pressure(nf, m, nrhs, ndof, _vp(phi_ptr + 16 * j0 * stp), ldp, stp,
                                                  _vp(om_t.data_ptr() + 8 * j0), rho, _vp(wdof), _vp(F), stream))
            if nhead > 0:
                _lib.check(lib.bem_froude_krylov(nf, m, ndof, nhead, _vp(k_t.data_ptr() + 8 * j0), rho, g,
                                                 float(water_depth), _vp(heads_t), _vp(dm.centers), _vp(wdof),
                                                 _vp(FK), stream))
        if events:
            events[4].record()
        host = out.cpu().numpy()
        flags = torch.cat([f.info[:nbs], r.flags]).cpu().numpy()
        if flags[nbs + 1] != 0:
            raise _lib.GreenFunctionEvaluationError(_lib.BEM_ERR_NAN, "Green function returned a NaN in the "
                                                    "interaction matrix.\nIt could be due to overlapping panels.")
        if np.any(flags[:nbs] != 0):
            raise _lib.SingularMatrixError(_lib.BEM_ERR_SINGULAR,
                                           f"zero pivot in the LU factorisation (info={flags[:nbs].tolist()})")
        if flags[nbs] != 0:
            raise _lib.BemError(_lib.BEM_ERR_TIMEOUT, "bounded wait in the triangular solve timed out")
        res, pos = [], 0
        for (m, ndof, sf), (_, sk) in zip(views, sizes):
            F_h = host[pos:pos + sf].reshape(m, nrhs, ndof)[:, :ndof + nhead]
            FK_h = host[pos + sf:pos + sf + sk].reshape(m, max(nhead, 1), ndof)[:, :nhead]
            pos += sf + sk
            res.append((F_h, FK_h))
        return res

    # ---- many bodies --------------------------------------------------------
    def solve_bodies(self, bodies, omegas: Sequence[float], *, wave_directions: Sequence[float] = (0.0,),
                     rho: float = 1000.0, g: float = 9.81, water_depth: float = np.inf, batch_bytes: float = 8e9,
                     sync_stats: bool = False, grouping: Optional[str] = None,
                     band: float = 1.3) -> List[FrequencyResults]:
        """Frequency sweeps of many bodies of uneven panel counts, batched
        across bodies.  Returns one FrequencyResults per body, in order (what
        solve_frequencies returns for that body); water_depth as in
        solve_frequencies.

        grouping "bands" (the default of the mixed engine): the (body, omega)
        pairs, largest bodies first, fill batches whose sizes lie within a
        factor `band` of the batch's largest; every matrix is identity-padded
        to that size and factored by the grouped LU
        (bem_clu_factor_grouped), whose tensor-core updates stop at each
        matrix's own size, so a small body in a batch costs the update flops
        of its own size.  The batch size per size class comes from
        BatchTuner (timed once per class, cached).
        grouping "size" (the float64 engine's): bodies whose size rounds up to
        the same multiple of the LU block form one group, factored together;
        with max_batch or more frequencies each body runs its own sweep."""
        if not water_depth > 0:
            raise ValueError(f"water_depth must be > 0 (got {water_depth})")
        omegas = np.asarray(omegas, dtype=float)
        grouping = grouping or ("bands" if self.precision == "mixed" else "size")
        if grouping not in ("bands", "size"):
            raise ValueError("grouping must be 'bands' or 'size'")
        if grouping == "bands" and self.precision != "mixed":
            raise ValueError("grouping='bands' needs the mixed engine (grouped LU)")
        if grouping == "size" and len(omegas) >= self.max_batch:
            return [self.solve_frequencies(b, omegas, wave_directions=wave_directions, rho=rho, g=g,
                                           water_depth=water_depth) for b in bodies]
        heads = np.asarray(wave_directions, dtype=float)
        nhead = len(heads)
        blk = 128 if self.precision == "mixed" else 64
        sizes = [-(-b.mesh_including_lid.nb_faces // blk) * blk for b in bodies]
        nq = len(omegas)
        plan = []  # (npad, nrhs, pairs, B, need, grouped)
        if grouping == "size":
            groups: Dict[int, List[int]] = {}
            for i, npad in enumerate(sizes):
                groups.setdefault(npad, []).append(i)
            for npad, idxs in sorted(groups.items()):
                nrhs = max(len(bodies[i].dofs) for i in idxs) + nhead
                pairs = [(i, q) for i in idxs for q in range(nq)]
                B = int(max(1, min(len(pairs), batch_bytes // _Factors.estimate_bytes(npad, 1, self.precision))))
                for c0 in range(0, len(pairs), B):
                    plan.append((npad, nrhs, pairs[c0:c0 + B], B, False))
        else:
            for npad, pairs in band_batches(sizes, nq, band,
                                            lambda top: self.batch_tuner.batch_for(self, top, batch_bytes)):
                plan.append((npad, max(len(bodies[i].dofs) for i, _ in pairs) + nhead, pairs, len(pairs), True))
        need = max(_Factors.estimate_bytes(npad, B, self.precision) + _Rhs.estimate_bytes(npad, npad, B, nrhs)
                   + 64 * (1 << 16) for npad, nrhs, _, B, _ in plan)
        F_all = [np.zeros((nq, len(b.dofs) + nhead, len(b.dofs)), dtype=np.complex128) for b in bodies]
        FK_all = [np.zeros((nq, max(nhead, 1), len(b.dofs)), dtype=np.complex128) for b in bodies]
        stats = {"groups": len({p[0] for p in plan}), "batches": 0, "assembly_ms": 0.0, "lu_ms": 0.0,
                 "solve_ms": 0.0, "grouping": grouping}
        arena = DeviceArena(need, self.device)  # one arena: no device allocation between batches
        shape = None
        f = r = release = None
        for npad, nrhs, chunk, B, grouped in plan:
            if shape != (npad, nrhs, B):
                if release is not None:
                    del f, r
                    release()  # the previous batches' work completed: their results reached the host
                alloc, release = arena.allocator()
                f = _Factors(npad, B, self.device, self.precision, alloc=alloc)
                r = _Rhs(npad, npad, B, nrhs, self.device, self.precision, alloc=alloc)
                shape = (npad, nrhs, B)
            self._solve_body_batch(bodies, omegas, heads, chunk, f, r, npad,
                                   [sizes[i] for i, _ in chunk] if grouped else None, rho, g, water_depth,
                                   stats, F_all, FK_all, sync_stats)
        if release is not None:
            del f, r
            release()
        return [self._coefficients(b, omegas, heads, F_all[i], FK_all[i], dict(stats)) for i, b in enumerate(bodies)]

    def _solve_body_batch(self, bodies, omegas, heads, chunk, f, r, npad, active, rho, g, water_depth, stats,
                          F_all, FK_all, sync_stats):
        """One batch of solve_bodies: the (body, omega) pairs of chunk, each
        body's matrices identity-padded to npad (active: each matrix's own
        padded size for the grouped LU, or None)."""
        import torch
        lib = _lib.load()
        stream = _lib.stream_ptr()
        nhead = len(heads)
        nb = len(chunk)
        segments = []
        for j, (i, q) in enumerate(chunk):
            if segments and segments[-1][0] is bodies[i]:
                segments[-1][2] += 1
            else:
                segments.append([bodies[i], j, 1])
        om = omegas[[q for _, q in chunk]]
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)] if sync_stats else None
        if ev:
            ev[0].record()
        r.flags.zero_()
        for body, j0, m in segments:
            mesh = body.mesh_including_lid
            self.assemble_stage(f, mesh, wavenumbers(om[j0:j0 + m], water_depth, g), nan_flag=r.nan,
                                first=j0, lds=npad, water_depth=water_depth)
            self.pad_stage(f, j0, m, mesh.nb_faces)
        if ev:
            ev[1].record()
        self.factor_stage(f, nb, r.err, active=active)
        if ev:
            ev[2].record()
        out = self._solve_segments(f, r, [tuple(sg) for sg in segments], om, heads, rho=rho, g=g,
                                   stats=stats, events=ev, water_depth=water_depth)
        for (body, j0, m), (F, FK) in zip(segments, out):
            i = chunk[j0][0]
            qs = [q for _, q in chunk[j0:j0 + m]]
            F_all[i][qs] = F
            FK_all[i][qs, :nhead] = FK
        stats["batches"] += 1
        if ev:
            torch.cuda.synchronize()
            stats["assembly_ms"] += ev[0].elapsed_time(ev[1])
            stats["lu_ms"] += ev[1].elapsed_time(ev[2])
            stats["solve_ms"] += ev[2].elapsed_time(ev[4])

    def _refine(self, f, r, nb, Bc, Xc, Rc, nc, stats, stream):
        """Refined solve of nc columns (B, X, R column pointers, batch stride
        npad * r.nrhs) with the float32 factors: classical refinement, or flexible
        GMRES right-preconditioned by the factors; the classical iteration continues
        with that GMRES when it stops contracting."""
        lib = _lib.load()
        n, npad, ld = f.n, f.npad, f.npad * r.nrhs
        iters, resid = ctypes.c_int32(0), ctypes.c_double(0.0)

        def gmres(cycles):
            return lib.bem_gmres_solve(_vp(f.K), n, n * n, n, npad, nb, Bc, Xc, npad, ld, nc, 0.0, self.refine_tol,
                                       self.gmres_restart, cycles, _vp(f.lu_work_ptr),
                                       _vp(r.gmres_work(self.gmres_restart)), _vp(r.err), ctypes.byref(iters),
                                       ctypes.byref(resid), stream)
        if self.refinement == "gmres":
            # relative residual refine_tol in every column: atol 0, rtol refine_tol
            status = gmres(max(1, -(-self.refine_max_iter // self.gmres_restart)))
        else:
            status = lib.bem_refine_solve(_vp(f.K), n, n * n, n, npad, nb, _vp(f.lu_work_ptr), _vp(f.piv), Bc, Xc, Rc,
                                          npad, ld, nc, self.refine_tol, self.refine_max_iter, _vp(r.ts_work),
                                          _vp(r.norms), _vp(r.err), ctypes.byref(iters), ctypes.byref(resid), stream)
            if status == _lib.BEM_ERR_NOT_CONVERGED:
                # x += (LU)^-1 r does not contract (K close to singular, e.g. near an
                # irregular frequency): GMRES on K, preconditioned by the same float32
                # factors, from x = 0 to the same tolerance.
                stats["escalated_to_gmres"] = stats.get("escalated_to_gmres", 0) + 1
                status = gmres(max(1, self.gmres_escalation_cycles))
        stats["refine_iters"] = max(stats.get("refine_iters", 0), iters.value)
        stats["refine_residual"] = max(stats.get("refine_residual", 0.0), resid.value)
        if status == _lib.BEM_ERR_NOT_CONVERGED:
            stats["not_converged"] = stats.get("not_converged", 0) + 1
            raise _lib.NotConvergedError(status, lib.bem_last_error().decode())
        _lib.check(status)

    def _solve_fp64(self, f, r, nb, Bc, Xc, Rc, nc, stats, stream):
        """Float64 LU solve of nc columns with its residual checked against K
        (bem_zlu_refine_solve): the block-local pivoting of the factorisation
        cannot lose accuracy unnoticed; stats carry the worst relative
        residual and the iterations (1 when the first solve already meets
        refine_tol)."""
        lib = _lib.load()
        n, npad, ld = f.n, f.npad, f.npad * r.nrhs
        iters, resid = ctypes.c_int32(0), ctypes.c_double(0.0)
        status = lib.bem_zlu_refine_solve(_vp(f.K), npad, npad * npad, n, _vp(f.LU), npad, npad, npad * npad, nb,
                                          _vp(f.piv), _vp(f.lu_work), Bc, Xc, Rc, npad, ld, nc, FP64_RESIDUAL_TOL,
                                          self.refine_max_iter, _vp(r.ts_work), _vp(r.norms), _vp(r.err),
                                          ctypes.byref(iters), ctypes.byref(resid), stream)
        stats["fp64_residual"] = max(stats.get("fp64_residual", 0.0), resid.value)
        stats["fp64_solve_iters"] = max(stats.get("fp64_solve_iters", 0), iters.value)
        if status == _lib.BEM_ERR_NOT_CONVERGED and resid.value <= self.refine_tol:
            status = _lib.BEM_OK  # at the float64 floor of an ill-conditioned K, below the accepted residual
        if status == _lib.BEM_ERR_NOT_CONVERGED:
            stats["not_converged"] = stats.get("not_converged", 0) + 1
            raise _lib.NotConvergedError(status, lib.bem_last_error().decode() +
                                         " (float64 LU with pivoting inside its diagonal blocks)")
        _lib.check(status)

    def _gmres_solve(self, f, r, nb, atol, rtol, precond_ptr, stats, stream, Bc, Xc, nc):
        """Plain float64 GMRES of nc RHS columns (column pointers Bc into Xc)
        with SciPy's settings: restart 20, at most 10 n cycles by default."""
        lib = _lib.load()
        n, npad = f.n, f.npad
        maxc = self.gmres_maxiter if self.gmres_maxiter is not None else 10 * n
        iters, resid = ctypes.c_int32(0), ctypes.c_double(0.0)
        status = lib.bem_gmres_solve(_vp(f.K), f.ldk, f.strideK, n, npad, nb, Bc, Xc, npad, npad * r.nrhs, nc, atol,
                                     rtol, self.gmres_restart, int(maxc), precond_ptr,
                                     _vp(r.gmres_work(self.gmres_restart)), _vp(r.err), ctypes.byref(iters),
                                     ctypes.byref(resid), stream)
        stats["gmres_iters"] = max(stats.get("gmres_iters", 0), iters.value)
        stats["gmres_residual"] = max(stats.get("gmres_residual", 0.0), resid.value)
        if status == _lib.BEM_ERR_NOT_CONVERGED:
            raise _lib.NotConvergedError(status, lib.bem_last_error().decode() +
                                         "\nThis can be due to overlapping panels or irregular frequencies.")
        _lib.check(status)

    @staticmethod
    def _coefficients(body, omegas, heads, F_all, FK_all, stats):
        """Added mass Re(F) / omega^2, damping Im(F) / omega and the wave forces
        (problems_and_results.py:583-592); at omega = 0 or infinity the forces
        were computed with omega = 1, the damping is zero and the wave forces
        are NaN (the reference's limit-frequency results, airy_waves.py:36-37)."""
        ndof = len(body.dofs)
        omegas = np.asarray(omegas, dtype=float)
        limit = (omegas == 0.0) | np.isinf(omegas)
        w = np.where(limit, 1.0, omegas)[:, None, None]
        rad = F_all[:, :ndof, :]
        added_mass = np.real(rad) / w ** 2
        damping = np.imag(rad) / w
        damping[limit] = 0.0
        diffraction = F_all[:, ndof:, :].copy()
        fk = FK_all[:, : len(heads), :].copy()
        diffraction[limit] = np.nan
        fk[limit] = np.nan
        return FrequencyResults(omegas=omegas, dofs=list(body.dofs), wave_directions=heads, added_mass=added_mass,
                                radiation_damping=damping, diffraction=diffraction, froude_krylov=fk,
                                excitation=diffraction + fk, stats=stats)

    # ------------------------------------------------------------------------
    # capytaine MatrixEngine interface
    def build_matrices(self, mesh1, mesh2, **gf_params):
        """bem/engines.py:273-298 with a single-entry cache (:258-270)."""
        key = (mesh1, mesh2, dict(gf_params))
        if key == self.last_computed_inputs:
            return self.last_computed_matrices
        self.last_computed_matrices = None
        params = dict(gf_params)
        params.setdefault("early_dot_product", True)
        st = _shared_structure(mesh1, mesh2) if params["early_dot_product"] else None
        if st is not None:
            # bem/engines.py:178-247: the whole first mesh against the reference
            # sub-mesh of the second, as block-circulant matrices
            import torch
            S, K = self.green_function.evaluate_device(mesh1.merged(), st.submesh, dtype=torch.complex128, **params)
            self.last_computed_inputs = key
            self.last_computed_matrices = (DeviceBlockCirculantMatrix(S, st, self),
                                           DeviceBlockCirculantMatrix(K, st, self))
            return self.last_computed_matrices
        S, K = self.green_function.evaluate_device(mesh1, mesh2, **params)
        self.last_computed_inputs = key
        self.last_computed_matrices = (DeviceMatrix(S, self), DeviceMatrix(K, self))
        return self.last_computed_matrices

    def build_S_matrix(self, points, mesh, **gf_params):
        S, _ = self.green_function.evaluate_device(points, mesh, **gf_params)
        return DeviceMatrix(S, self)

    def build_fullK_matrix(self, mesh1, mesh2, **gf_params):
        gf_params.setdefault("diagonal_term_in_double_layer", True)
        gf_params.setdefault("adjoint_double_layer", True)
        gf_params["early_dot_product"] = False
        _, K = self.green_function.evaluate_device(mesh1, mesh2, **gf_params)
        return K.cpu().numpy()

    def linear_solver(self, A, b):
        """bem/engines.py:300-346: LU of A on the device, cached on A (the cache
        entry replaces K, as the reference does), one RHS per call; or GMRES
        (bem/engines.py:74-89); or the user's callable."""
        if callable(self._linear_solver):
            x = self._linear_solver(A, b)
            if np.asarray(x).shape != np.asarray(b).shape:
                raise ValueError(f"Error in linear solver of {self}: the shape of the output is not the same "
                                 "as the shape of the RHS")
            return x
        if not isinstance(A, (DeviceMatrix, DeviceBlockCirculantMatrix)):
            A = DeviceMatrix(_to_device(np.asarray(A), self.device), self)
        if self._linear_solver == "gmres":
            x = A.gmres(np.asarray(b), atol=1e-6, rtol=1e-5, restart=self.gmres_restart, maxiter=self.gmres_maxiter)
        else:
            x = A.solve(np.asarray(b))
        if x.shape != np.asarray(b).shape:
            raise ValueError("linear solver output shape mismatch")
        return x

    def compute_ram_estimation(self, problem):
        """Device memory (GB) of S, K and the LU (bem/engines.py:348-398): for a
        mesh with symmetries the first block columns of S and K and the systems
        of S and K (LU in place)."""
        mesh = problem.body.mesh_including_lid if hasattr(problem.body, "mesh_including_lid") \
            else problem.body.mesh
        n = mesh.nb_faces
        st = block_structure(mesh)
        if st is not None:
            return 16 * (2 * n * st.n_sub + 2 * st.nsys * padded_size(st.n_sys) ** 2) / 1e9
        return 3 * 16 * padded_size(n) ** 2 / 1e9


def _to_device(a: np.ndarray, device):
    import torch
    t = torch.as_tensor(np.asfortranarray(a), device=device)
    return t


def _fp64_checked_solve(K_ptr, ldk, strideK, n, lu, batch, Bh, nrhs, tol=FP64_RESIDUAL_TOL, accept=1e-10,
                        max_iter=30):
    """X solving K X = B for `batch` systems with the float64 factors lu =
    (Kf, piv, work, npad) of bem_zlu_factor, the residual of every column
    checked (and refined) against the unfactored K at K_ptr (n x n,
    column-major, ldk, strideK apart) by bem_zlu_refine_solve.  Bh: (batch,
    nrhs, npad) complex128 device tensor, rows >= n zero.  A residual that
    stops decreasing above tol is accepted up to `accept`.  Returns X shaped
    like Bh."""
    import torch
    Kf, piv, work, npad = lu
    lib = _lib.load()
    stream = _lib.stream_ptr()
    X = torch.zeros_like(Bh)
    R = torch.empty_like(Bh)
    err = torch.zeros(1, dtype=torch.int32, device=Bh.device)
    for c0 in range(0, nrhs, RHS_CHUNK):
        nc = min(RHS_CHUNK, nrhs - c0)
        ts = torch.empty(int(lib.bem_zgemm_ts_workspace_bytes(n, n, nc, batch)), dtype=torch.uint8, device=Bh.device)
        norms = torch.zeros(2 * batch * nc + 2, dtype=torch.float64, device=Bh.device)
        iters, resid = ctypes.c_int32(0), ctypes.c_double(0.0)
        off = 16 * npad * c0
        status = lib.bem_zlu_refine_solve(_vp(K_ptr), ldk, strideK, n, _vp(Kf), npad, npad, npad * npad, batch,
                                          _vp(piv), _vp(work), _vp(Bh.data_ptr() + off), _vp(X.data_ptr() + off),
                                          _vp(R.data_ptr() + off), npad, npad * nrhs, nc, tol, max_iter, _vp(ts),
                                          _vp(norms), _vp(err), ctypes.byref(iters), ctypes.byref(resid), stream)
        if status == _lib.BEM_ERR_NOT_CONVERGED and resid.value <= accept:
            status = _lib.BEM_OK
        if status == _lib.BEM_ERR_NOT_CONVERGED:
            raise _lib.NotConvergedError(status, lib.bem_last_error().decode())
        _lib.check(status)
    if int(err.item()) != 0:
        raise _lib.BemError(_lib.BEM_ERR_TIMEOUT, "bounded wait in the triangular solve timed out")
    return X


class DeviceMatrix:
    """A device-resident influence matrix usable where capytaine expects an
    ndarray: ``M @ x`` and ``engine.linear_solver(M, b)`` run on the GPU."""

    def __init__(self, t, engine: B200Engine):
        self.t = t  # (n, N) view, column-major
        self.engine = engine
        self._lu = None

    @property
    def shape(self):
        return tuple(self.t.shape)

    @property
    def dtype(self):
        return np.dtype(str(self.t.dtype).replace("torch.", ""))

    def __array__(self, dtype=None, copy=None):
        a = self.t.cpu().numpy()
        return a.astype(dtype) if dtype is not None else a

    def __matmul__(self, x):
        import torch
        x = np.asarray(x)
        vec = x.ndim == 1
        X = x.reshape(x.shape[0], -1).astype(np.complex128)
        n, K = self.t.shape
        nrhs = X.shape[1]
        # Explicit column-major buffers: element (i, c) at i + c*ld (reported strides
        # of size-1 dimensions are not reliable leading dimensions).
        Acm = torch.empty((K, n), dtype=torch.complex128, device=self.t.device)  # Acm[j, i] = A[i, j]
        Acm.copy_(self.t.T)
        Xcm = torch.as_tensor(np.ascontiguousarray(X.T), device=Acm.device)   # Xcm[c, k] = X[k, c]
        Ycm = torch.empty((nrhs, n), dtype=torch.complex128, device=Acm.device)
        lib = _lib.load()
        for c0 in range(0, nrhs, 16):
            c1 = min(nrhs, c0 + 16)
            work = torch.empty(int(lib.bem_zgemm_ts_workspace_bytes(n, K, c1 - c0, 1)), dtype=torch.uint8,
                               device=Acm.device)
            _lib.check(lib.bem_zgemm_ts(n, K, c1 - c0, 1.0, 0.0, _vp(Acm), n, 0, _vp(Xcm[c0:c1]), K, 0, 0.0, 0.0,
                                        _vp(Ycm[c0:c1]), n, 0, 1, _vp(work), _lib.stream_ptr()))
        res = Ycm.T.cpu().numpy()
        if self.t.dtype == torch.complex64:
            res = res.astype(np.complex64)
        return res[:, 0] if vec else res.reshape((n,) + x.shape[1:])

    def _factor(self):
        import torch
        if self._lu is not None:
            return self._lu
        n = self.t.shape[0]
        npad = padded_size(n)
        dev = self.t.device
        lib = _lib.load()
        # Column-major npad x npad buffer: element (r, c) at r + c*npad, i.e. Kf.T[r, c].
        Kf = torch.zeros((npad, npad), dtype=torch.complex128, device=dev)
        Kf.T[:n, :n] = self.t.to(torch.complex128)
        _lib.check(lib.bem_zpad_identity(_vp(Kf), npad, npad * npad, 1, n, npad, _lib.stream_ptr()))
        piv = torch.empty(npad, dtype=torch.int32, device=dev)
        info = torch.zeros(1, dtype=torch.int32, device=dev)
        work = torch.empty(int(lib.bem_zlu_workspace_bytes(npad, 1)), dtype=torch.uint8, device=dev)
        _lib.check(lib.bem_zlu_factor(_vp(Kf), npad, npad, npad * npad, 1, _vp(piv), _vp(info), _vp(work),
                                      _lib.stream_ptr()))
        if int(info.item()) != 0:
            raise _lib.SingularMatrixError(_lib.BEM_ERR_SINGULAR, f"zero pivot at column {int(info.item())}")
        # the unfactored matrix, column-major complex128, for the residual checks
        Kcm = torch.empty((n, n), dtype=torch.complex128, device=dev)  # Kcm[j, i] = K[i, j]
        Kcm.copy_(self.t.to(torch.complex128).T)
        self._lu = (Kf, piv, work, npad)
        self._kcm = Kcm
        return self._lu

    def gmres(self, b: np.ndarray, *, atol=1e-6, rtol=1e-5, restart=20, maxiter=None) -> np.ndarray:
        """Restarted GMRES on the device (x0 = 0), SciPy's criterion
        |b - A x| <= max(atol, rtol |b|) per column; NotConvergedError (a
        RuntimeError) otherwise, as capytaine's solve_gmres (bem/engines.py:74-89)."""
        import torch
        b = np.asarray(b)
        vec = b.ndim == 1
        Bm = b.reshape(b.shape[0], -1).astype(np.complex128)
        n, nrhs = Bm.shape
        dev = self.t.device
        lib = _lib.load()
        A = self.t.to(torch.complex128)
        Acm = torch.empty((n, n), dtype=torch.complex128, device=dev)  # Acm[j, i] = A[i, j]: column-major
        Acm.copy_(A.T)
        maxc = int(maxiter) if maxiter is not None else 10 * n
        out = np.empty_like(Bm)
        for c0 in range(0, nrhs, 16):
            c1 = min(nrhs, c0 + 16)
            nc = c1 - c0
            Bd = torch.as_tensor(np.ascontiguousarray(Bm[:, c0:c1].T), device=dev)  # column-major n x nc
            Xd = torch.empty_like(Bd)
            nbytes = int(lib.bem_gmres_workspace_bytes(n, n, nc, 1, restart))
            work = torch.empty(nbytes + 256, dtype=torch.uint8, device=dev)
            wptr = (work.data_ptr() + 255) // 256 * 256
            iters, resid = ctypes.c_int32(0), ctypes.c_double(0.0)
            st = lib.bem_gmres_solve(_vp(Acm), n, 0, n, n, 1, _vp(Bd), _vp(Xd), n, 0, nc, float(atol), float(rtol),
                                     int(restart), maxc, None, _vp(wptr), None, ctypes.byref(iters),
                                     ctypes.byref(resid), _lib.stream_ptr())
            if st == _lib.BEM_ERR_NOT_CONVERGED:
                raise _lib.NotConvergedError(st, lib.bem_last_error().decode() +
                                             "\nThis can be due to overlapping panels or irregular frequencies.")
            _lib.check(st)
            out[:, c0:c1] = Xd.T.cpu().numpy()
        x = out[:, 0] if vec else out.reshape(b.shape)
        return x.astype(np.complex64) if self.t.dtype == torch.complex64 else x

    def solve(self, b: np.ndarray) -> np.ndarray:
        import torch
        Kf, piv, work, npad = self._factor()
        b = np.asarray(b)
        vec = b.ndim == 1
        Bm = b.reshape(b.shape[0], -1).astype(np.complex128)
        n, nrhs = Bm.shape
        dev = Kf.device
        Bd = torch.zeros((1, nrhs, npad), dtype=torch.complex128, device=dev)  # column-major npad x nrhs
        Bd[0, :, :n] = torch.as_tensor(Bm.T.copy(), device=dev)
        X = _fp64_checked_solve(self._kcm, n, 0, n, (Kf, piv, work, npad), 1, Bd, nrhs)
        out = X[0, :, :n].T.cpu().numpy()
        x = out[:, 0] if vec else out.reshape(b.shape)
        return x.astype(np.complex64) if self.t.dtype == torch.complex64 else x


def _structure_signature(mesh):
    """Kind, planes, order and axis of the symmetries of a mesh (None: plain)."""
    from .symmetric_meshes import ReflectionSymmetricMesh, RotationSymmetricMesh
    if isinstance(mesh, ReflectionSymmetricMesh):
        return ("reflection", mesh.plane, _structure_signature(mesh.half))
    if isinstance(mesh, RotationSymmetricMesh):
        return ("rotation", mesh.n, mesh.axis, _structure_signature(mesh.wedge))
    return None


def _shared_structure(mesh1, mesh2):
    """Block structure of the matrices of mesh1 (collocation) against mesh2
    (panels) when both have the same symmetries (the condition of
    bem/engines.py:181-235), else None."""
    if not hasattr(mesh1, "faces_centers"):
        return None
    sig = _structure_signature(mesh2)
    if sig is None or _structure_signature(mesh1) != sig:
        return None
    st = block_structure(mesh2)
    if st is None or mesh1.nb_faces != mesh2.nb_faces:
        return None
    return st


class DeviceBlockCirculantMatrix:
    """S or K between two meshes with the same symmetries, kept as its first
    block column on the device and the independent systems of its
    block-diagonalisation: what capytaine keeps as a BlockCirculantMatrix /
    NestedBlockCirculantMatrix (tools/block_circulant_matrices.py:42-301).
    ``M @ x`` applies the systems between the two transforms,
    ``engine.linear_solver(M, b)`` factors the systems (batched float64 LU,
    cached on the matrix, as LUDecomposedBlockCirculantMatrix) and solves, and
    ``np.asarray(M)`` is the dense matrix."""

    def __init__(self, cols, st, engine: B200Engine):
        import torch
        self.st, self.engine = st, engine
        self.n = st.nb_images * st.n_sub
        self.cols = cols  # (n, n_sub) column-major view: element (i, j) at i + j * n
        dev = cols.device
        self.W, self.Winv, self.src = _transform_tensors(st, dev)
        self.systems = torch.empty((st.nsys, st.n_sys * st.n_sys), dtype=torch.complex128, device=dev)
        _combine_first_column(st, self.W, self.src, cols.data_ptr(), self.n, 1, self.systems.data_ptr(), st.n_sys,
                              st.n_sys * st.n_sys, _lib.stream_ptr())
        self._lu = None

    @property
    def shape(self):
        return (self.n, self.n)

    @property
    def dtype(self):
        return np.dtype(np.complex64) if self.engine.green_function.floating_point_precision == "float32" \
            else np.dtype(np.complex128)

    def __array__(self, dtype=None, copy=None):
        st = self.st
        cols = self.cols.cpu().numpy()  # (n, n_sub)
        a = st.full_matrix(cols.reshape(st.nb_images, st.n_sub, st.n_sub))
        return a.astype(dtype if dtype is not None else self.dtype)

    def _columns(self, x):
        """(n, nrhs) complex128 right-hand side as a device (nrhs, n) tensor."""
        import torch
        x = np.asarray(x)
        X = x.reshape(x.shape[0], -1).astype(np.complex128)
        return torch.as_tensor(np.ascontiguousarray(X.T), device=self.systems.device), x.ndim == 1, x.shape

    def _to_systems(self, Xd, ld):
        """(nsys, nrhs, ld) device tensor of the right-hand sides of the systems (rows >= n_sys zero)."""
        import torch
        st = self.st
        nrhs = Xd.shape[0]
        Xh = torch.zeros((st.nsys, nrhs, ld), dtype=torch.complex128, device=Xd.device)
        _lib.check(_lib.load().bem_block_combine(_vp(Xd), 0, st.n_sys, self.n, _vp(Xh), 0, nrhs * ld, ld,
                                                 _vp(self.W), None, st.nsys, st.nsys, st.n_sys, nrhs, 1,
                                                 _lib.stream_ptr()))
        return Xh

    def _from_systems(self, Yh, ld):
        import torch
        st = self.st
        nrhs = Yh.shape[1]
        Y = torch.empty((nrhs, self.n), dtype=torch.complex128, device=Yh.device)
        _lib.check(_lib.load().bem_block_combine(_vp(Yh), 0, nrhs * ld, ld, _vp(Y), 0, st.n_sys, self.n,
                                                 _vp(self.Winv), None, st.nsys, st.nsys, st.n_sys, nrhs, 1,
                                                 _lib.stream_ptr()))
        return Y

    def _out(self, Y, vec, shape):
        res = Y.T.cpu().numpy()
        res = res.astype(self.dtype)
        return res[:, 0] if vec else res.reshape(shape)

    def __matmul__(self, x):
        import torch
        st = self.st
        Xd, vec, shape = self._columns(x)
        nrhs, ns = Xd.shape[0], st.n_sys
        Xh = self._to_systems(Xd, ns)
        Yh = torch.empty_like(Xh)
        lib = _lib.load()
        for c0 in range(0, nrhs, RHS_CHUNK):
            nc = min(RHS_CHUNK, nrhs - c0)
            work = torch.empty(int(lib.bem_zgemm_ts_workspace_bytes(ns, ns, nc, st.nsys)), dtype=torch.uint8,
                               device=Xh.device)
            _lib.check(lib.bem_zgemm_ts(ns, ns, nc, 1.0, 0.0, _vp(self.systems), ns, ns * ns,
                                        _vp(Xh.data_ptr() + 16 * ns * c0), ns, nrhs * ns, 0.0, 0.0,
                                        _vp(Yh.data_ptr() + 16 * ns * c0), ns, nrhs * ns, st.nsys, _vp(work),
                                        _lib.stream_ptr()))
        return self._out(self._from_systems(Yh, ns), vec, shape)

    def _factor(self):
        import torch
        if self._lu is not None:
            return self._lu
        st = self.st
        ns, npad = st.n_sys, padded_size(st.n_sys)
        dev = self.systems.device
        lib = _lib.load()
        Kf = torch.zeros((st.nsys, npad, npad), dtype=torch.complex128, device=dev)  # Kf[k].T: column-major
        Kf.transpose(1, 2)[:, :ns, :ns] = self.systems.view(st.nsys, ns, ns).transpose(1, 2)
        stream = _lib.stream_ptr()
        _lib.check(lib.bem_zpad_identity(_vp(Kf), npad, npad * npad, st.nsys, ns, npad, stream))
        piv = torch.empty((st.nsys, npad), dtype=torch.int32, device=dev)
        info = torch.zeros(st.nsys, dtype=torch.int32, device=dev)
        work = torch.empty(int(lib.bem_zlu_workspace_bytes(npad, st.nsys)), dtype=torch.uint8, device=dev)
        _lib.check(lib.bem_zlu_factor(_vp(Kf), npad, npad, npad * npad, st.nsys, _vp(piv), _vp(info), _vp(work),
                                      stream))
        bad = info.cpu().numpy()
        if np.any(bad != 0):
            raise _lib.SingularMatrixError(_lib.BEM_ERR_SINGULAR, f"zero pivot (info={bad.tolist()})")
        self._lu = (Kf, piv, work, npad)
        return self._lu

    def solve(self, b):
        import torch
        Kf, piv, work, npad = self._factor()
        st = self.st
        Xd, vec, shape = self._columns(b)
        nrhs = Xd.shape[0]
        Bh = self._to_systems(Xd, npad)
        X = _fp64_checked_solve(self.systems, st.n_sys, st.n_sys * st.n_sys, st.n_sys, (Kf, piv, work, npad),
                                st.nsys, Bh, nrhs)
        return self._out(self._from_systems(X, npad), vec, shape)

    def gmres(self, b, **kw):
        """capytaine's solve_gmres iterates on the whole operator: the dense
        matrix on the device, then DeviceMatrix.gmres."""
        import torch
        dense = torch.as_tensor(np.asfortranarray(np.asarray(self, dtype=np.complex128)), device=self.systems.device)
        return DeviceMatrix(dense, self.engine).gmres(b, **kw)
