"""ctypes binding of ``libcapytaine_b200.so`` (declared in include/capytaine_b200.h).

The product path always goes through this library.  There is no CPU fallback:
importing works without a GPU (so the library and its symbols can be
inspected), but every compute call raises when the library or a CUDA device is
missing.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcapytaine_b200.so")

BEM_OK = 0
BEM_ERR_INVALID_ARGUMENT = 1
BEM_ERR_CUDA = 2
BEM_ERR_NAN = 3
BEM_ERR_SINGULAR = 4
BEM_ERR_NOT_CONVERGED = 5
BEM_ERR_OUT_OF_MEMORY = 6
BEM_ERR_UNSUPPORTED = 7
BEM_ERR_TIMEOUT = 8

BEM_GRID_LEGACY, BEM_GRID_SCALED_NEMOH3 = 0, 1
BEM_GF_HIGH_FREQ, BEM_GF_LOW_FREQ, BEM_GF_LOW_FREQ_WITH_RANKINE_PART = 0, 1, 2
BEM_DTYPE_C128, BEM_DTYPE_C64 = 0, 1
BEM_PREC_FP64, BEM_PREC_MIXED = 0, 1


class BemError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"[bem status {code}] {message}")
        self.code = code


class GreenFunctionEvaluationError(BemError):
    """Same meaning as capytaine's GreenFunctionEvaluationError (NaN in a matrix)."""


class SingularMatrixError(BemError):
    pass


class NotConvergedError(BemError):
    pass


c_int, c_i64, c_double, c_void_p = ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p


class AssemblyArgs(ctypes.Structure):
    """Mirror of ``bem_assembly_args`` (include/capytaine_b200.h)."""
    _fields_ = [
        ("n", c_int), ("points_dev", c_void_p), ("dot_normals_dev", c_void_p),
        ("nb_faces", c_int), ("nb_vertices", c_int), ("vertices_dev", c_void_p), ("faces_dev", c_void_p),
        ("centers_dev", c_void_p), ("normals_dev", c_void_p), ("areas_dev", c_void_p), ("radii_dev", c_void_p),
        ("nb_quad_points", c_int), ("quad_points_dev", c_void_p), ("quad_weights_dev", c_void_p),
        ("tabulation_nb_integration_points", c_int), ("tabulation_grid_shape", c_int), ("nr", c_int), ("nz", c_int),
        ("r_range_dev", c_void_p), ("z_range_dev", c_void_p), ("table_dev", c_void_p), ("table32_dev", c_void_p),
        ("wavenumber", c_double), ("free_surface", c_double), ("gf_singularities", c_int),
        ("adjoint_double_layer", c_int), ("early_dot_product", c_int), ("diagonal_term", c_int), ("precision", c_int),
        ("out_dtype", c_int), ("S_dev", c_void_p), ("K_dev", c_void_p), ("lds", c_i64), ("ldk", c_i64),
        ("k_plane_stride", c_i64), ("nan_flag_dev", c_void_p), ("r_inv_den_dev", c_void_p),
        ("z_inv_den_dev", c_void_p),
    ]


class GreenFunctionParams(ctypes.Structure):
    """Mirror of ``bem_green_function_params``."""
    _fields_ = [("tabulation_nr", c_int), ("tabulation_rmax", c_double), ("tabulation_nz", c_int),
                ("tabulation_zmin", c_double), ("tabulation_nb_integration_points", c_int),
                ("tabulation_grid_shape", c_int), ("gf_singularities", c_int)]


class MeshDesc(ctypes.Structure):
    """Mirror of ``bem_mesh_desc`` (host pointers)."""
    _fields_ = [("nb_faces", c_int), ("nb_vertices", c_int), ("vertices", c_void_p), ("faces", c_void_p),
                ("centers", c_void_p), ("normals", c_void_p), ("areas", c_void_p), ("radii", c_void_p),
                ("hull_mask", c_void_p)]


class SolveStats(ctypes.Structure):
    """Mirror of ``bem_solve_stats``."""
    _fields_ = [("iterations", c_int), ("residual", c_double), ("escalated_to_gmres", c_int)]


BEM_PENDING = 9

_SIGNATURES = {
    "bem_last_error": ([], ctypes.c_char_p),
    "bem_version": ([], c_int),
    "bem_launch_count": ([], ctypes.c_longlong),
    "bem_kernel_timer_enable": ([ctypes.c_int], ctypes.c_int),
    "bem_kernel_timer_read": ([ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong)],
                              ctypes.c_int),
    "bem_kernel_class_name": ([ctypes.c_int], ctypes.c_char_p),
    "bem_default_r_spacing": ([c_int, c_double, c_int, c_void_p], c_int),
    "bem_default_z_spacing": ([c_int, c_double, c_int, c_void_p], c_int),
    "bem_construct_tabulation": ([c_void_p, c_int, c_void_p, c_int, c_int, c_void_p, c_void_p], c_int),
    "bem_tabulation_inverse_denominators": ([c_void_p, c_int, c_void_p], c_int),
    "bem_assemble": ([ctypes.POINTER(AssemblyArgs), c_void_p], c_int),
    "bem_assemble_rankine_part": ([ctypes.POINTER(AssemblyArgs), c_void_p, c_i64, c_void_p], c_int),
    "bem_assemble_wave_symmetric": ([ctypes.POINTER(AssemblyArgs), c_void_p, c_i64, c_void_p], c_int),
    "bem_assemble_wave_symmetric_batched": ([ctypes.POINTER(AssemblyArgs), c_void_p, c_i64, c_void_p, c_int, c_i64,
                                             c_i64, c_void_p], c_int),
    "bem_assemble_wave_symmetric_batched_lu": ([ctypes.POINTER(AssemblyArgs), c_void_p, c_i64, c_void_p, c_int,
                                                c_i64, c_i64, c_void_p, c_int, c_int, c_void_p], c_int),
    "bem_assemble_symmetric": ([ctypes.POINTER(AssemblyArgs), c_void_p], c_int),
    "bem_assemble_finite_depth": ([ctypes.POINTER(AssemblyArgs), c_double, c_int, c_void_p, c_int, c_void_p], c_int),
    "bem_assemble_wave_cached": ([ctypes.POINTER(AssemblyArgs), c_void_p, c_i64, c_void_p, c_int, c_i64, c_i64,
                                  c_void_p], c_int),
    "bem_zpad_identity": ([c_void_p, c_i64, c_i64, c_int, c_int, c_int, c_void_p], c_int),
    "bem_zgemm": ([c_int, c_int, c_int, c_double, c_void_p, c_i64, c_i64, c_void_p, c_i64, c_i64, c_double,
                   c_void_p, c_i64, c_i64, c_int, c_void_p], c_int),
    "bem_zlu_workspace_bytes": ([c_int, c_int], c_i64),
    "bem_zlu_factor": ([c_void_p, c_int, c_i64, c_i64, c_int, c_void_p, c_void_p, c_void_p, c_void_p], c_int),
    "bem_zlu_solve": ([c_void_p, c_int, c_i64, c_i64, c_int, c_void_p, c_void_p, c_void_p, c_i64, c_i64, c_int,
                       c_void_p, c_void_p], c_int),
    "bem_build_rhs": ([c_int, c_int, c_void_p, c_void_p, c_double, c_double, c_int, c_void_p, c_int, c_void_p,
                       c_void_p, c_void_p, c_void_p, c_void_p, c_i64, c_i64, c_void_p], c_int),
    "bem_zgemm_ts_workspace_bytes": ([c_int, c_int, c_int, c_int], c_i64),
    "bem_zgemm_ts": ([c_int, c_int, c_int, c_double, c_double, c_void_p, c_i64, c_i64, c_void_p, c_i64, c_i64,
                      c_double, c_double, c_void_p, c_i64, c_i64, c_int, c_void_p, c_void_p], c_int),
    "bem_integrate_pressure": ([c_int, c_int, c_int, c_int, c_void_p, c_i64, c_i64, c_void_p, c_double, c_void_p,
                                c_void_p, c_void_p], c_int),
    "bem_cgemm_tf32_update": ([c_void_p, c_i64, c_int, c_void_p, c_i64, c_int, c_int, c_void_p, c_void_p, c_i64,
                               c_i64, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p], c_int),
    "bem_clu_workspace_bytes": ([c_int, c_int], c_i64),
    "bem_clu_factor": ([c_void_p, c_i64, c_i64, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                        c_void_p], c_int),
    "bem_clu_factor_grouped": ([c_void_p, c_i64, c_i64, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                c_void_p, c_void_p], c_int),
    "bem_clu_factor_planes": ([c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p], c_int),
    "bem_clu_solve": ([c_void_p, c_int, c_int, c_void_p, c_void_p, c_i64, c_i64, c_int, c_void_p, c_void_p], c_int),
    "bem_clu_solve_bounded": ([c_void_p, c_int, c_int, c_void_p, c_void_p, c_i64, c_i64, c_int, ctypes.c_longlong,
                               c_int, c_void_p, c_void_p], c_int),
    "bem_zlu_refine_solve": ([c_void_p, c_i64, c_i64, c_int, c_void_p, c_int, c_i64, c_i64, c_int, c_void_p,
                              c_void_p, c_void_p, c_void_p, c_void_p, c_i64, c_i64, c_int, c_double, c_int, c_void_p,
                              c_void_p, c_void_p, ctypes.POINTER(c_int), ctypes.POINTER(c_double), c_void_p], c_int),
    "bem_refine_solve": ([c_void_p, c_i64, c_i64, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                          c_void_p, c_i64, c_i64, c_int, c_double, c_int, c_void_p, c_void_p, c_void_p,
                          ctypes.POINTER(c_int), ctypes.POINTER(c_double), c_void_p], c_int),
    "bem_gmres_workspace_bytes": ([c_int, c_int, c_int, c_int, c_int], c_i64),
    "bem_gmres_solve": ([c_void_p, c_i64, c_i64, c_int, c_int, c_int, c_void_p, c_void_p, c_i64, c_i64, c_int,
                         c_double, c_double, c_int, c_int, c_void_p, c_void_p, c_void_p, ctypes.POINTER(c_int),
                         ctypes.POINTER(c_double), c_void_p], c_int),
    "bem_zgemm_ts_static_capacity": ([], c_i64),
    "bem_zgemm_ts_static": ([c_int, c_int, c_int, c_double, c_double, c_void_p, c_i64, c_i64, c_void_p, c_i64, c_i64,
                             c_double, c_double, c_void_p, c_i64, c_i64, c_int, c_void_p], c_int),
    "bem_froude_krylov": ([c_int, c_int, c_int, c_int, c_void_p, c_double, c_double, c_double, c_void_p, c_void_p,
                           c_void_p, c_void_p, c_void_p], c_int),
    "bem_context_create": ([c_int, ctypes.POINTER(GreenFunctionParams), ctypes.POINTER(c_void_p)], c_int),
    "bem_context_tabulation": ([c_void_p, c_void_p, c_void_p, c_void_p], c_int),
    "bem_context_set_tabulation": ([c_void_p, c_void_p], c_int),
    "bem_solve_frequency": ([c_void_p, ctypes.POINTER(MeshDesc), c_int, c_void_p, c_int, c_void_p, c_int, c_void_p,
                             c_double, c_double, c_int, c_void_p, c_void_p, c_void_p, ctypes.POINTER(SolveStats)],
                            c_int),
    "bem_solve_submit": ([c_void_p, ctypes.POINTER(MeshDesc), c_int, c_void_p, c_int, c_void_p, c_int, c_void_p,
                          c_double, c_double, c_int, c_void_p, c_void_p, c_void_p, ctypes.POINTER(c_void_p)], c_int),
    "bem_request_poll": ([c_void_p, c_int, ctypes.POINTER(SolveStats)], c_int),
    "bem_lu_factor": ([c_void_p, c_void_p, c_i64, c_int, c_int, ctypes.POINTER(c_void_p)], c_int),
    "bem_lu_solve": ([c_void_p, c_void_p, c_i64, c_int, c_void_p, c_i64, ctypes.POINTER(SolveStats)], c_int),
    "bem_release": ([c_void_p], c_int),
    "bem_block_combine": ([c_void_p, c_i64, c_i64, c_i64, c_void_p, c_i64, c_i64, c_i64, c_void_p, c_void_p, c_int,
                           c_int, c_int, c_int, c_int, c_void_p], c_int),
}

_lock = threading.Lock()
_lib = None


def exported_symbols():
    """Names of the C-ABI entry points this binding declares."""
    return sorted(_SIGNATURES)


def load(build_if_missing: bool = False):
    """Load the shared library (optionally building it first)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            if build_if_missing:
                from . import build as _build
                _build.build()
            else:
                raise BemError(BEM_ERR_UNSUPPORTED,
                               f"{LIB_PATH} is missing: build it with `python -m capytaine_b200.build`")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
        return lib


def check(status: int):
    """Raise the exception matching a bem status code."""
    if status == BEM_OK:
        return
    msg = load().bem_last_error().decode(errors="replace")
    if status == BEM_ERR_NAN:
        raise GreenFunctionEvaluationError(status, msg or "Green function returned a NaN in the interaction matrix.")
    if status == BEM_ERR_SINGULAR:
        raise SingularMatrixError(status, msg or "singular matrix")
    if status == BEM_ERR_NOT_CONVERGED:
        raise NotConvergedError(status, msg or "iterative refinement did not converge")
    if status == BEM_ERR_OUT_OF_MEMORY:
        raise MemoryError(msg)
    raise BemError(status, msg)


def call(name, *args):
    check(getattr(load(), name)(*args))


def require_cuda(device=None):
    """Fail loudly when no CUDA device is usable: there is no CPU path."""
    import torch
    if not torch.cuda.is_available():
        raise BemError(BEM_ERR_UNSUPPORTED, "capytaine_b200 needs a CUDA device (sm_100a); none is available")
    load()
    return torch.device(device if device is not None else "cuda")


def current_stream_handle() -> int:
    """cudaStream_t of the current stream of the current device (torch's raw
    query, without the Stream object that torch.cuda.current_stream builds)."""
    import torch
    try:
        return torch._C._cuda_getCurrentRawStream(torch._C._cuda_getDevice())
    except AttributeError:  # a torch without the raw query
        return torch.cuda.current_stream().cuda_stream


def stream_ptr(stream=None):
    return ctypes.c_void_p(stream.cuda_stream if stream is not None else current_stream_handle())


class StreamShared:
    """Device tensors written on one CUDA stream and read from others (caches
    shared by the threads of a request server): a reader's stream waits for the
    writer's event, and the tensors are marked as in use by the reader's stream
    so that the caching allocator does not hand their memory out under it."""

    def __init__(self, *tensors):
        import torch
        self.tensors = tensors
        self.stream = torch.cuda.current_stream()
        self.event = torch.cuda.Event()
        self.event.record(self.stream)

    def acquire(self):
        import torch
        cur = torch.cuda.current_stream()
        if cur != self.stream:
            cur.wait_event(self.event)
            for t in self.tensors:
                t.record_stream(cur)
        return self


def upload(a, dtype, device):
    """Host array -> device tensor of `dtype` (see upload_many)."""
    return upload_many([(a, dtype)], device)[0]


def upload_many(arrays, device):
    """Host arrays -> device tensors [(array, torch dtype), ...] in one
    transfer on the current stream, without waiting for the stream's earlier
    work: the values are packed into one host buffer (256-byte aligned
    pieces) and copied asynchronously (the driver stages pageable memory
    before returning), into one device allocation that the returned tensors
    view.  Two CUDA calls per group of arrays: an allocation from the caching
    allocator and the copy."""
    import numpy as np
    import torch
    hosts = [np.ascontiguousarray(np.asarray(a), dtype=_NP_OF[dt]) for a, dt in arrays]
    if torch.device(device).type != "cuda":
        return [torch.from_numpy(h).to(device) for h in hosts]
    offs, total = [], 0
    for h in hosts:
        offs.append(total)
        total += -(-h.nbytes // 256) * 256
    buf = np.empty(max(total, 1), dtype=np.uint8)
    for h, o in zip(hosts, offs):
        buf[o:o + h.nbytes] = h.reshape(-1).view(np.uint8)
    dev = torch.from_numpy(buf).to(device, non_blocking=True)
    return [dev[o:o + h.nbytes].view(dt).view(h.shape) for h, o, (_, dt) in zip(hosts, offs, arrays)]


def _np_of():
    import numpy as np
    import torch
    return {torch.float64: np.float64, torch.float32: np.float32, torch.int32: np.int32, torch.int64: np.int64,
            torch.complex128: np.complex128, torch.complex64: np.complex64, torch.uint8: np.uint8}


class _NpOf(dict):
    def __missing__(self, key):
        self.update(_np_of())
        return dict.__getitem__(self, key)


_NP_OF = _NpOf()


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)
