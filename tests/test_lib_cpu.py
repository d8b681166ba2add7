"""CPU-side checks of the C ABI: the library loads, exports every symbol the
header declares, the ctypes mirror of each struct matches the C layout, and
the host-side grid functions agree bit for bit with the oracle."""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from capytaine_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "capytaine_b200.h")


def _declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bem_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    return _lib.load(build_if_missing=True)


def test_library_exports_every_declared_symbol(lib):
    declared = _declared_functions()
    assert declared, "no bem_* functions found in the header"
    missing = [name for name in declared if not hasattr(lib, name)]
    assert not missing, f"symbols declared in the header but not exported: {missing}"
    # and the Python binding declares exactly what the header declares
    assert sorted(_lib.exported_symbols()) == declared


def _prototypes():
    """{name: (return type, [parameter types])} of the header's functions."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for ret, name, params in re.findall(r"([\w\s\*]+?)\s*\b(bem_\w+)\s*\(([^)]*)\)\s*;", text):
        params = " ".join(params.split())
        plist = [] if params in ("", "void") else [p.strip() for p in params.split(",")]
        out[name] = (" ".join(ret.split()), plist)
    return out


def _c_kind(decl):
    """Argument class of a C declaration: pointer, double, int64 or int32."""
    if "*" in decl:
        return "pointer"
    words = decl.replace("const ", "").split()
    base = " ".join(words[:-1]) if len(words) > 1 else words[0]
    return {"double": "double", "int64_t": "int64", "long long": "int64", "int": "int32",
            "int32_t": "int32"}[base]


def _ctypes_kind(t):
    if t in (ctypes.c_void_p, ctypes.c_char_p) or (isinstance(t, type) and issubclass(t, ctypes._Pointer)):
        return "pointer"
    if t is ctypes.c_double:
        return "double"
    if ctypes.sizeof(t) == 8:
        return "int64"
    assert ctypes.sizeof(t) == 4, t
    return "int32"


def test_binding_signatures_match_header():
    """Every ctypes signature has the header prototype's number and classes of
    arguments and its return class: a mismatch would pass arguments in the
    wrong registers without any error."""
    protos = _prototypes()
    assert sorted(protos) == _declared_functions()
    for name, (argtypes, restype) in _lib._SIGNATURES.items():
        ret, params = protos[name]
        assert [_c_kind(p) for p in params] == [_ctypes_kind(t) for t in argtypes], name
        ret_kind = "pointer" if "*" in ret else _c_kind(ret + " r")
        assert ret_kind == _ctypes_kind(restype), name


def test_version_and_error_string(lib):
    assert lib.bem_version() >= 100
    assert isinstance(lib.bem_last_error(), bytes)


def test_invalid_arguments_are_rejected_without_gpu(lib):
    assert lib.bem_assemble(None, None) == _lib.BEM_ERR_INVALID_ARGUMENT
    assert b"null" in lib.bem_last_error()
    assert lib.bem_default_r_spacing(-1, 100.0, 1, None) == _lib.BEM_ERR_INVALID_ARGUMENT


def test_symmetric_assembly_preconditions_checked_on_host(lib):
    """The mesh-with-itself fast path refuses, before any launch, inputs it
    does not cover (the host falls back to bem_assemble for those)."""
    fake = 4096  # never dereferenced: every call below fails its host checks
    a = _lib.AssemblyArgs(n=10, points_dev=fake, dot_normals_dev=fake, nb_faces=12, nb_vertices=4,
                          vertices_dev=fake, faces_dev=fake, centers_dev=fake, normals_dev=fake, areas_dev=fake,
                          radii_dev=fake, nb_quad_points=1, quad_points_dev=fake, quad_weights_dev=fake,
                          wavenumber=1.0, free_surface=0.0, gf_singularities=_lib.BEM_GF_LOW_FREQ,
                          adjoint_double_layer=1, early_dot_product=1, diagonal_term=1,
                          precision=_lib.BEM_PREC_FP64, out_dtype=_lib.BEM_DTYPE_C128, S_dev=fake, K_dev=fake,
                          lds=12, ldk=12)
    assert lib.bem_assemble_wave_symmetric(a, fake, 12, None) == _lib.BEM_ERR_INVALID_ARGUMENT  # n != nb_faces
    assert b"one mesh" in lib.bem_last_error()
    a.n = 12
    a.points_dev = 8192  # collocation points not the quadrature points
    assert lib.bem_assemble_wave_symmetric(a, fake, 12, None) == _lib.BEM_ERR_INVALID_ARGUMENT
    a.points_dev = fake
    a.wavenumber = float("inf")
    assert lib.bem_assemble_wave_symmetric(a, fake, 12, None) == _lib.BEM_ERR_UNSUPPORTED
    a.wavenumber = 1.0
    a.gf_singularities = _lib.BEM_GF_LOW_FREQ_WITH_RANKINE_PART
    assert lib.bem_assemble_rankine_part(a, fake, 12, None) == _lib.BEM_ERR_UNSUPPORTED
    assert lib.bem_assemble_wave_symmetric(a, fake, 12, None) == _lib.BEM_ERR_UNSUPPORTED
    a.gf_singularities = _lib.BEM_GF_LOW_FREQ
    a.free_surface = float("inf")
    assert lib.bem_assemble_rankine_part(a, fake, 12, None) == _lib.BEM_ERR_UNSUPPORTED
    a.free_surface = 0.0
    assert lib.bem_assemble_rankine_part(a, fake, 11, None) == _lib.BEM_ERR_INVALID_ARGUMENT  # ld < n
    assert lib.bem_assemble_rankine_part(a, None, 12, None) == _lib.BEM_ERR_INVALID_ARGUMENT


def test_finite_depth_assembly_preconditions_checked_on_host(lib):
    """bem_assemble_finite_depth refuses bad depths, Prony sizes, methods and
    output formats before any launch."""
    fake = 4096  # never dereferenced: every call below fails its host checks
    a = _lib.AssemblyArgs(n=12, points_dev=fake, dot_normals_dev=fake, nb_faces=12, nb_vertices=4,
                          vertices_dev=fake, faces_dev=fake, centers_dev=fake, normals_dev=fake, areas_dev=fake,
                          radii_dev=fake, nb_quad_points=1, quad_points_dev=fake, quad_weights_dev=fake,
                          tabulation_nb_integration_points=101, wavenumber=1.0, free_surface=0.0,
                          gf_singularities=_lib.BEM_GF_LOW_FREQ, adjoint_double_layer=1, early_dot_product=1,
                          diagonal_term=1, precision=_lib.BEM_PREC_FP64, out_dtype=_lib.BEM_DTYPE_C128, S_dev=fake,
                          K_dev=fake, lds=12, ldk=12)
    bad, unsupported = _lib.BEM_ERR_INVALID_ARGUMENT, _lib.BEM_ERR_UNSUPPORTED
    assert lib.bem_assemble_finite_depth(None, 10.0, 1, fake, 4, None) == bad
    for depth in (0.0, -1.0, float("inf"), float("nan")):
        assert lib.bem_assemble_finite_depth(a, depth, 1, fake, 4, None) == bad
    assert b"depth" in lib.bem_last_error()
    assert lib.bem_assemble_finite_depth(a, 10.0, 1, fake, 65, None) == bad  # more than 64 exponentials
    assert lib.bem_assemble_finite_depth(a, 10.0, 1, None, 4, None) == bad  # no decomposition
    assert lib.bem_assemble_finite_depth(a, 10.0, 2, fake, 4, None) == bad  # unknown method
    a.gf_singularities = 7
    assert lib.bem_assemble_finite_depth(a, 10.0, 1, fake, 4, None) == bad
    a.gf_singularities = _lib.BEM_GF_LOW_FREQ
    a.free_surface = float("inf")
    assert lib.bem_assemble_finite_depth(a, 10.0, 1, fake, 4, None) == bad
    a.free_surface = 0.0
    a.out_dtype = 7
    assert lib.bem_assemble_finite_depth(a, 10.0, 1, fake, 4, None) == bad
    a.out_dtype = _lib.BEM_DTYPE_C128
    a.precision = _lib.BEM_PREC_MIXED
    assert lib.bem_assemble_finite_depth(a, 10.0, 1, fake, 4, None) == unsupported
    a.precision = _lib.BEM_PREC_FP64
    a.early_dot_product = 0
    a.k_plane_stride = 12 * 12 - 1  # gradient planes overlap
    assert lib.bem_assemble_finite_depth(a, 10.0, 1, fake, 4, None) == bad
    a.early_dot_product = 1
    a.ldk = 11
    assert lib.bem_assemble_finite_depth(a, 10.0, 1, fake, 4, None) == bad


def test_cached_wave_and_block_combine_preconditions_checked_on_host(lib):
    """Entry points of the symmetric engines refuse bad shapes before any launch."""
    import ctypes
    fake = 4096
    a = _lib.AssemblyArgs(n=40, points_dev=8192, dot_normals_dev=fake, nb_faces=10, nb_vertices=4,
                          vertices_dev=fake, faces_dev=fake, centers_dev=fake, normals_dev=fake, areas_dev=fake,
                          radii_dev=fake, nb_quad_points=1, quad_points_dev=12288, quad_weights_dev=fake,
                          wavenumber=1.0, free_surface=0.0, gf_singularities=_lib.BEM_GF_LOW_FREQ,
                          adjoint_double_layer=1, early_dot_product=1, diagonal_term=1,
                          precision=_lib.BEM_PREC_FP64, out_dtype=_lib.BEM_DTYPE_C128, S_dev=fake, K_dev=fake,
                          lds=40, ldk=40)
    ks = (ctypes.c_double * 2)(0.5, 1.0)
    # the centres must be the quadrature points (one point per face)
    assert lib.bem_assemble_wave_cached(a, fake, 40, ks, 2, 400, 400, None) == _lib.BEM_ERR_INVALID_ARGUMENT
    a.quad_points_dev = fake
    assert lib.bem_assemble_wave_cached(a, fake, 39, ks, 2, 400, 400, None) == _lib.BEM_ERR_INVALID_ARGUMENT  # ld
    assert lib.bem_assemble_wave_cached(a, fake, 40, ks, 2, 399, 400, None) == _lib.BEM_ERR_INVALID_ARGUMENT
    assert lib.bem_assemble_wave_cached(a, None, 40, ks, 2, 400, 400, None) == _lib.BEM_ERR_INVALID_ARGUMENT
    bad = (ctypes.c_double * 1)(float("inf"))
    assert lib.bem_assemble_wave_cached(a, fake, 40, bad, 1, 0, 0, None) == _lib.BEM_ERR_UNSUPPORTED
    # block combine: sizes, pointers, grid limits
    assert lib.bem_block_combine(fake, 0, 1, 8, fake, 0, 1, 8, fake, None, 2, 2, 8, 4, 0, None) == _lib.BEM_OK
    assert lib.bem_block_combine(None, 0, 1, 8, fake, 0, 1, 8, fake, None, 2, 2, 8, 4, 1, None) \
        == _lib.BEM_ERR_INVALID_ARGUMENT
    assert lib.bem_block_combine(fake, 0, 1, 8, fake, 0, 1, 8, fake, None, 0, 2, 8, 4, 1, None) \
        == _lib.BEM_ERR_INVALID_ARGUMENT
    assert lib.bem_block_combine(fake, 0, 1, 7, fake, 0, 1, 8, fake, None, 2, 2, 8, 4, 1, None) \
        == _lib.BEM_ERR_INVALID_ARGUMENT  # column stride < rows
    assert lib.bem_block_combine(fake, 0, 1, 8, fake, 0, 1, 8, fake, None, 2, 2, 8, 70000, 1, None) \
        == _lib.BEM_ERR_INVALID_ARGUMENT
    assert b"65535" in lib.bem_last_error()


_STRUCTS = {"bem_assembly_args": _lib.AssemblyArgs, "bem_green_function_params": _lib.GreenFunctionParams,
            "bem_mesh_desc": _lib.MeshDesc, "bem_solve_stats": _lib.SolveStats}


@pytest.mark.parametrize("cname", sorted(_STRUCTS))
def test_struct_layout_matches_header(cname):
    pystruct = _STRUCTS[cname]
    fields = [f for f, _ in pystruct._fields_]
    prog = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void) {",
            f'  printf("%zu\\n", sizeof({cname}));']
    for f in fields:
        prog.append(f'  printf("%zu\\n", offsetof({cname}, {f}));')
    prog.append("  return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        open(src, "w").write("\n".join(prog))
        subprocess.run(["gcc", "-o", exe, src], check=True)
        out = [int(x) for x in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    assert out[0] == ctypes.sizeof(pystruct)
    for f, off in zip(fields, out[1:]):
        assert getattr(pystruct, f).offset == off, f


@pytest.mark.parametrize("nr,rmax,grid", [(328, 100.0, 0), (676, 100.0, 1), (600, 120.0, 1), (0, 100.0, 1)])
def test_r_spacing_matches_oracle(lib, oracle_mod, nr, rmax, grid):
    out = np.zeros(nr)
    assert lib.bem_default_r_spacing(nr, rmax, grid, out.ctypes.data_as(ctypes.c_void_p)) == 0
    np.testing.assert_array_equal(out, oracle_mod.default_r_spacing(nr, rmax, grid))


@pytest.mark.parametrize("nz,zmin,grid", [(46, -16.0, 0), (372, -251.0, 1), (124, -100.0, 1)])
def test_z_spacing_matches_oracle(lib, oracle_mod, nz, zmin, grid):
    out = np.zeros(nz)
    assert lib.bem_default_z_spacing(nz, zmin, grid, out.ctypes.data_as(ctypes.c_void_p)) == 0
    np.testing.assert_array_equal(out, oracle_mod.default_z_spacing(nz, zmin, grid))


def test_green_function_host_settings_without_gpu():
    from capytaine_b200.green_function import Delhommeau
    gf = Delhommeau(tabulation_cache_dir=None)
    assert gf.tabulated_r_range.shape == (676,) and gf.tabulated_z_range.shape == (372,)
    assert gf.exportable_settings["tabulation_grid_shape"] == "scaled_nemoh3"
    assert str(gf) == "Delhommeau()"
    assert "tabulation_nr=328" in str(Delhommeau(tabulation_nr=328, tabulation_cache_dir=None))


def test_no_cpu_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from capytaine_b200.green_function import Delhommeau
    from capytaine_b200.meshes import mesh_sphere
    gf = Delhommeau(tabulation_cache_dir=None)
    mesh = mesh_sphere(resolution=(4, 4)).immersed_part()
    with pytest.raises(_lib.BemError):
        gf.evaluate(mesh, mesh, wavenumber=1.0)


def test_linear_algebra_arguments_checked_on_host(lib):
    """Bad shapes, null pointers and misaligned workspaces are refused with
    BEM_ERR_INVALID_ARGUMENT before anything reaches the device (the status
    capytaine's callers map to a ValueError through _lib.check)."""
    import ctypes
    fake = 1 << 20          # 1 MiB-aligned, never dereferenced: each call fails its host checks
    bad = _lib.BEM_ERR_INVALID_ARGUMENT
    it, res = ctypes.c_int32(0), ctypes.c_double(0.0)
    # identity padding: npad < n, lda < npad
    assert lib.bem_zpad_identity(fake, 64, 4096, 1, 65, 64, None) == bad
    assert lib.bem_zpad_identity(fake, 32, 4096, 1, 16, 64, None) == bad
    assert lib.bem_zpad_identity(fake, 64, 4096, 1, 64, 64, None) == _lib.BEM_OK  # nothing to pad
    assert lib.bem_zgemm(-1, 4, 4, 1.0, fake, 4, 16, fake, 4, 16, 0.0, fake, 4, 16, 1, None) == bad
    assert lib.bem_zgemm(4, 4, 4, 1.0, None, 4, 16, fake, 4, 16, 0.0, fake, 4, 16, 1, None) == bad
    # mixed LU: npad a multiple of 128 at least n, 1024-byte aligned workspace
    assert lib.bem_clu_factor(fake, 100, 10000, 100, 100, 1, fake, fake, fake, fake, None) == bad
    assert lib.bem_clu_factor(fake, 200, 40000, 200, 128, 1, fake, fake, fake, fake, None) == bad
    assert lib.bem_clu_factor(fake, 100, 10000, 100, 128, 1, fake, fake, fake + 512, fake, None) == bad
    assert b"1024-byte" in lib.bem_last_error()
    assert lib.bem_clu_solve(fake, 100, 1, fake, fake, 128, 128, 1, fake, None) == bad
    # refinement: nrhs in [1, 16], ldb >= npad
    args = (fake, 100, 10000, 100, 128, 1, fake, fake, fake, fake, fake)
    assert lib.bem_refine_solve(*args, 128, 128 * 17, 17, 1e-10, 10, fake, fake, fake, ctypes.byref(it),
                                ctypes.byref(res), None) == bad
    assert lib.bem_refine_solve(*args, 100, 100, 1, 1e-10, 10, fake, fake, fake, ctypes.byref(it),
                                ctypes.byref(res), None) == bad
    # GMRES: 256-byte aligned workspace, sizes
    assert lib.bem_gmres_solve(fake, 100, 10000, 100, 128, 1, fake, fake, 128, 128, 1, 0.0, 1e-5, 20, 5, None,
                               fake + 16, fake, ctypes.byref(it), ctypes.byref(res), None) == bad
    assert lib.bem_gmres_solve(fake, 50, 10000, 100, 128, 1, fake, fake, 128, 128, 1, 0.0, 1e-5, 20, 5, None,
                               fake, fake, ctypes.byref(it), ctypes.byref(res), None) == bad  # lda < n
    assert lib.bem_gmres_workspace_bytes(100, 128, 1, 1, 20) > 0
    # one more restart vector adds at least one complex128 column of npad rows
    # per system to the Krylov basis V and one to the kept preconditioned
    # basis Z of the flexible form
    for nrhs, batch in ((1, 1), (7, 3)):
        grow = (lib.bem_gmres_workspace_bytes(1000, 1024, nrhs, batch, 21)
                - lib.bem_gmres_workspace_bytes(1000, 1024, nrhs, batch, 20))
        assert grow >= 2 * 16 * 1024 * nrhs * batch
    # right-hand sides and forces: ldb < n, null outputs
    inf = float("inf")
    assert lib.bem_build_rhs(100, 1, fake, fake, 9.81, inf, 1, fake, 1, fake, fake, fake, None, fake, 99, 100 * 2,
                             None) == bad
    for depth in (0.0, -5.0, float("nan")):  # water depth must be > 0 (+inf: infinite depth)
        assert lib.bem_build_rhs(100, 1, fake, fake, 9.81, depth, 1, fake, 1, fake, fake, fake, None, fake, 100,
                                 100 * 2, None) == bad
        assert lib.bem_froude_krylov(100, 1, 1, 1, fake, 1000.0, 9.81, depth, fake, fake, fake, fake, None) == bad
    assert lib.bem_integrate_pressure(100, 1, 2, 1, fake, 99, 200, fake, 1000.0, fake, fake, None) == bad
    assert lib.bem_integrate_pressure(100, 1, 2, 1, fake, 100, 200, fake, 1000.0, fake, None, None) == bad
    assert lib.bem_froude_krylov(100, 1, 1, 0, fake, 1000.0, 9.81, inf, fake, fake, fake, fake, None) == bad


def test_frequency_solve_api_arguments_checked_on_host(lib):
    """The handle-based entry points refuse bad arguments before touching a
    device, and bem_release only frees handles of this library."""
    bad = _lib.BEM_ERR_INVALID_ARGUMENT
    out = ctypes.c_void_p()
    assert lib.bem_release(None) == _lib.BEM_OK
    junk = (ctypes.c_uint32 * 16)()  # not a handle
    assert lib.bem_release(ctypes.addressof(junk)) == bad
    assert lib.bem_context_create(0, None, ctypes.byref(out)) == bad and out.value is None
    p = _lib.GreenFunctionParams(676, 100.0, 372, -251.0, 1001, _lib.BEM_GRID_SCALED_NEMOH3,
                                 _lib.BEM_GF_LOW_FREQ_WITH_RANKINE_PART)
    assert lib.bem_context_create(0, ctypes.byref(p), ctypes.byref(out)) == bad
    assert b"gf_singularities" in lib.bem_last_error()
    mesh = _lib.MeshDesc()
    w = (ctypes.c_double * 1)(1.0)
    stats = _lib.SolveStats()
    assert lib.bem_solve_frequency(None, ctypes.byref(mesh), 1, w, 1, w, 0, None, 1000.0, 9.81, 0, w, w, None,
                                   ctypes.byref(stats)) == bad
    assert lib.bem_solve_submit(None, ctypes.byref(mesh), 1, w, 1, w, 0, None, 1000.0, 9.81, 0, w, w, None,
                                ctypes.byref(out)) == bad
    assert lib.bem_lu_factor(None, None, 4, 4, 0, ctypes.byref(out)) == bad
    assert lib.bem_lu_solve(ctypes.addressof(junk), None, 4, 1, None, 4, None) == bad
    assert lib.bem_request_poll(ctypes.addressof(junk), 0, None) == bad


def test_c_program_links_against_the_library(lib):
    """A plain C99 program (not C++) includes the header, links the shared
    library and calls host-side entry points: what a non-Python host does
    (a cgo or JNI shim compiles the same way)."""
    src = r'''
#include <stdio.h>
#include "capytaine_b200.h"
int main(void) {
  double r[676], z[372];
  if (bem_version() < 100) return 1;
  if (bem_default_r_spacing(676, 100.0, BEM_GRID_SCALED_NEMOH3, r) != BEM_OK) return 2;
  if (bem_default_z_spacing(372, -251.0, BEM_GRID_SCALED_NEMOH3, z) != BEM_OK) return 3;
  if (bem_assemble(NULL, NULL) != BEM_ERR_INVALID_ARGUMENT) return 4;
  if (bem_zgemm_ts_static_capacity() <= 0) return 5;
  if (bem_release(NULL) != BEM_OK) return 6;
  if (bem_context_create(0, NULL, NULL) != BEM_ERR_INVALID_ARGUMENT) return 7;
  printf("%.17g %.17g %s\n", r[675], z[0], bem_last_error());
  return 0;
}
'''
    libdir = os.path.dirname(_lib.LIB_PATH)
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "host.c")
        exe = os.path.join(d, "host")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.dirname(HEADER), "-o", exe, c,
                        "-L", libdir, "-lcapytaine_b200", f"-Wl,-rpath,{libdir}"], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    r = np.zeros(676)
    lib.bem_default_r_spacing(676, 100.0, _lib.BEM_GRID_SCALED_NEMOH3, r.ctypes.data_as(ctypes.c_void_p))
    assert float(out[0]) == r[-1]
