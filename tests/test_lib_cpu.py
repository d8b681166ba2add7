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


def test_version_and_error_string(lib):
    assert lib.bem_version() >= 100
    assert isinstance(lib.bem_last_error(), bytes)


def test_invalid_arguments_are_rejected_without_gpu(lib):
    assert lib.bem_assemble(None, None) == _lib.BEM_ERR_INVALID_ARGUMENT
    assert b"null" in lib.bem_last_error()
    assert lib.bem_default_r_spacing(-1, 100.0, 1, None) == _lib.BEM_ERR_INVALID_ARGUMENT


_STRUCTS = {"bem_assembly_args": _lib.AssemblyArgs}


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
