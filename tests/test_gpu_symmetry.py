"""Symmetric-mesh engines on the device: the block transform kernel against
NumPy, and B200Engine.solve_frequencies on meshes with one plane, two planes,
rotation and dihedral symmetry against the oracle's block-circulant solve
(capytaine's algorithm, bem/engines.py:178-247 and
tools/block_circulant_matrices.py) and against the engine's own dense solve of
the merged mesh."""
import ctypes

import numpy as np
import pytest

from capytaine_b200 import _lib
from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
from capytaine_b200.symmetry import block_structure

pytestmark = pytest.mark.gpu


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def test_block_combine_matches_numpy():
    """Matrix layout with an image map (dihedral macro-blocks), and the forward
    and inverse vector transforms, against einsum."""
    import torch
    lib = _lib.load()
    rng = np.random.default_rng(3)
    nf, mi, ns, q = 3, 5, 37, 2
    images = 2 * mi
    N = images * ns
    cols = rng.standard_normal((nf, ns, N)) + 1j * rng.standard_normal((nf, ns, N))  # [f][c][row]
    W = rng.standard_normal((mi, mi)) + 1j * rng.standard_normal((mi, mi))
    src = rng.integers(0, images, (mi, q, q)).astype(np.int32)
    nsys = q * ns
    ld_out = nsys + 5
    out = torch.zeros((nf * mi, nsys * ld_out), dtype=torch.complex128, device="cuda")
    cols_d = torch.as_tensor(cols, device="cuda")
    W_d = torch.as_tensor(W, device="cuda")
    for a in range(q):
        for b in range(q):
            s_d = torch.as_tensor(np.ascontiguousarray(src[:, a, b]), device="cuda")
            _lib.check(lib.bem_block_combine(_vp(cols_d), ns * N, ns, N,
                                             ctypes.c_void_p(out.data_ptr() + 16 * (a * ns + b * ns * ld_out)),
                                             mi * nsys * ld_out, nsys * ld_out, ld_out, _vp(W_d), _vp(s_d), mi, mi, ns,
                                             ns, nf, _lib.stream_ptr()))
    got = out.cpu().numpy().reshape(nf, mi, nsys, ld_out)[:, :, :, :nsys]  # [f][k][col][row]
    blocks = cols.reshape(nf, ns, images, ns).transpose(0, 2, 1, 3)      # [f][image][col][row]
    for a in range(q):
        for b in range(q):
            ref = np.einsum("ki,ficr->fkcr", W, blocks[:, src[:, a, b]])
            np.testing.assert_allclose(got[:, :, b * ns:(b + 1) * ns, a * ns:(a + 1) * ns], ref, rtol=0, atol=1e-12)
    # vectors: (nf, nrhs, N) -> (nf * mi, nrhs, ldv) and back with the inverse
    nrhs, ldv = 4, nsys + 3
    v = rng.standard_normal((nf, nrhs, mi * nsys)) + 1j * rng.standard_normal((nf, nrhs, mi * nsys))
    Winv = np.linalg.inv(W)
    v_d = torch.as_tensor(v, device="cuda")
    vh = torch.zeros((nf * mi, nrhs * ldv), dtype=torch.complex128, device="cuda")
    back = torch.zeros_like(v_d)
    _lib.check(lib.bem_block_combine(_vp(v_d), nrhs * mi * nsys, nsys, mi * nsys, _vp(vh), mi * nrhs * ldv,
                                     nrhs * ldv, ldv, _vp(W_d), None, mi, mi, nsys, nrhs, nf, _lib.stream_ptr()))
    Winv_d = torch.as_tensor(Winv, device="cuda")
    _lib.check(lib.bem_block_combine(_vp(vh), mi * nrhs * ldv, nrhs * ldv, ldv, _vp(back), nrhs * mi * nsys, nsys,
                                     mi * nsys, _vp(Winv_d), None, mi, mi, nsys, nrhs, nf, _lib.stream_ptr()))
    ref = np.einsum("ki,fcir->fkcr", W, v.reshape(nf, nrhs, mi, nsys))
    np.testing.assert_allclose(vh.cpu().numpy().reshape(nf, mi, nrhs, ldv)[..., :nsys], ref, rtol=0, atol=1e-12)
    np.testing.assert_allclose(back.cpu().numpy(), v, rtol=0, atol=1e-11)


def _oracle_ref(oracle_mod, gf, mesh, omegas, heads, lid=None):
    st = block_structure(mesh)
    full = mesh.merged()
    nested = st.kind in ("reflections", "dihedral")
    return [oracle_mod.solve_frequency_symmetric(gf, full, st.submesh, st.nb_images, nested,
                                                 oracle_mod.rigid_body_dofs(), w, wave_directions=heads,
                                                 hull_mask=lid) for w in omegas]


@pytest.mark.parametrize("kind", ["reflection", "reflections", "rotation", "dihedral"])
@pytest.mark.parametrize("precision,gate", [("fp64", 1e-6), ("mixed", 1e-5)])
def test_symmetric_engine_against_oracle(oracle_mod, default_oracle_gf, tmp_path, kind, precision, gate):
    from capytaine_b200.engine import B200Engine
    from test_gpu_mixed import _shared_table_gf
    from test_gpu_solve import coefficient_errors
    from test_symmetry_cpu import _symmetric_cases
    mesh = _symmetric_cases(exact=False)[kind]
    body = FloatingBody(mesh, rigid_body_dofs())
    omegas = np.linspace(0.4, 2.6, 4)
    heads = (0.0, 0.7)
    eng = B200Engine(green_function=_shared_table_gf(default_oracle_gf, tmp_path), precision=precision, max_batch=3)
    res = eng.solve_frequencies(body, omegas, wave_directions=heads)
    assert res.stats["symmetry"] == kind
    ref = _oracle_ref(oracle_mod, default_oracle_gf, mesh, omegas, heads)
    errs = coefficient_errors(res, ref, body.dofs)
    assert max(errs.values()) < gate, errs


@pytest.mark.parametrize("kind", ["reflection", "reflections", "rotation", "dihedral"])
def test_symmetric_engine_equals_dense_engine_on_exact_images(default_oracle_gf, tmp_path, kind):
    """For meshes whose faces and images have the same geometry the symmetric
    solve and the dense solve of the merged mesh are the same to rounding."""
    from capytaine_b200.engine import B200Engine
    from test_gpu_mixed import _shared_table_gf
    from test_symmetry_cpu import _symmetric_cases
    mesh = _symmetric_cases(exact=True)[kind]
    omegas = np.linspace(0.4, 2.6, 3)
    eng = B200Engine(green_function=_shared_table_gf(default_oracle_gf, tmp_path), max_batch=3)
    sym = eng.solve_frequencies(FloatingBody(mesh, rigid_body_dofs()), omegas)
    dense = eng.solve_frequencies(FloatingBody(mesh.merged(), rigid_body_dofs()), omegas)
    for name in ("added_mass", "radiation_damping", "excitation"):
        a, b = getattr(sym, name), getattr(dense, name)
        assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max(), name


def test_symmetric_engine_direct_method_and_lid(oracle_mod, default_oracle_gf, tmp_path):
    """Direct method on two planes; a lid of the same symmetry (indirect, mixed)."""
    from capytaine_b200.engine import B200Engine
    from test_gpu_mixed import _shared_table_gf
    from test_gpu_solve import coefficient_errors
    from test_symmetry_cpu import _symmetric_cases
    gf = _shared_table_gf(default_oracle_gf, tmp_path)
    mesh = _symmetric_cases(exact=True)["reflections"]
    omegas = np.array([0.8, 1.9])
    body = FloatingBody(mesh, rigid_body_dofs())
    direct = B200Engine(green_function=gf, method="direct").solve_frequencies(body, omegas)
    ref = [oracle_mod.solve_frequency(default_oracle_gf, mesh.merged(), oracle_mod.rigid_body_dofs(), w,
                                      method="direct") for w in omegas]
    errs = coefficient_errors(direct, ref, body.dofs)
    assert max(errs.values()) < 1e-6, errs
    cyl = _symmetric_cases(exact=False)["reflection"]
    lid = cyl.generate_lid()
    body = FloatingBody(cyl, rigid_body_dofs(), lid_mesh=lid)
    res = B200Engine(green_function=gf, precision="mixed").solve_frequencies(body, omegas)
    assert res.stats["symmetry"] == "reflection"
    ref = _oracle_ref(oracle_mod, default_oracle_gf, body.mesh_including_lid, omegas, (0.0,), lid=body.hull_mask)
    errs = coefficient_errors(res, ref, body.dofs)
    assert max(errs.values()) < 1e-5, errs


@pytest.mark.parametrize("kind", ["reflection", "reflections", "rotation", "dihedral"])
def test_matrix_engine_block_circulant_matrices(default_oracle_gf, tmp_path, kind):
    """build_matrices on a mesh with symmetries returns block-circulant device
    matrices (capytaine's _build_matrices_with_symmetries): dense form, product,
    LU solve and GMRES against the dense matrices of the merged mesh."""
    from capytaine_b200.engine import B200Engine, DeviceBlockCirculantMatrix
    from test_gpu_mixed import _shared_table_gf
    from test_symmetry_cpu import _symmetric_cases
    gf = _shared_table_gf(default_oracle_gf, tmp_path)
    mesh = _symmetric_cases(exact=True)[kind]
    eng = B200Engine(green_function=gf)
    S, K = eng.build_matrices(mesh, mesh, wavenumber=1.1)
    assert isinstance(S, DeviceBlockCirculantMatrix) and isinstance(K, DeviceBlockCirculantMatrix)
    assert K.shape == (mesh.nb_faces, mesh.nb_faces)
    full = mesh.merged()
    Sd, Kd = (np.asarray(m) for m in B200Engine(green_function=gf).build_matrices(full, full, wavenumber=1.1))
    for a, b in ((S, Sd), (K, Kd)):
        assert np.abs(np.asarray(a) - b).max() <= 1e-9 * np.abs(b).max()
    rng = np.random.default_rng(1)
    x = rng.standard_normal((mesh.nb_faces, 3)) + 1j * rng.standard_normal((mesh.nb_faces, 3))
    np.testing.assert_allclose(S @ x, Sd @ x, rtol=0, atol=1e-9 * np.abs(Sd @ x).max())
    ref = np.linalg.solve(Kd, x[:, 0])
    got = eng.linear_solver(K, x[:, 0])
    assert got.shape == x[:, 0].shape
    assert np.abs(got - ref).max() <= 1e-9 * np.abs(ref).max()
    got2 = eng.linear_solver(K, x)  # cached factors, several columns
    assert np.abs(got2 - np.linalg.solve(Kd, x)).max() <= 1e-9 * np.abs(ref).max()
    g = B200Engine(green_function=gf, linear_solver="gmres")
    _, Kg = g.build_matrices(mesh, mesh, wavenumber=1.1)
    xg = g.linear_solver(Kg, x[:, 0])
    assert np.linalg.norm(Kd @ xg - x[:, 0]) <= 1e-5 * np.linalg.norm(x[:, 0]) * 1.01
