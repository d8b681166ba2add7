"""Host-side dispatch of Delhommeau.assemble_into on the CPU: which C-ABI entry
point each call reaches, with which wavenumber, variant, output offset, depth,
method and Prony decomposition.  The library is replaced by a recorder and the
device by host memory; nothing is computed, so no GPU is needed."""
import ctypes

import numpy as np
import pytest

from capytaine_b200 import _lib
from capytaine_b200.meshes import mesh_sphere


class _Recorder:
    """Stands for the loaded library: every bem_* call is recorded with a copy
    of its assembly arguments and returns BEM_OK."""

    def __init__(self):
        self.calls = []

    def __getattr__(self, name):
        if not name.startswith("bem_"):
            raise AttributeError(name)

        def call(*args):
            rec = [name]
            for a in args:
                if isinstance(a, _lib.AssemblyArgs):
                    rec.append({f: getattr(a, f) for f, _ in a._fields_})
                elif hasattr(a, "_obj") and isinstance(a._obj, _lib.AssemblyArgs):  # byref
                    rec.append({f: getattr(a._obj, f) for f, _ in a._obj._fields_})
                else:
                    rec.append(a.value if isinstance(a, ctypes.c_void_p) else a)
            self.calls.append(rec)
            return _lib.BEM_OK
        return call


class _Shared:
    def __init__(self, *tensors):
        self.tensors = tensors

    def acquire(self):
        return self


@pytest.fixture
def host_gf(monkeypatch):
    import torch
    from capytaine_b200 import green_function as G
    rec = _Recorder()
    monkeypatch.setattr(_lib, "require_cuda", lambda device=None: torch.device("cpu"))
    monkeypatch.setattr(_lib, "load", lambda build_if_missing=False: rec)
    monkeypatch.setattr(_lib, "stream_ptr", lambda stream=None: ctypes.c_void_p(0))
    monkeypatch.setattr(_lib, "StreamShared", _Shared)

    def make(**kw):
        gf = G.Delhommeau(tabulation_cache_dir=None, **kw)
        r = torch.linspace(0.0, 1.0, 8, dtype=torch.float64)
        z = torch.linspace(-1.0, 0.0, 6, dtype=torch.float64)
        table = torch.zeros((8, 6, 5), dtype=torch.float64)
        gf._device_tabulation = lambda: (r, z, table, table.float())
        rec.calls.clear()  # the grid spacings of the constructor
        return gf
    return make, rec


def _buffers(n, nk):
    import torch
    S = torch.zeros((nk, n * n), dtype=torch.complex128)
    K = torch.zeros_like(S)
    return S, K


def test_finite_depth_sweep_launches_once_per_wavenumber(host_gf):
    make, rec = host_gf
    gf = make()
    mesh = mesh_sphere(resolution=(4, 6)).immersed_part()
    n = mesh.nb_faces
    ks = [0.3, 0.9, np.inf]
    S, K = _buffers(n, len(ks))
    gf.assemble_into(mesh, mesh, S[0], K[0], water_depth=4.0, wavenumber=ks[0], sweep=(ks, n * n, n * n))
    calls = [c for c in rec.calls if c[0] == "bem_assemble_finite_depth"]
    assert len(calls) == len(ks) and len(calls) == len(rec.calls)
    for i, (name, a, depth, method, prony_ptr, nexp, stream) in enumerate(calls):
        assert a["wavenumber"] == ks[i] and depth == 4.0 and method == 1
        assert a["S_dev"] == S.data_ptr() + 16 * i * n * n and a["K_dev"] == K.data_ptr() + 16 * i * n * n
        assert nexp == gf.find_best_exponential_decomposition(ks[i] * 4.0).shape[1]
        # low_freq for finite k, high_freq at k = infinity (delhommeau.py:466-490)
        want = _lib.BEM_GF_HIGH_FREQ if ks[i] == np.inf else _lib.BEM_GF_LOW_FREQ
        assert a["gf_singularities"] == want
        assert (a["nr"] > 0) == (0 < ks[i] < np.inf)  # the table only where there is a wave term
        assert a["early_dot_product"] == 1 and a["precision"] == _lib.BEM_PREC_FP64


def test_finite_depth_legacy_method_forces_low_freq(host_gf):
    make, rec = host_gf
    gf = make(finite_depth_method="legacy", gf_singularities="high_freq")
    mesh = mesh_sphere(resolution=(4, 6)).immersed_part()
    S, K = _buffers(mesh.nb_faces, 1)
    for k in (0.5, np.inf):
        gf.assemble_into(mesh, mesh, S[0], K[0], water_depth=3.0, wavenumber=k)
    assert [c[3] for c in rec.calls] == [0, 0]  # method 0: legacy
    assert [c[1]["gf_singularities"] for c in rec.calls] == [_lib.BEM_GF_LOW_FREQ] * 2


def test_finite_depth_output_formats(host_gf):
    """complex64 outputs and the three gradient planes reach the finite-depth
    entry point with their flags; mismatched dtypes and k h = 0 are refused on
    the host (no Prony decomposition at k h = 0, as capytaine)."""
    import torch
    make, rec = host_gf
    gf = make(gf_singularities="high_freq")
    mesh = mesh_sphere(resolution=(4, 6)).immersed_part()
    n = mesh.nb_faces
    S = torch.zeros((n, n), dtype=torch.complex64)
    gf.assemble_into(mesh, mesh, S, S.clone(), water_depth=3.0, wavenumber=1.0)
    K3 = torch.zeros((3, n, n), dtype=torch.complex128)
    S2 = torch.zeros((n, n), dtype=torch.complex128)
    gf.assemble_into(mesh, mesh, S2, K3, water_depth=3.0, wavenumber=1.0, early_dot_product=False,
                     k_plane_stride=n * n, adjoint_double_layer=False)
    (_, a64, *_), (_, a3, *_) = rec.calls
    assert a64["out_dtype"] == _lib.BEM_DTYPE_C64 and a64["early_dot_product"] == 1
    assert a3["out_dtype"] == _lib.BEM_DTYPE_C128 and a3["early_dot_product"] == 0
    assert a3["k_plane_stride"] == n * n and a3["adjoint_double_layer"] == 0
    assert a64["gf_singularities"] == a3["gf_singularities"] == _lib.BEM_GF_HIGH_FREQ
    rec.calls.clear()
    with pytest.raises(TypeError):
        gf.assemble_into(mesh, mesh, S, S2, water_depth=3.0, wavenumber=1.0)
    with pytest.raises(NotImplementedError):
        gf.assemble_into(mesh, mesh, S2, S2.clone(), water_depth=3.0, wavenumber=0.0)
    assert not rec.calls


def test_infinite_depth_sweep_with_limit_wavenumbers_takes_the_general_kernel(host_gf):
    make, rec = host_gf
    gf = make(gf_singularities="high_freq")
    mesh = mesh_sphere(resolution=(4, 6)).immersed_part()
    n = mesh.nb_faces
    ks = [0.0, 0.7, np.inf]
    S, K = _buffers(n, len(ks))
    gf.assemble_into(mesh, mesh, S[0], K[0], wavenumber=ks[0], sweep=(ks, n * n, n * n))
    assert [c[0] for c in rec.calls] == ["bem_assemble"] * 3
    args = [c[1] for c in rec.calls]
    assert [a["wavenumber"] for a in args] == ks
    # the variant of each wavenumber, not of the first one
    assert [a["gf_singularities"] for a in args] == [_lib.BEM_GF_LOW_FREQ, _lib.BEM_GF_HIGH_FREQ,
                                                     _lib.BEM_GF_HIGH_FREQ]
    assert all(a["nr"] > 0 for a in args)  # one finite wavenumber needs the table
    assert [a["S_dev"] - S.data_ptr() for a in args] == [16 * i * n * n for i in range(3)]


def test_infinite_depth_sweep_of_finite_wavenumbers_is_one_batched_launch(host_gf):
    make, rec = host_gf
    gf = make()
    mesh = mesh_sphere(resolution=(4, 6)).immersed_part()
    n = mesh.nb_faces
    ks = [0.2, 0.7, 1.9]
    S, K = _buffers(n, len(ks))
    gf.assemble_into(mesh, mesh, S[0], K[0], wavenumber=ks[0], sweep=(ks, n * n, n * n))
    names = [c[0] for c in rec.calls]
    assert names == ["bem_assemble_rankine_part", "bem_assemble_wave_symmetric_batched"]
    assert rec.calls[1][5] == len(ks)


def _doubles(ptr, n):
    return np.array((ctypes.c_double * n).from_address(ptr))


class _ReadingRecorder(_Recorder):
    """Also reads, at call time, the per-frequency arrays the right-hand-side and
    force entry points receive (host memory here)."""

    def __getattr__(self, name):
        call = super().__getattr__(name)

        def reading(*args):
            call(*args)
            rec = self.calls[-1]
            if name == "bem_build_rhs":     # (n, batch, omega, k, g, depth, ...)
                rec.append({"omega": _doubles(rec[3], rec[2]), "k": _doubles(rec[4], rec[2]), "depth": rec[6]})
            elif name == "bem_integrate_pressure":  # (n, batch, nrhs, ndof, phi, ldp, strideP, omega, ...)
                rec.append({"omega": _doubles(rec[8], rec[2])})
            elif name == "bem_froude_krylov":  # (n, batch, ndof, nhead, k, rho, g, depth, ...)
                rec.append({"k": _doubles(rec[5], rec[2]), "depth": rec[8]})
            return _lib.BEM_OK
        return reading


@pytest.fixture
def host_engine(host_gf, monkeypatch):
    from capytaine_b200.engine import B200Engine
    make, _ = host_gf
    rec = _ReadingRecorder()
    monkeypatch.setattr(_lib, "load", lambda build_if_missing=False: rec)
    return (lambda **kw: B200Engine(green_function=make(), **kw)), rec


def test_engine_limit_frequencies_use_omega_one_and_zero_wave(host_engine):
    """solve_frequencies at omega = 0, finite and infinity: the matrices at k = 0,
    omega^2/g and infinity; the right-hand sides and pressures with omega = 1 at
    the limits and the incident wave switched off there (k = 0); zero damping
    and NaN wave forces reported at the limits."""
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    new_engine, rec = host_engine
    body = FloatingBody(mesh_sphere(resolution=(4, 6)).immersed_part(), rigid_body_dofs(only=["Heave"]))
    res = new_engine().solve_frequencies(body, [0.0, 1.2, np.inf])
    k = 1.2 ** 2 / 9.81
    assembled = [c[1]["wavenumber"] for c in rec.calls if c[0] == "bem_assemble"] + \
        [c[1]["wavenumber"] for c in rec.calls if c[0] == "bem_assemble_wave_symmetric"]
    assert sorted(assembled) == [0.0, k, np.inf]
    rhs, = [c[-1] for c in rec.calls if c[0] == "bem_build_rhs"]
    np.testing.assert_array_equal(rhs["omega"], [1.0, 1.2, 1.0])
    np.testing.assert_array_equal(rhs["k"], [0.0, k, 0.0])
    assert rhs["depth"] == np.inf
    pres, = [c[-1] for c in rec.calls if c[0] == "bem_integrate_pressure"]
    np.testing.assert_array_equal(pres["omega"], [1.0, 1.2, 1.0])
    assert np.all(res.radiation_damping[[0, 2]] == 0.0)
    assert np.all(np.isnan(res.excitation[[0, 2]])) and not np.any(np.isnan(res.excitation[1]))


def test_engine_finite_depth_passes_the_depth_and_its_wavenumbers(host_engine):
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    from capytaine_b200.engine import wavenumbers
    new_engine, rec = host_engine
    body = FloatingBody(mesh_sphere(resolution=(4, 6)).immersed_part(), rigid_body_dofs(only=["Surge", "Heave"]))
    omegas = [0.8, 2.0, np.inf]
    new_engine(precision="mixed").solve_frequencies(body, omegas, water_depth=5.0)
    ks = wavenumbers(omegas, 5.0)
    fd = [c for c in rec.calls if c[0] == "bem_assemble_finite_depth"]
    assert [c[1]["wavenumber"] for c in fd] == list(ks) and all(c[2] == 5.0 for c in fd)
    assert all(c[1]["precision"] == _lib.BEM_PREC_FP64 for c in fd)  # float64 assembly in finite depth
    rhs, = [c[-1] for c in rec.calls if c[0] == "bem_build_rhs"]
    np.testing.assert_array_equal(rhs["k"], [ks[0], ks[1], 0.0])
    assert rhs["depth"] == 5.0
    fk, = [c[-1] for c in rec.calls if c[0] == "bem_froude_krylov"]
    np.testing.assert_array_equal(fk["k"], [ks[0], ks[1], 0.0])
    assert fk["depth"] == 5.0
    np.testing.assert_allclose(9.81 * ks[:2] * np.tanh(ks[:2] * 5.0), np.square(omegas[:2]), rtol=1e-14)


def test_symmetric_engine_first_block_column_in_finite_depth_and_at_limits(host_engine):
    """Meshes with symmetries: the first block column (all N points against the
    n_sub panels of the reference sub-mesh) assembled per wavenumber by the
    finite-depth kernel, or by the general kernel when a limit frequency is in
    the sweep, each into its own N x n_sub slot."""
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    from capytaine_b200.meshes import mesh_parallelepiped
    from capytaine_b200.symmetry import block_structure
    new_engine, rec = host_engine
    mesh = mesh_parallelepiped(size=(6, 4, 4), resolution=(4, 4, 4), reflection_symmetry=True).immersed_part()
    st = block_structure(mesh)
    N = mesh.nb_faces
    body = FloatingBody(mesh, rigid_body_dofs(only=["Heave"]))
    eng = new_engine()
    for depth, omegas, entry in ((5.0, [0.7, np.inf], "bem_assemble_finite_depth"),
                                 (np.inf, [0.0, 1.0], "bem_assemble")):
        rec.calls.clear()
        res = eng.solve_frequencies(body, omegas, water_depth=depth)
        assert res.stats["symmetry"] == "reflections"
        calls = [c for c in rec.calls if c[0] == entry]
        assert len(calls) == 2
        base = calls[0][1]["S_dev"]
        for i, c in enumerate(calls):
            a = c[1]
            assert a["n"] == N and a["nb_faces"] == st.n_sub and a["lds"] == N and a["ldk"] == N
            assert a["S_dev"] - base == 16 * i * N * st.n_sub
        assert not any(c[0] in ("bem_assemble_wave_cached", "bem_assemble_rankine_part") for c in rec.calls)
        rhs, = [c[-1] for c in rec.calls if c[0] == "bem_build_rhs"]
        assert rhs["depth"] == depth
        assert np.all(res.radiation_damping[np.isinf(omegas) | (np.asarray(omegas) == 0)] == 0.0)


def test_solve_bodies_in_finite_depth(host_engine):
    """solve_bodies batched across bodies of two padded sizes in finite depth:
    one finite-depth launch per (body, omega) into the padded slot of its
    group, and the depth on the right-hand sides of every batch."""
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    from capytaine_b200.engine import padded_size, wavenumbers
    new_engine, rec = host_engine
    bodies = [FloatingBody(mesh_sphere(resolution=res).immersed_part(), rigid_body_dofs(only=["Heave"]))
              for res in ((4, 6), (10, 16))]
    omegas = [0.9, 1.6]
    new_engine(max_batch=8).solve_bodies(bodies, omegas, water_depth=6.0)
    fd = [c[1] for c in rec.calls if c[0] == "bem_assemble_finite_depth"]
    assert len(fd) == len(bodies) * len(omegas)
    for body in bodies:
        n = body.mesh.nb_faces
        mine = [a for a in fd if a["nb_faces"] == n]
        assert [a["wavenumber"] for a in mine] == list(wavenumbers(omegas, 6.0))
        assert all(a["lds"] == padded_size(n) for a in mine)
    rhs = [c[-1] for c in rec.calls if c[0] == "bem_build_rhs"]
    assert rhs and all(r["depth"] == 6.0 for r in rhs)
