"""The mesh-with-itself fast path of the assembly (Rankine part computed once
and reused across wavenumbers; wave term evaluated once per unordered pair of
faces and mirrored) against the general kernel that evaluates every entry on
its own.  Both are float64; they differ only in rounding order, so the bar is
1e-13 relative to the largest entry.  Parity of the fast path with the oracle
is covered by test_gpu_assembly.py, whose mesh-with-itself cases take it."""
import os

import numpy as np
import pytest

from capytaine_b200.meshes import Mesh, mesh_sphere, mesh_rectangle, mesh_parallelepiped

pytestmark = pytest.mark.gpu

RTOL = 1e-13


def _gf(default_oracle_gf, tmp_path, **kw):
    from capytaine_b200.green_function import Delhommeau
    gf = Delhommeau(tabulation_cache_dir=str(tmp_path), **kw)
    np.savez(os.path.join(str(tmp_path), gf._cache_filename), r_range=default_oracle_gf.tabulated_r_range,
             z_range=default_oracle_gf.tabulated_z_range, values=default_oracle_gf.tabulated_integrals)
    return gf


def _close(a, b, rtol=RTOL):
    err = np.abs(a - b).max() / np.abs(b).max()
    assert err <= rtol, err


def _lid_mesh():
    hull = mesh_sphere(radius=2.0, resolution=(10, 16)).immersed_part()
    lid = mesh_rectangle(size=(1.6, 1.6), resolution=(4, 4), center=(0, 0, 0), normal=(0, 0, 1))
    return Mesh.join_meshes(hull, lid)


MESHES = {
    "hemisphere_lid": _lid_mesh,  # free-surface panels: self term of Green_wave.f90:128-158
    "barge_300": lambda: mesh_parallelepiped(size=(10, 3, 3), resolution=(20, 6, 6)).immersed_part(),
}


@pytest.mark.parametrize("mesh_name", sorted(MESHES))
@pytest.mark.parametrize("sing", ["low_freq", "high_freq"])
@pytest.mark.parametrize("adjoint", [True, False])
def test_symmetric_path_matches_general_kernel(default_oracle_gf, tmp_path, mesh_name, sing, adjoint):
    mesh = MESHES[mesh_name]()
    fast = _gf(default_oracle_gf, tmp_path, gf_singularities=sing)
    general = _gf(default_oracle_gf, tmp_path, gf_singularities=sing)
    general.rankine_cache_bytes = 0
    general.symmetric_assembly = False
    # small, medium and large k (the last one reaches the asymptotic branch)
    for k in (0.05, 1.3, 40.0):
        S, K = fast.evaluate(mesh, mesh, wavenumber=k, adjoint_double_layer=adjoint)
        S0, K0 = general.evaluate(mesh, mesh, wavenumber=k, adjoint_double_layer=adjoint)
        _close(S, S0)
        _close(K, K0)
    assert len(fast._rankine_cache) == 1 and len(general._rankine_cache) == 0


def test_rankine_cache_keys_and_budget(default_oracle_gf, tmp_path):
    mesh = MESHES["barge_300"]()
    gf = _gf(default_oracle_gf, tmp_path)
    n = mesh.nb_faces
    gf.evaluate(mesh, mesh, wavenumber=1.0)
    gf.evaluate(mesh, mesh, wavenumber=2.0)
    assert len(gf._rankine_cache) == 1
    gf.evaluate(mesh, mesh, wavenumber=2.0, adjoint_double_layer=False)
    assert len(gf._rankine_cache) == 2
    gf.evaluate(mesh, mesh, wavenumber=0.5)  # a hit
    assert len(gf._rankine_cache) == 2
    gf.rankine_cache_bytes = 16 * n * n  # room for one: a new mesh evicts both
    small = mesh_sphere(resolution=(6, 8)).immersed_part()
    gf.evaluate(small, small, wavenumber=0.5)
    assert len(gf._rankine_cache) == 1
    gf.clear_rankine_cache()
    assert len(gf._rankine_cache) == 0


def test_padded_leading_dimensions(default_oracle_gf, tmp_path):
    """The engine's padded layout (lds, ldk > n) through the fast path."""
    import torch
    mesh = MESHES["barge_300"]()
    gf = _gf(default_oracle_gf, tmp_path)
    n = mesh.nb_faces
    ld = n + 37
    S = torch.full((n, ld), complex(7, 7), dtype=torch.complex128, device="cuda")
    K = torch.full((n, ld), complex(7, 7), dtype=torch.complex128, device="cuda")
    gf.assemble_into(mesh, mesh, S, K, wavenumber=0.8, lds=ld, ldk=ld)
    S_ref, K_ref = gf.evaluate(mesh, mesh, wavenumber=0.8)
    # column-major (n x n) with leading dimension ld: column J at S[J, :n]
    _close(S[:, :n].cpu().numpy().T, S_ref)
    _close(K[:, :n].cpu().numpy().T, K_ref)
    assert torch.all(S[:, n:] == complex(7, 7)) and torch.all(K[:, n:] == complex(7, 7))


@pytest.mark.parametrize("mesh_name", sorted(MESHES))
def test_batched_wavenumbers_equal_single_calls(default_oracle_gf, tmp_path, mesh_name):
    """bem_assemble_wave_symmetric_batched (one launch for several wavenumbers,
    outputs strided, leading dimension larger than n) writes exactly what one
    call per wavenumber writes; the general kernel's sweep loop agrees too."""
    import torch
    mesh = MESHES[mesh_name]()
    n = mesh.nb_faces
    ld = n + 5
    ks = [0.05, 0.7, 1.3, 40.0]
    out = {}
    for name, cache in (("fast", 4 << 30), ("general", 0)):
        gf = _gf(default_oracle_gf, tmp_path)
        gf.rankine_cache_bytes = cache
        gf.symmetric_assembly = cache > 0
        S = torch.full((len(ks), ld * n), float("nan"), dtype=torch.complex128, device="cuda")
        K = torch.full_like(S, float("nan"))
        gf.assemble_into(mesh, mesh, S[0], K[0], wavenumber=ks[0], lds=ld, ldk=ld, sweep=(ks, ld * n, ld * n))
        S1, K1 = torch.empty_like(S), torch.empty_like(K)
        for i, k in enumerate(ks):
            gf.assemble_into(mesh, mesh, S1[i], K1[i], wavenumber=k, lds=ld, ldk=ld)
        torch.cuda.synchronize()
        sv = S.reshape(len(ks), n, ld)[:, :, :n]
        kv = K.reshape(len(ks), n, ld)[:, :, :n]
        assert torch.equal(sv, S1.reshape(len(ks), n, ld)[:, :, :n])
        assert torch.equal(kv, K1.reshape(len(ks), n, ld)[:, :, :n])
        out[name] = (sv.cpu().numpy(), kv.cpu().numpy())
    _close(out["fast"][0], out["general"][0])
    _close(out["fast"][1], out["general"][1])


@pytest.mark.parametrize("sing", ["low_freq", "high_freq"])
@pytest.mark.parametrize("adjoint", [True, False])
def test_cached_rankine_for_points_against_a_mesh(default_oracle_gf, tmp_path, sing, adjoint):
    """bem_assemble_wave_cached (the first block column of a mesh with
    symmetries across a sweep: whole mesh against its sub-mesh) against the
    general kernel at each wavenumber, with lid panels on the free surface and
    the diagonal entries of the first block."""
    import torch
    from capytaine_b200.symmetric_meshes import ReflectionSymmetricMesh
    from capytaine_b200.symmetry import block_structure
    keep_y_positive = dict(origin=(0.0, 0.0, 0.0), normal=(0.0, -1.0, 0.0))
    half = Mesh.join_meshes(
        mesh_sphere(radius=2.0, resolution=(10, 16)).immersed_part().clipped(**keep_y_positive),
        mesh_rectangle(size=(1.6, 1.6), resolution=(4, 4), normal=(0, 0, 1)).clipped(**keep_y_positive))
    mesh = ReflectionSymmetricMesh(half, plane="xOz")
    full, sub = mesh.merged(), block_structure(mesh).submesh
    fast = _gf(default_oracle_gf, tmp_path, gf_singularities=sing)
    general = _gf(default_oracle_gf, tmp_path, gf_singularities=sing)
    general.rankine_cache_bytes = 0
    general.symmetric_assembly = False
    ks = [0.05, 1.3, 40.0]
    n, N = full.nb_faces, sub.nb_faces
    S = torch.empty((len(ks), N * n), dtype=torch.complex128, device="cuda")
    K = torch.empty_like(S)
    fast.assemble_into(full, sub, S[0], K[0], wavenumber=ks[0], adjoint_double_layer=adjoint, lds=n, ldk=n,
                       sweep=(ks, N * n, N * n))
    assert len(fast._rankine_cache) == 1
    for i, k in enumerate(ks):
        S0, K0 = general.evaluate(full, sub, wavenumber=k, adjoint_double_layer=adjoint)
        _close(S[i].view(N, n).T.cpu().numpy(), S0)
        _close(K[i].view(N, n).T.cpu().numpy(), K0)


@pytest.mark.parametrize("mesh_name", sorted(MESHES))
@pytest.mark.parametrize("sing", ["low_freq", "high_freq"])
@pytest.mark.parametrize("adjoint", [True, False])
def test_in_place_symmetric_assembly_without_reuse(default_oracle_gf, tmp_path, mesh_name, sing, adjoint):
    """bem_assemble_symmetric (Rankine part written into K, wave term added in
    place, one wavenumber, nothing cached; the request server's assembly)
    against the general kernel, with leading dimensions larger than n."""
    import torch
    mesh = MESHES[mesh_name]()
    n = mesh.nb_faces
    ld = n + 3
    inplace = _gf(default_oracle_gf, tmp_path, gf_singularities=sing)
    general = _gf(default_oracle_gf, tmp_path, gf_singularities=sing)
    general.symmetric_assembly = False
    for k in (0.05, 1.3, 40.0):
        out = []
        for gf in (inplace, general):
            S = torch.full((n * ld,), float("nan"), dtype=torch.complex128, device="cuda")
            K = torch.full_like(S, float("nan"))
            gf.assemble_into(mesh, mesh, S, K, wavenumber=k, adjoint_double_layer=adjoint, lds=ld, ldk=ld,
                             reuse_rankine=False)
            out.append((S.view(n, ld)[:, :n].cpu().numpy(), K.view(n, ld)[:, :n].cpu().numpy()))
        _close(out[0][0], out[1][0])
        _close(out[0][1], out[1][1])
    assert len(inplace._rankine_cache) == 0
