"""Post-processing at points away from the body through the engine, as
capytaine's BEMSolver does it (bem/solver.py:426-561): the sources of a solved
problem (engine.build_matrices + engine.linear_solver, bem/solver.py:188-196),
then the potential S(points, mesh) @ sigma (compute_potential, :426-456, with
engine.build_S_matrix, bem/engines.py:142-164), the velocity from the three
gradient planes of build_fullK_matrix (bem/engines.py:166-176,
_compute_potential_gradient / compute_velocity, :458-503), the pressure
i omega rho phi (compute_pressure, :505-536) and the free-surface elevation
-(1/g) (-i omega) phi at points on z = 0 (compute_free_surface_elevation,
:539-561).  Every step is compared with the oracle doing the same with its own
matrices and SciPy's LU, float64 throughout."""
import numpy as np
import pytest

from capytaine_b200.meshes import mesh_sphere

pytestmark = pytest.mark.gpu

RHO, G = 1000.0, 9.81


def _field_points():
    rng = np.random.default_rng(2)
    pts = []
    while len(pts) < 300:  # in the fluid: below the free surface, outside the sphere
        p = rng.uniform((-4.0, -4.0, -3.0), (4.0, 4.0, -0.05))
        if np.linalg.norm(p) > 1.3:
            pts.append(p)
    fs = []
    while len(fs) < 60:  # on the free surface, outside the waterline
        p = np.append(rng.uniform((-4.0, -4.0), (4.0, 4.0)), 0.0)
        if np.linalg.norm(p) > 1.3:
            fs.append(p)
    return np.array(pts), np.array(fs)


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(b).max())


@pytest.mark.parametrize("omega", [0.7, 2.4])
def test_potential_velocity_pressure_elevation_at_field_points(oracle_mod, default_oracle_gf, tmp_path, omega):
    import scipy.linalg as sl
    from capytaine_b200.engine import B200Engine
    from test_gpu_mixed import _shared_table_gf
    mesh = mesh_sphere(radius=1.0, resolution=(12, 24)).immersed_part()
    k = omega ** 2 / G
    gfp = dict(free_surface=0.0, water_depth=np.inf, wavenumber=k)
    pts, fs = _field_points()
    bc = -1j * omega * mesh.faces_normals[:, 2]  # heave radiation
    # engine: sources, then the field quantities
    eng = B200Engine(green_function=_shared_table_gf(default_oracle_gf, tmp_path), precision="fp64")
    S, K = eng.build_matrices(mesh, mesh, **gfp)
    sigma = eng.linear_solver(K, bc)
    phi = eng.build_S_matrix(pts, mesh, **gfp) @ sigma
    gradG = eng.build_fullK_matrix(pts, mesh, **gfp)
    assert gradG.shape == (3, len(pts), mesh.nb_faces)
    vel = np.stack([gradG[i] @ sigma for i in range(3)], axis=-1)
    pressure = 1j * omega * RHO * phi
    eta = -1.0 / G * (-1j * omega) * (eng.build_S_matrix(fs, mesh, **gfp) @ sigma)
    # oracle
    So, Ko = default_oracle_gf.evaluate(mesh, mesh, **gfp)
    sigma_o = sl.lu_solve(sl.lu_factor(Ko), bc)
    phi_o = default_oracle_gf.evaluate(pts, mesh, **gfp)[0] @ sigma_o
    Go = default_oracle_gf.evaluate(pts, mesh, early_dot_product=False, **gfp)[1]
    vel_o = np.stack([Go[i] @ sigma_o for i in range(3)], axis=-1)
    eta_o = -1.0 / G * (-1j * omega) * (default_oracle_gf.evaluate(fs, mesh, **gfp)[0] @ sigma_o)
    assert _rel(sigma, sigma_o) < 1e-10
    assert _rel(phi, phi_o) < 1e-9
    assert _rel(vel, vel_o) < 1e-9
    assert _rel(pressure, 1j * omega * RHO * phi_o) < 1e-9
    assert _rel(eta, eta_o) < 1e-9
    # the potential on the body from the field-point path equals S @ sigma
    on_body = eng.build_S_matrix(mesh.faces_centers, mesh, **gfp) @ sigma
    assert _rel(on_body, S @ sigma) < 1e-12
