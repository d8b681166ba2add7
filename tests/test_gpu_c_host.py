"""The library-level entry points from a host that does not run Python.

A C99 program, compiled here with gcc against include/capytaine_b200.h and
linked to the shared library, runs the 800-panel hemisphere (heave radiation
+ diffraction at heading 0) through bem_context_create / bem_solve_frequency
(float64 and refined mixed) and through two concurrent bem_solve_submit
requests; the coefficients match the oracle's frequency-solve to 1e-6.  The LU
handle (bem_lu_factor / bem_lu_solve / bem_release) is checked through ctypes
against numpy's solve."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from capytaine_b200 import _lib

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

C_SOURCE = r'''
#include <stdio.h>
#include <stdlib.h>
#include "capytaine_b200.h"

static void* slurp(const char* dir, const char* name, size_t bytes) {
  char path[4096];
  snprintf(path, sizeof path, "%s/%s", dir, name);
  FILE* f = fopen(path, "rb");
  if (!f) { fprintf(stderr, "missing %s\n", path); exit(10); }
  void* p = malloc(bytes);
  if (fread(p, 1, bytes, f) != bytes) { fprintf(stderr, "short %s\n", path); exit(11); }
  fclose(f);
  return p;
}

static void spill(const char* dir, const char* name, const void* p, size_t bytes) {
  char path[4096];
  snprintf(path, sizeof path, "%s/%s", dir, name);
  FILE* f = fopen(path, "wb");
  fwrite(p, 1, bytes, f);
  fclose(f);
}

int main(int argc, char** argv) {
  const char* dir = argv[1];
  int nf = atoi(argv[2]), nv = atoi(argv[3]), nw = atoi(argv[4]);
  const int ndof = 1, nhead = 1;
  bem_mesh_desc mesh;
  mesh.nb_faces = nf;
  mesh.nb_vertices = nv;
  mesh.vertices = (const double*)slurp(dir, "vertices", sizeof(double) * 3 * nv);
  mesh.faces = (const int32_t*)slurp(dir, "faces", sizeof(int32_t) * 4 * nf);
  mesh.centers = (const double*)slurp(dir, "centers", sizeof(double) * 3 * nf);
  mesh.normals = (const double*)slurp(dir, "normals", sizeof(double) * 3 * nf);
  mesh.areas = (const double*)slurp(dir, "areas", sizeof(double) * nf);
  mesh.radii = (const double*)slurp(dir, "radii", sizeof(double) * nf);
  mesh.hull_mask = NULL;
  const double* dofn = (const double*)slurp(dir, "dofn", sizeof(double) * ndof * nf);
  const double* omegas = (const double*)slurp(dir, "omegas", sizeof(double) * nw);
  const double heading = 0.0;
  bem_green_function_params gp = {676, 100.0, 372, -251.0, 1001, BEM_GRID_SCALED_NEMOH3, BEM_GF_LOW_FREQ};
  bem_context* ctx = NULL;
  if (bem_context_create(0, &gp, &ctx) != BEM_OK) { fprintf(stderr, "%s\n", bem_last_error()); return 2; }
  double* am = malloc(sizeof(double) * 2 * nw * ndof * ndof);
  double* bd = malloc(sizeof(double) * 2 * nw * ndof * ndof);
  double* ex = malloc(sizeof(double) * 2 * nw * nhead * ndof * 2);
  const int precisions[2] = {BEM_PREC_FP64, BEM_PREC_MIXED};
  for (int p = 0; p < 2; ++p) {
    bem_solve_stats st;
    int s = bem_solve_frequency(ctx, &mesh, nw, omegas, ndof, dofn, nhead, &heading, 1000.0, 9.81, precisions[p],
                                am + p * nw, bd + p * nw, ex + p * nw * 2, &st);
    if (s != BEM_OK) { fprintf(stderr, "solve %d: %s\n", p, bem_last_error()); return 3; }
    printf("precision %d: iterations %d residual %.3e\n", p, st.iterations, st.residual);
  }
  spill(dir, "added_mass", am, sizeof(double) * 2 * nw);
  spill(dir, "damping", bd, sizeof(double) * 2 * nw);
  spill(dir, "excitation", ex, sizeof(double) * 2 * nw * 2);
  /* the same two solves as concurrent requests */
  double* am2 = malloc(sizeof(double) * 2 * nw);
  double* bd2 = malloc(sizeof(double) * 2 * nw);
  double* ex2 = malloc(sizeof(double) * 2 * nw * 2);
  bem_request* req[2];
  for (int p = 0; p < 2; ++p)
    if (bem_solve_submit(ctx, &mesh, nw, omegas, ndof, dofn, nhead, &heading, 1000.0, 9.81, precisions[p],
                         am2 + p * nw, bd2 + p * nw, ex2 + p * nw * 2, &req[p]) != BEM_OK) return 4;
  int pending = 2, polls = 0;
  while (pending) {
    pending = 0;
    for (int p = 0; p < 2; ++p) {
      int s = bem_request_poll(req[p], 0, NULL);
      if (s == BEM_PENDING) ++pending;
      else if (s != BEM_OK) { fprintf(stderr, "request %d: %s\n", p, bem_last_error()); return 5; }
    }
    ++polls;
  }
  for (int p = 0; p < 2; ++p) {
    if (bem_request_poll(req[p], 1, NULL) != BEM_OK) return 6;
    bem_release(req[p]);
  }
  spill(dir, "added_mass_async", am2, sizeof(double) * 2 * nw);
  spill(dir, "damping_async", bd2, sizeof(double) * 2 * nw);
  spill(dir, "excitation_async", ex2, sizeof(double) * 2 * nw * 2);
  if (bem_release(ctx) != BEM_OK) return 7;
  printf("ok %d polls\n", polls);
  return 0;
}
'''


def test_c99_host_runs_the_hemisphere_frequency_solves(oracle_mod, default_oracle_gf, tmp_path):
    from capytaine_b200.meshes import mesh_sphere
    mesh = mesh_sphere(radius=1.0, center=(0, 0, 0), resolution=(40, 40)).immersed_part()
    assert mesh.nb_faces == 800
    omegas = np.array([0.1, 1.3, 3.7])
    d = str(tmp_path)
    heave = mesh.faces_normals[:, 2].copy()  # heave: dof(x) . n = n_z
    arrays = {"vertices": mesh.vertices.astype(np.float64), "faces": mesh.faces.astype(np.int32),
              "centers": mesh.faces_centers, "normals": mesh.faces_normals, "areas": mesh.faces_areas,
              "radii": mesh.faces_radiuses, "dofn": heave, "omegas": omegas}
    for name, a in arrays.items():
        np.ascontiguousarray(a).tofile(os.path.join(d, name))
    libdir = os.path.dirname(_lib.LIB_PATH)
    exe = os.path.join(d, "host")
    src = os.path.join(d, "host.c")
    open(src, "w").write(C_SOURCE)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-o", exe, src,
                    "-L", libdir, "-lcapytaine_b200", f"-Wl,-rpath,{libdir}", "-lpthread"], check=True)
    run = subprocess.run([exe, d, str(mesh.nb_faces), str(len(mesh.vertices)), str(len(omegas))],
                         capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, run.stdout + run.stderr
    nw = len(omegas)
    am = np.fromfile(os.path.join(d, "added_mass")).reshape(2, nw)
    bd = np.fromfile(os.path.join(d, "damping")).reshape(2, nw)
    ex = np.fromfile(os.path.join(d, "excitation")).reshape(2, nw, 2)
    ex = ex[..., 0] + 1j * ex[..., 1]
    odofs = oracle_mod.rigid_body_dofs(only=["Heave"])
    ref = [oracle_mod.solve_frequency(default_oracle_gf, mesh, odofs, float(w)) for w in omegas]
    A = np.array([r["added_mass"]["Heave"]["Heave"] for r in ref])
    B = np.array([r["radiation_damping"]["Heave"]["Heave"] for r in ref])
    E = np.array([r["excitation"][0.0]["Heave"] for r in ref])
    for p, gate in ((0, 1e-6), (1, 1e-5)):
        for got, want in ((am[p], A), (bd[p], B), (ex[p], E)):
            floor = 1e-3 * np.abs(want).max()
            assert np.max(np.abs(got - want) / np.maximum(np.abs(want), floor)) < gate, (p, got, want)
    # the concurrent requests give the same numbers as the synchronous calls
    for name in ("added_mass", "damping", "excitation"):
        a = np.fromfile(os.path.join(d, name))
        b = np.fromfile(os.path.join(d, name + "_async"))
        assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max(), name


@pytest.mark.parametrize("precision,tol", [(_lib.BEM_PREC_FP64, 1e-12), (_lib.BEM_PREC_MIXED, 1e-9)])
def test_lu_handle_through_the_c_abi(precision, tol):
    import torch
    lib = _lib.load()
    rng = np.random.default_rng(3)
    n, nrhs = 700, 20  # two chunks of right-hand sides
    K = 10.0 * np.eye(n) + 0.3 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)
    b = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
    params = _lib.GreenFunctionParams(0, 100.0, 0, -251.0, 1001, _lib.BEM_GRID_SCALED_NEMOH3, _lib.BEM_GF_LOW_FREQ)
    ctx = ctypes.c_void_p()
    _lib.check(lib.bem_context_create(torch.cuda.current_device(), ctypes.byref(params), ctypes.byref(ctx)))
    ld = n + 5
    Kd = torch.zeros((n, ld), dtype=torch.complex128, device="cuda")  # column-major, leading dimension ld
    Kd[:, :n] = torch.as_tensor(K.T)
    Bd = torch.as_tensor(np.ascontiguousarray(b.T), device="cuda")
    Xd = torch.zeros_like(Bd)
    h = ctypes.c_void_p()
    _lib.check(lib.bem_lu_factor(ctx, ctypes.c_void_p(Kd.data_ptr()), ld, n, precision, ctypes.byref(h)))
    stats = _lib.SolveStats()
    _lib.check(lib.bem_lu_solve(h, ctypes.c_void_p(Bd.data_ptr()), n, nrhs, ctypes.c_void_p(Xd.data_ptr()), n,
                                ctypes.byref(stats)))
    x = Xd.cpu().numpy().T
    ref = np.linalg.solve(K, b)
    assert np.abs(x - ref).max() / np.abs(ref).max() < tol
    assert stats.iterations >= 1 and stats.residual <= 1e-10
    assert lib.bem_release(h) == _lib.BEM_OK
    assert lib.bem_release(ctx) == _lib.BEM_OK
