#!/usr/bin/env python
"""Frequency-solves per second of the B200 BEM engines on the 6084-panel barge.

Workload (one frequency-solve): assemble S and K of the Delhommeau Green
function at k = omega^2/g, factor K, solve the 6 rigid-body radiation problems
and the diffraction problem (heading 0), potentials S @ sigma, pressure
integration -> added mass, damping, excitation.  Barge 80 x 20 m, draft 10 m,
6084 panels, omega in linspace(0.05, 3, 60), infinite depth, rho 1000, g 9.81.
A step is one batch of `--batch` frequencies taken in order from the sweep.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--engine fp64|mixed]
    python bench.py --impl reference     # CPU reference (oracle port) arm

Multi-GPU (torchrun, one process per GPU): frequencies are independent units,
each rank solves its own share with no data-path collective (weak scaling);
the only collectives are the timing barrier and the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "freq solves/sec at N=6000, refined-mixed vs FP64 LU at 1e-5 err; p50/p99 latency"
UNIT = "freq-solves/s"
OMEGAS = np.linspace(0.05, 3.0, 60)
RHO, G = 1000.0, 9.81


def barge_body():
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    from capytaine_b200.meshes import mesh_parallelepiped
    mesh = mesh_parallelepiped(size=(80, 20, 20), resolution=(104, 26, 26)).immersed_part()
    return FloatingBody(mesh, rigid_body_dofs(rotation_center=(0.0, 0.0, 0.0)), name="barge")


def workload_config(args, n):
    return {"workload": "barge 80x20x10m, 6 dofs + diffraction (heading 0), omega linspace(0.05,3,60)",
            "nb_panels": int(n), "frequencies_per_step": int(args.batch), "engine": args.engine,
            "solver": (f"float32 tcgen05 LU + {args.refinement} refinement to 1e-10" if args.engine == "mixed"
                       else {"gmres": "float64 GMRES (atol 1e-6, rtol 1e-5, restart 20)",
                             "lu_decomposition": "float64 DMMA LU"}[args.linear_solver]),
            "depth": "infinite", "l2": "inputs larger than L2 (K: 604 MB complex128 per frequency)",
            "parallelism": f"frequency shards x{args.world}",
            "rankine_part": "computed once per sweep of the 60 frequencies (cache cleared at each sweep start)",
            "calls": "one solve_frequencies call per sweep of the body (4 steps of 15 frequencies)"}


RIGID_DOFS = ("Surge", "Sway", "Heave", "Roll", "Pitch", "Yaw")


def seeded_bodies(seed, count, panels=(500, 8000), all_dofs=False):
    """Seeded floating bodies with panel counts uniform in `panels`: even
    indices ellipsoids (semi-axes U[1, 10] m, centred on the free surface),
    odd indices vertical cylinders (radius U[1, 8] m, draft U[2, 15] m), the
    resolution chosen for the panel target; 1 to 6 rigid dofs about the origin
    (all 6 with all_dofs)."""
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    from capytaine_b200.meshes import mesh_ellipsoid, mesh_vertical_cylinder
    rng = np.random.default_rng(seed)
    bodies = []
    for i in range(count):
        target = rng.uniform(*panels)
        if i % 2 == 0:
            axes = rng.uniform(1.0, 10.0, 3)
            a = max(4, int(round(np.sqrt(target))))
            mesh = mesh_ellipsoid(semi_axes=tuple(axes), resolution=(a, 2 * a)).immersed_part()
        else:
            r, d = rng.uniform(1.0, 8.0), rng.uniform(2.0, 15.0)
            h = np.sqrt((2 * np.pi * r * d + 2 * np.pi * r * r) / target)  # side + bottom rings of nr x nth
            nth = max(8, int(round(2 * np.pi * r / h)))
            nz = max(1, int(round(d / h)))
            nr = max(1, int(round(r / h)))
            mesh = mesh_vertical_cylinder(length=2 * d, radius=r, resolution=(nr, nth, 2 * nz)).immersed_part()
        ndof = int(rng.integers(1, 7))
        dofs = [RIGID_DOFS[j] for j in sorted(rng.permutation(6)[:ndof])]
        if all_dofs:
            dofs = list(RIGID_DOFS)
        bodies.append(FloatingBody(mesh, rigid_body_dofs(only=dofs), name=f"body{i}"))
    return bodies


def scaled_body(body, factors, name):
    """A distinct body: the mesh of `body` stretched by `factors` along x, y, z
    (same topology, new geometry), same dofs; its host-side geometry computed."""
    from capytaine_b200.bodies import FloatingBody
    m = body.mesh.scaled(factors)
    for prop in ("faces_centers", "faces_normals", "faces_areas", "faces_radiuses", "quadrature_points",
                 "content_hash"):
        getattr(m, prop)
    return FloatingBody(m, body.dofs, name=name)


def run_serving(engine, bodies, *, rate, n_requests, seed, slots, repeat_frac=0.2, batch_max=1):
    """Poisson arrivals (mean `rate` per second, seeded) of frequency-solve
    requests on the SolveServer: each new request a distinct body (a body of
    the pool stretched by U[0.8, 1.25] along each axis) at omega ~ U[0.1, 4];
    with probability repeat_frac a repeat of one of the 16 most recent (body,
    omega) pairs, whose resident factors are reused.  Latency = completion -
    arrival on the host clock."""
    from capytaine_b200.serving import SolveServer
    rng = np.random.default_rng(seed)
    plan, recent = [], []
    for i in range(n_requests):
        if recent and rng.random() < repeat_frac:
            plan.append(recent[int(rng.integers(len(recent)))])
        else:
            base = bodies[int(rng.integers(len(bodies)))]
            pair = (scaled_body(base, rng.uniform(0.8, 1.25, 3), f"request{i}"), float(rng.uniform(0.1, 4.0)))
            plan.append(pair)
            recent = (recent + [pair])[-16:]
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_requests))
    with SolveServer(engine, slots=slots, batch_max=batch_max) as srv:
        warm = [srv.submit(b, 1.0) for b in bodies[:2 * slots]]  # kernels loaded, every slot used
        for f in warm:
            f.result()
        srv.release_resident()
        srv.counters.update(evicted=0, reused=0, max_inflight_requests=0, max_reserved_bytes=0)
        futs = []
        t0 = time.perf_counter()
        for (b, w), ta in zip(plan, arrivals):
            delay = t0 + ta - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            futs.append(srv.submit(b, w))
        res, errors = [], []
        for f in futs:
            try:
                res.append(f.result())
            except Exception as exc:  # reported in the line, not fatal to the run
                errors.append(repr(exc)[:200])
        counters = dict(srv.counters)
        arena_peak = srv._arena.peak
    lat = np.array([r.latency for r in res]) * 1e3
    first = min(r.arrival for r in res)
    last = max(r.finished for r in res)
    escalated = sum(1 for r in res if r.stats.get("escalated_to_gmres"))
    panels = np.array([b.mesh_including_lid.nb_faces for b, _ in plan])
    return {"arrival_rate_per_s": rate, "requests": n_requests, "slots": slots,
            "completed": len(res), "failed": len(errors), "first_error": errors[0] if errors else None,
            "escalated_to_gmres": escalated, "batched_requests": counters.get("batched", 0),
            "batch_max": batch_max,
            "solves_per_s": len(res) / (last - first), "offered_s": float(arrivals[-1]),
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "max": float(lat.max())},
            "reused_factors": int(sum(r.reused_factors for r in res)),
            "panels": {"min": int(panels.min()), "mean": float(panels.mean()), "max": int(panels.max())},
            "max_inflight_requests": counters["max_inflight_requests"],
            "max_reserved_gb": counters["max_reserved_bytes"] / 1e9, "evicted": counters["evicted"],
            "arena_peak_gb": arena_peak / 1e9, "body_pool": len(bodies), "seed": seed,
            "workload": "Poisson arrivals; distinct seeded bodies (ellipsoids / vertical cylinders of 500-8000 "
                        "panels stretched per request), 1-6 dofs, omega ~ U[0.1, 4], 20% repeats of resident "
                        "(mesh, omega) pairs"}


def run_bodies(args):
    """--workload bodies: 64 seeded bodies (ellipsoids and vertical cylinders,
    300-3000 panels, seed 0), 6 dofs + diffraction heading 0, 30 omega in
    linspace(0.1, 4): the refined mixed engine batched across bodies
    (solve_bodies) against one solve_frequencies sweep per body."""
    import torch
    from capytaine_b200.engine import B200Engine
    from capytaine_b200.green_function import Delhommeau
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    bodies = seeded_bodies(0, args.bodies, panels=(300, 3000), all_dofs=True)
    omegas = np.linspace(0.1, 4.0, 30)
    gf = Delhommeau(tabulation_cache_dir=None)
    eng = B200Engine(green_function=gf, precision="mixed", max_batch=16)
    eng.solve_bodies(bodies[:2], omegas[:2], grouping="size")  # warm-up
    # the batch-size tuner times each size class once, before the timed runs
    t_tune = time.perf_counter()
    eng.solve_bodies(bodies, omegas[:1])
    t_tune = time.perf_counter() - t_tune

    def timed(fn):
        gf.clear_rankine_cache()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record()
        res = fn()
        e1.record()
        torch.cuda.synchronize()
        return res, e0.elapsed_time(e1), time.perf_counter() - t0

    timings, out = {}, {}
    # 30 frequencies per body: each body fills its own batches (solve_bodies runs one sweep per body);
    # 3 frequencies per body: bodies of the same padded size share batches
    for name, oms, fn in (
            ("bands_30_omega", omegas, lambda: eng.solve_bodies(bodies, omegas, sync_stats=args.bodies_stats)),
            ("per_body_sweeps_30_omega", omegas, lambda: eng.solve_bodies(bodies, omegas, grouping="size")),
            ("bands_3_omega", omegas[::10], lambda: eng.solve_bodies(bodies, omegas[::10])),
            ("grouped_3_omega", omegas[::10], lambda: eng.solve_bodies(bodies, omegas[::10], grouping="size")),
            ("one_sweep_per_body_3_omega", omegas[::10],
             lambda: [eng.solve_frequencies(b, omegas[::10]) for b in bodies])):
        res, ms, wall = timed(fn)
        out[name] = res
        timings[name] = {"value": len(bodies) * len(oms) / (ms * 1e-3), "unit": UNIT, "ms": ms, "wall_s": wall}
    diff = 0.0
    for name in ("grouped_3_omega", "bands_3_omega"):
        for a, b in zip(out[name], out["one_sweep_per_body_3_omega"]):
            for c in ("added_mass", "radiation_damping", "excitation"):
                x, y = getattr(a, c), getattr(b, c)
                diff = max(diff, float(np.abs(x - y).max() / np.abs(y).max()))
    panels = [b.mesh.nb_faces for b in bodies]
    st = out["bands_30_omega"][0].stats
    line = {"metric": "freq solves/sec, 64 bodies of 300-3000 panels x 30 omega",
            "value": timings["bands_30_omega"]["value"], "unit": UNIT, "n_gpus": 1, "higher_is_better": True,
            "dtype": "c128 (assembly, residuals) / f32-tf32 (LU)", "data": "synthetic",
            "config": {"workload": "64 seeded bodies (ellipsoids semi-axes U[1,10] m / vertical cylinders r U[1,8] m, "
                                   "draft U[2,15] m), 6 dofs + diffraction heading 0, omega linspace(0.1, 4, 30)",
                       "bodies": len(bodies), "panels": {"min": min(panels), "mean": float(np.mean(panels)),
                                                         "max": max(panels)},
                       "groups": st.get("groups"), "batches": st.get("batches"),
                       "stages_ms": {k: round(st[k], 2) for k in ("assembly_ms", "lu_ms", "solve_ms") if st.get(k)}},
            **timings,
            "bands_over_per_body_sweeps_30_omega": (timings["bands_30_omega"]["value"]
                                                    / timings["per_body_sweeps_30_omega"]["value"]),
            "grouped_over_per_body_3_omega": (timings["grouped_3_omega"]["value"]
                                              / timings["one_sweep_per_body_3_omega"]["value"]),
            "max_rel_diff_grouped_vs_per_body": diff, "tuner_s": t_tune,
            "tuner_choices": dict(eng.batch_tuner._choice), "tuner_timings_ms": eng.batch_tuner.timings}
    print(json.dumps(line), flush=True)
    return 0


def cylinder_array_body():
    """3 x 3 vertical cylinders (radius 5 m, draft 20 m, spacing 30 m), each
    with rigid-body dofs about its own axis at the free surface and an interior
    lid for the removal of irregular frequencies: about 20000 panels."""
    from capytaine_b200.bodies import FloatingBody, join_bodies, rigid_body_dofs
    from capytaine_b200.meshes import mesh_vertical_cylinder
    hull0 = mesh_vertical_cylinder(length=40.0, radius=5.0, resolution=(8, 52, 64)).immersed_part()
    lid0 = hull0.generate_lid()
    bodies = []
    for i in range(3):
        for j in range(3):
            x, y = 30.0 * (i - 1), 30.0 * (j - 1)
            bodies.append(FloatingBody(hull0.translated((x, y, 0.0)), rigid_body_dofs(rotation_center=(x, y, 0.0)),
                                       lid_mesh=lid0.translated((x, y, 0.0)), name=f"cyl{3 * i + j}"))
    return join_bodies(*bodies, name="array3x3")


def run_array(args):
    """--workload array: frequency-solves/s of the 3 x 3 cylinder array (54
    dofs + diffraction heading 0, omega in linspace(0.1, 2, 40)), the refined
    mixed engine against the float64 GMRES engine (SciPy's settings), both on
    the device; coefficients of the two compared."""
    import torch
    from capytaine_b200.engine import B200Engine
    from capytaine_b200.green_function import Delhommeau
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    body = cylinder_array_body()
    n = body.mesh_including_lid.nb_faces
    omegas = np.linspace(0.1, 2.0, 40)[::max(1, 40 // args.array_frequencies)][:args.array_frequencies]
    gf = Delhommeau(tabulation_cache_dir=None)
    out = {}
    results = {}
    for name, eng in (("mixed", B200Engine(green_function=gf, precision="mixed", max_batch=args.array_batch)),
                      ("gmres_fp64", B200Engine(green_function=gf, precision="fp64", linear_solver="gmres",
                                                max_batch=args.array_batch))):
        eng.solve_frequencies(body, omegas[:1])  # warm-up
        gf.clear_rankine_cache()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        res = eng.solve_frequencies(body, omegas)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        results[name] = res
        out[name] = {"value": len(omegas) / (ms * 1e-3), "unit": UNIT, "ms_per_frequency": ms / len(omegas),
                     "stats": {k: v for k, v in res.stats.items() if not k.endswith("_ms")}}
        del eng
        torch.cuda.empty_cache()
    # float64 LU (DMMA) reference at the lowest and a middle frequency
    ref_omegas = [float(omegas[0]), float(omegas[len(omegas) // 2])]
    ref = B200Engine(green_function=gf, precision="fp64", max_batch=1).solve_frequencies(body, ref_omegas)
    torch.cuda.empty_cache()
    idx = [0, len(omegas) // 2]

    def rel(a, b):
        floor = 1e-3 * np.abs(b).max(axis=tuple(range(1, b.ndim)), keepdims=True)
        return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor)))
    diff = {}
    for name in ("mixed", "gmres_fp64"):
        diff[name] = {c: rel(getattr(results[name], c)[idx], getattr(ref, c))
                      for c in ("added_mass", "radiation_damping", "excitation")}
    line = {"metric": "freq solves/sec at N=20000 (3x3 cylinder array with lids), refined-mixed vs complex128 GMRES",
            "value": out["mixed"]["value"], "unit": UNIT, "n_gpus": 1, "higher_is_better": True,
            "dtype": "c128 (assembly, residuals) / f32-tf32 (LU)", "data": "synthetic",
            "config": {"workload": "3x3 vertical cylinders r=5 m, draft 20 m, spacing 30 m, interior lids, "
                                   "9x6 dofs + diffraction heading 0, omega linspace(0.1, 2, 40)",
                       "nb_panels": int(n), "nb_lid_panels": int(body.lid_mesh.nb_faces),
                       "frequencies": len(omegas), "batch": args.array_batch},
            "mixed": out["mixed"], "gmres_fp64": out["gmres_fp64"],
            "mixed_over_gmres": out["mixed"]["value"] / out["gmres_fp64"]["value"],
            "max_rel_err_vs_fp64_lu": diff, "reference_omegas": ref_omegas,
            "note": "errors against the float64 LU engine at two frequencies; GMRES stops at SciPy's tolerance "
                    "(|r| <= max(1e-6, 1e-5 |b|)), the mixed engine refines to 1e-10"}
    print(json.dumps(line), flush=True)
    return 0


def run_symmetric(args):
    """--workload symmetric: the barge of the headline workload built with its
    two symmetry planes (mesh_parallelepiped(reflection_symmetry=True): 4
    systems of 1521 panels per frequency), omega linspace(0.05, 3, 60), one
    solve_frequencies call per sweep: the refined mixed and the float64 engines
    on the symmetric mesh against the refined mixed engine on the same faces
    without symmetry; coefficients against the oracle's block-circulant solve
    (capytaine's algorithm) at omega = 1.05, which is also timed on the host
    cores as the CPU baseline."""
    import torch
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    from capytaine_b200.engine import B200Engine
    from capytaine_b200.green_function import Delhommeau
    from capytaine_b200.meshes import mesh_parallelepiped
    from capytaine_b200.symmetry import block_structure
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    mesh = mesh_parallelepiped(size=(80, 20, 20), resolution=(104, 26, 26), reflection_symmetry=True).immersed_part()
    body = FloatingBody(mesh, rigid_body_dofs(), name="barge_sym")
    plain = FloatingBody(mesh.merged(), rigid_body_dofs(), name="barge")
    st = block_structure(mesh)
    gf = Delhommeau(tabulation_cache_dir=None)
    out, results = {}, {}
    for name, b, prec in (("mixed_symmetric", body, "mixed"), ("fp64_symmetric", body, "fp64"),
                          ("mixed_plain", plain, "mixed")):
        eng = B200Engine(green_function=gf, precision=prec, max_batch=args.batch)
        eng.solve_frequencies(b, OMEGAS[:args.batch])  # warm-up
        ms = []
        for _ in range(max(1, args.sweeps)):
            gf.clear_rankine_cache()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            res = eng.solve_frequencies(b, OMEGAS)
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        results[name] = res
        t = float(np.median(ms))
        out[name] = {"value": len(OMEGAS) / (t * 1e-3), "unit": UNIT, "ms_per_sweep": t, "sweeps": len(ms)}
        eng.release()
        del eng
        torch.cuda.empty_cache()
    # accuracy and the CPU baseline: the oracle's block-circulant solve at omega = 1.05
    from oracle import oracle as O
    cores = len(os.sched_getaffinity(0))
    gfo = oracle_gf()
    idx = int(np.argmin(np.abs(OMEGAS - 1.05)))
    w = float(OMEGAS[idx])
    t0 = time.perf_counter()
    ref = O.solve_frequency_symmetric(gfo, mesh.merged(), st.submesh, st.nb_images, True, O.rigid_body_dofs(), w,
                                      rho=RHO, g=G, wave_directions=(0.0,))
    cpu_s = time.perf_counter() - t0
    errs = {name: coefficient_error(results[name], idx, ref) for name in results}
    line = {"metric": "freq solves/sec at N=6084 with two symmetry planes (4 systems of 1521)",
            "value": out["mixed_symmetric"]["value"], "unit": UNIT, "n_gpus": 1, "higher_is_better": True,
            "dtype": "c128 (assembly, residuals) / f32-tf32 (LU)", "data": "synthetic",
            "config": {"workload": "barge 80x20x10m with xOz and yOz symmetry, 6 dofs + diffraction (heading 0), "
                                   "omega linspace(0.05,3,60)", "nb_panels": int(mesh.nb_faces),
                       "systems_per_frequency": st.nsys, "system_size": st.n_sys, "frequencies_per_batch": args.batch,
                       "calls": "one solve_frequencies call per sweep of 60 frequencies"},
            **out,
            "symmetric_over_plain_mixed": out["mixed_symmetric"]["value"] / out["mixed_plain"]["value"],
            "mixed_over_fp64_symmetric": out["mixed_symmetric"]["value"] / out["fp64_symmetric"]["value"],
            "max_rel_err_vs_oracle_block_circulant": errs, "accuracy_omega": w,
            "cpu_baseline": {"value": 1.0 / cpu_s, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"1 block-circulant frequency-solve (omega={w:.3f}) of the symmetric barge"}}
    print(json.dumps(line), flush=True)
    return 0


def run_finite_depth(args):
    """--workload finite_depth: the headline barge (6084 panels, 6 dofs +
    diffraction) in 40 m of water, omega linspace(0.1, 3, 60) (k h > 0.1 at the
    lowest frequency), one solve_frequencies call per sweep: the refined mixed
    and the float64 engines (finite-depth assembly in float64 in both, one
    launch per frequency with its own Prony decomposition), coefficients
    against the oracle's finite-depth solve at omega = 1.05, which is also
    timed on the host cores as the CPU baseline."""
    import torch
    from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
    from capytaine_b200.engine import B200Engine
    from capytaine_b200.green_function import Delhommeau
    from capytaine_b200.meshes import mesh_parallelepiped
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    depth = 40.0
    omegas = np.linspace(0.1, 3.0, 60)
    mesh = mesh_parallelepiped(size=(80, 20, 20), resolution=(104, 26, 26)).immersed_part()
    body = FloatingBody(mesh, rigid_body_dofs(), name="barge")
    gf = Delhommeau(tabulation_cache_dir=None)
    out, results = {}, {}
    for prec in ("mixed", "fp64"):
        eng = B200Engine(green_function=gf, precision=prec, max_batch=args.batch)
        eng.solve_frequencies(body, omegas[:args.batch], water_depth=depth)  # warm-up
        ms = []
        for _ in range(max(1, args.sweeps)):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            res = eng.solve_frequencies(body, omegas, water_depth=depth)
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        results[prec] = res
        t = float(np.median(ms))
        # stage times of one batch, untimed (the stages synchronise to be read)
        stages = eng.solve_frequencies(body, omegas[:args.batch], water_depth=depth, sync_stats=True).stats
        out[prec] = {"value": len(omegas) / (t * 1e-3), "unit": UNIT, "ms_per_sweep": t, "sweeps": len(ms),
                     "stage_ms_one_batch": {k: v for k, v in stages.items() if k.endswith("_ms")}}
        eng.release()
        del eng
        torch.cuda.empty_cache()
    from oracle import oracle as O
    cores = len(os.sched_getaffinity(0))
    gfo = oracle_gf()
    idx = int(np.argmin(np.abs(omegas - 1.05)))
    w = float(omegas[idx])
    t0 = time.perf_counter()
    ref = O.solve_frequency(gfo, mesh, O.rigid_body_dofs(), w, rho=RHO, g=G, wave_directions=(0.0,),
                            water_depth=depth)
    cpu_s = time.perf_counter() - t0
    errs = {name: coefficient_error(results[name], idx, ref) for name in results}
    line = {"metric": "freq solves/sec at N=6084 in 40 m of water (finite-depth Green function)",
            "value": out["mixed"]["value"], "unit": UNIT, "n_gpus": 1, "higher_is_better": True,
            "dtype": "c128 (assembly, residuals) / f32-tf32 (LU)", "data": "synthetic",
            "config": {"workload": "barge 80x20x10m in 40 m of water, 6 dofs + diffraction (heading 0), "
                                   "omega linspace(0.1,3,60)", "nb_panels": int(mesh.nb_faces),
                       "water_depth": depth, "frequencies_per_batch": args.batch,
                       "calls": "one solve_frequencies call per sweep of 60 frequencies"},
            **out, "mixed_over_fp64": out["mixed"]["value"] / out["fp64"]["value"],
            "max_rel_err_vs_oracle": errs, "accuracy_omega": w,
            "cpu_baseline": {"value": 1.0 / cpu_s, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"1 finite-depth frequency-solve (omega={w:.3f}) of the barge"}}
    print(json.dumps(line), flush=True)
    return 0


def run_profile_case(case):
    """Small cases of the LU kernels for ncu captures (a few GB on the device at
    most, inputs of the update above L2): the launches are those of the
    6084-panel barge's LU at smaller batch."""
    import ctypes
    import torch
    from capytaine_b200 import _lib
    lib = _lib.load()
    s = _lib.stream_ptr()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")

    def vp(t):
        return ctypes.c_void_p(t.data_ptr())

    def factor(n, batch):
        K = 0.05 * torch.randn((batch, n, n), dtype=torch.complex128, device="cuda")
        K.diagonal(dim1=1, dim2=2).add_(3.0)
        work = torch.empty(int(lib.bem_clu_workspace_bytes(n, batch)) + 1024, dtype=torch.uint8, device="cuda")
        wv = work[(-work.data_ptr()) % 1024:]
        piv = torch.zeros((batch, n), dtype=torch.int32, device="cuda")
        info = torch.zeros(batch, dtype=torch.int32, device="cuda")
        _lib.check(lib.bem_clu_factor(vp(K), n, n * n, n, n, batch, vp(piv), vp(info), vp(wv), vp(err), s))
        return K, wv, piv

    if case == "gemm":
        m, kp, batch = 4480, 512, 2
        Aop = torch.randn((batch, m, kp), device="cuda", dtype=torch.float32)
        Bop = torch.randn((batch, 2 * m, kp), device="cuda", dtype=torch.float32)
        Cr = torch.randn((batch, m, m), device="cuda", dtype=torch.float32)
        Ci = torch.randn((batch, m, m), device="cuda", dtype=torch.float32)
        for _ in range(3):
            _lib.check(lib.bem_cgemm_tf32_update(vp(Aop), m, 0, vp(Bop), 2 * m, 0, kp, vp(Cr), vp(Ci), m, m * m,
                                                 0, 0, m, m, batch, vp(err), s))
    elif case == "gj":
        for _ in range(2):
            factor(1024, 2)
    else:
        n, batch, nrhs = 4096, 4, 7
        K, wv, piv = factor(n, batch)
        B = torch.ones((batch, nrhs, n), dtype=torch.complex128, device="cuda")
        for _ in range(2):
            _lib.check(lib.bem_clu_solve(vp(wv), n, batch, vp(piv), vp(B), n, n * nrhs, nrhs, vp(err), s))
    torch.cuda.synchronize()
    if int(err.item()) != 0:
        raise RuntimeError(f"profile case {case}: kernel error flag set")
    print(json.dumps({"profile_case": case, "ok": True}))
    return 0


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.device_index = device_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device_index)], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if self.proc is None:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return out
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        out["samples"] = len(rows)
        out["sm_mhz"] = float(np.median(sm)) if sm else None
        out["sm_max_mhz"] = float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for name, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        out["reasons"] = sorted(reasons)
        out["power_w_max"] = max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit()) \
            if any(r[3].replace(".", "").isdigit() for r in rows) else None
        return out


def measured_peaks():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def tf32_tensor_peak_tflops():
    """cuBLAS TF32 GEMM 8192^3 best of 5 in this run (TF32 has no entry in the
    measured-peaks file)."""
    import torch
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    a = torch.randn(8192, 8192, dtype=torch.float32, device="cuda")
    b = torch.randn(8192, 8192, dtype=torch.float32, device="cuda")
    best = 0.0
    for _ in range(6):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2 * 8192 ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    return best


def fp64_tensor_peak_tflops():
    """cuBLAS DGEMM 8192^3 best of 5 in this run: FP64 has no entry in the
    measured-peaks file, so the float64 roofline denominator is measured here."""
    import torch
    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    b = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    best = 0.0
    for _ in range(6):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2 * 8192 ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    return best


# DRAM bytes per algorithmic flop of the trailing-update GEMM, from one ncu
# capture of a full trailing update of two block steps (m = 4480, depth 256, 2
# matrices: 640.0 MB read + written for 82.2 GFLOP); the traffic of the
# average launch is scaled from it by its flops.
CGEMM_DRAM_BYTES_PER_FLOP = 640.0e6 / (8 * 4480 ** 2 * 256 * 2)


def lu_update_flops(npad, block):
    """Real flops of the trailing updates of one blocked complex LU: sum over
    the block steps of 8 m^2 b for an m x m update of depth b."""
    return sum(8.0 * (npad - kk - block) ** 2 * block for kk in range(0, npad - block, block))


def isolated_update_rate(n, batch):
    """TF/s of the tcgen05 update kernel on the largest trailing update of this
    LU (two block steps of 128: depth 256, m = npad - 256, `batch` matrices),
    launched alone on the current stream after the timed region; C (two
    float32 planes per matrix) is larger than L2, so every launch reads and
    writes it from HBM.  Average of 5 launches after 2 warm-up ones."""
    import ctypes
    import torch
    from capytaine_b200 import _lib
    lib = _lib.load()
    npad = -(-n // 128) * 128
    m, kp = npad - 256, 512
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    g = torch.Generator(device="cuda").manual_seed(3)
    Aop = torch.randn((batch, m, kp), device="cuda", dtype=torch.float32, generator=g)
    Bop = torch.randn((batch, 2 * m, kp), device="cuda", dtype=torch.float32, generator=g)
    Cr = torch.zeros((batch, m, m), device="cuda", dtype=torch.float32)
    Ci = torch.zeros((batch, m, m), device="cuda", dtype=torch.float32)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = _lib.stream_ptr()

    def launch():
        _lib.check(lib.bem_cgemm_tf32_update(vp(Aop), m, 0, vp(Bop), 2 * m, 0, kp, vp(Cr), vp(Ci), m, m * m,
                                             0, 0, m, m, batch, vp(err), s))
    for _ in range(2):
        launch()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(5):
        launch()
    e1.record()
    torch.cuda.synchronize()
    if int(err.item()) != 0:
        raise RuntimeError("isolated update: kernel error flag set")
    ms = e0.elapsed_time(e1) / 5
    flops = 8.0 * m * m * 256 * batch
    del Aop, Bop, Cr, Ci
    return {"m": m, "depth": 256, "batch": batch, "ms_per_launch": ms, "achieved": flops / (ms * 1e-3) / 1e12,
            "unit": "TFLOP/s"}


def kernel_roofline(kernels, n, frequencies, engine, peaks, peak_src, frequencies_per_step=15):
    """Roofline of the kernel class with the largest device time in the timed
    region: algorithmic work per launch / average launch duration."""
    name, k = max(kernels.items(), key=lambda kv: kv[1]["ms_total"])
    avg_s = k["ms_total"] / k["launches"] * 1e-3
    total_ms = sum(v["ms_total"] for v in kernels.values())
    base = {"kernel": name, "launches": k["launches"], "avg_launch_ms": avg_s * 1e3,
            "share_of_timed_kernels": k["ms_total"] / total_ms, "traffic": None}
    if name == "cgemm_tf32_update_kernel":
        npad = -(-n // 128) * 128
        flops = lu_update_flops(npad, 128) * frequencies / k["launches"]
        peak = tf32_tensor_peak_tflops()
        ach = flops / avg_s / 1e12
        iso = isolated_update_rate(n, frequencies_per_step)
        iso["frac"] = iso["achieved"] / peak
        iso["note"] = ("the largest trailing update of the same LU launched alone; the timed-region average "
                       "also counts the launches of the lookahead chain (diagonal block, strips, panel product, "
                       "U'), which run beside the Gauss-Jordan inverse and the pack on other streams and whose "
                       "event-timed durations include the wait for SMs held by those kernels")
        return base | {"bound": "tensor", "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak,
                       "isolated_largest_update": iso,
                       "peak_source": "cuBLAS TF32 GEMM 8192^3 measured in this run (TF32 has no entry in "
                                      "MEASURED_PEAKS.json)",
                       "algorithmic": "8 m^2 k real flops per complex update of m x m by depth k (the LU "
                                      "applies two block steps of 128 per pass: k = 256 beyond the strips)",
                       "traffic": flops * CGEMM_DRAM_BYTES_PER_FLOP,
                       "traffic_note": "DRAM bytes per launch, ncu capture of an m=4480 depth-256 launch scaled by flops",
                       "hbm_bound_frac": (flops * CGEMM_DRAM_BYTES_PER_FLOP / avg_s / 1e9) / peaks["hbm_gbs"]}
    if name == "zgemm_dmma_kernel":
        npad = -(-n // 64) * 64
        flops = lu_update_flops(npad, 64) * frequencies / k["launches"]
        peak = fp64_tensor_peak_tflops()
        ach = flops / avg_s / 1e12
        return base | {"bound": "tensor", "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak,
                       "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (float64 has no entry in "
                                      "MEASURED_PEAKS.json)",
                       "algorithmic": "8 m^2 64 real flops per complex update of m x m by depth 64"}
    if name == "ctrsm_persistent_kernel":
        npad = -(-n // 128) * 128
        # one forward and one backward sweep read the float32 planes once (8 bytes per entry)
        bytes_ = 8.0 * npad * npad / 2
        ach = bytes_ / avg_s / 1e9
        return base | {"bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                       "frac": ach / peaks["hbm_gbs"], "peak_source": f"{peak_src} hbm_gbs",
                       "algorithmic": "8 bytes per entry of one triangle of the float32 factors per sweep"}
    if name == "assemble_kernel":
        bytes_ = 32.0 * n * n
        ach = bytes_ / avg_s / 1e9
        return base | {"bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                       "frac": ach / peaks["hbm_gbs"], "peak_source": f"{peak_src} hbm_gbs",
                       "algorithmic": "32 bytes (complex128 S and K entries) per panel pair"}
    # latency-bound kernels: report the bytes they move against HBM
    if name == "clu_gj_kernel":
        bytes_ = 2 * 8.0 * 128 * 128
    else:
        bytes_ = 0.0
    ach = bytes_ / avg_s / 1e9
    return base | {"bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                   "frac": ach / peaks["hbm_gbs"], "peak_source": f"{peak_src} hbm_gbs",
                   "algorithmic": "bytes read and written per launch"}


# ---------------------------------------------------------------------------
def cpu_reference_solve(body, omega, gf_oracle):
    """One frequency-solve with the oracle port (C++ OpenMP assembly + SciPy LU)."""
    from oracle import oracle as O
    odofs = {name: O.Dof("translation" if type(d).__name__ == "TranslationDof" else "rotation", d.direction,
                         getattr(d, "rotation_center", (0.0, 0.0, 0.0))) for name, d in body.dofs.items()}
    return O.solve_frequency(gf_oracle, body.mesh, odofs, omega, rho=RHO, g=G, wave_directions=(0.0,))


def oracle_gf():
    from oracle import oracle as O
    O.build_oracle()
    return O.OracleDelhommeau(nthreads=0)


def coefficient_error(res, idx, ref):
    """Max over A, B, F_exc of |c - c_ref| / max(|c_ref|, 1e-3 max|C_ref|)."""
    dofs = list(res.dofs)
    A = np.array([[ref["added_mass"][i][j] for j in dofs] for i in dofs])
    B = np.array([[ref["radiation_damping"][i][j] for j in dofs] for i in dofs])
    E = np.array([[ref["excitation"][0.0][j] for j in dofs]])
    errs = {}
    for name, got, r in (("added_mass", res.added_mass[idx], A), ("radiation_damping", res.radiation_damping[idx], B),
                         ("excitation", res.excitation[idx], E)):
        floor = 1e-3 * np.abs(r).max()
        errs[name] = float(np.max(np.abs(got - r) / np.maximum(np.abs(r), floor)))
    return errs


def run_reference(args):
    """--impl reference: the oracle port on the host cores, one frequency per step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cores = len(os.sched_getaffinity(0))
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    body = barge_body()
    gf = oracle_gf()
    times = []
    for step in range(args.warmup + args.steps):
        w = float(OMEGAS[step % len(OMEGAS)])
        t0 = time.perf_counter()
        cpu_reference_solve(body, w, gf)
        dt = time.perf_counter() - t0
        if step >= args.warmup:
            times.append(dt)
    total = sum(times)
    value = len(times) / total
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {k: v for k, v in workload_config(args, body.mesh.nb_faces).items()
                       if k not in ("rankine_part", "calls")} | {
                "engine": "oracle port (C++ OpenMP + SciPy LU)",
                "solver": "SciPy zgetrf/zgetrs (complex128 LU, one right-hand side at a time), "
                          "C++ OpenMP assembly", "frequencies_per_step": 1},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{len(times)} frequency-solves of the 6084-panel barge, one per step"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=15)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--engine", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--fp64-steps", type=int, default=4,
                    help="timed steps of the float64 engine for the refined-mixed vs float64 comparison (0: skip)")
    ap.add_argument("--batch", type=int, default=15, help="frequencies per step (60 = 4 steps of 15 per sweep)")
    ap.add_argument("--refinement", default="classical", choices=["classical", "gmres"],
                    help="refinement of the mixed engine: x += (LU)^-1 r, or GMRES preconditioned by the LU")
    ap.add_argument("--linear-solver", default="lu_decomposition", choices=["lu_decomposition", "gmres"],
                    help="solver of the float64 engine (--engine fp64)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serving-requests", type=int, default=1000,
                    help="requests of the serving run (Poisson arrivals); 0 skips it")
    ap.add_argument("--arrival-rate", type=float, default=200.0)
    ap.add_argument("--slots", type=int, default=8)
    ap.add_argument("--serving-batch", type=int, default=4,
                    help="requests of similar sizes factored together by the server (1: one per factorisation)")
    ap.add_argument("--workload", default="barge",
                    choices=["barge", "array", "bodies", "symmetric", "finite_depth"],
                    help="array: the 3x3 cylinder array with lids (20000 panels), mixed vs float64 GMRES; "
                         "bodies: 64 bodies of 300-3000 panels batched across bodies; "
                         "symmetric: the barge with its two symmetry planes; "
                         "finite_depth: the barge in 40 m of water")
    ap.add_argument("--sweeps", type=int, default=3,
                    help="timed sweeps per engine of --workload symmetric and finite_depth")
    ap.add_argument("--bodies", type=int, default=64)
    ap.add_argument("--bodies-stats", action="store_true", help="per-stage device times of the batched sweep")
    ap.add_argument("--array-frequencies", type=int, default=40)
    ap.add_argument("--array-batch", type=int, default=4)
    ap.add_argument("--accuracy-stride", type=int, default=5,
                    help="the accuracy leg checks every n-th frequency of the sweep against the oracle")
    ap.add_argument("--profile-case", choices=["gemm", "gj", "trsm"],
                    help="run one small case for an ncu capture and exit: gemm = three trailing updates of "
                         "depth 256 (m = 4480, 2 matrices); gj = two mixed LUs of 2 x 1024 (16 Gauss-Jordan "
                         "inverses); trsm = a 4 x 4096 mixed LU and two solves of 7 right-hand sides")
    args = ap.parse_args()
    if args.profile_case:
        return run_profile_case(args.profile_case)
    args.world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "array":
        return run_array(args)
    if args.workload == "bodies":
        return run_bodies(args)
    if args.workload == "symmetric":
        return run_symmetric(args)
    if args.workload == "finite_depth":
        return run_finite_depth(args)

    import torch
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    world = args.world
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    from capytaine_b200 import _lib
    from capytaine_b200.engine import B200Engine
    from capytaine_b200.green_function import Delhommeau

    body = barge_body()
    n = body.mesh_including_lid.nb_faces
    gf = Delhommeau(tabulation_cache_dir=None)
    if args.engine == "mixed":
        engine = B200Engine(green_function=gf, precision="mixed", max_batch=args.batch, refinement=args.refinement)
    else:
        engine = B200Engine(green_function=gf, precision="fp64", max_batch=args.batch,
                            linear_solver=args.linear_solver)
    # this rank's share of the sweep: frequencies rank, rank + world, ...
    from capytaine_b200.sharding import frequency_shard, max_over_ranks
    my_omegas = OMEGAS[frequency_shard(OMEGAS, rank, world)]
    nb = args.batch
    batches = [my_omegas[(s * nb + np.arange(nb)) % len(my_omegas)] for s in range(args.warmup + args.steps)]

    def sweep_start(s):
        return (s * nb) % len(my_omegas) < nb

    def calls(s0, s1):
        """Steps s0..s1-1 grouped into one solve_frequencies call per sweep of the body."""
        out = []
        for s in range(s0, s1):
            if not out or sweep_start(s):
                out.append([])
            out[-1].append(s)
        return [(grp, np.concatenate([batches[s] for s in grp])) for grp in out]

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- device-resident timing (value) ----------------------------------
    lib = _lib.load()
    for grp, oms in calls(0, args.warmup):
        engine.solve_frequencies(body, oms, batch=nb)
    torch.cuda.synchronize()
    sampler = ClockSampler(local_rank)
    sampler.start()
    barrier()
    torch.cuda.synchronize()
    launches0 = lib.bem_launch_count()
    _lib.check(lib.bem_kernel_timer_enable(1))
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    step_ms = []
    ev0.record()
    for grp, oms in calls(args.warmup, args.warmup + args.steps):
        e_a, e_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e_a.record()
        if sweep_start(grp[0]):
            gf.clear_rankine_cache()  # the Rankine part is computed once per sweep of the body
        res = engine.solve_frequencies(body, oms, batch=nb)
        e_b.record()
        step_ms.append((e_a, e_b, len(grp)))
    ev1.record()
    torch.cuda.synchronize()
    launches = lib.bem_launch_count() - launches0
    barrier()
    clocks = sampler.stop()
    t_ms = ev0.elapsed_time(ev1)
    lat = np.array([a.elapsed_time(b) / cnt for a, b, cnt in step_ms])  # per step, averaged within a call
    t_ms = max_over_ranks(t_ms)
    total_solves = args.steps * nb * world
    value = total_solves / (t_ms * 1e-3)

    # ---- per-stage times and the roofline of the dominant kernel ----------
    kernels = {}
    for c in range(10):
        tot, cnt = ctypes.c_double(0.0), ctypes.c_longlong(0)
        _lib.check(lib.bem_kernel_timer_read(c, ctypes.byref(tot), ctypes.byref(cnt)))
        if cnt.value:
            kernels[lib.bem_kernel_class_name(c).decode()] = {"class": c, "ms_total": tot.value,
                                                              "launches": int(cnt.value)}
    _lib.check(lib.bem_kernel_timer_enable(0))
    # stage times averaged over this rank's whole sweep (the stages' costs vary
    # with the frequency: the wave term's table stencils and the refinement's
    # iterations near the irregular frequencies)
    nsweep = -(-len(my_omegas) // nb)
    st = engine.solve_frequencies(body, my_omegas, batch=nb, sync_stats=True).stats
    st = {k: (v / nsweep if k.endswith("_ms") else v) for k, v in st.items()}
    st["batches_averaged"] = nsweep
    peaks, peak_src = measured_peaks()
    roofline = kernel_roofline(kernels, n, nb * args.steps, args.engine, peaks, peak_src, nb)

    # ---- end to end through the public API with host buffers --------------
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    h2d = d2h = 0
    for grp, oms in calls(args.warmup, args.warmup + args.steps):
        gf._mesh_cache.clear()  # mesh arrays come from host memory every call
        engine._body_cache.clear()
        if sweep_start(grp[0]):
            gf.clear_rankine_cache()
        r = engine.solve_frequencies(body, oms, batch=nb)
        m = body.mesh_including_lid
        h2d += 8 * (m.vertices.size + 3 * 3 * m.nb_faces + 2 * m.nb_faces + 4 * m.nb_faces) + 4 * m.faces.size
        h2d += 8 * (2 * len(body.dofs) * m.nb_faces) + 4 * m.nb_faces
        h2d += len(grp) * 8 * (2 * nb + 1)
        d2h += len(grp) * (16 * nb * (len(body.dofs) + 1) * len(body.dofs) * 2 + 4 * (nb + 2))
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e = {"value": total_solves / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d / args.steps),
           "d2h_bytes_per_step": int(d2h / args.steps)}

    # ---- the float64 engine on the same batches (refined-mixed vs FP64 LU) -
    fp64 = None
    if args.engine == "mixed" and args.fp64_steps > 0:
        eng64 = B200Engine(green_function=gf, precision="fp64", max_batch=args.batch)
        eng64.solve_frequencies(body, batches[0])
        barrier()
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        for grp, oms in calls(args.warmup, args.warmup + args.fp64_steps):
            eng64.solve_frequencies(body, oms, batch=nb)
        f1.record()
        torch.cuda.synchronize()
        f_ms = max_over_ranks(f0.elapsed_time(f1))
        fp64 = {"value": args.fp64_steps * nb * world / (f_ms * 1e-3), "unit": UNIT, "steps": args.fp64_steps,
                "ms_per_step": f_ms / args.fp64_steps}
        fp64["mixed_over_fp64"] = value / fp64["value"]
        del eng64

    # ---- serving: Poisson request stream, p50 / p99 latency ---------------
    serving = None
    if args.serving_requests > 0:
        engine.release()  # the server allocates its own arena
        torch.cuda.empty_cache()
        pool = seeded_bodies(1000 + rank, 32)
        serving = run_serving(B200Engine(green_function=gf, precision=args.engine, refinement=args.refinement)
                              if args.engine == "mixed" else B200Engine(green_function=gf, precision="fp64"),
                              pool, rate=args.arrival_rate, n_requests=args.serving_requests, seed=7 + rank,
                              slots=args.slots, batch_max=args.serving_batch)

    # ---- CPU baseline (oracle port on the host cores) and accuracy --------
    cpu = None
    accuracy = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # every 5th frequency of the timed sweep (12 of the 60): timed on the
        # host cores as the CPU baseline, and the reference of the accuracy of
        # both GPU engines at each of them
        cores = len(os.sched_getaffinity(0))
        gfo = oracle_gf()
        sample = [float(w) for w in OMEGAS[::args.accuracy_stride]]
        t0 = time.perf_counter()
        refs = [cpu_reference_solve(body, w, gfo) for w in sample]
        cpu_s = time.perf_counter() - t0
        cpu = {"value": len(sample) / cpu_s, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{len(sample)} frequency-solves of the 6084-panel barge (every "
                         f"{args.accuracy_stride}th omega of the sweep, {sample[0]:.2f} to {sample[-1]:.2f} rad/s)"}

        def sweep_errors(res):
            per = [max(coefficient_error(res, i, ref).values()) for i, ref in enumerate(refs)]
            worst = int(np.argmax(per))
            fam = coefficient_error(res, worst, refs[worst])
            return {"max_rel_err_vs_oracle": fam, "worst": per[worst], "worst_omega": sample[worst],
                    "per_omega": {f"{w:.2f}": float(f"{e:.3e}") for w, e in zip(sample, per)}}
        got = engine.solve_frequencies(body, sample, batch=nb)
        accuracy = {"omegas": len(sample), **sweep_errors(got), "refine_iters": got.stats.get("refine_iters"),
                    "refine_residual": got.stats.get("refine_residual"),
                    "escalated_to_gmres": got.stats.get("escalated_to_gmres", 0),
                    "note": "GPU-built tabulation vs oracle-built tabulation; error per omega = max over added "
                            "mass, damping and excitation of |c - c_ref| / max(|c_ref|, 1e-3 max |C_ref|)"}
        if args.engine == "mixed":
            g64 = B200Engine(green_function=gf, precision="fp64", max_batch=nb).solve_frequencies(body, sample)
            accuracy["fp64_engine"] = sweep_errors(g64)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "c128" if args.engine == "fp64" else "c128 (assembly, residuals) / f32-tf32 (LU)",
                "data": "synthetic", "config": workload_config(args, n), "roofline": roofline,
                "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
                "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                               "unit": f"ms per step of {nb} frequencies"},
                "stages_ms_per_step": {k: (round(v, 3) if isinstance(v, float) else v) for k, v in st.items()},
                "kernels_timed_region": {k: {"ms_total": round(v["ms_total"], 3), "launches": v["launches"]}
                                         for k, v in kernels.items()},
                "fp64_engine": fp64, "accuracy": accuracy, "serving": serving}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
