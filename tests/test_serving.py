"""Request server: admission by device-memory footprint, residency and reuse of
factors, and results that are the same alone and in a mix of concurrent
requests.

The scheduler tests run on the host with a stand-in engine (no GPU); the
results tests run the real engine on the GPU."""
import threading
import time

import numpy as np
import pytest

from capytaine_b200.bodies import FloatingBody, rigid_body_dofs
from capytaine_b200.meshes import mesh_parallelepiped, mesh_sphere, mesh_vertical_cylinder


class _StandInEngine:
    """Engine stages that only record calls: F depends on the mesh and omega."""
    precision = "mixed"
    device = "cpu"
    gmres_restart = 20

    def __init__(self, delay=0.0):
        self.delay = delay
        self.lock = threading.Lock()
        self.calls = []
        self.running = 0
        self.max_running = 0

    def _enter(self, what):
        with self.lock:
            self.calls.append(what)
            self.running += 1
            self.max_running = max(self.max_running, self.running)
        time.sleep(self.delay)
        with self.lock:
            self.running -= 1

    def assemble_stage(self, f, mesh, ks, nan_flag=None, reuse_rankine=True, first=0, lds=None):
        self._enter(("assemble", mesh.nb_faces, float(ks[0])))

    def pad_stage(self, f, first, m, n_body):
        self.calls.append(("pad", first, n_body))

    def factor_stage(self, f, nb, err, active=None):
        self._enter(("factor", f.n) if active is None else ("factor_grouped", f.n, tuple(active)))

    def _solve_segments(self, f, r, segments, om, heads, rho=1000.0, g=9.81, stats=None):
        self._enter(("solve_batch", f.n, len(segments)))
        out = []
        for body, j0, m in segments:
            n = body.mesh_including_lid.nb_faces
            ndof, nhead = len(body.dofs), len(heads)
            out.append((np.full((m, ndof + nhead, ndof), n + 1j * om[j0]), np.full((m, nhead, ndof), 2.0 * n)))
        return out

    def solve_stage(self, f, r, body, om, heads, rho=1000.0, g=9.81, stats=None, events=None):
        self._enter(("solve", f.n, float(om[0])))
        ndof, nhead = len(body.dofs), len(heads)
        F = np.full((1, ndof + nhead, ndof), f.n + 1j * om[0])
        FK = np.full((1, nhead, ndof), 2.0 * f.n)
        return F, FK


def _body(n_side, dofs=("Heave",)):
    mesh = mesh_parallelepiped(size=(4, 4, 4), resolution=(n_side, n_side, n_side)).immersed_part()
    return FloatingBody(mesh, rigid_body_dofs(only=list(dofs)))


def _server(engine, **kw):
    from capytaine_b200.serving import SolveServer
    return SolveServer(engine, **kw)


def test_device_arena_first_fit_and_coalescing():
    import torch
    from capytaine_b200.serving import ArenaFull, DeviceArena
    ar = DeviceArena(1 << 20, "cpu", granule=1 << 12)
    a1, r1 = ar.allocator()
    a2, r2 = ar.allocator()
    x = a1((100,), torch.complex128, True)
    y = a2((1000,), torch.float32)
    z = a1((10, 10), torch.int32, True)
    assert x.dtype == torch.complex128 and float(x.abs().sum()) == 0.0 and z.shape == (10, 10)
    base = ar.buf.data_ptr()
    assert (x.data_ptr() - base) % 4096 == 0 and (y.data_ptr() - base) % 4096 == 0
    assert ar.used == 3 * 4096
    with pytest.raises(ArenaFull):
        a2(((1 << 20),), torch.uint8)
    r1()
    assert ar.used == 4096 and ar.largest_free == (1 << 20) - 2 * 4096
    r2()
    assert ar.used == 0 and ar.largest_free == 1 << 20 and ar.peak == 3 * 4096


def test_scheduler_reuses_resident_factors_and_counts():
    eng = _StandInEngine()
    with _server(eng, slots=2, memory_budget=1 << 28) as srv:
        b = _body(4)
        r1 = srv.solve(b, 1.0, timeout=60)
        r2 = srv.solve(b, 1.0, timeout=60)
        r3 = srv.solve(b, 2.0, timeout=60)
        assert not r1.reused_factors and r2.reused_factors and not r3.reused_factors
        assert np.array_equal(r1.added_mass, r2.added_mass)
        assert srv.counters["completed"] == 3 and srv.counters["reused"] == 1
        kinds = [c[0] for c in eng.calls]
        assert kinds.count("assemble") == 2 and kinds.count("factor") == 2 and kinds.count("solve") == 3


def test_scheduler_keeps_the_memory_budget_and_evicts():
    from capytaine_b200.engine import _Factors, _Rhs
    eng = _StandInEngine(delay=0.01)
    bodies = [_body(k) for k in (6, 8, 10, 12)]
    n_max = max(b.mesh.nb_faces for b in bodies)
    npad = -(-n_max // 128) * 128
    one = _Factors.estimate_bytes(n_max, 1, "mixed") + _Rhs.estimate_bytes(n_max, npad, 1, 2)
    budget = int(2.5 * one)
    with _server(eng, slots=4, memory_budget=budget) as srv:
        futs = [srv.submit(b, w) for w in (0.5, 1.0, 1.5) for b in bodies]
        res = [f.result(timeout=60) for f in futs]
        assert len(res) == 12
        assert srv.counters["max_reserved_bytes"] <= budget
        assert srv.counters["evicted"] > 0
        assert srv.resident_bytes <= budget


def test_scheduler_overlaps_requests_in_slots():
    eng = _StandInEngine(delay=0.02)
    with _server(eng, slots=4, memory_budget=1 << 28) as srv:
        futs = [srv.submit(_body(4 + (i % 3)), 0.3 + 0.1 * i) for i in range(8)]
        for f in futs:
            f.result(timeout=60)
    assert eng.max_running >= 2
    assert srv.counters["max_inflight_requests"] >= 2


def test_scheduler_rejects_a_request_above_the_budget():
    eng = _StandInEngine()
    with _server(eng, slots=1, memory_budget=1000) as srv:
        with pytest.raises(MemoryError):
            srv.solve(_body(6), 1.0, timeout=60)
        assert srv.counters["failed"] == 1


def test_a_failing_slot_fails_the_queue_instead_of_hanging():
    from capytaine_b200.serving import SolveServer

    class Broken(SolveServer):
        def _slot_stream(self):
            raise ValueError("no device")
    with pytest.raises(RuntimeError, match="slot failed"):
        srv = Broken(_StandInEngine(), slots=1, memory_budget=1 << 28)
        try:
            srv.submit(_body(4), 1.0).result(timeout=30)
        finally:
            srv.shutdown(wait=True)


def test_scheduler_admits_in_arrival_order():
    eng = _StandInEngine(delay=0.005)
    with _server(eng, slots=1, memory_budget=1 << 28) as srv:
        bodies = [_body(4 + i) for i in range(5)]
        futs = [srv.submit(b, 1.0) for b in bodies]
        order = [f.result(timeout=60).request_id for f in futs]
        admitted = [f.result().admitted for f in futs]
    assert order == sorted(order) and admitted == sorted(admitted)


def test_scheduler_batches_waiting_requests_of_similar_sizes():
    """With batch_max > 1, a slot that admits a new request takes waiting new
    requests whose padded sizes lie within the band into one grouped
    factorisation; requests of other sizes, repeats of resident factors and
    other headings stay out; every request gets its own result."""
    eng = _StandInEngine(delay=0.2)
    same = [_body(10), _body(9), _body(10, dofs=("Heave", "Surge"))]  # 300, 297, 300 panels
    far = _body(24)
    for b in same + [far]:  # geometry and hashes ready, so that the submissions below are quick
        _ = b.mesh_including_lid.content_hash
    with _server(eng, slots=1, memory_budget=1 << 30, batch_max=4) as srv:
        blocker = srv.submit(_body(4), 0.1)  # occupies the slot while the others queue
        time.sleep(0.02)
        futs = [srv.submit(b, 0.5 + 0.1 * i) for i, b in enumerate(same)]
        f_far = srv.submit(far, 0.9)
        f_head = srv.submit(same[0], 1.7, wave_directions=(0.0, 1.0))  # other headings
        res = [f.result(timeout=60) for f in futs]
        blocker.result(timeout=60)
        r_far, r_head = f_far.result(timeout=60), f_head.result(timeout=60)
    grouped = [c for c in eng.calls if c[0] == "factor_grouped"]
    assert len(grouped) == 1 and len(grouped[0][2]) == 3
    for b, r in zip(same, res):
        n = b.mesh_including_lid.nb_faces
        assert r.stats["batched"] == 3 and r.radiation_damping.shape == (len(b.dofs), len(b.dofs))
        assert np.all(r.added_mass == n / r.omega ** 2)
    assert "batched" not in r_far.stats and "batched" not in r_head.stats
    assert srv.counters["batched"] == 3 and srv.counters["completed"] == 6


# ---------------------------------------------------------------------------
@pytest.mark.gpu
def test_results_same_alone_and_in_the_mix(oracle_mod, default_oracle_gf, tmp_path):
    """Each request's coefficients in a mix of concurrent requests (different
    meshes, repeats, several slots) equal those of the same request run alone,
    and those of the engine's frequency sweep."""
    from capytaine_b200.engine import B200Engine
    from capytaine_b200.serving import SolveServer
    from test_gpu_mixed import _shared_table_gf
    gf = _shared_table_gf(default_oracle_gf, tmp_path)
    bodies = [
        FloatingBody(mesh_sphere(radius=1.0, resolution=(10, 20)).immersed_part(), rigid_body_dofs()),
        FloatingBody(mesh_parallelepiped(size=(8, 3, 4), resolution=(16, 6, 8)).immersed_part(),
                     rigid_body_dofs(only=["Surge", "Heave", "Pitch"])),
        FloatingBody(mesh_vertical_cylinder(length=6.0, radius=2.0, resolution=(4, 24, 12)).immersed_part(),
                     rigid_body_dofs(only=["Heave"])),
    ]
    reqs = [(b, w) for w in (0.4, 1.3, 2.6) for b in bodies]
    eng = B200Engine(green_function=gf, precision="mixed")
    with SolveServer(eng, slots=1, memory_budget=4 << 30) as alone:
        solo = [alone.solve(b, w, timeout=300) for b, w in reqs]
    with SolveServer(eng, slots=4, memory_budget=4 << 30) as mix:
        futs = [mix.submit(b, w) for b, w in reqs + reqs[::-1]]
        got = [f.result(timeout=600) for f in futs]
        assert mix.counters["max_inflight_requests"] >= 2
        assert mix.counters["reused"] >= 1
    got = got[:len(reqs)] + got[len(reqs):][::-1]
    for i, (b, w) in enumerate(reqs):
        for g in (got[i], got[len(reqs) + i]):
            for name in ("added_mass", "radiation_damping", "excitation"):
                a, s = getattr(g, name), getattr(solo[i], name)
                assert np.abs(a - s).max() <= 1e-12 * np.abs(s).max(), (i, name)
    for b in bodies:
        ws = [w for bb, w in reqs if bb is b]
        sweep = eng.solve_frequencies(b, ws)
        for j, w in enumerate(ws):
            s = solo[reqs.index((b, w))]
            for name in ("added_mass", "radiation_damping", "excitation"):
                a = getattr(sweep, name)[j]
                assert np.abs(a - getattr(s, name)).max() <= 1e-8 * np.abs(a).max(), name


@pytest.mark.gpu
def test_batched_requests_same_as_alone(oracle_mod, default_oracle_gf, tmp_path):
    """Requests factored together (batch_max 4: waiting requests of similar
    sizes share one grouped factorisation, identity-padded to the largest)
    give each request's result alone within the refinement tolerance."""
    from capytaine_b200.engine import B200Engine
    from capytaine_b200.serving import SolveServer
    from test_gpu_mixed import _shared_table_gf
    gf = _shared_table_gf(default_oracle_gf, tmp_path)
    bodies = [
        FloatingBody(mesh_sphere(radius=1.0, resolution=(10, 20)).immersed_part(), rigid_body_dofs()),
        FloatingBody(mesh_sphere(radius=1.5, resolution=(10, 22)).immersed_part(),
                     rigid_body_dofs(only=["Surge", "Heave", "Pitch"])),
        FloatingBody(mesh_vertical_cylinder(length=6.0, radius=2.0, resolution=(3, 20, 10)).immersed_part(),
                     rigid_body_dofs(only=["Heave"])),
    ]
    reqs = [(b, w) for w in (0.4, 1.3, 2.6) for b in bodies]
    eng = B200Engine(green_function=gf, precision="mixed")
    with SolveServer(eng, slots=1, memory_budget=4 << 30) as alone:
        solo = [alone.solve(b, w, timeout=300) for b, w in reqs]
    with SolveServer(eng, slots=1, memory_budget=4 << 30, batch_max=4, keep_factors=False) as srv:
        blocker = srv.submit(bodies[0], 3.3)  # the others queue behind it and are batched
        futs = [srv.submit(b, w) for b, w in reqs]
        got = [f.result(timeout=600) for f in futs]
        blocker.result(timeout=600)
        assert srv.counters.get("batched", 0) >= 4
    for i in range(len(reqs)):
        for name in ("added_mass", "radiation_damping", "excitation"):
            a, s = getattr(got[i], name), getattr(solo[i], name)
            assert np.abs(a - s).max() <= 1e-8 * np.abs(s).max(), (i, name)


@pytest.mark.gpu
def test_server_against_the_oracle(oracle_mod, default_oracle_gf, tmp_path):
    from capytaine_b200.engine import B200Engine
    from capytaine_b200.serving import SolveServer
    from test_gpu_mixed import _shared_table_gf
    gf = _shared_table_gf(default_oracle_gf, tmp_path)
    mesh = mesh_sphere(radius=1.0, resolution=(12, 24)).immersed_part()
    body = FloatingBody(mesh, rigid_body_dofs())
    omegas = [0.5, 2.0]
    with SolveServer(B200Engine(green_function=gf, precision="mixed"), slots=2, memory_budget=2 << 30) as srv:
        res = [f.result(timeout=600) for f in [srv.submit(body, w) for w in omegas]]
    for w, r in zip(omegas, res):
        ref = oracle_mod.solve_frequency(default_oracle_gf, mesh, oracle_mod.rigid_body_dofs(), w)
        A = np.array([[ref["added_mass"][i][j] for j in body.dofs] for i in body.dofs])
        E = np.array([ref["excitation"][0.0][j] for j in body.dofs])
        assert np.max(np.abs(r.added_mass - A) / np.maximum(np.abs(A), 1e-3 * np.abs(A).max())) < 1e-5
        assert np.max(np.abs(r.excitation[0] - E) / np.maximum(np.abs(E), 1e-3 * np.abs(E).max())) < 1e-5


def test_server_rejects_limit_frequencies_before_queueing():
    eng = _StandInEngine()
    with _server(eng, slots=1, memory_budget=1 << 28) as srv:
        for omega in (0.0, np.inf, -1.0, np.nan):
            with pytest.raises(ValueError):
                srv.submit(_body(4), omega)
        assert srv.counters["submitted"] == 0 and not eng.calls
