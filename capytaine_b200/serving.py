"""Request server for frequency-solves on one B200: continuous batching.

A request is one frequency-solve of one body: assemble S and K at
k = omega^2/g, factor K, solve every radiation and diffraction problem, S @
sigma, forces -> added mass, radiation damping, excitation (what capytaine's
``BEMSolver.solve_all`` does for one (body, omega) group, bem/solver.py:268-372).
capytaine itself has no server; this is the request loop around the same
engine stages (``B200Engine.assemble_stage`` / ``factor_stage`` /
``solve_stage``).

Scheduling
* ``submit`` queues a request and returns a ``concurrent.futures.Future``.
* ``slots`` worker threads, each with its own CUDA stream: requests admitted
  while others run are enqueued on their own stream, so their kernels overlap
  on the device (different mesh sizes run side by side).
* Admission by device-memory footprint: a request is admitted (in arrival
  order) when a slot is free and the bytes of its matrices, factors and
  right-hand sides fit in ``memory_budget`` next to what is in flight and what
  is resident; resident factors not in use are evicted (least recently used)
  to make room.  A request that alone exceeds the budget fails with
  MemoryError.
* Device memory: one arena of ``memory_budget`` bytes is allocated when the
  server starts and every buffer of a request is a view of it, so serving
  never calls the CUDA allocator (whose frees synchronise the whole device)
  between requests.
* Residency: the factors of every solved (mesh, omega) stay on the device
  (with S and K) until evicted; a later request for the same mesh and omega
  only solves its right-hand sides with them.  Device meshes and the
  tabulation are resident in the Green function's caches.

Results do not depend on what else runs: every kernel is deterministic and
requests share no mutable device memory.
"""
from __future__ import annotations

import concurrent.futures as cf
import logging
import threading
import time
from collections import OrderedDict, deque
from dataclasses import dataclass, field
from typing import Deque, Dict, List, Optional, Sequence

import numpy as np

from . import _lib
from .arena import ArenaFull, DeviceArena  # noqa: F401  (re-exported)
from .engine import B200Engine, _Factors, _Rhs

LOG = logging.getLogger(__name__)


@dataclass
class SolveResult:
    """Coefficients of one frequency-solve: added_mass / radiation_damping
    [radiating_dof, influenced_dof], diffraction / froude_krylov / excitation
    [heading, influenced_dof]; host clock times (time.perf_counter) of arrival,
    admission and completion; whether resident factors were reused."""
    request_id: int
    omega: float
    dofs: List[str]
    wave_directions: np.ndarray
    added_mass: np.ndarray
    radiation_damping: np.ndarray
    diffraction: np.ndarray
    froude_krylov: np.ndarray
    excitation: np.ndarray
    arrival: float
    admitted: float
    finished: float
    reused_factors: bool
    stats: Dict[str, float] = field(default_factory=dict)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


@dataclass
class _Request:
    rid: int
    body: object
    omega: float
    heads: np.ndarray
    rho: float
    g: float
    arrival: float
    future: cf.Future
    key: tuple = ()
    n: int = 0
    nrhs: int = 0


class _Resident:
    """S, K and the factors of one (mesh, omega) kept on the device between requests."""

    def __init__(self, f: _Factors, nbytes: int, release):
        self.f = f
        self.nbytes = nbytes
        self.release = release  # frees the arena blocks of f
        self.users = 0
        self.lock = threading.Lock()


class SolveServer:
    """Continuous-batching request loop (see the module docstring).

    engine: a B200Engine (its precision, refinement and Green function are
    used; default: the refined mixed-precision engine).  memory_budget: device
    bytes for in-flight requests plus resident factors (default 60% of the
    device memory).  slots: concurrent requests on the device.  keep_factors:
    keep the factors of solved (mesh, omega) pairs resident for reuse.
    """

    def __init__(self, engine: Optional[B200Engine] = None, *, slots: int = 4, memory_budget: Optional[int] = None,
                 keep_factors: bool = True, batch_max: int = 1, band: float = 1.3):
        import torch
        self.engine = engine if engine is not None else B200Engine(precision="mixed")
        dev = torch.device(self.engine.device)
        if dev.type == "cuda" and dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        if memory_budget is None:
            total = torch.cuda.get_device_properties(self.device).total_memory
            memory_budget = int(0.6 * total)
        self.memory_budget = int(memory_budget)
        self.keep_factors = bool(keep_factors)
        # continuous batching of factorisations: a slot that admits a new
        # request also takes up to batch_max - 1 waiting ones of similar size
        # (padded sizes within a factor `band`, same headings, rho and g) and
        # factors them together with the grouped LU (mixed engine only)
        self.batch_max = max(1, int(batch_max)) if self.engine.precision == "mixed" else 1
        self.band = float(band)
        self._arena = DeviceArena(self.memory_budget, self.device)
        self._cv = threading.Condition()
        self._pending: Deque[_Request] = deque()
        self._resident: "OrderedDict[tuple, _Resident]" = OrderedDict()
        self._resident_bytes = 0
        self._inflight_bytes = 0
        self._next_id = 0
        self._closed = False
        self._failure: Optional[BaseException] = None
        self.counters = {"submitted": 0, "completed": 0, "failed": 0, "reused": 0, "evicted": 0,
                         "max_reserved_bytes": 0, "max_inflight_requests": 0}
        self._inflight = 0
        self._workers = [threading.Thread(target=self._worker, name=f"bem-slot-{i}", daemon=True)
                         for i in range(int(slots))]
        for t in self._workers:
            t.start()

    # ---- public API ---------------------------------------------------------
    def submit(self, body, omega: float, *, wave_directions: Sequence[float] = (0.0,), rho: float = 1000.0,
               g: float = 9.81) -> cf.Future:
        if not 0.0 < float(omega) < np.inf:
            raise ValueError("the request server solves finite, non-zero frequencies; omega = 0 or infinity "
                             "goes through B200Engine.solve_frequencies")
        heads = np.asarray(wave_directions, dtype=float)
        mesh = body.mesh_including_lid
        nrhs = len(body.dofs) + len(heads)
        fut: cf.Future = cf.Future()
        with self._cv:
            if self._failure is not None:
                raise RuntimeError(f"request server slot failed: {self._failure!r}")
            if self._closed:
                raise RuntimeError("server is shut down")
            rid = self._next_id
            self._next_id += 1
            req = _Request(rid, body, float(omega), heads, float(rho), float(g), time.perf_counter(), fut)
            req.key = (mesh.content_hash, float(omega), float(g))
            req.n = mesh.nb_faces
            req.nrhs = nrhs
            self._pending.append(req)
            self.counters["submitted"] += 1
            self._cv.notify_all()
        return fut

    def solve(self, body, omega: float, *, timeout: Optional[float] = None, **kw) -> SolveResult:
        """Submit and wait (at most `timeout` seconds when given)."""
        return self.submit(body, omega, **kw).result(timeout=timeout)

    def shutdown(self, wait: bool = True):
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        if wait:
            for t in self._workers:
                t.join()
            self.release_resident()
            self._arena = None  # the device memory goes back to torch's allocator

    def release_resident(self):
        """Drop every resident factorisation not in use."""
        with self._cv:
            for key in [k for k, e in self._resident.items() if e.users == 0]:
                self._drop_locked(key)

    @property
    def resident_bytes(self) -> int:
        return self._resident_bytes

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.shutdown()

    # ---- admission ----------------------------------------------------------
    def _footprint(self, req: _Request, reuse: bool) -> int:
        """Device bytes a request holds while it runs: its S, K and factors
        (unless resident factors are reused) and its right-hand sides."""
        prec = self.engine.precision
        blk = 128 if prec == "mixed" else 64
        npad = -(-req.n // blk) * blk
        f_bytes = 0 if reuse else _Factors.estimate_bytes(req.n, 1, prec)
        g_bytes = 0
        if prec == "mixed":
            g_bytes = int(_lib.load().bem_gmres_workspace_bytes(req.n, npad, req.nrhs, 1,
                                                                self.engine.gmres_restart)) + 256
        return f_bytes + g_bytes + _Rhs.estimate_bytes(req.n, npad, 1, req.nrhs)

    def _drop_locked(self, key):
        e = self._resident.pop(key)
        self._resident_bytes -= e.nbytes
        e.release()
        self.counters["evicted"] += 1

    def _make_room_locked(self, need: int) -> bool:
        while self._inflight_bytes + self._resident_bytes + need > self.memory_budget:
            victim = next((k for k, e in self._resident.items() if e.users == 0), None)
            if victim is None:
                return False
            self._drop_locked(victim)
        return True

    @staticmethod
    def _padded(n: int) -> int:
        return -(-n // 128) * 128

    def _batch_footprint(self, reqs: List[_Request]) -> int:
        """Device bytes of one grouped batch of new requests (all identity-padded
        to the largest), with the GMRES workspace of the refinement fallback."""
        npad = max(self._padded(q.n) for q in reqs)
        nrhs = max(q.nrhs for q in reqs)
        B = len(reqs)
        g_bytes = int(_lib.load().bem_gmres_workspace_bytes(npad, npad, min(nrhs, 16), B,
                                                            self.engine.gmres_restart)) + 256
        return _Factors.estimate_bytes(npad, B, "mixed") + g_bytes + _Rhs.estimate_bytes(npad, npad, B, nrhs)

    def _companions_locked(self, head: _Request) -> List[_Request]:
        """Waiting new requests that can share head's factorisation."""
        if self.batch_max <= 1:
            return []
        p0 = self._padded(head.n)
        out = []
        for q in list(self._pending)[1:]:
            if len(out) + 1 >= self.batch_max:
                break
            p = self._padded(q.n)
            if (q.key in self._resident or q.key == head.key or any(q.key == o.key for o in out)
                    or max(p, p0) > self.band * min(p, p0) or q.rho != head.rho or q.g != head.g
                    or q.heads.shape != head.heads.shape or not np.array_equal(q.heads, head.heads)):
                continue
            out.append(q)
        return out

    def _take_locked(self):
        """Admission in arrival order: the head of the queue when it fits (with
        the waiting requests that join its factorisation, when batching)."""
        if not self._pending:
            return None
        head = self._pending[0]
        res = self._resident.get(head.key)
        if res is None:
            extra = self._companions_locked(head)
            while extra:
                need = self._batch_footprint([head] + extra)
                if need <= self.memory_budget and self._make_room_locked(need):
                    self._pending.popleft()
                    for q in extra:
                        self._pending.remove(q)
                    return [head] + extra, None, need
                extra.pop()
        need = self._footprint(head, res is not None)
        if need > self.memory_budget:
            self._pending.popleft()
            head.future.set_exception(MemoryError(
                f"request of {head.n} panels needs {need / 1e9:.2f} GB, above the server budget "
                f"{self.memory_budget / 1e9:.2f} GB"))
            self.counters["failed"] += 1
            return "retry"
        if res is not None:
            res.users += 1  # pinned before making room, so it is not evicted
            self._resident.move_to_end(head.key)
        if not self._make_room_locked(need):
            if res is not None:
                res.users -= 1
            return None
        self._pending.popleft()
        return [head], res, need

    def _slot_stream(self):
        """Context placing the calling thread's work on its own CUDA stream."""
        import contextlib
        import torch
        dev = torch.device(self.device)
        if dev.type != "cuda":  # host-side tests of the scheduler with a stand-in engine
            return contextlib.nullcontext()
        torch.cuda.set_device(dev.index)
        return torch.cuda.stream(torch.cuda.Stream(device=dev))

    def _worker(self):
        try:
            self._serve()
        except BaseException as exc:  # a slot that cannot run fails the queue instead of hanging it
            with self._cv:
                self._closed = True
                self._failure = exc
                while self._pending:
                    req = self._pending.popleft()
                    if not req.future.done():
                        req.future.set_exception(RuntimeError(f"request server slot failed: {exc!r}"))
                self._cv.notify_all()
            LOG.error("request server slot failed: %r", exc)

    def _serve(self):
        slot = self._slot_stream()
        while True:
            with self._cv:
                while True:
                    if self._closed and not self._pending:
                        return
                    got = self._take_locked()
                    if got == "retry":
                        continue
                    if got is not None:
                        break
                    self._cv.wait()
                reqs, res, need = got
                self._inflight_bytes += need
                self._inflight += len(reqs)
                self.counters["max_inflight_requests"] = max(self.counters["max_inflight_requests"], self._inflight)
                self.counters["max_reserved_bytes"] = max(self.counters["max_reserved_bytes"],
                                                          self._inflight_bytes + self._resident_bytes)
            admitted = time.perf_counter()
            keep = results = error = None
            try:
                with slot:
                    if len(reqs) == 1:
                        result, keep = self._run(reqs[0], res, admitted)
                        results = [result]
                    else:
                        results = self._run_batch(reqs, admitted)
            except BaseException as exc:  # the requests fail, the server goes on
                error = exc
            finally:
                with self._cv:
                    self._inflight_bytes -= need
                    self._inflight -= len(reqs)
                    if res is not None:
                        res.users -= 1
                    if keep is not None:
                        f, release = keep
                        key = reqs[0].key
                        if key not in self._resident and self._make_room_locked(f.nbytes):
                            self._resident[key] = _Resident(f, f.nbytes, release)
                            self._resident_bytes += f.nbytes
                        else:
                            release()
                    if error is None:
                        self.counters["completed"] += len(reqs)
                        if res is not None:
                            self.counters["reused"] += 1
                        if len(reqs) > 1:
                            self.counters["batched"] = self.counters.get("batched", 0) + len(reqs)
                    else:
                        self.counters["failed"] += len(reqs)
                    self._cv.notify_all()
            # the callers see the results after the bookkeeping above
            for i, req in enumerate(reqs):
                if error is None:
                    req.future.set_result(results[i])
                else:
                    req.future.set_exception(error)

    def _buffers(self, build):
        """build(alloc) with arena views, all or nothing: when the arena has no
        block large enough, evict an unused resident factorisation, or wait
        for a running request to free its buffers, and retry."""
        while True:
            arena = self._arena
            if arena is None:
                raise RuntimeError("server is shut down")
            alloc, release = arena.allocator()
            try:
                return build(alloc), release
            except ArenaFull:
                release()
                with self._cv:
                    victim = next((k for k, e in self._resident.items() if e.users == 0), None)
                    if victim is not None:
                        self._drop_locked(victim)
                    else:
                        self._cv.wait(timeout=0.05)

    def _run_batch(self, reqs: List[_Request], admitted: float) -> List[SolveResult]:
        """New requests of similar sizes in one grouped factorisation: each
        request's S and K are assembled into its slot of a batch padded to the
        largest (identity padding), the grouped LU factors them at the cost of
        their own sizes, the right-hand sides of every request are solved
        together and the forces integrated per request.  No factors are kept
        resident (they share one allocation)."""
        eng = self.engine
        npad = max(self._padded(q.n) for q in reqs)
        nrhs = max(q.nrhs for q in reqs)
        B = len(reqs)
        stats: Dict[str, float] = {}
        f, release = self._buffers(lambda a: _Factors(npad, B, self.device, "mixed", alloc=a))
        try:
            def rhs(alloc):
                r = _Rhs(npad, npad, B, nrhs, self.device, "mixed", alloc=alloc)
                r.gmres_work(eng.gmres_restart)
                return r
            r, release_r = self._buffers(rhs)
            try:
                r.flags.zero_()
                om = np.array([q.omega for q in reqs])
                for j, q in enumerate(reqs):
                    mesh = q.body.mesh_including_lid
                    eng.assemble_stage(f, mesh, [q.omega ** 2 / q.g], nan_flag=r.nan, reuse_rankine=False,
                                       first=j, lds=npad)
                    eng.pad_stage(f, j, 1, mesh.nb_faces)
                eng.factor_stage(f, B, r.err, active=[self._padded(q.n) for q in reqs])
                out = eng._solve_segments(f, r, [(q.body, j, 1) for j, q in enumerate(reqs)], om, reqs[0].heads,
                                          rho=reqs[0].rho, g=reqs[0].g, stats=stats)
            finally:
                release_r()
        finally:
            release()
        finished = time.perf_counter()
        results = []
        for q, (F, FK) in zip(reqs, out):
            ndof = len(q.body.dofs)
            w = q.omega
            rad, dif, fk = F[0, :ndof, :], F[0, ndof:, :], FK[0]
            results.append(SolveResult(
                request_id=q.rid, omega=w, dofs=list(q.body.dofs), wave_directions=q.heads,
                added_mass=np.real(rad) / w ** 2, radiation_damping=np.imag(rad) / w, diffraction=dif,
                froude_krylov=fk, excitation=dif + fk, arrival=q.arrival, admitted=admitted, finished=finished,
                reused_factors=False, stats=dict(stats, batched=B)))
        return results

    def _run(self, req: _Request, res: Optional[_Resident], admitted: float):
        """Enqueue the request's work on the current (slot) stream and wait
        for it; returns the result and (factors, release) to keep resident, if any."""
        eng = self.engine
        body = req.body
        mesh = body.mesh_including_lid
        om = np.array([req.omega])
        stats: Dict[str, float] = {}
        # GMRES workspace up front: the refined solve may escalate to it
        gmres = eng.precision == "mixed"

        def rhs(alloc, n, npad):
            r = _Rhs(n, npad, 1, req.nrhs, self.device, eng.precision, alloc=alloc)
            if gmres:
                r.gmres_work(eng.gmres_restart)
            return r
        if res is not None:
            with res.lock:  # repeats of one entry take turns on its buffers
                r, release_r = self._buffers(lambda a: rhs(a, res.f.n, res.f.npad))
                try:
                    F, FK = eng.solve_stage(res.f, r, body, om, req.heads, rho=req.rho, g=req.g, stats=stats)
                finally:
                    release_r()
            keep = None
        else:
            f, release = self._buffers(lambda a: _Factors(req.n, 1, self.device, eng.precision, alloc=a))
            try:
                r, release_r = self._buffers(lambda a: rhs(a, f.n, f.npad))
                try:
                    eng.assemble_stage(f, mesh, om ** 2 / req.g, nan_flag=r.nan, reuse_rankine=False)
                    eng.factor_stage(f, 1, r.err)
                    F, FK = eng.solve_stage(f, r, body, om, req.heads, rho=req.rho, g=req.g, stats=stats)
                finally:
                    release_r()
            except BaseException:
                release()
                raise
            keep = (f, release) if self.keep_factors else None  # S, K and factors stay with `release`
            if keep is None:
                release()
        finished = time.perf_counter()
        ndof = len(body.dofs)
        w = req.omega
        rad, dif, fk = F[0, :ndof, :], F[0, ndof:, :], FK[0]
        result = SolveResult(
            request_id=req.rid, omega=w, dofs=list(body.dofs), wave_directions=req.heads,
            added_mass=np.real(rad) / w ** 2, radiation_damping=np.imag(rad) / w, diffraction=dif,
            froude_krylov=fk, excitation=dif + fk, arrival=req.arrival, admitted=admitted, finished=finished,
            reused_factors=res is not None, stats=dict(stats))
        return result, keep
