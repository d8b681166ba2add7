"""Frequency shards across ranks (one process per GPU in production), checked
with two gloo ranks on the host and a stand-in engine: every frequency is solved
by exactly one rank, every rank ends with the whole sweep in order, and the
timing reduction takes the maximum over the ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from capytaine_b200.sharding import frequency_shard, merge_shards


class _StandIn:
    def __init__(self, rank):
        self.rank = rank

    def solve_frequencies(self, body, omegas, **kw):
        from capytaine_b200.engine import FrequencyResults
        w = np.asarray(omegas)
        ndof = 2
        am = np.stack([np.full((ndof, ndof), x) for x in w])
        exc = (w[:, None, None] * np.ones((len(w), 1, ndof))).astype(complex) + 1j * self.rank
        return FrequencyResults(omegas=w, dofs=["Heave", "Pitch"], wave_directions=np.array([0.0]),
                                added_mass=am, radiation_damping=2 * am, diffraction=exc,
                                froude_krylov=0 * exc, excitation=exc)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, omegas, out):
    import torch.distributed as dist
    from capytaine_b200.sharding import max_over_ranks, solve_frequencies_sharded
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = solve_frequencies_sharded(_StandIn(rank), None, omegas)
        t = max_over_ranks(10.0 + rank)
        out.put((rank, res.added_mass[:, 0, 0].tolist(), res.excitation[:, 0, 0].imag.tolist(), t))
    finally:
        dist.destroy_process_group()


def test_frequency_shard_partitions_the_sweep():
    for n, world in ((60, 1), (60, 2), (61, 8), (3, 4)):
        parts = [frequency_shard(np.zeros(n), r, world) for r in range(world)]
        assert sorted(np.concatenate(parts).tolist()) == list(range(n))
    with pytest.raises(ValueError):
        frequency_shard(np.zeros(4), 2, 2)


def test_merge_shards_orders_the_sweep():
    omegas = np.linspace(0.1, 1.0, 7)
    parts = [(frequency_shard(omegas, r, 3), _StandIn(r).solve_frequencies(None, omegas[frequency_shard(omegas, r, 3)]))
             for r in range(3)]
    full = merge_shards(omegas, parts)
    assert np.allclose(full.added_mass[:, 0, 0], omegas)


def test_two_gloo_ranks():
    omegas = np.linspace(0.05, 3.0, 11)
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, omegas, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = [out.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, am, exc_im, t in got:
        assert np.allclose(am, omegas)  # every rank holds the whole sweep, in order
        owner = [frequency_shard(omegas, r, 2) for r in range(2)]
        for r, idx in enumerate(owner):
            assert np.allclose(np.asarray(exc_im)[idx], r)  # solved by its owner
        assert t == 11.0  # maximum over the ranks
