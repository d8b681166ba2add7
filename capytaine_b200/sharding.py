"""Frequency-solves across GPUs: one process per GPU, frequencies sharded.

Frequency-solves of a sweep share nothing but the read-only mesh and table, so
each rank solves its own share (round robin over the sweep: ranks get
interleaved frequencies, which balances the cost when it grows with omega)
with no collective on the data path.  The only collectives are a gather of the
small coefficient arrays at the end and, for measurements, the maximum of the
ranks' times.  Works with any torch.distributed backend (NCCL between GPUs,
gloo on the host).
"""
from __future__ import annotations

from typing import Sequence

import numpy as np


def frequency_shard(omegas: Sequence[float], rank: int, world: int) -> np.ndarray:
    """Indices of the frequencies that `rank` solves: rank, rank + world, ..."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    return np.arange(rank, len(omegas), world)


def max_over_ranks(value: float) -> float:
    """Largest value over the ranks (a no-op without an initialised process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def solve_frequencies_sharded(engine, body, omegas: Sequence[float], **kw):
    """engine.solve_frequencies on this rank's share of omegas, then every
    rank receives the coefficients of the whole sweep (a FrequencyResults in
    the order of omegas).  Without a process group this is solve_frequencies."""
    import torch.distributed as dist
    omegas = np.asarray(omegas, dtype=float)
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return engine.solve_frequencies(body, omegas, **kw)
    rank, world = dist.get_rank(), dist.get_world_size()
    idx = frequency_shard(omegas, rank, world)
    local = engine.solve_frequencies(body, omegas[idx], **kw) if len(idx) else None
    parts = [None] * world
    dist.all_gather_object(parts, (idx, local))
    return merge_shards(omegas, parts)


def merge_shards(omegas, parts):
    """Coefficients of the whole sweep from the (indices, FrequencyResults)
    shards of the ranks."""
    from .engine import FrequencyResults
    full = None
    for idx, res in parts:
        if res is None:
            continue
        if full is None:
            shape = lambda a: (len(omegas),) + a.shape[1:]  # noqa: E731
            full = {k: np.zeros(shape(getattr(res, k)), dtype=getattr(res, k).dtype)
                    for k in ("added_mass", "radiation_damping", "diffraction", "froude_krylov", "excitation")}
            dofs, heads = res.dofs, res.wave_directions
        for k in full:
            full[k][idx] = getattr(res, k)
    if full is None:
        raise ValueError("no rank solved any frequency")
    return FrequencyResults(omegas=np.asarray(omegas), dofs=dofs, wave_directions=heads, **full)
