"""Batch-size autotuner of the grouped factorisation.

``B200Engine.solve_bodies`` (grouping "bands") puts the (body, omega) pairs of
many bodies into batches factored by one grouped LU.  How many matrices a
batch should hold depends on their size: small matrices need many per launch
to fill the GPU (the tensor-core updates of one 512-panel matrix are a few
tiles), large ones saturate it with few and only cost memory.  The tuner
times the grouped LU of synthetic diagonally dominant batches of each
candidate size for a size class (padded sizes rounded up to a multiple of
512), once per (device, precision, class), and keeps the candidate with the
least time per matrix (the smaller one when within 5%).  Choices are kept in
memory and, with ``cache_path``, in a JSON file that later processes read
instead of timing again.
"""
from __future__ import annotations

import json
import math
import os
import threading
from typing import Dict, Optional, Sequence

from . import _lib

CLASS = 512  # size classes: padded sizes rounded up to a multiple of this


class BatchTuner:
    def __init__(self, candidates: Sequence[int] = (8, 16, 32, 64), cache_path: Optional[str] = None,
                 measure: bool = True, default: int = 16):
        self.candidates = tuple(sorted(int(c) for c in candidates))
        self.cache_path = cache_path
        self.measure = measure
        self.default = int(default)
        self._lock = threading.Lock()
        self._choice: Dict[str, int] = {}
        self.timings: Dict[str, Dict[int, float]] = {}
        if cache_path and os.path.exists(cache_path):
            try:
                with open(cache_path) as fh:
                    self._choice.update({k: int(v) for k, v in json.load(fh).items()})
            except (OSError, ValueError):
                pass

    @staticmethod
    def size_class(npad: int) -> int:
        return max(CLASS, int(math.ceil(npad / CLASS) * CLASS))

    def _key(self, engine, cls: int) -> str:
        import torch
        name = torch.cuda.get_device_name(engine.device).replace(" ", "_")
        return f"{name}/{engine.precision}/{cls}"

    def batch_for(self, engine, npad: int, batch_bytes: float) -> int:
        """Matrices per grouped factorisation for matrices of padded size npad
        (at most what batch_bytes holds)."""
        from .engine import _Factors
        cap = int(max(1, batch_bytes // _Factors.estimate_bytes(npad, 1, engine.precision)))
        cls = self.size_class(npad)
        key = self._key(engine, cls)
        with self._lock:
            choice = self._choice.get(key)
            if choice is None:
                choice = self._time(engine, cls, batch_bytes) if self.measure else self.default
                self._choice[key] = choice
                if self.cache_path:
                    try:
                        with open(self.cache_path, "w") as fh:
                            json.dump(self._choice, fh, indent=1, sort_keys=True)
                    except OSError:
                        pass
        return max(1, min(choice, cap))

    def _time(self, engine, npad: int, batch_bytes: float) -> int:
        """Time per matrix of the grouped LU of each candidate batch size."""
        import torch
        from .engine import _Factors, _vp
        lib = _lib.load()
        dev = engine.device
        stream = _lib.stream_ptr()
        per = {}
        for B in self.candidates:
            if _Factors.estimate_bytes(npad, B, engine.precision) > batch_bytes:
                break
            f = _Factors(npad, B, dev, engine.precision)
            g = torch.Generator(device=dev).manual_seed(B)
            K = f.K.view(B, npad, npad)
            for b in range(B):  # one matrix at a time: no batch-sized temporary
                K[b].copy_(0.05 * torch.randn((npad, npad), dtype=torch.complex128, device=dev, generator=g))
            K.diagonal(dim1=1, dim2=2).add_(10.0)
            err = torch.zeros(1, dtype=torch.int32, device=dev)
            act = (_lib.c_int * B)(*([npad] * B))
            best = math.inf
            for rep in range(3):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                if engine.precision == "mixed":
                    _lib.check(lib.bem_clu_factor_grouped(_vp(f.K), npad, npad * npad, npad, npad, B, act,
                                                          _vp(f.piv), _vp(f.info), _vp(f.lu_work_ptr), _vp(err),
                                                          stream))
                else:
                    _lib.check(lib.bem_zlu_factor(_vp(f.K), npad, npad, npad * npad, B, _vp(f.piv), _vp(f.info),
                                                  _vp(f.lu_work), stream))
                e1.record()
                torch.cuda.synchronize()
                if rep > 0:  # the first launch of a shape loads and configures kernels
                    best = min(best, e0.elapsed_time(e1) / B)
            per[B] = best
            del f, K
        torch.cuda.empty_cache()
        if not per:
            return 1
        fastest = min(per.values())
        self.timings[f"{npad}"] = per
        return min(B for B, t in per.items() if t <= 1.05 * fastest)


DEFAULT_TUNER = BatchTuner()
