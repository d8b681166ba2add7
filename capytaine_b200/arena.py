"""Device memory arena: one allocation carved into aligned blocks.

The request server and the many-body sweep take every buffer of a request or
of a group of bodies from one arena allocated up front, so that no
cudaMalloc / cudaFree (which synchronise the whole device) happens between
requests or groups.
"""
from __future__ import annotations

import threading


class ArenaFull(MemoryError):
    """No free block of the requested size in the arena (retry after frees)."""


class DeviceArena:
    """One device allocation carved into `granule`-aligned blocks, first fit
    with coalescing of free neighbours.  ``allocator()`` returns an
    (alloc, release) pair: alloc(shape, dtype, zero=False) hands out tensor
    views (zeroed on the caller's current stream when asked), release() frees
    every block handed out by that pair."""

    def __init__(self, nbytes: int, device, granule: int = 1 << 16):
        import torch
        self.granule = int(granule)
        self.size = int(nbytes) // self.granule * self.granule
        self.buf = torch.empty(self.size, dtype=torch.uint8, device=device)
        self._free = [(0, self.size)]  # (offset, size), sorted by offset
        self._lock = threading.Lock()
        self.used = 0
        self.peak = 0

    def allocate(self, nbytes: int) -> int:
        size = max(self.granule, -(-int(nbytes) // self.granule) * self.granule)
        with self._lock:
            for i, (off, sz) in enumerate(self._free):
                if sz >= size:
                    if sz == size:
                        self._free.pop(i)
                    else:
                        self._free[i] = (off + size, sz - size)
                    self.used += size
                    self.peak = max(self.peak, self.used)
                    return off
        raise ArenaFull(f"no free block of {size} bytes in the device arena")

    def release(self, off: int, nbytes: int):
        size = max(self.granule, -(-int(nbytes) // self.granule) * self.granule)
        with self._lock:
            self.used -= size
            fl = self._free
            lo, hi = 0, len(fl)
            while lo < hi:  # insertion point by offset
                mid = (lo + hi) // 2
                if fl[mid][0] < off:
                    lo = mid + 1
                else:
                    hi = mid
            fl.insert(lo, (off, size))
            if lo + 1 < len(fl) and fl[lo][0] + fl[lo][1] == fl[lo + 1][0]:
                fl[lo] = (fl[lo][0], fl[lo][1] + fl[lo + 1][1])
                fl.pop(lo + 1)
            if lo > 0 and fl[lo - 1][0] + fl[lo - 1][1] == fl[lo][0]:
                fl[lo - 1] = (fl[lo - 1][0], fl[lo - 1][1] + fl[lo][1])
                fl.pop(lo)

    @property
    def largest_free(self) -> int:
        with self._lock:
            return max((sz for _, sz in self._free), default=0)

    def allocator(self):
        import torch
        blocks = []

        def alloc(shape, dtype, zero=False):
            count = 1
            for d in shape:
                count *= int(d)
            nbytes = count * torch.empty((), dtype=dtype).element_size()
            off = self.allocate(nbytes)
            blocks.append((off, nbytes))
            t = self.buf[off:off + nbytes].view(dtype).view(tuple(shape))
            if zero:
                t.zero_()
            return t

        def release():
            while blocks:
                self.release(*blocks.pop())
        return alloc, release
