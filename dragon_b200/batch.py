"""Many independent grids advanced together (include/dragon_batch.h).

The reference runs independent problems one after another (a loop of
Grid::advance, DRAGON/Hydro/CFL/CFL.cpp:151-213). A Batch holds grid objects of
uneven sizes - 1D hydro and 2D MHD - each with its own configuration,
boundaries, CFL dt and retries, and advances them all with one persistent
kernel per step over a device work queue, replayed from a CUDA graph. Each
FP64 member ends in exactly the state its own advance_steps would give. The
members share one precision; in a mixed FP32/FP64 batch the 1D members end
exactly where their own mixed advance ends and the 2D MHD members to FP32
rounding of it.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

from . import _lib

ORDER_PHASE_MAJOR, ORDER_1D_FIRST, ORDER_LARGEST_FIRST, ORDER_WAVEFRONT = 0, 1, 2, 3


@dataclass
class Tuning:
    tile_1d: int = 254
    ctas_per_sm: int = 0     # 0: as many as fit
    order: int = ORDER_PHASE_MAJOR
    graph_steps: int = 32
    mhd_tiles: int = 8       # 32 x 8 tiles of a 2D MHD phase per work item
    wave: int = 1            # ORDER_WAVEFRONT: 2D MHD grids per wavefront group

    def to_c(self):
        return _lib.BatchTuning(self.tile_1d, self.ctas_per_sm, self.order, self.graph_steps, self.mhd_tiles,
                                self.wave)

    @staticmethod
    def from_c(t):
        return Tuning(t.tile_1d, t.ctas_per_sm, t.order, t.graph_steps, t.mhd_tiles or 1, t.wave or 1)


class Batch:
    def __init__(self, grids=()):
        self._lib = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(self._lib.dragon_gpu_batch_create(ctypes.byref(h)))
        self._h = h
        self.members = []
        for g in grids:
            self.add(g)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.dragon_gpu_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, grid) -> int:
        """Adds a Grid1D (hydro) or Grid2D (MHD); returns its index."""
        grid._to_device()
        idx = ctypes.c_int()
        _lib.check(self._lib.dragon_gpu_batch_add_instance(self._h, grid._h, ctypes.byref(idx)))
        self.members.append(grid)
        return idx.value

    def __len__(self):
        return len(self.members)

    @property
    def tuning(self) -> Tuning:
        t = _lib.BatchTuning()
        _lib.check(self._lib.dragon_gpu_batch_get_tuning(self._h, ctypes.byref(t)))
        return Tuning.from_c(t)

    @tuning.setter
    def tuning(self, t: Tuning) -> None:
        c = t.to_c()
        _lib.check(self._lib.dragon_gpu_batch_set_tuning(self._h, ctypes.byref(c)))

    def autotune(self, steps_per_candidate: int = 4):
        """Times every launch shape on the members' states (restored) and keeps the fastest."""
        for g in self.members:
            g._to_device()
        t = _lib.BatchTuning()
        ms = ctypes.c_double()
        _lib.check(self._lib.dragon_gpu_batch_autotune(self._h, int(steps_per_candidate), ctypes.byref(t),
                                                       ctypes.byref(ms)))
        return Tuning.from_c(t), ms.value

    def advance_steps(self, nsteps: int) -> dict:
        """Every member takes nsteps CFL-limited steps."""
        for g in self.members:
            g._to_device()
        st = _lib.BatchStats()
        rc = self._lib.dragon_gpu_batch_advance_steps(self._h, int(nsteps), ctypes.byref(st))
        for g in self.members:
            g._device_ran()
        _lib.check(rc)
        return {name: getattr(st, name) for name, _ in st._fields_}
