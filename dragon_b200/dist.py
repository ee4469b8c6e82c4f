"""DistGrid1D / DistGrid2D / DistGrid3D over several GPUs: one process per
GPU, the grid cut into slabs along x, a halo exchange per step.

The reference's DistGrid (DRAGON/Refinement/DistGrid.cpp:58-346) splits a
root grid into child grids on pthreads: every step the root fills its ghosts
and takes the CFL time over the whole grid, copies each child its block with
ghosts (pushToChildren, :115-204), the children step concurrently, and the
interiors come back (loadFromChildren, :208-289); if any child fails, no child
commits and the root retries with half the step (:292-304, :349-360, with
DRAGONWING's all-or-nothing checkpoints). The result is bit-identical to the
serial grid as long as every child has the ghost width the scheme needs
(validGhosts, :27-39).

Here there is no root copy of the grid. Rank r holds slab r of the x axis
(sizes by computeChildSize, :21-25) on its own GPU, and one step is:

1. The boundary list, restricted to the faces of the global box this slab
   touches, fills the slab's ghosts on the device. An x-periodic element
   becomes an exchange between the first and the last slab at the element's
   place in the list.
2. Halo exchange: each slab sends its outer ``ghosts`` layers (cells, and
   face-centred B for MHD) to its x neighbours, who write them into their
   ghost layers. After it every ghost cell of every slab holds what the
   serial grid holds at that position.
3. Each rank's CFL time over its slab and one-cell ring, then an all-reduce
   MIN: CFL_coeff / max_speed is monotone in max_speed, so the minimum over
   slabs is exactly the serial grid's CFL time.
4. Every slab steps with the same dt; an all-reduce of the success flags
   commits all or none (a slab that succeeded undoes its step with
   dragon_gpu_step_rollback) and the step is retried at half the dt.

Cutting only x keeps every halo a set of whole layers, contiguous in memory
per field, and makes each boundary element's fill along y and z local to a
slab (a y or z ghost is filled from cells of the same x layer), so the fill
order of the serial list is kept exactly. With 180 GB of HBM per GPU, slabs are
wide and halos are a small fraction of a step's traffic.

Boundary elements with a host ``apply()`` (user GhostFill subclasses) are not
supported on a distributed grid.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch
import torch.distributed as tdist

from . import _lib
from .boundary import IGNORE, OUTFLOW, PERIODIC, USER, X, X_negative, X_positive, BoundaryList, as_list
from .grid import AdvanceResult, Config, Grid1D, Grid2D, Grid3D, StepFailed

ALL_FACES = 63


def child_size(n: int, parts: int, i: int) -> int:
    """computeChildSize (DistGrid.cpp:21-25): the first n % parts slabs get one more cell."""
    return n // parts + (1 if i < n % parts else 0)


def valid_ghosts(ghosts: int, mhd: bool) -> int:
    """validGhosts (DistGrid.cpp:27-39) for the unsplit scheme: 3 with MHD (CTU
    + constrained transport), else 2."""
    return max(int(ghosts), 3 if mhd else 2)


def _normalised_faces(e) -> int:
    f = e.get_faces() & ALL_FACES
    if e.kind == PERIODIC:  # Periodic.cpp:14-15: an axis always covers both faces
        g = 0
        for a in range(3):
            if f & (3 << (2 * a)):
                g |= 3 << (2 * a)
        f = g
    return f


class SlabProgram:
    """The boundary list of slab `rank` of `parts`: device entries
    (type, faces, corners, state) and the place of the x-periodic exchange.

    The entries are the global list's, in order, after the implicit Outflow
    over the globally uncovered faces (BoundaryList.hpp:97-104), each masked to
    the faces of the global box the slab touches. An element periodic in x
    leaves an Ignore placeholder where the exchange runs (its y / z part stays
    a device entry right after it). A device user fill (DeviceGhostFill) stays
    a device entry that fills the global faces the slab touches; the slab's
    grid carries its global origin for the fill's coordinates. A final Ignore
    over every face keeps the device from adding an implicit Outflow on faces
    between slabs.
    """

    def __init__(self, blist: BoundaryList, rank: int, parts: int, dim: int):
        self.entries: list[tuple[int, int, int, list[float]]] = []
        # device user fills by entry: (element, the faces it fills on this slab)
        self.fills: dict[int, tuple[object, int]] = {}
        self.wrap_at: int | None = None
        self.wrap_corners = True
        own = ALL_FACES & ~X
        if rank == 0:
            own |= X_negative
        if rank == parts - 1:
            own |= X_positive
        els = list(blist)
        if any(e.is_custom for e in els):
            raise NotImplementedError("boundary elements with a host apply() are not supported on a DistGrid")
        uncovered = ALL_FACES
        for e in els:
            uncovered &= ~_normalised_faces(e)
        if uncovered & own:
            self.entries.append((OUTFLOW, uncovered & own, 1, [0.0] * 8))
        for e in els:
            f = _normalised_faces(e)
            st = list(e.state()) + [0.0] * 8
            if e.kind == PERIODIC and f & X:
                if self.wrap_at is not None:
                    raise NotImplementedError("more than one element periodic in x")
                self.wrap_at = len(self.entries)
                self.wrap_corners = bool(e.corners)
                self.entries.append((IGNORE, 0, 1, [0.0] * 8))
                rest = f & ~X
                if rest and dim > 1:
                    self.entries.append((PERIODIC, rest, int(e.corners), [0.0] * 8))
            elif e.kind == USER:
                # a device fill visits the faces of the global box this slab touches
                self.fills[len(self.entries)] = (e, e.fill_faces & own)
                self.entries.append((USER, f & own, int(e.corners), [0.0] * 8))
            else:
                self.entries.append((e.kind, f & own, int(e.corners), st[:8]))
        self.entries.append((IGNORE, ALL_FACES, 1, [0.0] * 8))


class GpuSlab:
    """One slab resident on this process's GPU: a Grid1D/2D/3D and the C ABI
    calls the distributed step uses (ranged boundary fill, halo pack / unpack,
    step with rollback)."""

    def __init__(self, dim, n, d, ghosts, config: Config):
        cls = {1: Grid1D, 2: Grid2D, 3: Grid3D}[dim]
        self.grid = cls(*n, *d, ghosts=ghosts, config=config)
        self.L = self.grid._lib
        self.h = self.grid._h
        self.dim = dim
        self.n = self.grid.n
        self.ghosts = self.grid.ghosts
        self.has_faces = self.grid._B is not None
        self.on_device = torch.cuda.is_available()

    def set_origin(self, offset):
        """The slab's place in the global grid, for its device user fills."""
        o = list(offset) + [0] * (3 - len(offset))
        _lib.check(self.L.dragon_gpu_set_origin(self.h, int(o[0]), int(o[1]), int(o[2])))

    def set_entries(self, entries, fills=None):
        arr = (_lib.BCDesc * max(1, len(entries)))()
        for k, (t, faces, corners, st) in enumerate(entries):
            arr[k].type = t
            arr[k].faces = faces
            arr[k].corners = corners
            for q in range(8):
                arr[k].state[q] = st[q]
        _lib.check(self.L.dragon_gpu_set_boundary(self.h, arr, len(entries)))
        if int(self.L.dragon_gpu_boundary_entries(self.h)) != len(entries):
            raise RuntimeError("device boundary list does not match the slab program")
        for k, (el, ff) in (fills or {}).items():
            el.bind(self.L, self.h, k, fill_faces=ff)

    def apply_range(self, first, count):
        if count <= 0:
            return
        self.grid._to_device()
        _lib.check(self.L.dragon_gpu_apply_boundary_range(self.h, int(first), int(count)))
        self.grid._device_ran()

    def halo_count(self, layers, faces, corners) -> int:
        out = ctypes.c_longlong()
        _lib.check(self.L.dragon_gpu_halo_size(self.h, 0, int(layers), int(faces), int(corners), ctypes.byref(out)))
        return out.value

    def pack(self, first, layers, faces, corners, buf: torch.Tensor):
        self.grid._to_device()
        _lib.check(self.L.dragon_gpu_halo_pack(self.h, 0, int(first), int(layers), int(faces), int(corners),
                                               ctypes.c_void_p(buf.data_ptr()), int(buf.is_cuda)))

    def unpack(self, first, layers, faces, corners, buf: torch.Tensor):
        self.grid._to_device()
        if buf.is_cuda:
            torch.cuda.current_stream(buf.device).synchronize()  # a receive may still be landing
        _lib.check(self.L.dragon_gpu_halo_unpack(self.h, 0, int(first), int(layers), int(faces), int(corners),
                                                 ctypes.c_void_p(buf.data_ptr()), int(buf.is_cuda)))
        self.grid._device_ran()

    def cfl_time(self):
        """This slab's CFL time, or None when its signal speeds are all zero."""
        self.grid._to_device()
        out = ctypes.c_double()
        rc = self.L.dragon_gpu_cfl_time(self.h, ctypes.byref(out))
        if rc == 4:
            return None
        _lib.check(rc)
        return out.value

    def try_step(self, dt) -> bool:
        self.grid._to_device()
        st = _lib.StepStatus()
        rc = self.L.dragon_gpu_unsplit_step(self.h, float(dt), ctypes.byref(st))
        if rc == 3:
            return False
        _lib.check(rc)
        self.grid._device_ran()
        return True

    def rollback(self):
        _lib.check(self.L.dragon_gpu_step_rollback(self.h))
        self.grid._device_ran()

    def initialize_B_fields(self):
        self.grid._to_device()
        _lib.check(self.L.dragon_gpu_initialize_B_fields(self.h))
        self.grid._device_ran()

    def get_w(self):
        return self.grid.w.copy()

    def set_w(self, a):
        self.grid.w[...] = a

    def get_B(self):
        return self.grid.B.copy()

    def set_B(self, a):
        self.grid.B[...] = a


class _DistBase:
    dim = 0

    def __init__(self, n, d, ghosts, config, group, slab_factory):
        self.config = config or Config()
        self.group = group
        self.rank = tdist.get_rank(group)
        self.parts = tdist.get_world_size(group)
        self.N = tuple(int(x) for x in n)
        self.d = tuple(float(x) for x in d)
        self.ghosts = valid_ghosts(ghosts, self.config.mhd)
        g = self.ghosts
        sizes = [child_size(self.N[0], self.parts, r) for r in range(self.parts)]
        if min(sizes) < g:
            raise ValueError(f"slabs of {min(sizes)} cells are thinner than the {g} ghost layers")
        self.sizes = sizes
        self.offset = sum(sizes[: self.rank])
        nl = (sizes[self.rank],) + self.N[1:]
        make = slab_factory or GpuSlab
        self.slab = make(self.dim, nl, tuple(d), g, self.config)
        if self.slab.ghosts != g:
            raise RuntimeError("slab ghost width differs from the distributed grid's")
        self.nl = sizes[self.rank]
        if hasattr(self.slab, "set_origin"):
            self.slab.set_origin((self.offset,))
        self.has_faces = self.slab.has_faces
        nccl = tdist.get_backend(group) == "nccl"
        self.comm_device = torch.device("cuda", torch.cuda.current_device()) if nccl else torch.device("cpu")
        self._boundary = BoundaryList()
        self._program = SlabProgram(self._boundary, self.rank, self.parts, self.dim)
        self.slab.set_entries(self._program.entries, self._program.fills)
        self._bufs = {}

    # -- topology -------------------------------------------------------------
    def _peer(self, r):
        return r if self.group is None else tdist.get_global_rank(self.group, r)

    @property
    def local(self):
        """This rank's slab (a Grid1D/2D/3D on the GPU for the default slab)."""
        return self.slab

    # -- boundary -------------------------------------------------------------
    @property
    def boundary(self) -> BoundaryList:
        return self._boundary

    @boundary.setter
    def boundary(self, b):
        self._boundary = as_list(b)
        self._program = SlabProgram(self._boundary, self.rank, self.parts, self.dim)
        self.slab.set_entries(self._program.entries, self._program.fills)

    # -- halo exchange ----------------------------------------------------------
    def _buf(self, key, count):
        t = self._bufs.get(key)
        if t is None or t.numel() != count:
            t = torch.empty(count, dtype=torch.float64, device=self.comm_device)
            if t.device.type == "cpu" and torch.cuda.is_available():
                t = t.pin_memory()
            self._bufs[key] = t
        return t

    def _layers(self, side, role, wrap):
        """(cell first, cell layers, face first, face layers) of the layers slab
        sends to / receives from its neighbour on `side` (0 low x, 1 high x).
        Between slabs, the high neighbour's faces [0, g] (its first face is the
        shared one, which the reference takes from the higher child,
        DistGrid.cpp:222-250) land on faces [nl, nl + g]; the periodic wrap
        moves g layers of faces like Periodic.cpp:55-62."""
        g, nl = self.ghosts, self.nl
        high_faces = g if wrap else g + 1
        if role == "send":
            if side == 0:
                return (0, g, 0, high_faces)
            return (nl - g, g, nl - g, g)
        if side == 0:
            return (-g, g, -g, g)
        return (nl, g, nl, high_faces)

    def _message(self, side, role, wrap, corners):
        c0, cn, f0, fn = self._layers(side, role, wrap)
        nc = self.slab.halo_count(cn, 0, corners)
        nfc = self.slab.halo_count(fn, 1, corners) if self.has_faces else 0
        return (c0, cn, f0, fn, nc, nfc)

    def _pack(self, msg, corners, buf):
        c0, cn, f0, fn, nc, nfc = msg
        self.slab.pack(c0, cn, 0, corners, buf[:nc])
        if nfc:
            self.slab.pack(f0, fn, 1, corners, buf[nc:nc + nfc])

    def _unpack(self, msg, corners, buf):
        c0, cn, f0, fn, nc, nfc = msg
        self.slab.unpack(c0, cn, 0, corners, buf[:nc])
        if nfc:
            self.slab.unpack(f0, fn, 1, corners, buf[nc:nc + nfc])

    def _exchange(self, pairs, wrap, corners):
        """pairs: [(side, peer)]: send to and receive from `peer` across `side`."""
        ops, recvs = [], []
        for side, peer in pairs:
            smsg = self._message(side, "send", wrap, corners)
            rmsg = self._message(side, "recv", wrap, corners)
            sbuf = self._buf(("s", side, wrap, corners), smsg[4] + smsg[5])
            rbuf = self._buf(("r", side, wrap, corners), rmsg[4] + rmsg[5])
            self._pack(smsg, corners, sbuf)
            ops.append(tdist.P2POp(tdist.isend, sbuf, self._peer(peer), self.group))
            ops.append(tdist.P2POp(tdist.irecv, rbuf, self._peer(peer), self.group))
            recvs.append((rmsg, rbuf))
        for req in tdist.batch_isend_irecv(ops):
            req.wait()
        for rmsg, rbuf in recvs:
            self._unpack(rmsg, corners, rbuf)

    def _wrap_exchange(self):
        """The x-periodic element's fill, at its place in the list: the first
        and the last slab exchange their outer layers."""
        P, r, c = self.parts, self.rank, int(self._program.wrap_corners)
        if P == 1:
            # a single slab wraps onto itself; low ghosts take the high layers and back
            self._exchange_self(c)
            return
        if r == 0:
            self._exchange([(0, P - 1)], True, c)
        elif r == P - 1:
            self._exchange([(1, 0)], True, c)

    def _exchange_self(self, corners):
        lo_send = self._message(1, "send", True, corners)   # layers [nl-g, nl) -> ghosts [-g, 0)
        hi_send = self._message(0, "send", True, corners)   # layers [0, g) -> ghosts [nl, nl+g)
        lo_recv = self._message(0, "recv", True, corners)
        hi_recv = self._message(1, "recv", True, corners)
        b1 = self._buf(("self", 1, corners), lo_send[4] + lo_send[5])
        b0 = self._buf(("self", 0, corners), hi_send[4] + hi_send[5])
        self._pack(lo_send, corners, b1)
        self._pack(hi_send, corners, b0)
        self._unpack(lo_recv, corners, b1)
        self._unpack(hi_recv, corners, b0)

    def _internal_exchange(self):
        pairs = []
        if self.rank > 0:
            pairs.append((0, self.rank - 1))
        if self.rank < self.parts - 1:
            pairs.append((1, self.rank + 1))
        if pairs:
            self._exchange(pairs, False, 1)

    def apply_boundary(self):
        """BoundaryList::apply on the distributed grid: the slab's part of the
        list, the x-periodic wrap at its place, then the halo exchange."""
        prog = self._program
        n = len(prog.entries)
        if prog.wrap_at is None:
            self.slab.apply_range(0, n)
        else:
            self.slab.apply_range(0, prog.wrap_at)
            self._wrap_exchange()
            self.slab.apply_range(prog.wrap_at + 1, n - prog.wrap_at - 1)
        self._internal_exchange()

    # -- reductions ---------------------------------------------------------------
    def _allreduce_min(self, v: float) -> float:
        t = torch.tensor([v], dtype=torch.float64, device=self.comm_device)
        tdist.all_reduce(t, op=tdist.ReduceOp.MIN, group=self.group)
        return float(t.item())

    def cfl_time(self) -> float:
        """CFL::cfl_time over the whole grid (CFL.cpp:88-137) on the current
        ghosts: the minimum of the slabs' CFL times."""
        local = self.slab.cfl_time()
        dt = self._allreduce_min(math.inf if local is None else local)
        if math.isinf(dt):
            raise RuntimeError("CFL timestep failed: max signal speed is zero")
        return dt

    # -- stepping -------------------------------------------------------------------
    def unsplit_step(self, dt: float):
        """DistGrid<T>::step (DistGrid.cpp:292-304): every slab steps or none
        does; raises StepFailed when any slab failed."""
        ok = self.slab.try_step(dt)
        if self._allreduce_min(1.0 if ok else 0.0) < 1.0:
            if ok:
                self.slab.rollback()
            raise StepFailed("a slab of the distributed grid failed its step", None)

    def _step_with_retry(self, t1: float, res: AdvanceResult) -> float:
        tol = self.config.timestep_tol
        while True:
            try:
                self.unsplit_step(t1)
                return t1
            except StepFailed:
                res.retries += 1
                t1 *= 0.5
                if t1 < tol:
                    raise

    def advance(self, dt: float, check_cfl: bool = True) -> AdvanceResult:
        """Grid::advance_unsplit (CFL.cpp:188-213) on the distributed grid."""
        res = AdvanceResult()
        tol = self.config.timestep_tol
        while dt > tol:
            self.apply_boundary()
            t1 = min(dt, self.cfl_time()) if check_cfl else dt
            t1 = self._step_with_retry(t1, res)
            dt -= t1
            res.steps += 1
            res.last_dt = t1
            res.time_advanced += t1
        return res

    def advance_steps(self, nsteps: int) -> AdvanceResult:
        """nsteps CFL-limited steps (the serial grid's advance_steps)."""
        res = AdvanceResult()
        for _ in range(int(nsteps)):
            self.apply_boundary()
            t1 = self._step_with_retry(self.cfl_time(), res)
            res.steps += 1
            res.last_dt = t1
            res.time_advanced += t1
        return res

    def initialize_B_fields(self):
        """Grid::initialize_B_fields (B_fields.cpp:117-149) after the
        distributed ghost fill."""
        if not self.has_faces:
            raise AttributeError("grid has no face-centred B")
        self.apply_boundary()
        self.slab.initialize_B_fields()

    # -- parent <-> slabs ---------------------------------------------------------------
    def scatter(self, w_full: np.ndarray, B_full: np.ndarray | None = None):
        """pushToChildren (DistGrid.cpp:115-204): this rank's slab of a padded
        global array, ghosts included (every rank passes the same array)."""
        g, o, nl = self.ghosts, self.offset, self.nl
        self.slab.set_w(np.ascontiguousarray(w_full[o:o + nl + 2 * g]))
        if self.has_faces:
            if B_full is None:
                raise ValueError("an MHD grid needs its face-centred B")
            self.slab.set_B(np.ascontiguousarray(B_full[o:o + nl + 2 * g + 1]))

    def gather(self):
        """loadFromChildren (DistGrid.cpp:208-289) onto every rank: the padded
        global cell array (and face B), x ghosts from the outer slabs."""
        g = self.ghosts
        w = self.slab.get_w()
        lo = 0 if self.rank == 0 else g
        hi = w.shape[0] if self.rank == self.parts - 1 else g + self.nl
        parts = self._allgather(w[lo:hi])
        w_full = np.concatenate(parts, axis=0)
        if not self.has_faces:
            return w_full
        B = self.slab.get_B()
        hi = B.shape[0] if self.rank == self.parts - 1 else g + self.nl
        B_full = np.concatenate(self._allgather(B[lo:hi]), axis=0)
        return w_full, B_full

    def _allgather(self, a: np.ndarray):
        outs = [None] * self.parts
        tdist.all_gather_object(outs, np.ascontiguousarray(a), group=self.group)
        return outs


class DistGrid1D(_DistBase):
    """DistGrid1D(nx, dx, ghosts=3) (DistGrid.hpp:30-47) across the ranks of `group`."""

    dim = 1

    def __init__(self, nx, dx, ghosts=3, config: Config | None = None, group=None, slab_factory=None):
        super().__init__((nx,), (dx,), ghosts, config, group, slab_factory)


class DistGrid2D(_DistBase):
    """DistGrid2D(nx, ny, dx, dy, ghosts=3) (DistGrid.hpp:49-66) across the ranks of `group`."""

    dim = 2

    def __init__(self, nx, ny, dx, dy, ghosts=3, config: Config | None = None, group=None, slab_factory=None):
        super().__init__((nx, ny), (dx, dy), ghosts, config, group, slab_factory)


class DistGrid3D(_DistBase):
    """DistGrid3D(nx, ny, nz, dx, dy, dz, ghosts=3) (DistGrid.hpp:68-86) across the ranks of `group`."""

    dim = 3

    def __init__(self, nx, ny, nz, dx, dy, dz, ghosts=3, config: Config | None = None, group=None,
                 slab_factory=None):
        super().__init__((nx, ny, nz), (dx, dy, dz), ghosts, config, group, slab_factory)
