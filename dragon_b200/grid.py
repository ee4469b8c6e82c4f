"""Grid1D / Grid2D / Grid3D resident on the GPU, mirroring DRAGON's Grid API.

The classes keep the reference's constructor arguments, ghost policy,
``boundary`` member, ``advance(dt, check_cfl=True)``, ``unsplit_step(dt)``,
``initialize_B_fields()`` and cell access with ghost coordinates
(DRAGON/Hydro/Grid.hpp:19-144). A host mirror of the padded array in the
reference's memory order (last index fastest, ghosts included) is synced
lazily: reads after a device step download, writes mark the mirror dirty and
the next device call uploads it.

Errors follow the reference: a failing step raises (``StepFailed``), and the
CFL-zero and timestep-underflow cases raise too, where the reference throws or
exits (CFL.cpp:102-117,205-208).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .boundary import IGNORE, USER, BoundaryList, as_list

# Config ids (DRAGON/Config.h)
RIEMANN_EXACT, RIEMANN_HLL, RIEMANN_HLLC, RIEMANN_HLLD, RIEMANN_HLLE, RIEMANN_HLLX, RIEMANN_ROE = range(7)
LIMITER_MINMOD, LIMITER_MC, LIMITER_VANLEER, LIMITER_SUPERBEE, LIMITER_VANALBADA = range(5)
CFL_MAX, CFL_ADD = 0, 1
CT_CONSV_TOTAL_E, CT_CONSV_THERMAL, CT_CONSV_BETA_GATED = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
GUESS_MEAN, GUESS_ANALYTIC, GUESS_LEARNED, GUESS_PERFECT = 0, 1, 2, 3


@dataclass
class Config:
    """Runtime form of DRAGON/Config.h's switches; defaults are the shipped ones."""

    mhd: bool = False
    riemann: int = RIEMANN_HLLX
    limiter: int = LIMITER_MC
    cfl: int = CFL_ADD
    ct_energy: int = CT_CONSV_BETA_GATED
    exact_max_iters: int = 6
    exact_tol: float = 1e-12
    cfl_coeff: float = 0.3
    timestep_tol: float = 1e-14
    precision: int = PREC_FP64
    exact_guess: int = GUESS_MEAN
    perfect_guess_err_exp: int = 0

    def to_c(self) -> _lib.DragonConfig:
        c = _lib.DragonConfig()
        c.mhd = int(self.mhd)
        c.riemann = self.riemann
        c.limiter = self.limiter
        c.cfl = self.cfl
        c.ct_energy = self.ct_energy
        c.exact_max_iters = self.exact_max_iters
        c.exact_tol = self.exact_tol
        c.cfl_coeff = self.cfl_coeff
        c.timestep_tol = self.timestep_tol
        c.precision = self.precision
        c.exact_guess = self.exact_guess
        c.perfect_guess_err_exp = self.perfect_guess_err_exp
        return c


class StepFailed(RuntimeError):
    """Grid::unsplit_step threw (unphysical state / no physical flux)."""

    def __init__(self, msg, status):
        super().__init__(msg)
        self.status = status


@dataclass
class AdvanceResult:
    steps: int = 0
    retries: int = 0
    last_dt: float = 0.0
    time_advanced: float = 0.0
    pivots_exact: int = 0
    hlld_to_hlle: int = 0
    newton_iters: int = 0
    exact_calls: int = 0
    trrs: int = 0
    muscl_first_order: int = 0
    extra: dict = field(default_factory=dict)


def _result(st: _lib.AdvanceStats) -> AdvanceResult:
    return AdvanceResult(st.steps, st.retries, st.last_dt, st.time_advanced, st.pivots_exact, st.hlld_to_hlle,
                         st.newton_iters, st.exact_calls, st.trrs, st.muscl_first_order)


def custom_slabs(n, g, faces, reach=None):
    """(axis, first, layers) per face in the mask `faces` of a grid with
    interior extents n and g ghosts: the face's g ghost layers and `reach`
    interior layers next to them (None: g). None when the slabs of an axis
    would cover it end to end (a full round trip is then as cheap)."""
    r = g if reach is None else int(reach)
    out = []
    for a, na in enumerate(n):
        neg, pos = faces & (1 << (2 * a)), faces & (1 << (2 * a + 1))
        if (neg or pos) and (bool(neg) + bool(pos)) * (g + r) >= na + 2 * g - 1:
            return None
        if neg:
            out.append((a, -g, g + r))
        if pos:
            out.append((a, na - r, g + r))
    return out


def _slab_index(dim, axis, first, layers, g):
    sl = [slice(None)] * dim
    sl[axis] = slice(first + g, first + g + layers)
    return tuple(sl)


def slab_to_buffer(arr, dim, axis, first, layers, g):
    """Layers [first, first + layers) along `axis` of a padded host array (last
    axis: fields) in the order of dragon_gpu_halo_pack's buffer with corners:
    field, layer, then the transverse axes over their padded extent (last
    fastest)."""
    return np.ascontiguousarray(np.moveaxis(np.moveaxis(arr[_slab_index(dim, axis, first, layers, g)], axis, 0), -1, 0))


def buffer_to_slab(buf, arr, dim, axis, first, layers, g):
    """The inverse of slab_to_buffer: writes a halo buffer into those layers of arr."""
    nf = arr.shape[-1]
    trans = [arr.shape[b] for b in range(dim) if b != axis]
    arr[_slab_index(dim, axis, first, layers, g)] = np.moveaxis(np.moveaxis(buf.reshape(nf, layers, *trans), 0, -1), 0, axis)


class _SlabView:
    """The grid as a user GhostFill element sees it on the ghost-slab path
    (_GridBase._apply_custom): w, B, grid[i, j] and the geometry read and
    write the host mirror directly, which is current only in the slabs along
    the element's faces. Everything else is the grid's."""

    def __init__(self, grid):
        object.__setattr__(self, "_grid", grid)

    @property
    def w(self) -> np.ndarray:
        return self._grid._w

    @property
    def B(self) -> np.ndarray:
        if self._grid._B is None:
            raise AttributeError("grid has no face-centred B")
        return self._grid._B

    def _B_(self):
        return self.B

    def __getitem__(self, idx):
        return self._grid._w[self._grid._index(idx)]

    def __setitem__(self, idx, value):
        self._grid._w[self._grid._index(idx)] = np.asarray(value, dtype=np.float64)[: self._grid.nfields]

    def __getattr__(self, name):
        return getattr(self._grid, name)


class _GridBase:
    dim = 0

    def __init__(self, n, d, ghosts, config: Config | None):
        self.config = config or Config()
        self._lib = _lib.load()
        n3 = list(n) + [1] * (3 - len(n))
        d3 = list(d) + [0.0] * (3 - len(d))
        h = ctypes.c_void_p()
        cfg = self.config.to_c()
        _lib.check(self._lib.dragon_gpu_grid_create(self.dim, n3[0], n3[1], n3[2], d3[0], d3[1], d3[2], int(ghosts),
                                                    ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        dim = ctypes.c_int()
        nn = (ctypes.c_int * 3)()
        g = ctypes.c_int()
        nf = ctypes.c_int()
        _lib.check(self._lib.dragon_gpu_grid_info(h, ctypes.byref(dim), nn, ctypes.byref(g), ctypes.byref(nf)))
        self.n = tuple(nn[i] for i in range(self.dim))
        self.ghosts = g.value
        self.nfields = nf.value
        shape = tuple(x + 2 * self.ghosts for x in self.n) + (self.nfields,)
        self._w = np.zeros(shape, dtype=np.float64)
        self._B = None
        if self.config.mhd and self.dim >= 2:
            self._B = np.zeros(tuple(x + 1 + 2 * self.ghosts for x in self.n) + (3,), dtype=np.float64)
        self._host_dirty = True      # host mirror newer than device
        self._dev_dirty = False      # device newer than host mirror
        self._boundary = BoundaryList()
        self._push_boundary()

    # -- lifecycle ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.dragon_gpu_grid_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- sync --------------------------------------------------------------
    def _ptr(self, a):
        return a.ctypes.data_as(_lib.c_double_p)

    def upload(self):
        _lib.check(self._lib.dragon_gpu_upload_prim(self._h, self._ptr(self._w)))
        if self._B is not None:
            _lib.check(self._lib.dragon_gpu_upload_faceB(self._h, self._ptr(self._B)))
        self._host_dirty = False

    def download(self):
        _lib.check(self._lib.dragon_gpu_download_prim(self._h, self._ptr(self._w)))
        if self._B is not None:
            _lib.check(self._lib.dragon_gpu_download_faceB(self._h, self._ptr(self._B)))
        self._dev_dirty = False

    def _to_device(self):
        if self._host_dirty:
            self.upload()

    def _device_ran(self):
        self._dev_dirty = True

    @property
    def w(self) -> np.ndarray:
        """The padded primitive array (host mirror; modifications are uploaded
        before the next device call)."""
        if self._dev_dirty:
            self.download()
        self._host_dirty = True
        return self._w

    @property
    def B(self) -> np.ndarray:
        """Face-centred B, padded (n+1 per axis), 3 components (MHD 2D/3D)."""
        if self._B is None:
            raise AttributeError("grid has no face-centred B")
        if self._dev_dirty:
            self.download()
        self._host_dirty = True
        return self._B

    def _B_(self):
        return self.B

    def interior(self) -> np.ndarray:
        g = self.ghosts
        sl = tuple(slice(g, g + x) for x in self.n)
        return self.w[sl]

    def _index(self, idx):
        if not isinstance(idx, tuple):
            idx = (idx,)
        if len(idx) != self.dim:
            raise IndexError(f"{self.dim}D grid needs {self.dim} indices")
        g = self.ghosts
        out = []
        for i, n in zip(idx, self.n):
            if not (-g <= i < n + g):
                raise IndexError(f"index {i} outside [-{g}, {n + g})")
            out.append(i + g)
        return tuple(out)

    def __getitem__(self, idx):
        return self.w[self._index(idx)]

    def __setitem__(self, idx, value):
        self.w[self._index(idx)] = np.asarray(value, dtype=np.float64)[: self.nfields]

    # -- boundary ------------------------------------------------------------
    @property
    def boundary(self) -> BoundaryList:
        return self._boundary

    @boundary.setter
    def boundary(self, b):
        self._boundary = as_list(b)
        self._push_boundary()

    def _push_boundary(self):
        els = list(self._boundary)
        arr = (_lib.BCDesc * max(1, len(els)))()
        for k, e in enumerate(els):
            # user elements run on the host; on the device they only cover their faces
            arr[k].type = IGNORE if e.is_custom else e.kind
            arr[k].faces = e.get_faces()
            arr[k].corners = int(e.corners)
            st = list(e.state()) + [0.0] * 8
            for q in range(8):
                arr[k].state[q] = st[q]
        _lib.check(self._lib.dragon_gpu_set_boundary(self._h, arr, len(els)))
        for k, e in enumerate(els):
            if e.kind == USER:
                e.bind(self._lib, self._h, k)

    def _apply_boundary_host(self):
        """BoundaryList::apply (BoundaryList.hpp:79-93) with user elements: the
        device applies the runs of built-in entries (the implicit Outflow first),
        each user element's apply(grid) runs on the host between them, on the
        slabs along its faces only (_apply_custom)."""
        els = list(self._boundary)
        off = int(self._lib.dragon_gpu_boundary_entries(self._h)) - len(els)
        start = 0  # first device entry not yet applied
        for k, e in enumerate(els + [None]):
            if e is not None and not e.is_custom:
                continue
            stop = off + k
            if stop > start:
                self._to_device()
                _lib.check(self._lib.dragon_gpu_apply_boundary_range(self._h, start, stop - start))
                self._device_ran()
            if e is not None:
                self._apply_custom(e)
            start = off + k + 1

    def _custom_slabs(self, e):
        """The layers a user element sees, per face of its mask: its ghost
        layers and the `reach` interior layers next to them (GhostFill.reach,
        default the ghost width), over the whole padded transverse extent.
        Returns (axis, first, layers) in interior coordinates, or None when the
        slabs would cover an axis end to end."""
        return custom_slabs(self.n, self.ghosts, e.get_faces(), e.reach)

    def _slab_copy(self, axis, first, layers, faces, down):
        """Copies layers [first, first + layers) along `axis` (cells, or face B
        with faces = 1) between the device state and the host mirror, over the
        padded transverse extent: down = True device to host."""
        arr = self._B if faces else self._w
        count = ctypes.c_longlong()
        _lib.check(self._lib.dragon_gpu_halo_size(self._h, axis, layers, faces, 1, ctypes.byref(count)))
        if down:
            buf = np.empty(count.value)
            _lib.check(self._lib.dragon_gpu_halo_pack(self._h, axis, first, layers, faces, 1, self._ptr(buf), 0))
            buffer_to_slab(buf, arr, self.dim, axis, first, layers, self.ghosts)
        else:
            buf = slab_to_buffer(arr, self.dim, axis, first, layers, self.ghosts)
            _lib.check(self._lib.dragon_gpu_halo_unpack(self._h, axis, first, layers, faces, 1, self._ptr(buf), 0))

    def _apply_custom(self, e):
        """One user element on the host. When the device holds the newer state,
        only the slabs along the element's faces cross the host link: they are
        copied into the host mirror, the element's apply runs on a view of the
        mirror that triggers no transfer, and the same slabs go back (cells,
        and face B for MHD grids). Slabs that would span a whole axis fall
        back to apply on the grid itself (a full round trip)."""
        slabs = self._custom_slabs(e)
        if slabs is None:
            e.apply(self)
            return
        self._to_device()
        if self._dev_dirty:
            for a, first, layers in slabs:
                self._slab_copy(a, first, layers, 0, True)
                if self._B is not None:
                    self._slab_copy(a, first, layers + 1, 1, True)
        e.apply(_SlabView(self))
        for a, first, layers in slabs:
            self._slab_copy(a, first, layers, 0, False)
            if self._B is not None:
                self._slab_copy(a, first, layers + 1, 1, False)

    def _advance_host(self, dt: float, check_cfl: bool, split: bool) -> AdvanceResult:
        """Grid::advance_unsplit / advance_split (CFL.cpp:160-213) driven from
        the host, for boundary lists with user elements."""
        tol = self.config.timestep_tol
        res = AdvanceResult()
        while dt > tol:
            self._apply_boundary_host()
            t1 = min(dt, self.cfl_time()) if check_cfl else dt
            while True:
                try:
                    (self.split_step if split else self.unsplit_step)(t1)
                    break
                except StepFailed:
                    res.retries += 1
                    t1 *= 0.5
                    if t1 < tol:
                        raise
            dt -= t1
            res.steps += 1
            res.last_dt = t1
            res.time_advanced += t1
        return res

    def apply_boundary(self):
        if self._boundary.has_custom():
            self._push_boundary()
            self._apply_boundary_host()
            return
        self._push_boundary()
        self._to_device()
        _lib.check(self._lib.dragon_gpu_apply_boundary(self._h))
        self._device_ran()

    # -- stepping --------------------------------------------------------------
    def cfl_time(self) -> float:
        """CFL::cfl_time on the current ghosts (CFL.cpp:88-137)."""
        self._to_device()
        out = ctypes.c_double()
        _lib.check(self._lib.dragon_gpu_cfl_time(self._h, ctypes.byref(out)))
        return out.value

    def unsplit_step(self, dt: float):
        """Grid::unsplit_step (Unsplit.cpp:28-206): raises StepFailed, committing
        nothing, when the reference would throw."""
        self._to_device()
        st = _lib.StepStatus()
        rc = self._lib.dragon_gpu_unsplit_step(self._h, float(dt), ctypes.byref(st))
        if rc == 3:
            raise StepFailed(self._lib.dragon_gpu_last_error().decode(), st)
        _lib.check(rc)
        self._device_ran()

    def split_step(self, dt: float):
        """Grid::split_step (Splitting.cpp:118-217): Strang sequence of 1D
        sweeps (hydro); raises StepFailed, committing nothing, on failure."""
        self._to_device()
        st = _lib.StepStatus()
        rc = self._lib.dragon_gpu_split_step(self._h, float(dt), ctypes.byref(st))
        if rc == 3:
            raise StepFailed(self._lib.dragon_gpu_last_error().decode(), st)
        _lib.check(rc)
        self._device_ran()

    def advance_split(self, dt: float, check_cfl: bool = True) -> AdvanceResult:
        """Grid::advance_split (CFL.cpp:160-184): the advance loop around split_step."""
        if self._boundary.has_custom():
            return self._advance_host(dt, check_cfl, split=True)
        self._to_device()
        st = _lib.AdvanceStats()
        rc = self._lib.dragon_gpu_advance_split(self._h, float(dt), int(bool(check_cfl)), ctypes.byref(st))
        self._device_ran()
        _lib.check(rc)
        return _result(st)

    def advance(self, dt: float, check_cfl: bool = True) -> AdvanceResult:
        """Grid::advance (CFL.cpp:151-213), run entirely on the device (on the
        host-driven path when the boundary list has user elements)."""
        if self._boundary.has_custom():
            return self._advance_host(dt, check_cfl, split=False)
        self._to_device()
        st = _lib.AdvanceStats()
        rc = self._lib.dragon_gpu_advance(self._h, float(dt), int(bool(check_cfl)), ctypes.byref(st))
        self._device_ran()
        _lib.check(rc)
        return _result(st)

    advance_unsplit = advance

    def advance_steps(self, nsteps: int) -> AdvanceResult:
        """nsteps CFL-limited steps (each the reference's advance(cfl_time()))."""
        if self._boundary.has_custom():
            res = AdvanceResult()
            for _ in range(int(nsteps)):
                self._apply_boundary_host()
                r = self._advance_host(self.cfl_time(), True, split=False)
                res.steps += r.steps
                res.retries += r.retries
                res.last_dt = r.last_dt
                res.time_advanced += r.time_advanced
            return res
        self._to_device()
        st = _lib.AdvanceStats()
        rc = self._lib.dragon_gpu_advance_steps(self._h, int(nsteps), ctypes.byref(st))
        self._device_ran()
        _lib.check(rc)
        return _result(st)

    def advance_steps_async(self, nsteps: int) -> None:
        """Enqueues nsteps CFL-limited steps on the grid's stream and returns
        without waiting for the device; advance_wait() completes them (retries
        included). The grid takes no other call in between."""
        if self._boundary.has_custom():
            raise RuntimeError("boundary lists with user elements advance from the host")
        self._to_device()
        _lib.check(self._lib.dragon_gpu_advance_steps_async(self._h, int(nsteps)))

    def advance_wait(self) -> AdvanceResult:
        st = _lib.AdvanceStats()
        rc = self._lib.dragon_gpu_advance_wait(self._h, ctypes.byref(st))
        self._device_ran()
        _lib.check(rc)
        return _result(st)

    def initialize_B_fields(self):
        """Grid::initialize_B_fields (B_fields.cpp:117-149)."""
        self._push_boundary()
        self._to_device()
        _lib.check(self._lib.dragon_gpu_initialize_B_fields(self._h))
        self._device_ran()

    def launch_count(self) -> int:
        return int(self._lib.dragon_gpu_launch_count(self._h))

    # -- exact solver: Newton statistics, sample log, learned guess ----------
    def newton_stats(self, reset: bool = False) -> dict:
        """Exact-solver counters summed over every step since creation / reset."""
        st = _lib.NewtonStats()
        _lib.check(self._lib.dragon_gpu_newton_stats(self._h, ctypes.byref(st), int(bool(reset))))
        return {name: int(getattr(st, name)) for name, _ in st._fields_}

    def newton_log(self, capacity: int, stride: int = 1):
        """Starts logging converged Newton solves (every stride-th, up to capacity rows); 0 stops."""
        _lib.check(self._lib.dragon_gpu_newton_log_enable(self._h, int(capacity), int(stride)))

    def newton_log_rows(self, max_rows: int | None = None) -> np.ndarray:
        """Stored log rows: rhoL, vxL, pL, rhoR, vxR, pR, p*, iterations (face-normal frame)."""
        rows_p = ctypes.c_void_p()
        n = ctypes.c_longlong()
        _lib.check(self._lib.dragon_gpu_newton_log_device(self._h, ctypes.byref(rows_p), ctypes.byref(n)))
        m = n.value if max_rows is None else min(n.value, int(max_rows))
        out = np.zeros((m, 8))
        got = ctypes.c_longlong()
        if m:
            _lib.check(self._lib.dragon_gpu_newton_log_read(self._h, self._ptr(out), m, ctypes.byref(got)))
        return out[:got.value] if m else out

    def set_network(self, net) -> None:
        """Copies a learned-guess network (dragon_b200.learned.Network) into the grid."""
        _lib.check(self._lib.dragon_gpu_grid_set_mlp(self._h, net._h))

    def getGhosts(self) -> int:
        return self.ghosts


class Grid1D(_GridBase):
    """Grid1D(size, dx, ghosts=1) (Grid.hpp:40-59)."""

    dim = 1

    def __init__(self, size: int, dx: float, ghosts: int = 1, config: Config | None = None):
        super().__init__((size,), (dx,), ghosts, config)
        self.dx = dx

    def getSize(self):
        return self.n[0]


class Grid2D(_GridBase):
    """Grid2D(nx, ny, dx, dy, ghosts=1) (Grid.hpp:61-101)."""

    dim = 2

    def __init__(self, nx: int, ny: int, dx: float, dy: float, ghosts: int = 1, config: Config | None = None):
        super().__init__((nx, ny), (dx, dy), ghosts, config)
        self.dx, self.dy = dx, dy

    def getSizeX(self):
        return self.n[0]

    def getSizeY(self):
        return self.n[1]


class Grid3D(_GridBase):
    """Grid3D(nx, ny, nz, dx, dy, dz, ghosts=2) (Grid.hpp:103-144)."""

    dim = 3

    def __init__(self, nx, ny, nz, dx, dy, dz, ghosts: int = 2, config: Config | None = None):
        super().__init__((nx, ny, nz), (dx, dy, dz), ghosts, config)
        self.dx, self.dy, self.dz = dx, dy, dz

    def getSizeX(self):
        return self.n[0]

    def getSizeY(self):
        return self.n[1]

    def getSizeZ(self):
        return self.n[2]
