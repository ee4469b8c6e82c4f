"""Python handle on the C restatement of the reference (oracle/liboracle_*.so).

Test infrastructure: the parity oracle used by tests/, the smoke check and the
bench's CPU leg when the reference library itself (oracle/_ref) is not
available. Same interface as oracle.refgrid.RefGrid. The libraries are built
from committed C sources (``make -C oracle port``), so they exist wherever the
repository is built.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_dp = ctypes.POINTER(ctypes.c_double)
_libs: dict[bool, ctypes.CDLL] = {}


def lib_path(mhd: bool) -> str:
    return os.path.join(HERE, f"liboracle_{'mhd' if mhd else 'hydro'}.so")


def load(mhd: bool) -> ctypes.CDLL:
    if mhd in _libs:
        return _libs[mhd]
    p = lib_path(mhd)
    if not os.path.exists(p):
        subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
    L = ctypes.CDLL(p)
    L.ora_set_options.argtypes = [ctypes.c_int] * 5 + [ctypes.c_double] * 3
    L.ora_grid_new.restype = ctypes.c_void_p
    L.ora_grid_new.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 3 + [ctypes.c_int]
    for fn in ("ora_grid_free", "ora_grid_ghosts", "ora_boundary_clear", "ora_boundary_apply",
               "ora_initialize_B_fields"):
        getattr(L, fn).argtypes = [ctypes.c_void_p]
    for fn in ("ora_grid_set_prim", "ora_grid_get_prim", "ora_grid_set_faceB", "ora_grid_get_faceB"):
        getattr(L, fn).argtypes = [ctypes.c_void_p, _dp]
    L.ora_boundary_add.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp]
    L.ora_cfl_time.argtypes = [ctypes.c_void_p, _dp]
    L.ora_unsplit_step.argtypes = [ctypes.c_void_p, ctypes.c_double]
    L.ora_advance.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                              ctypes.POINTER(ctypes.c_int)]
    L.ora_limiter.restype = ctypes.c_double
    L.ora_limiter.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double]
    L.ora_muscl.argtypes = [_dp, _dp, _dp, ctypes.c_double, _dp, _dp, _dp]
    L.ora_riemann_flux.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_double, ctypes.c_int, _dp]
    L.ora_exact_star.argtypes = [_dp, _dp, ctypes.c_double, _dp, _dp, ctypes.POINTER(ctypes.c_int)]
    L.ora_exact_log_start.argtypes = [_dp, ctypes.c_long]
    L.ora_exact_log_stop.restype = ctypes.c_long
    _libs[mhd] = L
    return L


def _p(a):
    return a.ctypes.data_as(_dp)


class PortError(RuntimeError):
    pass


class PortGrid:
    """Same interface as oracle.refgrid.RefGrid, backed by the C restatement."""

    def __init__(self, dim, n, d, ghosts=1, mhd=False, riemann=5, limiter=1, cfl=1, ct_energy=2, exact_max_iters=6,
                 exact_tol=1e-12, cfl_coeff=0.3, timestep_tol=1e-14, **_ignored):
        self.L = load(mhd)
        self.mhd = mhd
        self.dim = dim
        self.opts = (riemann, limiter, cfl, ct_energy, exact_max_iters, exact_tol, cfl_coeff, timestep_tol)
        n3 = list(n) + [1] * (3 - len(n))
        d3 = list(d) + [0.0] * (3 - len(d))
        self.n = tuple(n3[:dim])
        self.h = self.L.ora_grid_new(dim, n3[0], n3[1], n3[2], d3[0], d3[1], d3[2], int(ghosts))
        self.ghosts = self.L.ora_grid_ghosts(self.h)
        self.nf = 8 if mhd else 5
        self.shape = tuple(x + 2 * self.ghosts for x in self.n) + (self.nf,)
        self.bshape = tuple(x + 1 + 2 * self.ghosts for x in self.n) + (3,)

    def _o(self):
        self.L.ora_set_options(*self.opts)

    def close(self):
        if self.h:
            self.L.ora_grid_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_prim(self):
        a = np.zeros(self.shape)
        self.L.ora_grid_get_prim(self.h, _p(a))
        return a

    def set_prim(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.shape == self.shape
        self.L.ora_grid_set_prim(self.h, _p(a))

    def get_faceB(self):
        a = np.zeros(self.bshape)
        self.L.ora_grid_get_faceB(self.h, _p(a))
        return a

    def set_faceB(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.shape == self.bshape
        self.L.ora_grid_set_faceB(self.h, _p(a))

    def set_boundary(self, entries):
        self.L.ora_boundary_clear(self.h)
        for (t, faces, corners, state) in entries:
            st = np.zeros(8)
            if state is not None:
                st[: len(state)] = state
            if self.L.ora_boundary_add(self.h, int(t), int(faces), int(corners), _p(st)):
                raise PortError("bad boundary entry")

    def apply_boundary(self):
        self._o()
        self.L.ora_boundary_apply(self.h)

    def initialize_B_fields(self):
        self._o()
        if self.L.ora_initialize_B_fields(self.h):
            raise PortError("initialize_B_fields needs a 2D/3D MHD grid")

    def cfl_time(self):
        self._o()
        out = ctypes.c_double()
        if self.L.ora_cfl_time(self.h, ctypes.byref(out)):
            raise PortError("CFL timestep failed: max signal speed is zero")
        return out.value

    def unsplit_step(self, dt):
        self._o()
        if self.L.ora_unsplit_step(self.h, float(dt)):
            raise PortError("Unphysical state would be produced")

    def advance(self, dt, check_cfl=True):
        self._o()
        steps, retries = ctypes.c_int(), ctypes.c_int()
        rc = self.L.ora_advance(self.h, float(dt), int(check_cfl), ctypes.byref(steps), ctypes.byref(retries))
        if rc:
            raise PortError({2: "CFL timestep failed: max signal speed is zero",
                             3: "Timestep has fallen below minimum"}.get(rc, "advance failed"))
        return steps.value, retries.value

    def step_cfl(self):
        self.apply_boundary()
        dt = self.cfl_time()
        self.advance(dt)
        return dt


def run_steps_2d(w0, dx, dy, steps, riemann=5, limiter=1, boundary=(), ghosts=2):
    """Convenience: a 2D hydro grid advanced `steps` CFL steps; returns the padded array."""
    g = ghosts
    nx, ny = w0.shape[0] - 2 * g, w0.shape[1] - 2 * g
    P = PortGrid(2, (nx, ny), (dx, dy), ghosts=g, riemann=riemann, limiter=limiter)
    P.set_prim(w0)
    P.set_boundary(boundary)
    for _ in range(steps):
        P.step_cfl()
    return P.get_prim()


class ExactLog:
    """Context manager recording the hydro oracle's Newton-branch exact solves:
    rows (rhoL, vxL, pL, rhoR, vxR, pR, p*, iterations) in the face-normal frame; the
    iteration count is negated when the cap ended the solve."""

    def __init__(self, cap=1 << 20):
        self.buf = np.zeros((cap, 8))
        self.n = 0

    def __enter__(self):
        load(False).ora_exact_log_start(_p(self.buf), self.buf.shape[0])
        return self

    def __exit__(self, *exc):
        self.n = load(False).ora_exact_log_stop()
        return False

    @property
    def rows(self):
        return self.buf[:min(self.n, self.buf.shape[0])]
