"""Python handle on the DRAGON reference compiled as a library (oracle/_ref).

Test infrastructure: the parity tests and the CPU-baseline leg of bench.py use
this to run the reference's own Grid / DistGrid / Boundary / CFL code through
oracle/ref_shim.cpp. It is never on the product path.

Libraries (built by ``make -C oracle ref`` from the reference sources):
  libdragon_ref_hydro.so   hydro build
  libdragon_ref_mhd.so     MHD build, CT energy BETA_GATED (shipped form)
  libdragon_ref_mhd_rt.so  MHD build, CT energy chosen at run time
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_dp = ctypes.POINTER(ctypes.c_double)
_cache: dict[str, ctypes.CDLL] = {}


def ref_lib_path(variant: str) -> str:
    return os.path.join(REF_DIR, f"libdragon_ref_{variant}.so")


def available(variant: str = "hydro") -> bool:
    return os.path.exists(ref_lib_path(variant))


def load(variant: str) -> ctypes.CDLL:
    if variant in _cache:
        return _cache[variant]
    p = ref_lib_path(variant)
    if not os.path.exists(p):
        raise FileNotFoundError(f"{p} not built (make -C oracle ref)")
    L = ctypes.CDLL(p)
    L.ref_grid_new.restype = ctypes.c_void_p
    L.ref_grid_new.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 3 + [ctypes.c_int, ctypes.c_int]
    for fn in ("ref_grid_free", "ref_grid_ghosts", "ref_boundary_clear", "ref_boundary_commit",
               "ref_boundary_apply"):
        getattr(L, fn).argtypes = [ctypes.c_void_p]
    L.ref_grid_get_prim.argtypes = [ctypes.c_void_p, _dp]
    L.ref_grid_set_prim.argtypes = [ctypes.c_void_p, _dp]
    L.ref_boundary_add.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp]
    L.ref_cfl_time.argtypes = [ctypes.c_void_p, _dp, ctypes.c_char_p, ctypes.c_int]
    L.ref_unsplit_step.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_char_p, ctypes.c_int]
    L.ref_advance.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
    L.ref_split_step.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_char_p, ctypes.c_int]
    L.ref_advance_split.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
    L.ref_config.argtypes = [ctypes.c_int] * 5
    L.ref_cfl_speed.restype = ctypes.c_double
    L.ref_cfl_speed.argtypes = [_dp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
    L.ref_limiter.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp]
    L.ref_muscl.argtypes = [_dp, _dp, _dp, ctypes.c_double, _dp, _dp, _dp]
    L.ref_riemann_flux.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_double, ctypes.c_int, _dp, ctypes.c_char_p,
                                   ctypes.c_int]
    L.ref_face_mask.argtypes = [ctypes.c_char_p]
    if L.ref_is_mhd():
        L.ref_grid_get_faceB.argtypes = [ctypes.c_void_p, _dp]
        L.ref_grid_set_faceB.argtypes = [ctypes.c_void_p, _dp]
        L.ref_initialize_B_fields.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
    else:
        L.ref_exact_star.argtypes = [_dp, _dp, ctypes.c_double, _dp, _dp]
        L.ref_exact_sample.argtypes = [_dp, _dp, ctypes.c_double, _dp]
    _cache[variant] = L
    return L


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class RefError(RuntimeError):
    pass


class RefGrid:
    """A reference Grid{1,2,3}D (or DistGrid) with numpy access to its padded arrays."""

    def __init__(self, dim, n, d, ghosts=1, mhd=False, dist=False, ct_runtime=False, riemann=5, limiter=1, cfl=1,
                 ct_energy=2, core_count=0):
        self.variant = ("mhd_rt" if ct_runtime else "mhd") if mhd else "hydro"
        self.L = load(self.variant)
        self.dim = dim
        self.mhd = mhd
        self.cfgargs = (riemann, limiter, cfl, ct_energy, core_count)
        self.L.ref_config(*self.cfgargs)
        n3 = list(n) + [1] * (3 - len(n))
        d3 = list(d) + [0.0] * (3 - len(d))
        self.n = tuple(n3[:dim])
        self.h = self.L.ref_grid_new(dim, n3[0], n3[1], n3[2], d3[0], d3[1], d3[2], int(ghosts), int(dist))
        self.ghosts = self.L.ref_grid_ghosts(self.h)
        self.nf = 8 if mhd else 5
        self.shape = tuple(x + 2 * self.ghosts for x in self.n) + (self.nf,)
        self.bshape = tuple(x + 1 + 2 * self.ghosts for x in self.n) + (3,)

    def close(self):
        if self.h:
            self.L.ref_grid_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _cfg(self):
        self.L.ref_config(*self.cfgargs)

    def get_prim(self) -> np.ndarray:
        a = np.zeros(self.shape)
        self.L.ref_grid_get_prim(self.h, _p(a))
        return a

    def set_prim(self, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.shape == self.shape, (a.shape, self.shape)
        self.L.ref_grid_set_prim(self.h, _p(a))

    def get_faceB(self) -> np.ndarray:
        a = np.zeros(self.bshape)
        self.L.ref_grid_get_faceB(self.h, _p(a))
        return a

    def set_faceB(self, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.shape == self.bshape
        self.L.ref_grid_set_faceB(self.h, _p(a))

    def set_boundary(self, entries):
        """entries: iterable of (type, faces, corners, state-or-None) like dragon_bc_desc."""
        self.L.ref_boundary_clear(self.h)
        for (t, faces, corners, state) in entries:
            st = np.zeros(8)
            if state is not None:
                st[: len(state)] = state
            if self.L.ref_boundary_add(self.h, int(t), int(faces), int(corners), _p(st)) != 0:
                raise RefError("bad boundary type")
        self.L.ref_boundary_commit(self.h)

    def apply_boundary(self):
        self._cfg()
        self.L.ref_boundary_apply(self.h)

    def initialize_B_fields(self):
        msg = ctypes.create_string_buffer(256)
        if self.L.ref_initialize_B_fields(self.h, msg, 256):
            raise RefError(msg.value.decode())

    def cfl_time(self) -> float:
        self._cfg()
        out = ctypes.c_double()
        msg = ctypes.create_string_buffer(256)
        if self.L.ref_cfl_time(self.h, ctypes.byref(out), msg, 256):
            raise RefError(msg.value.decode())
        return out.value

    def unsplit_step(self, dt: float):
        self._cfg()
        msg = ctypes.create_string_buffer(256)
        if self.L.ref_unsplit_step(self.h, float(dt), msg, 256):
            raise RefError(msg.value.decode())

    def advance(self, dt: float, check_cfl: bool = True):
        self._cfg()
        msg = ctypes.create_string_buffer(256)
        if self.L.ref_advance(self.h, float(dt), int(check_cfl), msg, 256):
            raise RefError(msg.value.decode())

    def split_step(self, dt: float):
        self._cfg()
        msg = ctypes.create_string_buffer(256)
        if self.L.ref_split_step(self.h, float(dt), msg, 256):
            raise RefError(msg.value.decode())

    def advance_split(self, dt: float, check_cfl: bool = True):
        self._cfg()
        msg = ctypes.create_string_buffer(256)
        if self.L.ref_advance_split(self.h, float(dt), int(check_cfl), msg, 256):
            raise RefError(msg.value.decode())

    def step_cfl(self) -> float:
        """One step of advance(cfl_time()): ghost fill, CFL dt, one step."""
        self.apply_boundary()
        dt = self.cfl_time()
        self.advance(dt)
        return dt


def bc_entries_from(boundary_list):
    """Converts a dragon_b200.boundary list into RefGrid.set_boundary entries."""
    out = []
    for e in boundary_list:
        st = list(e.state()) if e.state() else None
        out.append((e.kind, e.get_faces(), e.corners, st))
    return out
