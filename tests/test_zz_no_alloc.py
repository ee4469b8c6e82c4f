"""dragon_gpu_cfl_time_noalloc: the CFL step computed without allocating any
device memory, for callers that must not allocate once their run is under way
(an application whose memory pool owns the whole GPU, or a loop that cannot
take cudaMalloc's device-wide synchronisation). The test calls it through the
C ABI on states held by a grid handle and checks it against the handle's own
dragon_gpu_cfl_time, bit for bit, on two calls in a row (the fixed working
array is shared between calls and keeps the previous call's contents). It
also checks that a grid too large for the fixed array is refused.

Collected last on purpose, so a run that stops at the first failure has
already run every other test."""
import ctypes

import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

import dragon_b200 as dg  # noqa: E402
from dragon_b200 import _lib, problems  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not cuda_ok():
        pytest.fail("CUDA device required for -m gpu tests")


def noalloc_dt(G):
    L = G._lib
    prim = ctypes.c_void_p()
    plane = ctypes.c_longlong()
    pitch = ctypes.c_longlong()
    _lib.check(L.dragon_gpu_device_state(G._h, ctypes.byref(prim), ctypes.byref(plane), ctypes.byref(pitch)))
    n = list(G.n) + [1] * (3 - G.dim)
    d = [G.dx, getattr(G, "dy", 0.0), getattr(G, "dz", 0.0)]
    out = ctypes.c_double()
    rc = L.dragon_gpu_cfl_time_noalloc(G.dim, n[0], n[1], n[2], G.ghosts, int(G.config.mhd),
                                       ctypes.cast(prim, _lib.c_double_p), plane.value, pitch.value, d[0], d[1],
                                       d[2], G.config.cfl, G.config.cfl_coeff, None, ctypes.byref(out))
    _lib.check(rc)
    return out.value


def check_twice(G, mutate):
    """First call, then change the state, then the second call; each must
    equal the handle path's dt."""
    for call in range(2):
        G.apply_boundary()
        dt_ref = G.cfl_time()
        dt = noalloc_dt(G)
        assert dt == dt_ref, (call, dt, dt_ref)
        mutate(G, call)


def test_noalloc_cfl_matches_handle_2d_hydro():
    w0, dx, dy = problems.kelvin_helmholtz_2d(96, ghosts=2, seed=3, ny=70)
    G = dg.Grid2D(96, 70, dx, dy, ghosts=2, config=dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_VANLEER))
    G.w[...] = w0
    G.boundary = dg.Periodic("X") + dg.Outflow("Y")
    check_twice(G, lambda g, k: g.advance_steps(3))


def test_noalloc_cfl_matches_handle_1d_and_3d_and_mhd():
    w1, dx = problems.sod_1d(3000, ghosts=2)
    G1 = dg.Grid1D(3000, dx, ghosts=2, config=dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_MINMOD))
    G1.w[...] = w1
    G1.boundary = dg.Outflow()
    check_twice(G1, lambda g, k: g.advance_steps(5))

    rng = np.random.default_rng(1)
    w3, dx3 = problems.blast_3d(20, ghosts=2)
    w3[..., 2:5] = rng.uniform(-0.3, 0.3, w3.shape[:-1] + (3,))
    w3[..., 0] = np.where(w3[..., 0] > 0, w3[..., 0], 1.0)
    w3[..., 1] = np.where(w3[..., 1] > 0, w3[..., 1], 0.1)
    G3 = dg.Grid3D(20, 20, 20, dx3, dx3 * 1.5, dx3 * 0.5, ghosts=2, config=dg.Config(cfl=dg.CFL_MAX))

    def bump3(g, k):
        w = g.w
        w[..., 1] *= 1.7

    G3.w[...] = w3
    G3.boundary = dg.Reflective()
    check_twice(G3, bump3)

    wm, Bm, dxm = problems.blast_2d_mhd(40, ghosts=3)
    Gm = dg.Grid2D(40, 40, dxm, dxm, ghosts=3, config=dg.Config(mhd=True))
    Gm.w[...] = wm
    Gm.B[...] = Bm
    Gm.boundary = dg.Periodic()
    Gm.initialize_B_fields()

    def bumpm(g, k):
        g.B[..., 0] *= 3.0
        g.initialize_B_fields()

    check_twice(Gm, bumpm)


def test_noalloc_refuses_oversized_grid():
    G = dg.Grid2D(8, 8, 0.1, 0.1, ghosts=2)
    G.w[..., 0] = 1.0
    G.w[..., 1] = 1.0
    G.apply_boundary()
    L = G._lib
    prim = ctypes.c_void_p()
    plane = ctypes.c_longlong()
    pitch = ctypes.c_longlong()
    _lib.check(L.dragon_gpu_device_state(G._h, ctypes.byref(prim), ctypes.byref(plane), ctypes.byref(pitch)))
    out = ctypes.c_double(-1.0)
    rc = L.dragon_gpu_cfl_time_noalloc(2, 20000, 8, 1, 2, 0, ctypes.cast(prim, _lib.c_double_p), 1 << 40, 1 << 20,
                                       0.1, 0.1, 0.0, 1, 0.3, None, ctypes.byref(out))
    assert rc == 1
    assert b"too large" in L.dragon_gpu_last_error()
    assert out.value == -1.0
