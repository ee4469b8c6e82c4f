"""The per-step prologue of 2D / 3D grids (ghost fill in list order, ring CFL,
dt), run as one cooperative launch with bounded grid barriers.

* Failure path: a test hook makes one CTA return before the first grid
  barrier, so every other CTA's bounded wait runs out. The advance must fail
  with DRAGON_GPU_ECUDA and the barrier message, within seconds (one wait
  limit, not one per enqueued step), commit nothing, and leave a grid that
  steps bit for bit like one that never failed.
* The separate-launch prologue (devices without cooperative launch; forced
  by a test hook) must give the same states bit for bit, corner ghosts and
  MHD face ghosts included.
"""
import time

import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

import dragon_b200 as dg  # noqa: E402
from dragon_b200 import _lib, problems  # noqa: E402

DEBUG_STALL_CTA, DEBUG_NO_COOP = 1, 2  # include/dragon_gpu.h
ECUDA = 2


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not cuda_ok():
        pytest.fail("CUDA device required for -m gpu tests")


def kh(n=256):
    w0, dx, dy = problems.kelvin_helmholtz_2d(n, ghosts=2, seed=21)
    G = dg.Grid2D(n, n, dx, dy, ghosts=2, config=dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_VANLEER))
    G.w[...] = w0
    G.boundary = dg.Periodic()
    return G


def test_barrier_wait_that_runs_out_fails_the_advance_and_recovers():
    G, H = kh(), kh()
    G.advance_steps(2)
    H.advance_steps(2)
    before = G.w.copy()
    _lib.check(G._lib.dragon_gpu_debug_set(G._h, DEBUG_STALL_CTA, 1))
    t0 = time.perf_counter()
    with pytest.raises(_lib.DragonGPUError) as exc:
        G.advance_steps(5)
    elapsed = time.perf_counter() - t0
    assert exc.value.code == ECUDA
    assert "grid barrier" in str(exc.value)
    assert elapsed < 30.0, elapsed   # one wait limit, not one per enqueued prologue
    g = 2
    assert np.array_equal(G.w[g:-g, g:-g], before[g:-g, g:-g])  # no step was committed
    _lib.check(G._lib.dragon_gpu_debug_set(G._h, DEBUG_STALL_CTA, -1))
    res = G.advance_steps(5)
    H.advance_steps(5)
    assert res.steps == 5
    assert np.array_equal(G.w, H.w)


def pair(make, steps, advance=None):
    A, B = make(), make()
    _lib.check(B._lib.dragon_gpu_debug_set(B._h, DEBUG_NO_COOP, 1))
    la, lb = A.launch_count(), B.launch_count()
    for X in (A, B):
        if advance is None:
            X.advance_steps(steps)
        else:
            advance(X)
    assert B.launch_count() - lb > A.launch_count() - la  # the fallback really ran (more launches)
    assert np.array_equal(A.w, B.w)
    if A._B is not None:
        assert np.array_equal(A.B, B.B)


def test_fallback_prologue_hydro_2d_walls_and_periodic_without_corners():
    def make():
        n, ny = 70, 45
        w0, dx, dy = problems.kelvin_helmholtz_2d(n, ghosts=2, seed=5, ny=ny)
        # corner ghosts no element fills keep their initial value: make it a valid state
        w0[w0[..., 0] == 0] = (1.0, 2.5, 0.0, 0.0, 0.0)
        G = dg.Grid2D(n, ny, dx, dy, ghosts=2, config=dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_MC))
        G.w[...] = w0
        G.boundary = dg.Reflective("X-") + dg.Outflow.Gated("X+", corner_ghosts=False) + \
            dg.Periodic("Y", corner_ghosts=False)
        return G
    pair(make, 12)


def test_fallback_prologue_mhd_orszag_tang():
    def make():
        n = 64
        w0, B0, dx, dy = problems.orszag_tang_2d(n, ghosts=3)
        G = dg.Grid2D(n, n, dx, dy, ghosts=3, config=dg.Config(mhd=True, riemann=dg.RIEMANN_HLLX))
        G.w[...] = w0
        G.B[...] = B0
        G.boundary = dg.Periodic()
        G.initialize_B_fields()
        return G
    pair(make, 10)


def test_fallback_prologue_mhd_blast_outflow_reflective():
    def make():
        n = 48
        w0, B0, dx = problems.blast_2d_mhd(n, ghosts=3)[:3]
        G = dg.Grid2D(n, n, dx, dx, ghosts=3, config=dg.Config(mhd=True, riemann=dg.RIEMANN_HLLX))
        G.w[...] = w0
        G.B[...] = B0
        G.boundary = dg.Reflective("Y", corner_ghosts=False) + dg.Outflow("X")
        G.initialize_B_fields()
        return G
    pair(make, 10)


def test_fallback_prologue_hydro_3d():
    def make():
        n = 24
        w, d = problems.blast_3d(n, ghosts=2, p_in=10.0)
        w[w[..., 0] == 0] = (1.0, 0.1, 0.0, 0.0, 0.0)  # edge ghosts no element fills
        G = dg.Grid3D(n, n, n, d, d, d, ghosts=2, config=dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_MC))
        G.w[...] = w
        G.boundary = dg.Reflective("Z") + dg.Periodic("XY", corner_ghosts=False)
        return G
    pair(make, 5)
