"""dragon_gpu_advance_steps_async / dragon_gpu_advance_wait: the two halves of
advance_steps give the same state and statistics, and the handle refuses other
calls while an advance is in flight."""
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


def _kh(n=96, seed=4):
    w0, dx, dy = problems.kelvin_helmholtz_2d(n, ghosts=2, seed=seed)
    G = dg.Grid2D(n, n, dx, dy, ghosts=2, config=dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_VANLEER))
    G.w[...] = w0
    G.boundary = dg.Periodic()
    return G


@pytest.mark.parametrize("steps", [1, 7, 130])
def test_async_equals_sync(steps):
    A, B = _kh(), _kh()
    ra = A.advance_steps(steps)
    B.advance_steps_async(steps)
    rb = B.advance_wait()
    np.testing.assert_array_equal(A.w, B.w)
    assert (ra.steps, ra.retries, ra.last_dt) == (rb.steps, rb.retries, rb.last_dt)


def test_async_refuses_other_calls_until_wait():
    G = _kh()
    L, h = G._lib, G._h
    G.advance_steps_async(3)
    buf = np.zeros(G.w.shape)
    assert L.dragon_gpu_download_prim(h, buf.ctypes.data_as(_lib.c_double_p)) == 1
    assert L.dragon_gpu_advance_steps_async(h, 1) == 1
    st = _lib.StepStatus()
    assert L.dragon_gpu_unsplit_step(h, 1e-4, ctypes.byref(st)) == 1
    r = G.advance_wait()
    assert r.steps == 3
    assert L.dragon_gpu_advance_wait(h, None) == 1  # nothing in flight any more
    G.advance_steps(1)  # usable again


def test_async_strong_shock_matches_sync():
    """A 1D shock tube with a 1e5 pressure ratio: the async halves give the
    same state, step count and retry count as the synchronous advance."""
    w0, dx = problems.riemann_1d(256, (1.0, 0.0, 1000.0), (1.0, 0.0, 0.01))
    out = []
    for mode in ("sync", "async"):
        G = dg.Grid1D(256, dx, ghosts=2, config=dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_SUPERBEE))
        G.w[...] = w0
        if mode == "sync":
            r = G.advance_steps(20)
        else:
            G.advance_steps_async(20)
            r = G.advance_wait()
        out.append((G.w.copy(), r.steps, r.retries))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    assert out[0][1:] == out[1][1:]
