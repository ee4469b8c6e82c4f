"""User GhostFill elements (the reference's Jet pattern, Jets.hpp:12-39) on the
host-driven path: built-in elements stay on the device, the user's apply(grid)
runs on the host between them in list order. Checked bit for bit against the
oracle driven through the same sequence (ghost fill, user fill, CFL dt, step)."""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

import dragon_b200 as dg  # noqa: E402
from dragon_b200 import problems  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not cuda_ok():
        pytest.fail("CUDA device required for -m gpu tests")


class Jet(dg.GhostFill):
    """Inflow through part of the X- face (a jet of fixed state where
    |y - y0| < r), outflow elsewhere on that face."""

    def __init__(self, state, y0, r, dy, ghosts):
        super().__init__("X-", True)
        self.jet_state = np.asarray(state, dtype=np.float64)
        self.y0, self.r, self.dy, self.g = y0, r, dy, ghosts

    def fill(self, w):
        g = self.g
        ys = (np.arange(w.shape[1]) - g + 0.5) * self.dy
        jet = np.abs(ys - self.y0) < self.r
        for gl in range(1, g + 1):
            w[g - gl] = w[g]
            w[g - gl, jet] = self.jet_state

    def apply(self, grid):
        self.fill(grid.w)


def oracle(**kw):
    from oracle import port, refgrid
    return refgrid.RefGrid(**kw) if refgrid.available("hydro") else port.PortGrid(**kw)


def test_jet_inflow_matches_oracle():
    n = 32
    w0, dx, dy = problems.kelvin_helmholtz_2d(n, ghosts=2, seed=5)
    w0[..., 2] = 0.0
    jet = Jet([2.0, 3.0, 1.5, 0.0, 0.0], 0.5, 0.15, dy, 2)
    bl = dg.Periodic("Y") + jet
    G = dg.Grid2D(n, n, dx, dy, ghosts=2, config=dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_VANLEER))
    G.w[...] = w0
    G.boundary = bl
    assert G.boundary.has_custom()
    res = G.advance(0.03)
    assert res.steps > 2

    R = oracle(dim=2, n=(n, n), d=(dx, dy), ghosts=2, riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_VANLEER)
    R.set_prim(w0)
    from oracle.refgrid import bc_entries_from
    R.set_boundary(bc_entries_from([dg.Periodic("Y"), dg.Ignore("X-")]))
    t = 0.03
    steps = 0
    while t > 1e-14:
        R.apply_boundary()
        a = R.get_prim()
        jet.fill(a)
        R.set_prim(a)
        dt = min(t, R.cfl_time())
        R.unsplit_step(dt)
        t -= dt
        steps += 1
    assert steps == res.steps
    np.testing.assert_array_equal(G.w[2:-2, 2:-2], R.get_prim()[2:-2, 2:-2])
    # the jet really enters
    assert G.w[2, n // 2, 2] > 0.5


def test_custom_between_builtins_keeps_list_order():
    """A user element between two built-ins runs after the first and before
    the second (the second overwrites what it filled on shared faces)."""
    n = 12
    w0, dx, dy = problems.kelvin_helmholtz_2d(n, ghosts=2, seed=9)
    calls = []

    class Marker(dg.GhostFill):
        def apply(self, grid):
            calls.append(float(grid.w[0, 5, 0]))
            grid.w[0:2, :, 0] = 7.0

    G = dg.Grid2D(n, n, dx, dy, ghosts=2)
    G.w[...] = w0
    G.boundary = dg.Outflow("Y") + Marker("X-") + dg.Periodic("X")
    G.apply_boundary()
    assert len(calls) == 1
    # Periodic X comes last: it overwrites the marker's X- ghosts
    np.testing.assert_array_equal(G.w[0:2, 2:-2, 0], G.w[n:n + 2, 2:-2, 0])
