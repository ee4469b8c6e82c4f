"""User GhostFill elements (the reference's Jet pattern, Jets.hpp:12-39) on the
host-driven path: built-in elements stay on the device, the user's apply(grid)
runs on the host between them in list order, and only the slabs along the
element's faces cross the host link. Checked bit for bit against the oracle
driven through the same sequence (ghost fill, user fill, CFL dt, step), and
against a full round trip of the state."""
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


class FixedInflow(dg.GhostFill):
    """A user element that writes a fixed state into every ghost cell (and,
    on MHD grids, every ghost face) of its faces, reading the first interior
    layer for the transverse velocity like an inflow that carries the shear."""

    def __init__(self, faces, state, reach=None):
        super().__init__(faces, True)
        self.st = np.asarray(state, dtype=np.float64)
        if reach is not None:
            self.reach = reach

    def apply(self, grid):
        g = grid.ghosts
        w = grid.w
        w[:g] = self.st[: w.shape[-1]]
        w[:g, :, 3] = w[g, :, 3]          # the first interior layer's vy
        if grid.config.mhd:
            grid.B[:g, :, 1] = 0.25       # transverse face field in the ghost faces


@pytest.mark.parametrize("mhd", [False, True])
def test_ghost_slab_path_equals_full_round_trip(mhd):
    """The ghost-slab path (only the element's slabs cross the host link)
    gives the same state bit for bit as a full round trip of the state
    (forced by a reach that spans the axis)."""
    n = 96
    if mhd:
        w0, B0, dx, dy = problems.orszag_tang_2d(n, ghosts=3)
        st = [0.3, 0.2, 0.5, 0.0, 0.0, 0.2, 0.1, 0.0]
        cfg = dg.Config(mhd=True, riemann=dg.RIEMANN_HLLX)
    else:
        w0, dx, dy = problems.kelvin_helmholtz_2d(n, ghosts=2, seed=13)
        B0 = None
        st = [2.0, 3.0, 1.5, 0.0, 0.0]
        cfg = dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_VANLEER)
    out = []
    for reach in (None, 10 * n):
        G = dg.Grid2D(n, n, dx, dy, ghosts=3 if mhd else 2, config=cfg)
        G.w[...] = w0
        if mhd:
            G.B[...] = B0
        G.boundary = dg.Periodic("Y") + FixedInflow("X-", st, reach)
        if mhd:
            G.initialize_B_fields()
        el = list(G.boundary)[-1]
        assert (G._custom_slabs(el) is None) == (reach is not None)
        res = G.advance_steps(6)
        assert res.steps == 6
        out.append((G.w.copy(), G.B.copy() if mhd else None))
        G.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    if mhd:
        np.testing.assert_array_equal(out[0][1], out[1][1])
