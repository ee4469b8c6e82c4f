"""User ghost fills compiled for the device (DeviceGhostFill): the reference's
Jet pattern (Examples/CollidingFlows/Jets/Jets.hpp:12-39, Jet.cpp) written as a
device function runs inside the device advance loop and gives bit for bit what
the same fill gives as a host apply() (test_gpu_custom_bc.py checks that path
against the oracle); device fills that restate built-in elements give what
those elements give, in 1D, 2D and 3D."""
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


# params: y0, r, rho, p, vx
JET_SRC = """
__device__ void jet(const dragon_fill_ctx& c, int i, int j, int k) {
    for (int f = 0; f < c.nf; f++) c.set(f, i, j, k, c.get(f, 0, j, k));
    const double y = (j + 0.5) * c.d[1];
    if (fabs(y - c.params[0]) < c.params[1]) {
        c.set(DRAGON_RHO, i, j, k, c.params[2]);
        c.set(DRAGON_P, i, j, k, c.params[3]);
        c.set(DRAGON_VX, i, j, k, c.params[4]);
        c.set(DRAGON_VY, i, j, k, 0.0);
        c.set(DRAGON_VZ, i, j, k, 0.0);
    }
}
"""


class HostJet(dg.GhostFill):
    """The same jet as a host apply (outflow copy of the first interior layer,
    then the jet state where |y - y0| < r), over the whole padded X- slab."""

    def __init__(self, y0, r, state, dy, g):
        super().__init__("X-", True)
        self.y0, self.r, self.state_, self.dy, self.g = y0, r, np.asarray(state, float), dy, g

    def apply(self, grid):
        w, g = grid.w, self.g
        ys = (np.arange(w.shape[1]) - g + 0.5) * self.dy
        jet = np.abs(ys - self.y0) < self.r
        for gl in range(1, g + 1):
            w[g - gl] = w[g]
            w[g - gl, jet] = self.state_


def _kh(n, ghosts=2):
    w0, dx, dy = problems.kelvin_helmholtz_2d(n, ghosts=ghosts, seed=5)
    w0[..., 2] = 0.0
    return w0, dx, dy


def _grid(n, dx, dy, w0, bl):
    G = dg.Grid2D(n, n, dx, dy, ghosts=2, config=dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_VANLEER))
    G.w[...] = w0
    G.boundary = bl
    return G


@pytest.mark.parametrize("n", [32, 100])
def test_device_jet_equals_host_jet(n):
    w0, dx, dy = _kh(n)
    y0, r, state = 0.5, 0.15, [2.0, 3.0, 1.5, 0.0, 0.0]
    host = _grid(n, dx, dy, w0, dg.Periodic("Y") + HostJet(y0, r, state, dy, 2))
    dev = _grid(n, dx, dy, w0, dg.Periodic("Y") + dg.DeviceGhostFill(JET_SRC, "jet", faces="X-",
                                                                         params=[y0, r, state[0], state[1], state[2]]))
    assert host.boundary.has_custom() and not dev.boundary.has_custom()
    rh = host.advance(0.03)
    rd = dev.advance(0.03)
    assert rh.steps == rd.steps > 2
    np.testing.assert_array_equal(dev.w, host.w)
    g = 2
    ys = (np.arange(n) + 0.5) * dy
    assert np.all(dev.w[g:g + 2, g:-g][:, np.abs(ys - y0) < r / 2, 2] > 0)  # the jet has entered
    host.close()
    dev.close()


def test_device_jet_over_claimed_faces_like_the_reference():
    """The reference's Jet claims no faces (GhostFill(0, true)): the implicit
    Outflow covers X- too, and the jet overrides it inside the radius."""
    n = 48
    w0, dx, dy = _kh(n)
    jet = dg.DeviceGhostFill(JET_SRC, "jet", faces=0, fill_faces="X-", params=[0.5, 0.1, 2.0, 3.0, 1.5])
    a = _grid(n, dx, dy, w0, dg.Periodic("Y") + jet)
    b = _grid(n, dx, dy, w0, dg.Periodic("Y") + HostJet(0.5, 0.1, [2.0, 3.0, 1.5, 0.0, 0.0], dy, 2))
    ra, rb = a.advance_steps(12), b.advance_steps(12)
    assert ra.steps == rb.steps == 12
    np.testing.assert_array_equal(a.w, b.w)
    a.close()
    b.close()


# A device restatement of Reflective on one face (Reflective.cpp: mirror cell,
# normal velocity flipped), for every dimension.
REFLECT_SRC = """
__device__ void mirror(const dragon_fill_ctx& c, int i, int j, int k) {
    int q[3] = {i, j, k};
    const int a = c.axis, gl = c.side == 0 ? -q[a] : q[a] - (c.n[a] - 1);
    q[a] = c.side == 0 ? gl - 1 : c.n[a] - gl;
    for (int f = 0; f < c.nf; f++) {
        double v = c.get(f, q[0], q[1], q[2]);
        if (f == DRAGON_VX + a) v *= -1;
        c.set(f, i, j, k, v);
    }
}
"""


def _random_state(n, g, seed):
    """A physical primitive state (rho, p in [0.5, 2], |v| < 0.3) on the padded grid."""
    rng = np.random.default_rng(seed)
    shape = tuple(x + 2 * g for x in n)
    w = np.empty(shape + (5,))
    w[..., 0] = rng.uniform(0.5, 2.0, shape)
    w[..., 1] = rng.uniform(0.5, 2.0, shape)
    w[..., 2:] = rng.uniform(-0.3, 0.3, shape + (3,))
    return w


@pytest.mark.parametrize("dim,faces", [(1, "X-"), (1, "X"), (2, "X-"), (2, "X"), (2, "Y+"), (3, "X-"), (3, "X"),
                                       (3, "Y+"), (3, "Z")])
def test_device_reflective_equals_builtin(dim, faces):
    n = {1: (64,), 2: (24, 20), 3: (12, 10, 14)}[dim]
    ds = (1.0 / n[0],) * dim
    w0 = _random_state(n, 2, seed=dim)
    cls = {1: dg.Grid1D, 2: dg.Grid2D, 3: dg.Grid3D}[dim]
    cfg = dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_MC)
    grids = []
    for el in (dg.Reflective(faces, corner_ghosts=True),
               dg.DeviceGhostFill(REFLECT_SRC, "mirror", faces=faces, corner_ghosts=True)):
        G = cls(*n, *ds, ghosts=2, config=cfg)
        G.w[...] = w0
        G.boundary = dg.Outflow() + el
        grids.append(G)
    for G in grids:
        G.apply_boundary()
    np.testing.assert_array_equal(grids[1].w, grids[0].w)
    assert not np.array_equal(grids[1].w, w0)  # the fills ran
    r0, r1 = grids[0].advance_steps(4), grids[1].advance_steps(4)
    assert r0.steps == r1.steps == 4
    np.testing.assert_array_equal(grids[1].w, grids[0].w)
    for G in grids:
        G.close()


def test_unbound_user_entry_fails_the_advance():
    n = 16
    w0, dx, dy = _kh(n)
    G = dg.Grid2D(n, n, dx, dy, ghosts=2)
    G.w[...] = w0
    arr = (_lib.BCDesc * 1)()
    arr[0].type = dg.boundary.USER
    arr[0].faces = dg.X_negative
    arr[0].corners = 1
    _lib.check(G._lib.dragon_gpu_set_boundary(G._h, arr, 1))
    G._to_device()
    st = _lib.AdvanceStats()
    rc = G._lib.dragon_gpu_advance_steps(G._h, 2, ctypes.byref(st))
    assert rc == 1 and "no fill bound" in G._lib.dragon_gpu_last_error().decode()
    G.close()
