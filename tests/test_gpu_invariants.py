"""The reference's invariant suites, run on the device path at full size
(sizes where the oracle would take minutes).

* Dimension match (Testing/Core/Godunov/HydroDimMatch_Tests.cpp:17-219,
  MHDDimMatch_Tests.cpp): a 2D or 3D grid whose state varies along one axis
  only steps like a 1D grid of that axis (velocities and fields swapped into
  the 1D frame), to the reference's expect_close bar (1e-15 relative,
  1e-18 absolute). Hydro at 1024^2 and 128^3, MHD (the Dai-Woodward shock
  tube) at 1024 x 32.
* CTU blast symmetry (HydroCTU_Tests.cpp:153-279): a centred blast keeps its
  mirror symmetry about every axis, stays physical, conserves mass to 1e-10
  and depressurises its centre, to t = 0.05 (2D) and t = 0.02 (3D). At the
  reference's sizes (64^2, 64^3) the symmetry bar is the reference's 1e-14;
  at 1024^2 and 128^3 the runs take 16x / 2x more steps, and the rounding
  that breaks the mirror image (operations are not evaluated in mirrored
  order) accumulates to ~1e-13, so the bar there is 1e-12 relative to the
  field's largest value. The device path is bit-identical to the reference,
  so the reference shows the same deviations at these sizes.
"""
import math

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


def approx(a, b, rel=1e-15, ab=1e-18):
    """Testing/Core/FluidElement_Tests.cpp:83-85, elementwise."""
    return np.abs(a - b) <= ab + rel * np.maximum(np.abs(a), np.abs(b))


def assert_close(a, b, what, rel=1e-15, ab=1e-18):
    ok = approx(a, b, rel, ab)
    if not ok.all():
        k = np.argwhere(~ok)[0]
        raise AssertionError(f"{what}: {np.count_nonzero(~ok)} values off, first at {k.tolist()}: "
                             f"{a[tuple(k)]} vs {b[tuple(k)]}")


def profile_1d(n, g):
    """A smooth profile with one jump, positive density and pressure, all
    three velocity components non-zero."""
    x = (np.arange(n) + 0.5) / n
    w = np.zeros((n + 2 * g, 5))
    w[g:-g, 0] = 1 + 0.5 * (x > 0.5) + 0.2 * np.sin(6 * np.pi * x)
    w[g:-g, 1] = 2 + 0.5 * (x < 0.5) + 0.3 * np.sin(4 * np.pi * x)
    w[g:-g, 2] = 0.3 * np.cos(2 * np.pi * x)
    w[g:-g, 3] = 0.1 * np.sin(4 * np.pi * x)
    w[g:-g, 4] = -0.05
    return w


def rotate_to(w1, axis):
    """The 1D frame (normal velocity first) into a grid's frame whose varying axis is `axis`."""
    w = w1.copy()
    if axis == 1:
        w[..., [2, 3]] = w1[..., [3, 2]]
    elif axis == 2:
        w[..., [2, 4]] = w1[..., [4, 2]]
    return w


def one_d_grid(n, cfg, w1):
    G = dg.Grid1D(n, 1.0 / n, ghosts=2, config=cfg)
    G.w[...] = w1
    G.boundary = dg.Outflow()
    return G


@pytest.mark.parametrize("dim,axis", [(2, 0), (2, 1), (3, 0), (3, 1), (3, 2)])
def test_hydro_dimension_match(dim, axis):
    n = 1024 if dim == 2 else 128
    t = 32 if dim == 2 else 16   # transverse extent (periodic)
    g = 2
    cfg = dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_MC)
    w1 = profile_1d(n, g)
    E = one_d_grid(n, cfg, w1)
    shape = [t] * dim
    shape[axis] = n
    wf = rotate_to(w1, axis)
    # broadcast the profile along the transverse axes of the padded array
    idx = [None] * dim
    idx[axis] = slice(None)
    w = np.broadcast_to(wf[tuple(idx) + (slice(None),)], tuple(s + 2 * g for s in shape) + (5,)).copy()
    d = [1.0 / n] * dim
    G = (dg.Grid2D if dim == 2 else dg.Grid3D)(*shape, *d, ghosts=g, config=cfg)
    G.w[...] = w
    transverse = "".join("XYZ"[a] for a in range(dim) if a != axis)
    G.boundary = dg.Outflow("XYZ"[axis]) + dg.Periodic(transverse)
    E.apply_boundary()
    dt = 0.5 * E.cfl_time()
    for step in range(2):
        E.advance(dt, check_cfl=False)
        G.advance(dt, check_cfl=False)
        expect = rotate_to(E.w[g:-g], axis)
        inner = G.w[(slice(g, -g),) * dim]
        exp_b = np.broadcast_to(expect[tuple(idx) + (slice(None),)], inner.shape)
        assert_close(inner, exp_b, f"{dim}D axis {axis} step {step}")


DW = dict(rL=1.08, rR=1.0, vx=1.2, vy=0.01, vz=0.5, Bx=2.0, ByL=3.6, ByR=4.0, Bz=2.0, pL=0.95, pR=1.0)


@pytest.mark.parametrize("axis", [0, 1])
def test_mhd_dimension_match_dai_woodward(axis):
    """MHDDimMatch_Tests.cpp:68-140: the Dai-Woodward shock tube along x (or
    y) of a 2D MHD grid against the 1D MHD grid, one step at the smaller CFL
    time of the two."""
    n, t, g = 1024, 32, 3
    q = DW
    dx = 1.0 / n
    left = np.arange(n) < n // 2
    w1 = np.zeros((n + 2 * g, 8))
    w1[g:-g, 0] = np.where(left, q["rL"], q["rR"])
    w1[g:-g, 1] = np.where(left, q["pL"], q["pR"])
    w1[g:-g, 2] = np.where(left, q["vx"], 0.0)
    w1[g:-g, 3] = np.where(left, q["vy"], 0.0)
    w1[g:-g, 4] = np.where(left, q["vz"], 0.0)
    w1[g:-g, 5] = q["Bx"]
    w1[g:-g, 6] = np.where(left, q["ByL"], q["ByR"])
    w1[g:-g, 7] = q["Bz"]
    cfg = dg.Config(mhd=True, riemann=dg.RIEMANN_HLLD, limiter=dg.LIMITER_MC)
    E = dg.Grid1D(n, dx, ghosts=g, config=cfg)
    E.w[...] = w1
    E.boundary = dg.Outflow("X") + dg.Periodic("YZ")
    shape = (n, t) if axis == 0 else (t, n)
    G = dg.Grid2D(*shape, dx, dx, ghosts=g, config=cfg)
    wf = w1.copy()
    if axis == 1:
        wf[..., [2, 3]] = w1[..., [3, 2]]
        wf[..., [5, 6]] = w1[..., [6, 5]]
    w = np.zeros((shape[0] + 2 * g, shape[1] + 2 * g, 8))
    B = np.zeros((shape[0] + 1 + 2 * g, shape[1] + 1 + 2 * g, 3))
    k = np.arange(n + 1)
    by = np.where(k < n // 2, q["ByL"], q["ByR"])
    if axis == 0:
        w[:, :, :] = wf[:, None, :]
        B[g:g + n + 1, g:g + t + 1, 0] = q["Bx"]
        B[g:g + n + 1, g:g + t + 1, 1] = by[:, None]
        G.boundary = dg.Outflow("X") + dg.Periodic("YZ")
    else:
        w[:, :, :] = wf[None, :, :]
        B[g:g + t + 1, g:g + n + 1, 0] = by[None, :]
        B[g:g + t + 1, g:g + n + 1, 1] = q["Bx"]
        G.boundary = dg.Periodic("X") + dg.Outflow("Y") + dg.Periodic("Z")
    B[g:g + shape[0] + 1, g:g + shape[1] + 1, 2] = q["Bz"]
    G.w[...] = w
    G.B[...] = B
    G.apply_boundary()
    G.initialize_B_fields()
    E.apply_boundary()
    dt = min(G.cfl_time(), E.cfl_time())
    E.advance(dt)
    G.advance(dt)
    e = E.w[g:-g]
    gi = G.w[g:-g, g:-g]
    if axis == 1:
        gi = gi.transpose(1, 0, 2).copy()
        gi[..., [2, 3]] = gi[..., [3, 2]].copy()
        gi[..., [5, 6]] = gi[..., [6, 5]].copy()
    eb = np.broadcast_to(e[:, None, :], gi.shape)

    def energy(x):
        return x[..., 1] / (5.0 / 3.0 - 1.0) + 0.5 * x[..., 0] * (x[..., 2:5] ** 2).sum(-1) + \
            (x[..., 5:8] ** 2).sum(-1) / (8 * math.pi)
    assert_close(gi[..., 0], eb[..., 0], "rho")
    assert_close(energy(gi), energy(eb), "energy", rel=1e-14)  # energy recombined in numpy
    assert_close(gi[..., 5], eb[..., 5], "normal B")
    assert_close(gi[..., 2:5], eb[..., 2:5], "velocity")


def mirror_check(w, axis, tol):
    """expect_blast_mirror_{x,y,z} (HydroCTU_Tests.cpp:113-150): every cell
    against its mirror image about the centre plane normal to `axis`; the
    normal velocity flips sign."""
    m = np.flip(w, axis=axis).copy()
    m[..., 2 + axis] *= -1
    assert_close(w, m, f"mirror symmetry about axis {axis}", rel=tol, ab=tol)


def mirror_check_scaled(w, axis, tol):
    """The same mirror image, each field's deviation relative to its largest value."""
    m = np.flip(w, axis=axis).copy()
    m[..., 2 + axis] *= -1
    scale = np.max(np.abs(w), axis=tuple(range(w.ndim - 1)))
    dev = np.max(np.abs(w - m), axis=tuple(range(w.ndim - 1))) / np.where(scale > 0, scale, 1)
    assert np.all(dev <= tol), f"mirror symmetry about axis {axis}: max deviation per field {dev}"


@pytest.mark.parametrize("dim,n", [(2, 64), (3, 64), (2, 1024), (3, 128)])
def test_ctu_blast_symmetry_and_conservation(dim, n):
    T = 0.05 if dim == 2 else 0.02
    g = 2
    if dim == 2:
        x = (np.arange(n) + 0.5) / n - 0.5
        X, Y = np.meshgrid(x, x, indexing="ij")
        w = np.zeros((n + 2 * g, n + 2 * g, 5))
        w[g:-g, g:-g, 0] = 1.0
        w[g:-g, g:-g, 1] = np.where(np.sqrt(X * X + Y * Y) < 0.1, 10.0, 0.1)
        G = dg.Grid2D(n, n, 1.0 / n, 1.0 / n, ghosts=g)
    else:
        w, d = problems.blast_3d(n, ghosts=g, p_in=10.0)
        G = dg.Grid3D(n, n, n, d, d, d, ghosts=g)
    G.w[...] = w
    G.boundary = dg.Outflow()
    inner0 = w[(slice(g, -g),) * dim]
    res = G.advance(T)
    assert res.steps > 10
    inner = G.w[(slice(g, -g),) * dim]
    assert np.all(inner[..., 0] > 0) and np.all(inner[..., 1] > 0) and np.all(np.isfinite(inner))
    m0, m1 = inner0[..., 0].sum(), inner[..., 0].sum()
    assert abs(m1 - m0) <= 1e-10 + 1e-10 * max(abs(m0), abs(m1))
    c = (n // 2,) * dim
    assert inner[c + (1,)] < 10.0
    for a in range(dim):
        if n == 64:
            mirror_check(inner, a, 1e-14)
        else:
            mirror_check_scaled(inner, a, 1e-12)
