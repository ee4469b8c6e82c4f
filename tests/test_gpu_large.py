"""Full-size properties that need no oracle run (the oracle is too slow at
these sizes): with periodic boundaries the update is translation invariant,
so a problem shifted by (a, b) cells must give the shifted result bit for bit
(every face runs the same arithmetic, whichever tile computes it), and the
conserved totals stay constant to FP64 roundoff. Sizes are ragged (not
multiples of the tile shapes) so edge tiles are covered."""
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


def _interior(a, g, dim):
    return a[tuple(slice(g, -g) for _ in range(dim))]


def _conserved(w):
    rho, p = w[..., 0], w[..., 1]
    v2 = w[..., 2] ** 2 + w[..., 3] ** 2 + w[..., 4] ** 2
    E = p / (2.0 / 3.0) + 0.5 * rho * v2
    return np.array([rho.sum(), (rho * w[..., 2]).sum(), (rho * w[..., 3]).sum(), E.sum()])


def _run2d(w_int, g, steps, shift=(0, 0), precision=dg.PREC_FP64):
    nx, ny = w_int.shape[:2]
    G = dg.Grid2D(nx, ny, 1.0 / nx, 1.0 / ny, ghosts=g,
                  config=dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_VANLEER, precision=precision))
    w = np.zeros(G.w.shape)
    w[g:-g, g:-g] = np.roll(w_int, shift, axis=(0, 1))
    G.w[...] = w
    G.boundary = dg.Periodic()
    res = G.advance_steps(steps)
    out = _interior(G.w, g, 2).copy()
    G.close()
    return out, res


@pytest.mark.parametrize("precision", [dg.PREC_FP64, dg.PREC_MIXED])
def test_2d_translation_invariance_full_size(precision):
    nx, ny, g = 4099, 2053, 2
    w0, _, _ = problems.kelvin_helmholtz_2d(nx, ghosts=g, seed=31, ny=ny)
    w_int = w0[g:-g, g:-g]
    a, ra = _run2d(w_int, g, 3, precision=precision)
    b, rb = _run2d(w_int, g, 3, shift=(1234, 567), precision=precision)
    assert ra.last_dt == rb.last_dt
    if precision == dg.PREC_FP64:
        np.testing.assert_array_equal(np.roll(a, (1234, 567), axis=(0, 1)), b)
    else:
        # the mixed HLLC tile's pressure reference is the tile's minimum, which
        # depends on where the tile boundaries fall: equal to FP32 roundoff
        rel = problems.rel_l1(np.roll(a, (1234, 567), axis=(0, 1)), b)
        assert np.all(rel[:3] < 1e-6), rel


def test_2d_conservation_full_size():
    nx, ny, g = 4099, 2053, 2
    w0, _, _ = problems.kelvin_helmholtz_2d(nx, ghosts=g, seed=32, ny=ny)
    before = _conserved(w0[g:-g, g:-g])
    after, res = _run2d(w0[g:-g, g:-g], g, 4)
    c = _conserved(after)
    assert res.steps == 4
    assert abs(c[0] - before[0]) / abs(before[0]) < 1e-13
    assert abs(c[3] - before[3]) / abs(before[3]) < 1e-13
    # x momentum of the shear layer sums to (2 x 0.5 x 1/2 - 1 x 0.5 x 1/2) per column: nonzero
    assert abs(c[1] - before[1]) / abs(before[1]) < 1e-12
    assert abs(c[2] - before[2]) < 1e-12 * abs(before[0])


def test_3d_translation_invariance():
    n, g = (130, 97, 67), 2
    rng = np.random.default_rng(5)
    w = np.zeros(n + (5,))
    w[..., 0] = 1.0 + 0.3 * rng.random(n)
    w[..., 1] = 1.0 + 0.5 * rng.random(n)
    w[..., 2:5] = 0.2 * (rng.random(n + (3,)) - 0.5)
    outs = []
    for shift in [(0, 0, 0), (37, 11, 50)]:
        G = dg.Grid3D(*n, 1.0 / n[0], 1.0 / n[1], 1.0 / n[2], ghosts=g,
                      config=dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_MC))
        full = np.zeros(G.w.shape)
        full[g:-g, g:-g, g:-g] = np.roll(w, shift, axis=(0, 1, 2))
        G.w[...] = full
        G.boundary = dg.Periodic()
        G.advance_steps(2)
        outs.append(_interior(G.w, g, 3).copy())
        G.close()
    np.testing.assert_array_equal(np.roll(outs[0], (37, 11, 50), axis=(0, 1, 2)), outs[1])


def test_mhd_2d_translation_invariance_and_divb():
    n, g = 1030, 3
    w0, B0, dx, dy = problems.orszag_tang_2d(n, ghosts=g)
    shift = (301, 77)
    res = []
    for s in [(0, 0), shift]:
        G = dg.Grid2D(n, n, dx, dy, ghosts=g, config=dg.Config(mhd=True, riemann=dg.RIEMANN_HLLX))
        w = np.zeros(G.w.shape)
        w[g:-g, g:-g] = np.roll(w0[g:-g, g:-g], s, axis=(0, 1))
        B = np.zeros(G.B.shape)
        # periodic faces: face n is face 0, so the n interior faces roll as a block
        B[g:g + n, g:g + n] = np.roll(B0[g:g + n, g:g + n], s, axis=(0, 1))
        B[g + n, g:g + n] = B[g, g:g + n]
        B[g:g + n + 1, g + n] = B[g:g + n + 1, g]
        G.w[...] = w
        G.B[...] = B
        G.boundary = dg.Periodic()
        G.initialize_B_fields()
        G.advance_steps(3)
        Bf = G.B.copy()
        div = ((Bf[g + 1:g + n + 1, g:g + n, 0] - Bf[g:g + n, g:g + n, 0]) / dx
               + (Bf[g:g + n, g + 1:g + n + 1, 1] - Bf[g:g + n, g:g + n, 1]) / dy)
        assert np.abs(div).max() * dx < 1e-13
        res.append((_interior(G.w, g, 2).copy(), Bf[g:g + n, g:g + n].copy()))
        G.close()
    np.testing.assert_array_equal(np.roll(res[0][0], shift, axis=(0, 1)), res[1][0])
    np.testing.assert_array_equal(np.roll(res[0][1], shift, axis=(0, 1)), res[1][1])
