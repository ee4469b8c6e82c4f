"""GPU checks of the batched step: uneven 1D hydro and 2D MHD grids advanced
together by the persistent work-queue kernel end bit for bit where each grid's
own advance_steps ends, for every launch shape the autotuner may pick; the
autotuner leaves the states untouched."""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

import dragon_b200 as dg  # noqa: E402
from dragon_b200 import batch, problems  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not cuda_ok():
        pytest.fail("CUDA device required for -m gpu tests")


def make_grids(one, two, solver=dg.RIEMANN_HLLX):
    grids = []
    for k, spec in enumerate(one):
        G = dg.Grid1D(spec["n"], spec["dx"], ghosts=2,
                      config=dg.Config(riemann=solver, limiter=dg.LIMITER_MINMOD if k % 2 else dg.LIMITER_MC))
        G.w[...] = spec["w"]
        if k % 3 == 0:
            G.boundary = dg.Periodic()
        grids.append(G)
    for spec in two:
        n = spec["n"]
        G = dg.Grid2D(n, n, spec["dx"], spec["dx"], ghosts=3, config=dg.Config(mhd=True, riemann=dg.RIEMANN_HLLX))
        G.w[...] = spec["w"]
        G.B[...] = spec["B"]
        G.boundary = dg.Periodic()
        G.initialize_B_fields()
        grids.append(G)
    return grids


@pytest.fixture(scope="module")
def workload():
    return problems.batch_instances(n1d=24, n2d=4, seed=3, sizes_1d=(16, 700), sizes_2d=(16, 24, 40))


def states(grids):
    return [(G.w.copy(), G.B.copy() if G._B is not None else None) for G in grids]


def assert_same(a, b):
    for (w1, b1), (w2, b2) in zip(a, b):
        np.testing.assert_array_equal(w1, w2)
        if b1 is not None:
            np.testing.assert_array_equal(b1, b2)


@pytest.mark.parametrize("tile,order,per_sm,group", [(256, 0, 0, 1), (128, 1, 1, 1), (256, 2, 2, 1), (256, 0, 0, 2),
                                                     (128, 2, 1, 4), (256, 1, 2, 8)])
def test_batch_matches_single_grid_advance(workload, tile, order, per_sm, group):
    one, two = workload
    steps = 9
    ref = make_grids(one, two)
    for G in ref:
        G.advance_steps(steps)
    grids = make_grids(one, two)
    b = batch.Batch(grids)
    b.tuning = batch.Tuning(tile_1d=tile, ctas_per_sm=per_sm, order=order, graph_steps=4, mhd_tiles=group)
    st = b.advance_steps(steps)
    assert st["spin_timeouts"] == 0 and st["graph_replays"] >= 3
    assert_same(states(grids), states(ref))
    # a second advance continues from there like the grids' own
    for G in ref:
        G.advance_steps(3)
    b.advance_steps(3)
    assert_same(states(grids), states(ref))


def test_batch_exact_solver_members(workload):
    one, _ = workload
    ref = make_grids(one[:10], [], solver=dg.RIEMANN_EXACT)
    for G in ref:
        G.advance_steps(5)
    grids = make_grids(one[:10], [], solver=dg.RIEMANN_EXACT)
    batch.Batch(grids).advance_steps(5)
    for G, R in zip(grids, ref):
        np.testing.assert_array_equal(G.w, R.w)


def test_autotune_keeps_states(workload):
    one, two = workload
    grids = make_grids(one, two)
    before = states(grids)
    b = batch.Batch(grids)
    t, ms = b.autotune(2)
    assert ms > 0 and t.tile_1d in (128, 256) and t.order in (0, 1, 2)
    assert_same(states(grids), before)
    ref = make_grids(one, two)
    for G in ref:
        G.advance_steps(4)
    b.advance_steps(4)
    assert_same(states(grids), states(ref))


def test_batch_rejects_unsupported_members():
    b = batch.Batch()
    with pytest.raises(dg.grid._lib.DragonGPUError):
        b.add(dg.Grid2D(8, 8, 0.1, 0.1))           # 2D hydro
    b.add(dg.Grid1D(32, 1 / 32, config=dg.Config(riemann=dg.RIEMANN_HLLC)))
    with pytest.raises(dg.grid._lib.DragonGPUError):
        b.add(dg.Grid1D(32, 1 / 32, config=dg.Config(riemann=dg.RIEMANN_HLLE)))  # second 1D solver
