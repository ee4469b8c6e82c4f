"""GPU checks of the batched step: uneven 1D hydro and 2D MHD grids advanced
together by the persistent work-queue kernel end bit for bit where each grid's
own advance_steps ends, for every launch shape the autotuner may pick; a mixed
FP32/FP64 batch ends where its members' own mixed advances end (1D bit for bit,
2D MHD to FP32 rounding) and within the mixed bar of the FP64 batch; the
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


def make_grids(one, two, solver=dg.RIEMANN_HLLX, precision=dg.PREC_FP64):
    grids = []
    for k, spec in enumerate(one):
        G = dg.Grid1D(spec["n"], spec["dx"], ghosts=2,
                      config=dg.Config(riemann=solver, limiter=dg.LIMITER_MINMOD if k % 2 else dg.LIMITER_MC,
                                       precision=precision))
        G.w[...] = spec["w"]
        if k % 3 == 0:
            G.boundary = dg.Periodic()
        grids.append(G)
    for spec in two:
        n = spec["n"]
        G = dg.Grid2D(n, n, spec["dx"], spec["dx"], ghosts=3,
                      config=dg.Config(mhd=True, riemann=dg.RIEMANN_HLLX, precision=precision))
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


@pytest.mark.parametrize("tile,order,per_sm,group,wave", [(254, 0, 0, 1, 1), (126, 1, 1, 1, 1), (254, 2, 2, 1, 1),
                                                          (254, 0, 0, 2, 1), (126, 2, 1, 4, 1), (254, 1, 2, 8, 1),
                                                          (254, 3, 2, 8, 1), (126, 3, 0, 2, 3)])
def test_batch_matches_single_grid_advance(workload, tile, order, per_sm, group, wave):
    one, two = workload
    steps = 9
    ref = make_grids(one, two)
    for G in ref:
        G.advance_steps(steps)
    grids = make_grids(one, two)
    b = batch.Batch(grids)
    b.tuning = batch.Tuning(tile_1d=tile, ctas_per_sm=per_sm, order=order, graph_steps=4, mhd_tiles=group, wave=wave)
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
    assert ms > 0 and t.tile_1d in (126, 254) and t.order in (0, 1, 2, 3)
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


TOL_MIXED = 1e-5
TOL_MIXED_BATCH_MHD = 1e-6  # relative L1, mixed batch vs single-grid mixed, 9 steps


@pytest.mark.parametrize("tile,order,per_sm,group,wave", [(254, 0, 0, 1, 1), (126, 2, 1, 8, 1), (254, 3, 2, 8, 2)])
def test_mixed_batch_matches_single_grid_mixed_advance(workload, tile, order, per_sm, group, wave):
    one, two = workload
    steps = 9
    ref = make_grids(one, two, precision=dg.PREC_MIXED)
    for G in ref:
        G.advance_steps(steps)
    grids = make_grids(one, two, precision=dg.PREC_MIXED)
    b = batch.Batch(grids)
    b.tuning = batch.Tuning(tile_1d=tile, ctas_per_sm=per_sm, order=order, graph_steps=4, mhd_tiles=group, wave=wave)
    st = b.advance_steps(steps)
    assert st["spin_timeouts"] == 0
    for G, R in zip(grids, ref):
        if G.dim == 1:  # the same tile body and tiling: bit for bit
            np.testing.assert_array_equal(G.w, R.w)
            continue
        # 2D MHD: the phase bodies are inlined into a different kernel, where
        # the compiler may fuse other FP32 multiply-adds
        g = G.ghosts
        for a, r in ((G.w, R.w), (G.B, R.B)):
            l1 = problems.rel_l1(a[g:-g, g:-g].reshape(-1, a.shape[-1]), r[g:-g, g:-g].reshape(-1, r.shape[-1]))
            assert np.all(l1 <= TOL_MIXED_BATCH_MHD), (G.n, l1)


def test_mixed_batch_within_the_mixed_bar_of_fp64():
    """Members of the 2048 1D + 256 2D MHD batch's sizes (1D N in [64, 1024], MHD blasts 64^2
    and 128^2): every field of every member within the mixed bar of its FP64
    batch state after 20 steps."""
    one, two = problems.batch_instances(n1d=16, n2d=3, seed=4, sizes_1d=(64, 1024), sizes_2d=(64, 128))
    steps = 20
    fp64 = make_grids(one, two)
    batch.Batch(fp64).advance_steps(steps)
    mixed = make_grids(one, two, precision=dg.PREC_MIXED)
    batch.Batch(mixed).advance_steps(steps)
    differs = False
    for G, R in zip(mixed, fp64):
        g = G.ghosts
        sl = tuple(slice(g, g + n) for n in G.n)
        a, r = G.w[sl], R.w[sl]
        differs |= bool(np.any(a != r))
        l1 = problems.rel_l1(a.reshape(-1, a.shape[-1]), r.reshape(-1, r.shape[-1]))
        assert np.all(l1 <= TOL_MIXED), (G.n, l1)
    assert differs  # really the FP32 path


def test_mixed_batch_exact_solver_members(workload):
    one, _ = workload
    ref = make_grids(one[:10], [], solver=dg.RIEMANN_EXACT, precision=dg.PREC_MIXED)
    for G in ref:
        G.advance_steps(5)
    grids = make_grids(one[:10], [], solver=dg.RIEMANN_EXACT, precision=dg.PREC_MIXED)
    batch.Batch(grids).advance_steps(5)
    for G, R in zip(grids, ref):
        np.testing.assert_array_equal(G.w, R.w)


def test_batch_members_share_one_precision():
    b = batch.Batch()
    b.add(dg.Grid1D(32, 1 / 32, config=dg.Config(riemann=dg.RIEMANN_HLLC, precision=dg.PREC_MIXED)))
    with pytest.raises(dg.grid._lib.DragonGPUError):
        b.add(dg.Grid1D(32, 1 / 32, config=dg.Config(riemann=dg.RIEMANN_HLLC)))
