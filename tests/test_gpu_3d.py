"""GPU parity of the 3D unsplit CTU hydro step (12-solve corner transport)
against the reference. Solvers without pow are bit-identical; the exact
solver (CUDA pow vs glibc pow) is held to 1e-12 relative L1."""
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


def oracle_grid(**kw):
    from oracle import port, refgrid
    if refgrid.available("hydro"):
        return refgrid.RefGrid(**kw)
    return port.PortGrid(**kw)


def check(a, b, exact, what):
    if exact:
        bad = np.argwhere(a != b)
        assert bad.size == 0, f"{what}: {len(bad)} mismatches, first {bad[:3].tolist()}"
    else:
        l1 = problems.rel_l1(a, b)
        assert np.all(l1 <= 1e-12), f"{what}: rel L1 {l1}"


def blast(n, seed=0, p_in=10.0):
    w, d = problems.blast_3d(n, ghosts=2, p_in=p_in)
    rng = np.random.default_rng(seed)
    w[..., 2:5] = rng.uniform(-0.1, 0.1, w.shape[:-1] + (3,))
    w[..., 0] = np.where(w[..., 0] > 0, w[..., 0], 1.0)
    w[..., 1] = np.where(w[..., 1] > 0, w[..., 1], 0.1)
    return w, d


def pair(n, d, w0, boundary, riemann, limiter, ns=None):
    ns = ns or (n, n, n)
    ds = (d, d * 1.25, d * 0.8)
    cfg = dg.Config(riemann=riemann, limiter=limiter)
    G = dg.Grid3D(*ns, *ds, ghosts=2, config=cfg)
    R = oracle_grid(dim=3, n=ns, d=ds, ghosts=2, riemann=riemann, limiter=limiter)
    G.w[...] = w0
    R.set_prim(w0)
    G.boundary = boundary
    from oracle.refgrid import bc_entries_from
    R.set_boundary(bc_entries_from(dg.boundary.as_list(boundary)))
    return G, R


@pytest.mark.parametrize("riemann", [dg.RIEMANN_HLLC, dg.RIEMANN_HLL, dg.RIEMANN_HLLE, dg.RIEMANN_ROE,
                                     dg.RIEMANN_EXACT])
def test_3d_blast_solvers(riemann):
    n = 12
    w0, d = blast(n, seed=riemann)
    G, R = pair(n, d, w0, dg.Outflow(), riemann, dg.LIMITER_MC)
    for _ in range(4):
        R.step_cfl()
    res = G.advance_steps(4)
    assert res.steps == 4
    check(G.w, R.get_prim(), riemann != dg.RIEMANN_EXACT, f"3d s{riemann}")


@pytest.mark.parametrize("limiter", [0, 2, 3, 4])
def test_3d_limiters_ragged_mixed_boundaries(limiter):
    ns = (9, 13, 7)
    w0 = np.zeros((ns[0] + 4, ns[1] + 4, ns[2] + 4, 5))
    rng = np.random.default_rng(limiter)
    w0[..., 0] = 10 ** rng.uniform(-0.3, 0.3, w0.shape[:-1])
    w0[..., 1] = 10 ** rng.uniform(-0.3, 0.3, w0.shape[:-1])
    w0[..., 2:5] = rng.uniform(-0.3, 0.3, w0.shape[:-1] + (3,))
    b = dg.Reflective("X") + dg.Periodic("YZ")
    G, R = pair(ns[0], 0.1, w0, b, dg.RIEMANN_HLLC, limiter, ns=ns)
    R.advance(0.02)
    res = G.advance(0.02)
    assert res.steps >= 1
    check(G.w, R.get_prim(), True, f"3d l{limiter}")


def test_3d_exact_solver_statistics():
    """The exact solver's Newton statistics are reported (cap 6 iterations)."""
    n = 10
    w0, d = blast(n, p_in=100.0)
    G, _ = pair(n, d, w0, dg.Outflow(), dg.RIEMANN_EXACT, dg.LIMITER_MC)
    res = G.advance_steps(2)
    assert res.exact_calls > 0
    assert 0 < res.newton_iters <= 6 * res.exact_calls
