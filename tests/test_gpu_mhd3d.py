"""GPU parity of the 3D MHD CTU + CT step (6-solve ctu_sweep_MHD, 3D edge E
with Gardiner-Stone upwinding, 3D Faraday) against the reference: bit for bit
on random and blast states, every solver and CT energy mode, ragged grids and
mixed boundaries; div B at roundoff for a divergence-free start."""
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


def oracle(ns, ds, riemann, limiter, ct):
    from oracle import port, refgrid
    kw = dict(dim=3, n=ns, d=ds, ghosts=3, mhd=True, riemann=riemann, limiter=limiter, ct_energy=ct)
    variant = "mhd" if ct == 2 else "mhd_rt"
    if refgrid.available(variant):
        return refgrid.RefGrid(ct_runtime=(ct != 2), **kw)
    return port.PortGrid(**kw)


def same(a, b, what):
    bad = np.argwhere(~((a == b) | (np.isnan(a) & np.isnan(b))))
    assert bad.size == 0, f"{what}: {len(bad)} mismatches, first {bad[:3].tolist()}"


def pair(w0, B0, ns, ds, boundary, riemann=dg.RIEMANN_HLLX, limiter=dg.LIMITER_MC, ct=2):
    G = dg.Grid3D(*ns, *ds, ghosts=3, config=dg.Config(mhd=True, riemann=riemann, limiter=limiter, ct_energy=ct))
    R = oracle(ns, ds, riemann, limiter, ct)
    G.w[...] = w0
    G.B[...] = B0
    R.set_prim(w0)
    R.set_faceB(B0)
    G.boundary = boundary
    from oracle.refgrid import bc_entries_from
    R.set_boundary(bc_entries_from(dg.boundary.as_list(boundary)))
    G.initialize_B_fields()
    R.initialize_B_fields()
    same(G.w, R.get_prim(), "initialize_B_fields cells")
    same(G.B, R.get_faceB(), "initialize_B_fields faces")
    return G, R


def random_state(ns, seed, g=3):
    rng = np.random.default_rng(seed)
    shape = tuple(n + 2 * g for n in ns)
    w = np.zeros(shape + (8,))
    w[..., 0] = 10 ** rng.uniform(-0.3, 0.3, shape)
    w[..., 1] = 10 ** rng.uniform(-0.3, 0.3, shape)
    w[..., 2:5] = rng.uniform(-0.3, 0.3, shape + (3,))
    b = np.zeros(tuple(n + 1 + 2 * g for n in ns) + (3,))
    b[..., 0], b[..., 1], b[..., 2] = 0.3, -0.2, 0.1
    b += rng.uniform(-0.01, 0.01, b.shape)
    return w, b


def blast_mhd_3d(n, p_in=10.0, B=(0.5, 0.3, 0.2), g=3):
    w5, d = problems.blast_3d(n, ghosts=g, p_in=p_in)
    w = np.zeros(w5.shape[:-1] + (8,))
    w[..., :5] = w5
    w[..., 0] = np.where(w[..., 0] > 0, w[..., 0], 1.0)
    w[..., 1] = np.where(w[..., 1] > 0, w[..., 1], 0.1)
    b = np.zeros(tuple(n + 1 + 2 * g for _ in range(3)) + (3,))
    b[..., 0], b[..., 1], b[..., 2] = B
    return w, b, d


def divb_max(B, g, n):
    nx, ny, nz = n
    s = (slice(g, g + nx), slice(g, g + ny), slice(g, g + nz))
    d = (B[g + 1:g + nx + 1, g:g + ny, g:g + nz, 0] - B[s + (0,)]) + \
        (B[g:g + nx, g + 1:g + ny + 1, g:g + nz, 1] - B[s + (1,)]) + \
        (B[g:g + nx, g:g + ny, g + 1:g + nz + 1, 2] - B[s + (2,)])
    return np.abs(d).max()


@pytest.mark.parametrize("riemann", [dg.RIEMANN_HLLD, dg.RIEMANN_HLL, dg.RIEMANN_HLLE])
@pytest.mark.parametrize("ct", [0, 1, 2])
def test_mhd3d_random_periodic(riemann, ct):
    ns = (7, 8, 6)
    w0, B0 = random_state(ns, seed=riemann * 3 + ct)
    G, R = pair(w0, B0, ns, (0.1, 0.12, 0.09), dg.Periodic(), riemann=riemann, ct=ct)
    for _ in range(3):
        R.step_cfl()
    res = G.advance_steps(3)
    assert res.steps == 3
    same(G.w, R.get_prim(), f"cells s{riemann} ct{ct}")
    same(G.B, R.get_faceB(), f"faces s{riemann} ct{ct}")


@pytest.mark.parametrize("limiter", [dg.LIMITER_MINMOD, dg.LIMITER_VANLEER])
def test_mhd3d_blast_divb(limiter):
    n = 14
    w0, B0, d = blast_mhd_3d(n)
    G, R = pair(w0, B0, (n, n, n), (d, d, d), dg.Outflow(), limiter=limiter)
    R.advance(0.01)
    res = G.advance(0.01)
    assert res.steps >= 2
    same(G.w, R.get_prim(), "blast cells")
    same(G.B, R.get_faceB(), "blast faces")
    assert divb_max(G.B, 3, (n, n, n)) < 1e-13


def test_mhd3d_ragged_mixed_boundaries():
    ns = (9, 6, 11)
    w0, B0 = random_state(ns, seed=42)
    b = dg.Reflective("X") + dg.Periodic("YZ")
    G, R = pair(w0, B0, ns, (0.1, 0.1, 0.1), b, limiter=dg.LIMITER_SUPERBEE)
    R.advance(0.02)
    res = G.advance(0.02)
    assert res.steps >= 1
    same(G.w, R.get_prim(), "ragged cells")
    same(G.B, R.get_faceB(), "ragged faces")
