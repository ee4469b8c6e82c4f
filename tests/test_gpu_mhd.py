"""GPU parity of the MHD path (2D CTU + constrained transport, 1D HLLD sweep)
against the reference's MHD builds. HLLD / HLL / HLLE use no pow, so the
device results must be bit-identical to the reference's; div B of the face
field stays at FP64 roundoff."""
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
    variant = ("mhd_rt" if kw.get("ct_runtime") else "mhd")
    if refgrid.available(variant):
        return refgrid.RefGrid(**kw)
    kw.pop("ct_runtime", None)
    return port.PortGrid(**kw)


def same(a, b, what):
    bad = np.argwhere(~((a == b) | (np.isnan(a) & np.isnan(b))))
    assert bad.size == 0, f"{what}: {len(bad)} mismatches, first {bad[:3].tolist()}: {a[tuple(bad[0])]} vs " \
                          f"{b[tuple(bad[0])]}"


def divb_max(B, g, n, dx, dy):
    d = (B[g + 1:g + n + 1, g:g + n, 0] - B[g:g + n, g:g + n, 0]) / dx + \
        (B[g:g + n, g + 1:g + n + 1, 1] - B[g:g + n, g:g + n, 1]) / dy
    return np.abs(d).max()


def mhd_pair(w0, B0, n, dx, dy, boundary, riemann=dg.RIEMANN_HLLX, limiter=dg.LIMITER_MC, ct=2):
    cfg = dg.Config(mhd=True, riemann=riemann, limiter=limiter, ct_energy=ct)
    G = dg.Grid2D(n, n, dx, dy, ghosts=3, config=cfg)
    R = oracle_grid(dim=2, n=(n, n), d=(dx, dy), ghosts=3, mhd=True, ct_runtime=(ct != 2), riemann=riemann,
                    limiter=limiter, ct_energy=ct)
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


def test_orszag_tang_bitwise_and_divb():
    """BASELINE 2D MHD setup (Orszag-Tang, HLLD, MC, CTU+CT, BETA_GATED) at 48^2."""
    n = 48
    w0, B0, dx, dy = problems.orszag_tang_2d(n, ghosts=3)
    G, R = mhd_pair(w0, B0, n, dx, dy, dg.Periodic())
    dts = [R.step_cfl() for _ in range(12)]
    res = G.advance_steps(12)
    assert res.steps == 12 and res.last_dt == dts[-1]
    same(G.w, R.get_prim(), "OT cells")
    same(G.B, R.get_faceB(), "OT faces")
    assert divb_max(G.B, 3, n, dx, dy) * dx < 1e-13


@pytest.mark.parametrize("riemann", [dg.RIEMANN_HLLD, dg.RIEMANN_HLL, dg.RIEMANN_HLLE])
@pytest.mark.parametrize("ct", [0, 1, 2])
def test_mhd_solvers_and_energy_modes(riemann, ct):
    n = 20
    w0, B0, dx, dy = problems.orszag_tang_2d(n, ghosts=3, B0=0.9)
    G, R = mhd_pair(w0, B0, n, dx, dy, dg.Periodic(), riemann=riemann, limiter=dg.LIMITER_VANLEER, ct=ct)
    for _ in range(5):
        R.step_cfl()
    G.advance_steps(5)
    same(G.w, R.get_prim(), f"cells s{riemann} ct{ct}")
    same(G.B, R.get_faceB(), f"faces s{riemann} ct{ct}")


@pytest.mark.parametrize("bc", ["outflow", "reflective", "mixed"])
def test_mhd_blast_boundaries(bc):
    n = 24
    w0, B0, dx = problems.blast_2d_mhd(n, ghosts=3)
    b = {"outflow": dg.Outflow(), "reflective": dg.Reflective(),
         "mixed": dg.Reflective("X") + dg.Outflow("Y+") + dg.Fixed([1.0, 0.1, 0, 0, 0, 0.5, 0.5, 0.0], "Y-", False)}[bc]
    G, R = mhd_pair(w0, B0, n, dx, dx, b, limiter=dg.LIMITER_MINMOD)
    R.advance(0.02)
    res = G.advance(0.02)
    assert res.steps > 1
    same(G.w, R.get_prim(), f"blast cells {bc}")
    same(G.B, R.get_faceB(), f"blast faces {bc}")


def test_mhd_blast_ignore_keeps_ghosts():
    """Ignore on the x faces (Ignore.cpp): those ghost cells and faces are
    never filled, so every step must carry them over from the state it read
    (the step writes only the interior; its output buffers take the rest of
    the input's cells and faces) exactly as the reference, which never
    touches them."""
    n = 24
    g = 3
    w0, B0, dx = problems.blast_2d_mhd(n, ghosts=g)
    # ghosts start as copies of the nearest interior cell / face
    w0 = np.pad(w0[g:g + n, g:g + n], ((g, g), (g, g), (0, 0)), mode="edge")
    B0 = np.pad(B0[g:g + n + 1, g:g + n + 1], ((g, g), (g, g), (0, 0)), mode="edge")
    b = dg.Ignore("X") + dg.Periodic("Y")
    G, R = mhd_pair(w0, B0, n, dx, dx, b, limiter=dg.LIMITER_MC)
    w_init, B_init = np.array(G.w), np.array(G.B)
    R.advance(0.02)
    res = G.advance(0.02)
    assert res.steps > 1
    same(G.w, R.get_prim(), "blast cells, ignore x")
    same(G.B, R.get_faceB(), "blast faces, ignore x")
    # the x ghost layers are exactly what initialize_B_fields left there
    np.testing.assert_array_equal(G.w[:g, g:-g], w_init[:g, g:-g])
    np.testing.assert_array_equal(G.w[-g:, g:-g], w_init[-g:, g:-g])
    np.testing.assert_array_equal(G.B[:g, g:-g], B_init[:g, g:-g])


def test_mhd_1d_hlld_sweep():
    """Brio-Wu-like shock tube through the 1D sweep with HLLD (cell B only)."""
    n = 256
    g = 3
    w = np.zeros((n + 2 * g, 8))
    x = (np.arange(n) + 0.5) / n
    L = x < 0.5
    w[g:g + n, 0] = np.where(L, 1.0, 0.125)
    w[g:g + n, 1] = np.where(L, 1.0, 0.1)
    w[g:g + n, 5] = 0.75 * np.sqrt(4 * np.pi)
    w[g:g + n, 6] = np.where(L, 1.0, -1.0) * np.sqrt(4 * np.pi)
    cfg = dg.Config(mhd=True, riemann=dg.RIEMANN_HLLD, limiter=dg.LIMITER_MC)
    G = dg.Grid1D(n, 1.0 / n, ghosts=3, config=cfg)
    R = oracle_grid(dim=1, n=(n,), d=(1.0 / n,), ghosts=3, mhd=True, riemann=dg.RIEMANN_HLLD, limiter=1)
    G.w[...] = w
    R.set_prim(w)
    R.advance(0.05)
    G.advance(0.05)
    same(G.w, R.get_prim(), "1D MHD")
