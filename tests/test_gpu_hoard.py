"""Output and restart from device buffers (DRAGONHOARD, HDF5Output.cpp /
HDF5Restart.cpp) on the GPU.

* Snapshots written by the device pack match the oracle's restatement of
  writeToFile (oracle/hoard_port.py) bit for bit, for 1D / 2D / 3D, hydro and
  MHD, every write option, redundant-value precision, ghosts on and off,
  deflated and contiguous files; read back with the test-side HDF5 reader.
* Asynchronous snapshots taken between steps hold the state of the moment
  they were taken, with two files in flight.
* Restart: the reference's round trips (Testing/Core/IO_Tests.cpp:46-272,
  tagged states on 5, 3x4 and 3x4x5 grids with 2 ghosts), its dimension and
  size checks, the conservative restart, and a run continued from a file that
  ends where the uninterrupted run ends.
"""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

import dragon_b200 as dg  # noqa: E402
from dragon_b200 import hoard, problems  # noqa: E402
import h5subset  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not cuda_ok():
        pytest.fail("CUDA device required for -m gpu tests")


@pytest.fixture(autouse=True)
def _outdir(tmp_path, monkeypatch):
    monkeypatch.setattr(hoard, "output_dir", str(tmp_path))
    monkeypatch.setattr(hoard, "options", hoard.Options())
    return tmp_path


def _port():
    from oracle import hoard_port
    return hoard_port


SHAPES = {1: (37,), 2: (19, 45), 3: (9, 13, 11)}


def _grid(dim, mhd, ghosts=2, seed=0):
    n = SHAPES[dim]
    d = (0.1, 0.2, 0.3)[:dim]
    cfg = dg.Config(mhd=mhd, riemann=dg.RIEMANN_HLLD if mhd else dg.RIEMANN_HLLC)
    G = {1: dg.Grid1D, 2: dg.Grid2D, 3: dg.Grid3D}[dim](*n, *d, ghosts=ghosts, config=cfg)
    rng = np.random.default_rng(seed)
    w = G.w
    w[...] = rng.uniform(-1, 1, w.shape)
    w[..., 0] = rng.uniform(0.5, 2.0, w.shape[:-1])
    w[..., 1] = rng.uniform(0.1, 3.0, w.shape[:-1])
    if mhd and dim > 1:
        G.B[...] = rng.uniform(-1, 1, G.B.shape)
    return G, n, d


def _files(path):
    f = h5subset.File(path)
    out = {}

    def walk(g, prefix):
        for k in g.keys():
            o = g[k]
            if isinstance(o, h5subset.Group):
                walk(o, prefix + "/" + k)
            else:
                out[prefix + "/" + k] = o.read()
    walk(f, "")
    return f, out


def _check_file(path, G, n, d, dim, mhd, t, cycle, opt, red, ghosts):
    P = _port()
    f, got = _files(path)
    want = P.expected_datasets(G.w, G.B if (mhd and dim > 1) else None, dim, mhd, ghosts, G.ghosts, opt, red)
    assert sorted(got) == sorted(want)
    for k, v in want.items():
        assert got[k].dtype == v.dtype, k
        assert got[k].shape == v.shape, k
        np.testing.assert_array_equal(got[k], v, err_msg=k)
    attrs = P.expected_attrs(dim, mhd, n, d, ghosts, G.ghosts, t, cycle, opt)
    assert {k: f.attrs[k] for k in f.attrs} == attrs


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("mhd", [False, True])
@pytest.mark.parametrize("opt,red,ghosts,level", [(3, 1, False, 4), (7, 2, True, 0), (6, 0, False, 9),
                                                  (1, 1, True, 4), (3, 0, False, 0), (3, 2, False, 1)])
def test_snapshot_matches_oracle(tmp_path, dim, mhd, opt, red, ghosts, level):
    G, n, d = _grid(dim, mhd, seed=dim * 10 + opt)
    o = hoard.Options(write_option=opt, redundant_vals=red, compression_level=level, write_ghosts=ghosts)
    hoard.write_to_file(G, 0.666, 666, "snap", opts=o)
    _check_file(str(tmp_path / "snap.h5"), G, n, d, dim, mhd, 0.666, 666, opt, red, ghosts)
    G.close()


def test_snapshot_after_steps_is_the_stepped_state(tmp_path):
    """The pack reads the buffer the last step wrote (the double buffer flips)."""
    n = 64
    w0, dx, dy = problems.kelvin_helmholtz_2d(n, ghosts=2, seed=5)
    G = dg.Grid2D(n, n, dx, dy, ghosts=2)
    G.w[...] = w0
    G.boundary = dg.Periodic()
    for steps in (1, 2, 3):
        G.advance_steps(1)
        hoard.write_to_file(G, float(steps), steps, f"kh_{hoard.cycle_string(steps)}")
        _check_file(str(tmp_path / f"kh_{hoard.cycle_string(steps)}.h5"), G, (n, n), (dx, dy), 2, False,
                    float(steps), steps, 3, 1, False)


def test_async_snapshots_hold_their_moment(tmp_path):
    """Snapshots every 3 steps with two in flight: each file holds the state of
    the moment it was taken, not a later one."""
    n = 96
    w0, B0, dx, dy = problems.orszag_tang_2d(n, ghosts=3)
    G = dg.Grid2D(n, n, dx, dy, ghosts=3, config=dg.Config(mhd=True))
    G.w[...] = w0
    G.B[...] = B0
    G.boundary = dg.Periodic()
    G.initialize_B_fields()
    expect = []
    for k in range(5):
        hoard.write_to_file(G, 0.1 * k, k, f"ot_{k}", wait=False, opts=hoard.Options(write_option=7, redundant_vals=2))
        expect.append((G.w.copy(), G.B.copy()))
        G.advance_steps(3)
    hoard.wait(G)
    P = _port()
    for k, (w, B) in enumerate(expect):
        _, got = _files(str(tmp_path / f"ot_{k}.h5"))
        want = P.expected_datasets(w, B, 2, True, False, 3, 7, 2)
        for key, v in want.items():
            np.testing.assert_array_equal(got[key], v, err_msg=f"frame {k} {key}")


def test_async_failure_surfaces_on_wait(tmp_path):
    G, n, d = _grid(2, False)
    G._to_device()
    rc = G._lib.dragon_gpu_hoard_write_async(G._h, 0.0, 0, str(tmp_path / "no" / "such" / "dir.h5").encode(), None)
    assert rc == 0
    with pytest.raises(dg.grid._lib.DragonGPUError):
        hoard.wait(G)
    hoard.write_to_file(G, 0.0, 0, "fine")  # the grid stays usable
    _check_file(str(tmp_path / "fine.h5"), G, n, d, 2, False, 0.0, 0, 3, 1, False)


def test_invalid_write_option_is_refused():
    G, _, _ = _grid(2, False)
    for opt in (0, 2):
        with pytest.raises(dg.grid._lib.DragonGPUError):
            hoard.write_to_file(G, 0.0, 0, "bad", opts=hoard.Options(write_option=opt))


def _tag(G, dim, mhd):
    """IO_Tests.cpp: make_tagged_state(i*0.1 + j*0.01 + k*0.001) in every cell,
    make_tagged_A(...) on every face."""
    g = G.ghosts
    idx = np.meshgrid(*[np.arange(s) - g for s in G.w.shape[:dim]], indexing="ij")
    tag = sum(c * s for c, s in zip((0.1, 0.01, 0.001), idx))
    nf = G.nfields
    for f in range(nf):
        G.w[..., f] = tag + 10 * f
    G.w[..., 0] += 1.0  # positive density and pressure
    G.w[..., 1] += 1.0
    if mhd and dim > 1:
        fidx = np.meshgrid(*[np.arange(s) - g for s in G.B.shape[:dim]], indexing="ij")
        ftag = sum(c * s for c, s in zip((0.1, 0.01, 0.001), fidx))
        for c in range(3):
            G.B[..., c] = ftag + 100 * (c + 1)


@pytest.mark.parametrize("dim,n,d", [(1, (5,), (0.1,)), (2, (3, 4), (0.1, 0.2)), (3, (3, 4, 5), (0.1, 0.2, 0.3))])
@pytest.mark.parametrize("mhd", [False, True])
@pytest.mark.parametrize("ghosts", [False, True])
def test_reference_io_round_trip(dim, n, d, mhd, ghosts):
    """IO_Tests.cpp:46-203: write a tagged grid, read it into a fresh grid of
    the same extents (spacing 0): t, cycle and spacing come back, the cells of
    the file's range match (B within float precision when stored as float),
    face B matches, and writing left the grid unchanged."""
    cls = {1: dg.Grid1D, 2: dg.Grid2D, 3: dg.Grid3D}[dim]
    cfg = dg.Config(mhd=mhd)
    G = cls(*n, *d, ghosts=2, config=cfg)
    _tag(G, dim, mhd)
    w_before = G.w.copy()
    B_before = G.B.copy() if (mhd and dim > 1) else None
    hoard.options = hoard.Options(write_ghosts=ghosts)
    hoard.write_to_file(G, 0.666, 666, "TEMP_IO")
    np.testing.assert_array_equal(G.w, w_before)
    if B_before is not None:
        np.testing.assert_array_equal(G.B, B_before)
    G2 = cls(*n, *([0.0] * dim), ghosts=2, config=cfg)
    t, cyc = hoard.load_from_file(G2, "TEMP_IO" if dim == 1 else "TEMP_IO.h5")
    assert t == 0.666 and cyc == 666
    assert [getattr(G2, k) for k in ("dx", "dy", "dz")[:dim]] == list(d)
    g = 0 if ghosts else G.ghosts  # MHD grids raise the ghost width to 3 (validGhosts)
    sl = tuple(slice(g, s - g) for s in G.w.shape[:dim])
    a, b = G.w[sl], G2.w[sl]
    np.testing.assert_array_equal(a[..., :5], b[..., :5])
    if mhd:
        if dim == 1:
            np.testing.assert_array_equal(a[..., 5:], b[..., 5:])
        else:
            np.testing.assert_allclose(b[..., 5:], a[..., 5:], rtol=10 * np.finfo(np.float32).eps, atol=1e-7)
            fs = tuple(slice(g, s - g) for s in G.B.shape[:dim])
            np.testing.assert_array_equal(G.B[fs], G2.B[fs])
    if not ghosts:  # cells outside the file's range keep the fresh grid's zeros
        assert np.all(G2.w[(slice(0, G.ghosts),) + (slice(None),) * (dim - 1)] == 0)


def test_reference_io_dimension_and_size_checks():
    """IO_Tests.cpp:205-272: loading into a grid of another dimension or size fails."""
    G = dg.Grid2D(3, 4, 0.1, 0.2, ghosts=2)
    _tag(G, 2, False)
    hoard.write_to_file(G, 0.666, 666, "TEMP_IO")
    for other in (dg.Grid1D(12, 0.1, ghosts=2), dg.Grid3D(3, 4, 1, 0.1, 0.2, 0.3, ghosts=2)):
        with pytest.raises(dg.grid._lib.DragonGPUError, match="Expected"):
            hoard.load_from_file(other, "TEMP_IO")
    for other in (dg.Grid2D(4, 3, 0.1, 0.2, ghosts=2), dg.Grid2D(3, 5, 0.1, 0.2, ghosts=2)):
        with pytest.raises(dg.grid._lib.DragonGPUError, match="File size does not match"):
            hoard.load_from_file(other, "TEMP_IO")
    M = dg.Grid2D(3, 4, 0.1, 0.2, ghosts=2, config=dg.Config(mhd=True))
    _tag(M, 2, True)
    hoard.write_to_file(M, 0.0, 0, "TEMP_MHD")
    with pytest.raises(dg.grid._lib.DragonGPUError, match="MHD"):
        hoard.load_from_file(G, "TEMP_MHD")


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("mhd", [False, True])
@pytest.mark.parametrize("opt,red,ghosts", [(6, 1, False), (7, 0, True), (3, 0, False), (1, 2, True)])
def test_restart_matches_oracle(tmp_path, dim, mhd, opt, red, ghosts):
    """The restored state equals the oracle's restatement of loadFromFile,
    including the conservative restart (rho, momentum, E -> primitive) and
    omitted cell B."""
    G, n, d = _grid(dim, mhd, seed=dim + opt)
    o = hoard.Options(write_option=opt, redundant_vals=red, write_ghosts=ghosts)
    hoard.write_to_file(G, 1.5, 9, "r", opts=o)
    H, _, _ = _grid(dim, mhd, seed=99)
    w0 = H.w.copy()
    B0 = H.B.copy() if (mhd and dim > 1) else None
    t, cyc = hoard.load_from_file(H, "r")
    assert (t, cyc) == (1.5, 9)
    _, files = _files(str(tmp_path / "r.h5"))
    w, B = _port().restored_state(w0, B0, files, dim, mhd, mhd, H.ghosts, H.ghosts if ghosts else 0, opt)
    np.testing.assert_array_equal(H.w, w)
    if B is not None:
        np.testing.assert_array_equal(H.B, B)


@pytest.mark.parametrize("mhd", [False, True])
def test_continued_run_ends_where_the_uninterrupted_run_ends(mhd):
    """Advance 6 steps, write (double redundant values), restart a fresh grid
    from the file, advance 6 more: the state equals 12 uninterrupted steps."""
    n = 64
    if mhd:
        w0, B0, dx, dy = problems.orszag_tang_2d(n, ghosts=3)
        cfg, g = dg.Config(mhd=True), 3
    else:
        w0, dx, dy = problems.kelvin_helmholtz_2d(n, ghosts=2, seed=3)
        B0, cfg, g = None, dg.Config(), 2

    def fresh():
        G = dg.Grid2D(n, n, dx, dy, ghosts=g, config=cfg)
        G.boundary = dg.Periodic()
        return G

    A = fresh()
    A.w[...] = w0
    if mhd:
        A.B[...] = B0
        A.initialize_B_fields()
    A.advance_steps(6)
    hoard.write_to_file(A, 0.0, 6, "mid", opts=hoard.Options(write_option=1, redundant_vals=2))
    A.advance_steps(6)
    C = fresh()
    hoard.load_from_file(C, "mid")
    C.advance_steps(6)
    np.testing.assert_array_equal(C.w[g:-g, g:-g], A.w[g:-g, g:-g])
    if mhd:
        np.testing.assert_array_equal(C.B[g:-g, g:-g], A.B[g:-g, g:-g])


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("mhd", [False, True])
def test_device_pack_equals_host_writer(tmp_path, dim, mhd):
    """The file written from the device state and the file the host writer
    builds from the same state's host arrays hold the same datasets and
    attributes, bit for bit (write option 7, float redundant values)."""
    G, n, d = _grid(dim, mhd, seed=40 + dim)
    o = hoard.Options(write_option=7, redundant_vals=1, write_ghosts=True)
    hoard.write_to_file(G, 0.5, 5, "dev", opts=o)
    hoard.write_arrays(str(tmp_path / "host.h5"), dim, mhd, n, G.ghosts, d, 0.5, 5, G.w,
                       G.B if (mhd and dim > 1) else None, o)
    fa, a = _files(str(tmp_path / "dev.h5"))
    fb, b = _files(str(tmp_path / "host.h5"))
    assert sorted(a) == sorted(b)
    for k in a:
        assert a[k].dtype == b[k].dtype
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    assert {k: fa.attrs[k] for k in fa.attrs} == {k: fb.attrs[k] for k in fb.attrs}


def test_restart_waits_for_the_grids_own_file(tmp_path):
    """A restart that names a file the same grid is still writing reads the
    complete file: the load waits for the grid's writers first."""
    G, n, d = _grid(3, True, seed=77)
    w0, B0 = G.w.copy(), G.B.copy()
    hoard.write_to_file(G, 2.0, 4, "inflight", wait=False,
                        opts=hoard.Options(write_option=1, redundant_vals=2, compression_level=9))
    G.w[...] = 1.0  # changed after the snapshot, restored by the restart below
    t, cycle = hoard.load_from_file(G, "inflight")
    assert (t, cycle) == (2.0, 4)
    g = G.ghosts
    sl = (slice(g, -g),) * 3
    np.testing.assert_array_equal(G.w[sl], w0[sl])
    np.testing.assert_array_equal(G.B[sl], B0[sl])
    hoard.wait(G)


def test_full_size_snapshot_round_trip(tmp_path):
    """The 1024^2 shear layer (the benchmark's grid) after 3 steps: a deflated
    file (1024 chunks of 32 x 32 per dataset, two-level chunk B-trees) restarts
    a fresh grid to the same interior bit for bit, and equals the host
    writer's file of the same state."""
    n = 1024
    w0, dx, dy = problems.kelvin_helmholtz_2d(n, ghosts=2, seed=1234)
    G = dg.Grid2D(n, n, dx, dy, ghosts=2)
    G.w[...] = w0
    G.boundary = dg.Periodic()
    G.advance_steps(3)
    o = hoard.Options(write_option=1, compression_level=4)
    hoard.write_to_file(G, 0.01, 3, "big", opts=o)
    H = dg.Grid2D(n, n, dx, dy, ghosts=2)
    t, cycle = hoard.load_from_file(H, "big")
    assert (t, cycle) == (0.01, 3)
    np.testing.assert_array_equal(H.w[2:-2, 2:-2], G.w[2:-2, 2:-2])
    hoard.write_arrays(str(tmp_path / "host.h5"), 2, False, (n, n), 2, (dx, dy), 0.01, 3, G.w, None, o)
    _, a = _files(str(tmp_path / "big.h5"))
    _, b = _files(str(tmp_path / "host.h5"))
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
