"""DistGrid over several ranks == the serial grid, bit for bit.

CPU: gloo ranks whose slabs run on the oracle's C restatement (the halo
exchange, the slab boundary programs, the CFL all-reduce and the
all-or-nothing commit are the host logic of dragon_b200.dist, the same code
the GPU slabs use). The reference's own check is DistGrid vs Grid at rel 1e-26
(Testing/DistGrid_Tests.cpp:18-159); here the arrays are compared exactly.
"""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, build_oracle

sys.path.insert(0, os.path.join(ROOT, "tests"))
import dist_worker  # noqa: E402

from dragon_b200 import boundary as bd  # noqa: E402
from dragon_b200 import dist  # noqa: E402

ALL_CASES = ["kh2d_periodic", "kh2d_mixed", "kh2d_walls", "blast3d", "ot2d_mhd", "blast2d_mhd_walls",
             "blast3d_mhd", "sod1d"]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(world, cases, out, slab="port", fail_rank=-1, timeout=600):
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                   LOCAL_RANK=str(r))
        cmd = [sys.executable, os.path.join(ROOT, "tests", "dist_worker.py"), "--slab", slab, "--cases",
               ",".join(cases), "--out", str(out), "--fail-rank", str(fail_rank)]
        procs.append(subprocess.Popen(cmd, env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT))
    logs = []
    for p in procs:
        try:
            o, _ = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        logs.append(o.decode(errors="replace"))
    for p, log in zip(procs, logs):
        assert p.returncode == 0, log[-3000:]
    return {c: np.load(os.path.join(out, f"{c}.npz")) for c in cases}


@pytest.fixture(scope="module")
def oracle_built():
    build_oracle()


def _check(name, got, serial):
    w, B = serial
    np.testing.assert_array_equal(got["w"], w, err_msg=name)
    if B is not None:
        np.testing.assert_array_equal(got["B"], B, err_msg=name)


@pytest.mark.parametrize("world", [2, 3])
def test_dist_matches_serial(world, tmp_path, oracle_built):
    got = run_ranks(world, ALL_CASES, tmp_path)
    for name in ALL_CASES:
        _check(name, got[name], dist_worker.serial_run(name))
        assert int(got[name]["retries"]) == 0


def test_dist_single_rank_periodic_wrap(tmp_path, oracle_built):
    """One slab periodic in x wraps onto itself through the pack / unpack path."""
    cases = ["kh2d_periodic", "kh2d_mixed", "ot2d_mhd"]
    got = run_ranks(1, cases, tmp_path)
    for name in cases:
        _check(name, got[name], dist_worker.serial_run(name))


def test_dist_all_or_nothing_retry(tmp_path, oracle_built):
    """A slab that fails its first step makes every slab undo theirs and retry
    at half the step (DistGrid.cpp:292-304 with DRAGONWING's checkpoints)."""
    got = run_ranks(2, ["kh2d_retry"], tmp_path, fail_rank=1)["kh2d_retry"]
    assert int(got["retries"]) == 1
    _check("kh2d_retry", got, dist_worker.serial_run("kh2d_retry", fail_first=True))


def test_dist_output_and_restart(tmp_path, oracle_built):
    """DRAGONHOARD on a distributed grid (2 gloo ranks, oracle slabs): rank 0
    writes the gathered grid, and the file holds exactly what the serial
    grid's state writes; a fresh distributed grid restarted from it and
    advanced again ends where the uninterrupted serial run ends, bit for bit."""
    import h5subset
    from dragon_b200 import hoard
    cases = ["kh2d_periodic", "ot2d_mhd", "blast3d"]
    got = run_ranks(2, ["hoard_" + c for c in cases], tmp_path)
    opts = hoard.Options(write_option=7, redundant_vals=2)
    for name in cases:
        dim, n, d, g, cfg, _, _, B0, _, steps = dist_worker.case(name)
        w, B = dist_worker.serial_run(name)
        ref_path = str(tmp_path / f"serial_{name}.h5")
        hoard.write_arrays(ref_path, dim, cfg.mhd, n, g, d, 0.5, steps, w, B, opts)
        fa = h5subset.File(str(tmp_path / f"{name}_{hoard.cycle_string(steps)}.h5"))
        fb = h5subset.File(ref_path)
        assert {k: fa.attrs[k] for k in fa.attrs} == {k: fb.attrs[k] for k in fb.attrs}
        keys = ["/fluid/rho", "/fluid/p", "/fluid/E", "/fluid/v/x", "/fluid/momentum/y"] + \
            (["/fluid/Bf/x", "/fluid/B/z"] if cfg.mhd else [])
        for k in keys:
            np.testing.assert_array_equal(fa[k].read(), fb[k].read(), err_msg=f"{name} {k}")
        _check("hoard_" + name, got["hoard_" + name], dist_worker.serial_run(name, steps=2 * steps))


def test_child_sizes_and_ghosts():
    assert [dist.child_size(10, 3, i) for i in range(3)] == [4, 3, 3]
    assert sum(dist.child_size(1001, 7, i) for i in range(7)) == 1001
    assert dist.valid_ghosts(1, False) == 2 and dist.valid_ghosts(1, True) == 3 and dist.valid_ghosts(4, False) == 4


def test_slab_program_masks_faces():
    b = bd.Outflow("Y-", corner_ghosts=False) + bd.Periodic("XZ") + bd.Reflective("X-")
    # middle slab: no x faces of its own; the periodic element's x part is the wrap exchange
    p = dist.SlabProgram(b, 1, 3, 3)
    assert p.wrap_at is not None
    kinds = [(t, f) for (t, f, c, s) in p.entries]
    # implicit outflow over Y+ (uncovered, every slab touches it)
    assert kinds[0] == (bd.OUTFLOW, bd.Y_positive)
    assert kinds[1] == (bd.OUTFLOW, bd.Y_negative)
    assert kinds[p.wrap_at] == (bd.IGNORE, 0)
    assert kinds[p.wrap_at + 1] == (bd.PERIODIC, bd.Z)
    assert kinds[p.wrap_at + 2] == (bd.REFLECTIVE, 0)  # X- belongs to slab 0 only
    assert kinds[-1] == (bd.IGNORE, 63)
    p0 = dist.SlabProgram(b, 0, 3, 3)
    assert [(t, f) for (t, f, c, s) in p0.entries][p0.wrap_at + 2] == (bd.REFLECTIVE, bd.X_negative)
