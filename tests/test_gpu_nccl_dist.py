"""DistGrid over an NCCL process group, and bench.py's sharded-grid section.

Every GPU call here has one GPU, and NCCL refuses two ranks on one device, so
the group has one rank: the halo buffers then live on the device and the
x-periodic wrap, the CFL all-reduce MIN and the commit all-reduce go through
NCCL, which the gloo tests do not reach. The run is a child process so that
the NCCL group never outlives the test.
"""
import os
import socket
import subprocess
import sys
import textwrap

import pytest

from conftest import ROOT, cuda_ok

pytestmark = pytest.mark.gpu

SCRIPT = textwrap.dedent(r"""
    import json, sys
    sys.path.insert(0, ROOT)
    import numpy as np, torch, torch.distributed as dist
    import dragon_b200 as dg
    from dragon_b200 import problems
    from dragon_b200.dist import DistGrid2D
    import bench

    torch.cuda.set_device(0)
    dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=60))
    out = {}
    cfg = dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_VANLEER)
    w0, dx, dy = problems.kelvin_helmholtz_2d(64, ghosts=2, seed=5, ny=48)
    D = DistGrid2D(64, 48, dx, dy, ghosts=2, config=cfg)
    D.boundary = dg.Periodic()
    D.scatter(w0)
    out["comm_device"] = str(D.comm_device)
    rd = D.advance_steps(6)
    wd = D.gather()
    S = dg.Grid2D(64, 48, dx, dy, ghosts=2, config=cfg)
    S.boundary = dg.Periodic()
    S.w[...] = w0
    rs = S.advance_steps(6)
    out["equal"] = bool(np.array_equal(wd[2:-2, 2:-2], S.w[2:-2, 2:-2]))
    out["time"] = [rd.time_advanced, rs.time_advanced]
    D.local.grid.close()
    S.close()
    out["bench"] = bench.dist_report(1, torch.device("cuda", 0), n=256, steps=3, warmup=1)
    print("RESULT " + json.dumps(out))
    dist.destroy_process_group()
""")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_nccl_one_rank_distgrid_and_bench_section():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0", MASTER_ADDR="127.0.0.1",
               MASTER_PORT=str(_free_port()), NCCL_NVLS_ENABLE="0")
    p = subprocess.run([sys.executable, "-c", f"ROOT = {ROOT!r}\n" + SCRIPT], env=env, cwd=ROOT,
                       capture_output=True, text=True, timeout=240)
    assert p.returncode == 0, p.stderr[-3000:]
    line = [x for x in p.stdout.splitlines() if x.startswith("RESULT ")][-1]
    import json
    r = json.loads(line[len("RESULT "):])
    assert r["comm_device"].startswith("cuda")
    assert r["equal"]
    assert r["time"][0] == r["time"][1]
    b = r["bench"]
    assert b["scaling"] == "strong" and b["steps"] == 3
    assert b["value"] > 0 and b["ms_per_step"] > 0
