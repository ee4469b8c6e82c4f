"""Named workloads of the hot path, runnable from the command line (for
profiling and quick checks on a GPU):

    python -m dragon_b200.workloads kh      --n 1024 --steps 5 [--mixed]
    python -m dragon_b200.workloads ot      --n 512  --steps 5 [--mixed]
    python -m dragon_b200.workloads blast3d --n 128  --steps 3 [--riemann exact] [--mhd] [--mixed]
    python -m dragon_b200.workloads batch   --n1d 256 --n2d 32 --steps 5 [--mixed]
    python -m dragon_b200.workloads hoard   --n 2048 --steps 2 [--level 4]

kh: 2D shear layer (HLLC, van Leer, periodic); ot: 2D MHD Orszag-Tang (HLLD,
MC, CT, periodic); blast3d: 3D blast (MC, outflow; HLLC by default, or the
exact solver, or MHD with a uniform field; --mixed for either); batch: uneven 1D hydro + 2D MHD
grids advanced by the batched step; hoard: the kh grid written to `steps`
files from its device state (write option 3, deflate at --level, 0 for
contiguous datasets) in a temporary directory. Prints one line with steps and
wall time.
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from . import batch as _batch
from . import grid as _grid
from . import problems
from .boundary import Periodic


def kh(n, steps, mixed):
    w0, dx, dy = problems.kelvin_helmholtz_2d(n, ghosts=2, seed=1234)
    cfg = _grid.Config(riemann=_grid.RIEMANN_HLLC, limiter=_grid.LIMITER_VANLEER,
                       precision=_grid.PREC_MIXED if mixed else _grid.PREC_FP64)
    G = _grid.Grid2D(n, n, dx, dy, ghosts=2, config=cfg)
    G.w[...] = w0
    G.boundary = Periodic()
    return G


def ot(n, steps, mixed):
    w0, B0, dx, dy = problems.orszag_tang_2d(n, ghosts=3)
    cfg = _grid.Config(mhd=True, riemann=_grid.RIEMANN_HLLX, precision=_grid.PREC_MIXED if mixed else _grid.PREC_FP64)
    G = _grid.Grid2D(n, n, dx, dy, ghosts=3, config=cfg)
    G.w[...] = w0
    G.B[...] = B0
    G.boundary = Periodic()
    G.initialize_B_fields()
    return G


def blast3d(n, riemann, mhd, mixed=False):
    w5, d = problems.blast_3d(n, ghosts=3 if mhd else 2, p_in=10.0)
    if not mhd:
        cfg = _grid.Config(riemann=riemann, limiter=_grid.LIMITER_MC,
                           precision=_grid.PREC_MIXED if mixed else _grid.PREC_FP64)
        G = _grid.Grid3D(n, n, n, d, d, d, ghosts=2, config=cfg)
        G.w[...] = w5
        return G
    w = np.zeros(w5.shape[:-1] + (8,))
    w[..., :5] = w5
    G = _grid.Grid3D(n, n, n, d, d, d, ghosts=3, config=_grid.Config(mhd=True, riemann=_grid.RIEMANN_HLLX,
                                                                    limiter=_grid.LIMITER_MC,
                                                                    precision=_grid.PREC_MIXED if mixed else
                                                                    _grid.PREC_FP64))
    G.w[...] = w
    B = G.B
    B[..., 0], B[..., 1], B[..., 2] = 0.5, 0.3, 0.2
    G.initialize_B_fields()
    return G


def batch(n1d, n2d, mixed=False):
    one, two = problems.batch_instances(n1d=n1d, n2d=n2d)
    prec = _grid.PREC_MIXED if mixed else _grid.PREC_FP64
    grids = []
    for spec in one:
        G = _grid.Grid1D(spec["n"], spec["dx"], ghosts=2, config=_grid.Config(riemann=_grid.RIEMANN_HLLX,
                                                                                precision=prec))
        G.w[...] = spec["w"]
        grids.append(G)
    for spec in two:
        n = spec["n"]
        G = _grid.Grid2D(n, n, spec["dx"], spec["dx"], ghosts=3, config=_grid.Config(mhd=True, precision=prec))
        G.w[...] = spec["w"]
        G.B[...] = spec["B"]
        G.boundary = Periodic()
        G.initialize_B_fields()
        grids.append(G)
    return _batch.Batch(grids), grids


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("workload", choices=["kh", "ot", "blast3d", "batch", "hoard"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--mhd", action="store_true")
    ap.add_argument("--riemann", default="hllc", choices=["hllc", "exact", "hll", "hlle", "roe"])
    ap.add_argument("--n1d", type=int, default=256)
    ap.add_argument("--n2d", type=int, default=32)
    ap.add_argument("--level", type=int, default=0, help="hoard: deflate level (0: contiguous)")
    a = ap.parse_args(argv)
    rs = {"hllc": _grid.RIEMANN_HLLC, "exact": _grid.RIEMANN_EXACT, "hll": _grid.RIEMANN_HLL,
          "hlle": _grid.RIEMANN_HLLE, "roe": _grid.RIEMANN_ROE}[a.riemann]
    if a.workload == "batch":
        b, grids = batch(a.n1d, a.n2d, a.mixed)
        b.advance_steps(1)
        t = time.perf_counter()
        st = b.advance_steps(a.steps)
        print(f"batch members={len(grids)} steps={a.steps} wall_s={time.perf_counter() - t:.4f} "
              f"replay_ms={st['replay_ms']:.3f}")
        return
    if a.workload == "hoard":
        import shutil
        import tempfile

        from . import hoard
        G = kh(a.n, a.steps, False)
        G.advance_steps(2)
        d = tempfile.mkdtemp(prefix="hoard_")
        hoard.output_dir = d
        t = time.perf_counter()
        for k in range(a.steps):
            hoard.write_to_file(G, 0.0, k, f"frame_{hoard.cycle_string(k)}",
                                opts=hoard.Options(compression_level=a.level))
        print(f"hoard n={a.n} files={a.steps} wall_s={time.perf_counter() - t:.4f}")
        shutil.rmtree(d, ignore_errors=True)
        return
    G = {"kh": lambda: kh(a.n, a.steps, a.mixed), "ot": lambda: ot(a.n, a.steps, a.mixed),
         "blast3d": lambda: blast3d(a.n, rs, a.mhd, a.mixed)}[a.workload]()
    G.advance_steps(1)
    G.w  # noqa: B018  (synchronises)
    t = time.perf_counter()
    r = G.advance_steps(a.steps)
    G.w  # noqa: B018
    print(f"{a.workload} n={a.n} steps={r.steps} wall_s={time.perf_counter() - t:.4f}")


if __name__ == "__main__":
    main()
