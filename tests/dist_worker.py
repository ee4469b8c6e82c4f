"""One rank of a distributed-grid parity run (test infrastructure).

    RANK=r WORLD_SIZE=P MASTER_ADDR=127.0.0.1 MASTER_PORT=... \\
        python tests/dist_worker.py --slab port|gpu --cases a,b --out DIR

Each rank builds dragon_b200.dist.DistGrid{1,2,3}D for every named case with
slabs of the oracle's C restatement (--slab port, CPU) or of the GPU grid
(--slab gpu), loads the case's initial state, advances it and gathers the
global arrays; rank 0 writes DIR/<case>.npz. The serial runs the results are
compared with are in serial_run() below, so the test and the workers share
one definition of each case.
"""
from __future__ import annotations

import argparse
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from dragon_b200 import boundary as bd  # noqa: E402
from dragon_b200 import grid as gr  # noqa: E402
from dragon_b200 import problems  # noqa: E402

IGNORE_ALL = (bd.IGNORE, 63, 1, [0.0] * 8)


def _blast3d_mhd(n, g):
    w5, d = problems.blast_3d(n, ghosts=g, p_in=10.0)
    w = np.zeros(w5.shape[:-1] + (8,))
    w[..., :5] = w5
    B = np.zeros(tuple(x + 1 for x in w5.shape[:-1]) + (3,))
    B[..., 0], B[..., 1], B[..., 2] = 0.5, 0.3, 0.2
    return w, B, d


def _edge_ghosts(w, g):
    """Ghosts copied from the nearest interior cell, so that corner ghosts an
    element without corner_ghosts leaves alone still hold a physical state."""
    inner = w[tuple(slice(g, s - g) for s in w.shape[:-1])]
    return np.pad(inner, [(g, g)] * (w.ndim - 1) + [(0, 0)], mode="edge")


# Device user fills for the distributed-grid case below: the y faces take the
# nearest interior row with vy set from the global x position (c.off[0] is the
# slab's place in the grid), the X- face is a jet of fixed state where
# |y - 0.5| < 0.2.
Y_FILL = """
__device__ void yfill(const dragon_fill_ctx& c, int i, int j, int k) {
    const int js = c.side == 0 ? 0 : c.n[1] - 1;
    for (int f = 0; f < c.nf; f++) c.set(f, i, j, k, c.get(f, i, js, k));
    const double x = (c.off[0] + i + 0.5) * c.d[0];
    c.set(DRAGON_VY, i, j, k, c.params[0] * x * (1.0 - x));
}
"""
JET_FILL = """
__device__ void jet(const dragon_fill_ctx& c, int i, int j, int k) {
    for (int f = 0; f < c.nf; f++) c.set(f, i, j, k, c.get(f, 0, j, k));
    if (fabs((j + 0.5) * c.d[1] - 0.5) < 0.2) {
        c.set(DRAGON_RHO, i, j, k, 2.0);
        c.set(DRAGON_P, i, j, k, 3.0);
        c.set(DRAGON_VX, i, j, k, 1.5);
    }
}
"""


def case(name):
    """(dim, n, d, ghosts, Config, boundary, w0, B0 or None, init_B, steps)."""
    if name == "kh2d_device_fills":
        w, dx, dy = problems.kelvin_helmholtz_2d(24, ghosts=2, seed=9, ny=20)
        w = _edge_ghosts(w, 2)
        cfg = gr.Config(riemann=gr.RIEMANN_HLLC, limiter=gr.LIMITER_MC)
        b = (bd.DeviceGhostFill(Y_FILL, "yfill", faces="Y", params=[0.4]) +
             bd.DeviceGhostFill(JET_FILL, "jet", faces="X-") + bd.Outflow("X+"))
        return 2, (24, 20), (dx, dy), 2, cfg, b, w, None, False, 4
    if name == "kh2d_periodic":
        w, dx, dy = problems.kelvin_helmholtz_2d(24, ghosts=2, seed=7, ny=20)
        cfg = gr.Config(riemann=gr.RIEMANN_HLLC, limiter=gr.LIMITER_VANLEER)
        return 2, (24, 20), (dx, dy), 2, cfg, bd.Periodic(), w, None, False, 3
    if name == "kh2d_mixed":
        w, dx, dy = problems.kelvin_helmholtz_2d(24, ghosts=2, seed=8, ny=20)
        w = _edge_ghosts(w, 2)
        cfg = gr.Config(riemann=gr.RIEMANN_HLLC, limiter=gr.LIMITER_MC)
        b = bd.Outflow("Y-", corner_ghosts=False) + bd.Periodic("X", corner_ghosts=False) + bd.Reflective("Y+")
        return 2, (24, 20), (dx, dy), 2, cfg, b, w, None, False, 3
    if name == "kh2d_walls":
        w, dx, dy = problems.kelvin_helmholtz_2d(24, ghosts=2, seed=9, ny=20)
        w = _edge_ghosts(w, 2)
        cfg = gr.Config(riemann=gr.RIEMANN_HLLX, limiter=gr.LIMITER_MINMOD)
        b = bd.Outflow("Y", corner_ghosts=False) + bd.Reflective("X")
        return 2, (24, 20), (dx, dy), 2, cfg, b, w, None, False, 3
    if name == "blast3d":
        w, d = problems.blast_3d(12, ghosts=2, p_in=10.0)
        cfg = gr.Config(riemann=gr.RIEMANN_HLLC, limiter=gr.LIMITER_MC)
        return 3, (12, 12, 12), (d, d, d), 2, cfg, bd.BoundaryList(), w, None, False, 2
    if name == "ot2d_mhd":
        w, B, dx, dy = problems.orszag_tang_2d(24, ghosts=3)
        cfg = gr.Config(mhd=True, riemann=gr.RIEMANN_HLLX)
        return 2, (24, 24), (dx, dy), 3, cfg, bd.Periodic(), w, B, True, 3
    if name == "blast2d_mhd_walls":
        w, B, d = problems.blast_2d_mhd(24, ghosts=3)
        cfg = gr.Config(mhd=True, riemann=gr.RIEMANN_HLLD, limiter=gr.LIMITER_MINMOD)
        b = bd.Reflective("X") + bd.Periodic("Y")
        return 2, (24, 24), (d, d), 3, cfg, b, w, B, True, 3
    if name == "blast3d_mhd":
        w, B, d = _blast3d_mhd(12, 3)
        cfg = gr.Config(mhd=True, riemann=gr.RIEMANN_HLLX)
        return 3, (12, 12, 12), (d, d, d), 3, cfg, bd.BoundaryList(), w, B, True, 2
    if name == "sod1d":
        w, dx = problems.sod_1d(48, ghosts=2)
        cfg = gr.Config(riemann=gr.RIEMANN_HLLC, limiter=gr.LIMITER_MINMOD)
        return 1, (48,), (dx,), 2, cfg, bd.BoundaryList(), w, None, False, 5
    if name == "kh2d_retry":
        w, dx, dy = problems.kelvin_helmholtz_2d(24, ghosts=2, seed=10, ny=20)
        cfg = gr.Config(riemann=gr.RIEMANN_HLLC, limiter=gr.LIMITER_VANLEER)
        return 2, (24, 20), (dx, dy), 2, cfg, bd.Periodic(), w, None, False, 2
    raise KeyError(name)


def bc_entries(blist):
    out = []
    for e in bd.as_list(blist):
        st = list(e.state()) + [0.0] * 8
        out.append((e.kind, e.get_faces(), int(e.corners), st[:8]))
    return out


class PortSlab:
    """A slab on the CPU oracle with the interface dragon_b200.dist expects of
    a slab (the GPU slab is dragon_b200.dist.GpuSlab)."""

    fail_calls = ()  # try_step call numbers (from 1) that report a failure without stepping

    def __init__(self, dim, n, d, ghosts, config):
        from oracle.port import PortGrid
        c = config
        self.P = PortGrid(dim, n, d, ghosts=ghosts, mhd=c.mhd, riemann=c.riemann, limiter=c.limiter, cfl=c.cfl,
                          ct_energy=c.ct_energy, exact_max_iters=c.exact_max_iters, exact_tol=c.exact_tol,
                          cfl_coeff=c.cfl_coeff, timestep_tol=c.timestep_tol)
        self.dim = dim
        self.n = tuple(n)
        self.ghosts = self.P.ghosts
        self.has_faces = bool(c.mhd) and dim >= 2
        self.entries = []
        self.saved = None
        self.calls = 0

    def set_entries(self, entries, fills=None):
        if fills:
            raise NotImplementedError("device user fills need GPU slabs")
        self.entries = list(entries)

    def apply_range(self, first, count):
        if count <= 0:
            return
        self.P.set_boundary(self.entries[first:first + count] + [IGNORE_ALL])
        self.P.apply_boundary()

    def _slices(self, first, layers, faces, corners):
        g = self.ghosts
        sl = [slice(first + g, first + g + layers)]
        for b in range(1, self.dim):
            nb = self.n[b] + (1 if faces else 0)
            sl.append(slice(0, nb + 2 * g) if corners else slice(g, g + nb))
        return tuple(sl)

    def _array(self, faces):
        return self.P.get_faceB() if faces else self.P.get_prim()

    def halo_count(self, layers, faces, corners):
        a = self._array(faces)
        return int(a[self._slices(0, layers, faces, corners)].size)

    def pack(self, first, layers, faces, corners, buf):
        import torch
        blk = np.moveaxis(self._array(faces)[self._slices(first, layers, faces, corners)], -1, 0)
        buf.copy_(torch.from_numpy(np.ascontiguousarray(blk).ravel()))

    def unpack(self, first, layers, faces, corners, buf):
        a = self._array(faces)
        sl = self._slices(first, layers, faces, corners)
        shape = a[sl].shape
        blk = buf.cpu().numpy().reshape((shape[-1],) + shape[:-1])
        a[sl] = np.moveaxis(blk, 0, -1)
        (self.P.set_faceB if faces else self.P.set_prim)(a)

    def cfl_time(self):
        from oracle.port import PortError
        try:
            return self.P.cfl_time()
        except PortError:
            return None

    def _state(self):
        return (self.P.get_prim(), self.P.get_faceB() if self.has_faces else None)

    def _restore(self, s):
        self.P.set_prim(s[0])
        if s[1] is not None:
            self.P.set_faceB(s[1])

    def try_step(self, dt):
        from oracle.port import PortError
        self.calls += 1
        if self.calls in self.fail_calls:
            return False
        self.saved = self._state()
        try:
            self.P.unsplit_step(dt)
        except PortError:
            self._restore(self.saved)
            return False
        return True

    def rollback(self):
        self._restore(self.saved)

    def initialize_B_fields(self):
        self.P.set_boundary(self.entries + [IGNORE_ALL])
        self.P.initialize_B_fields()

    def get_w(self):
        return self.P.get_prim()

    def set_w(self, a):
        self.P.set_prim(a)

    def get_B(self):
        return self.P.get_faceB()

    def set_B(self, a):
        self.P.set_faceB(a)


def run_case(name, slab_factory, group=None):
    from dragon_b200 import dist
    dim, n, d, g, cfg, blist, w0, B0, init_B, steps = case(name)
    cls = {1: dist.DistGrid1D, 2: dist.DistGrid2D, 3: dist.DistGrid3D}[dim]
    G = cls(*n, *d, ghosts=g, config=cfg, group=group, slab_factory=slab_factory)
    if G.ghosts != g:
        raise RuntimeError(f"case {name}: ghost width {G.ghosts} != {g}")
    G.scatter(w0, B0)
    G.boundary = blist
    if init_B:
        G.initialize_B_fields()
    res = G.advance_steps(steps)
    out = G.gather()
    w, B = (out if isinstance(out, tuple) else (out, None))
    return w, B, res


def run_hoard_case(name, slab_factory, out_dir, group=None):
    """Output and restart of a distributed grid: the case's steps, a frame
    written from the distributed grid, a fresh distributed grid restarted
    from it and advanced by the case's steps again."""
    from dragon_b200 import dist, hoard
    dim, n, d, g, cfg, blist, w0, B0, init_B, steps = case(name)
    cls = {1: dist.DistGrid1D, 2: dist.DistGrid2D, 3: dist.DistGrid3D}[dim]
    hoard.output_dir = out_dir
    G = cls(*n, *d, ghosts=g, config=cfg, group=group, slab_factory=slab_factory)
    G.scatter(w0, B0)
    G.boundary = blist
    if init_B:
        G.initialize_B_fields()
    G.advance_steps(steps)
    hoard.write_to_file(G, 0.5, steps, f"{name}_{hoard.cycle_string(steps)}",
                        opts=hoard.Options(write_option=7, redundant_vals=2))
    H = cls(*n, *d, ghosts=g, config=cfg, group=group, slab_factory=slab_factory)
    H.boundary = blist
    t, cycle = hoard.load_from_file(H, f"{name}_{hoard.cycle_string(steps)}")
    if (t, cycle) != (0.5, steps):
        raise RuntimeError(f"restart returned t={t} cycle={cycle}")
    res = H.advance_steps(steps)
    out = H.gather()
    w, B = (out if isinstance(out, tuple) else (out, None))
    return w, B, res


def serial_run(name, backend="port", fail_first=False, steps=None):
    """The serial grid's run of a case: per step the boundary fill, the CFL
    time, then the step (halved once on the first step when fail_first);
    `steps` overrides the case's step count."""
    dim, n, d, g, cfg, blist, w0, B0, init_B, case_steps = case(name)
    steps = case_steps if steps is None else steps
    if backend == "port":
        from oracle.port import PortGrid
        c = cfg
        P = PortGrid(dim, n, d, ghosts=g, mhd=c.mhd, riemann=c.riemann, limiter=c.limiter, cfl=c.cfl,
                     ct_energy=c.ct_energy, exact_max_iters=c.exact_max_iters, exact_tol=c.exact_tol,
                     cfl_coeff=c.cfl_coeff, timestep_tol=c.timestep_tol)
        P.set_prim(w0)
        if B0 is not None:
            P.set_faceB(B0)
        P.set_boundary(bc_entries(blist))
        if init_B:
            P.initialize_B_fields()
        for s in range(steps):
            P.apply_boundary()
            dt = P.cfl_time()
            if fail_first and s == 0:
                dt *= 0.5
            P.unsplit_step(dt)
        return P.get_prim(), (P.get_faceB() if B0 is not None else None)
    cls = {1: gr.Grid1D, 2: gr.Grid2D, 3: gr.Grid3D}[dim]
    G = cls(*n, *d, ghosts=g, config=cfg)
    G.w[...] = w0
    if B0 is not None:
        G.B[...] = B0
    G.boundary = blist
    if init_B:
        G.initialize_B_fields()
    G.advance_steps(steps)
    return G.w.copy(), (G.B.copy() if B0 is not None else None)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--slab", choices=["port", "gpu"], default="port")
    ap.add_argument("--cases", required=True)
    ap.add_argument("--out", required=True)
    ap.add_argument("--fail-rank", type=int, default=-1)
    a = ap.parse_args()
    import torch.distributed as tdist
    tdist.init_process_group("gloo", init_method="env://")
    rank = tdist.get_rank()
    factory = None
    if a.slab == "port":
        factory = PortSlab
        if rank == a.fail_rank:
            class FailingSlab(PortSlab):
                fail_calls = (1,)
            factory = FailingSlab
    for name in a.cases.split(","):
        if name.startswith("hoard_"):
            w, B, res = run_hoard_case(name[len("hoard_"):], factory, a.out)
        else:
            w, B, res = run_case(name, factory)
        if rank == 0:
            np.savez(os.path.join(a.out, f"{name}.npz"), w=w, B=B if B is not None else np.zeros(0),
                     steps=res.steps, retries=res.retries, last_dt=res.last_dt)
    tdist.barrier()
    tdist.destroy_process_group()


if __name__ == "__main__":
    main()
