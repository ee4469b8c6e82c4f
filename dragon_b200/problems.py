"""Initial conditions of the standard test problems, as padded numpy arrays in
the reference's memory order (cells i slowest, ghosts included, NF primitive
fields rho, p, vx, vy, vz[, Bx, By, Bz]).

These restate the workloads the path is measured on: the 1D Sod tube, the 2D
Kelvin-Helmholtz shear layer, the 2D Orszag-Tang vortex and the 3D blast. Cell
centres sit at (i + 1/2) * dx from the domain origin; ghosts are left zero
(the boundary fill sets them).
"""
from __future__ import annotations

import math

import numpy as np


def _centres(n, lo, hi):
    d = (hi - lo) / n
    return lo + (np.arange(n) + 0.5) * d, d


def sod_1d(n=512, ghosts=2, x0=0.5, left=(1.0, 0.0, 1.0), right=(0.125, 0.0, 0.1)):
    """1D two-state Riemann problem on [0,1]: (rho, u, p) left / right of x0."""
    x, dx = _centres(n, 0.0, 1.0)
    w = np.zeros((n + 2 * ghosts, 5))
    L = x < x0
    w[ghosts:ghosts + n, 0] = np.where(L, left[0], right[0])
    w[ghosts:ghosts + n, 2] = np.where(L, left[1], right[1])
    w[ghosts:ghosts + n, 1] = np.where(L, left[2], right[2])
    return w, dx


def kelvin_helmholtz_2d(n=1024, ghosts=2, seed=1234, amp=0.01, ny=None):
    """Periodic unit-square shear layer: rho=2, vx=+0.5 for |y-0.5|<0.25, else
    rho=1, vx=-0.5; p=2.5; vy uniform noise of amplitude amp per cell from a
    seeded generator (numpy PCG64, seed)."""
    ny = ny or n
    x, dx = _centres(n, 0.0, 1.0)
    y, dy = _centres(ny, 0.0, 1.0)
    rng = np.random.Generator(np.random.PCG64(seed))
    vy = rng.uniform(-amp, amp, size=(n, ny))
    inner = np.abs(y - 0.5) < 0.25
    w = np.zeros((n + 2 * ghosts, ny + 2 * ghosts, 5))
    sl = (slice(ghosts, ghosts + n), slice(ghosts, ghosts + ny))
    w[sl + (0,)] = np.where(inner[None, :], 2.0, 1.0)
    w[sl + (1,)] = 2.5
    w[sl + (2,)] = np.where(inner[None, :], 0.5, -0.5)
    w[sl + (3,)] = vy
    return w, dx, dy


def orszag_tang_2d(n=1024, ghosts=3, B0=1.0 / math.sqrt(4.0 * math.pi)):
    """Periodic [0,1]^2 Orszag-Tang vortex in DRAGON's Gaussian units:
    rho = 25/(36 pi), p = 5/(12 pi), v = (-sin 2 pi y, sin 2 pi x),
    face B = B0 (-sin 2 pi y, sin 4 pi x). Bx lives on x-faces at
    (i dx, (j+1/2) dy), By on y-faces at ((i+1/2) dx, j dy). Returns the cell
    array (cell B left zero: initialize_B_fields fills it) and the face array."""
    x, dx = _centres(n, 0.0, 1.0)
    y, dy = _centres(n, 0.0, 1.0)
    g = ghosts
    w = np.zeros((n + 2 * g, n + 2 * g, 8))
    sl = (slice(g, g + n), slice(g, g + n))
    X, Y = np.meshgrid(x, y, indexing="ij")
    w[sl + (0,)] = 25.0 / (36.0 * math.pi)
    w[sl + (1,)] = 5.0 / (12.0 * math.pi)
    w[sl + (2,)] = -np.sin(2 * math.pi * Y)
    w[sl + (3,)] = np.sin(2 * math.pi * X)
    B = np.zeros((n + 1 + 2 * g, n + 1 + 2 * g, 3))
    xf = np.arange(n + 1) * dx
    yf = np.arange(n + 1) * dy
    Xf, Yc = np.meshgrid(xf, np.concatenate([y, [y[-1] + dy]]), indexing="ij")
    B[g:g + n + 1, g:g + n + 1, 0] = -B0 * np.sin(2 * math.pi * Yc)
    Xc, Yf = np.meshgrid(np.concatenate([x, [x[-1] + dx]]), yf, indexing="ij")
    B[g:g + n + 1, g:g + n + 1, 1] = B0 * np.sin(4 * math.pi * Xc)
    return w, B, dx, dy


def blast_3d(n=256, ghosts=2, p_in=10.0, p_out=0.1, r0=0.1):
    """Blast on [-0.5,0.5]^3: rho=1, v=0, p=p_in inside r<r0, else p_out."""
    x, dx = _centres(n, -0.5, 0.5)
    g = ghosts
    w = np.zeros((n + 2 * g,) * 3 + (5,))
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    r = np.sqrt(X * X + Y * Y + Z * Z)
    sl = (slice(g, g + n),) * 3
    w[sl + (0,)] = 1.0
    w[sl + (1,)] = np.where(r < r0, p_in, p_out)
    return w, dx


def blast_2d_mhd(n=128, ghosts=3, p_in=10.0, p_out=0.1, r0=0.1, B=(1.0 / math.sqrt(2.0), 1.0 / math.sqrt(2.0), 0.0)):
    """2D MHD blast on [-0.5,0.5]^2 with uniform B (cell and face values)."""
    x, dx = _centres(n, -0.5, 0.5)
    g = ghosts
    w = np.zeros((n + 2 * g, n + 2 * g, 8))
    X, Y = np.meshgrid(x, x, indexing="ij")
    r = np.sqrt(X * X + Y * Y)
    sl = (slice(g, g + n),) * 2
    w[sl + (0,)] = 1.0
    w[sl + (1,)] = np.where(r < r0, p_in, p_out)
    Bf = np.zeros((n + 1 + 2 * g, n + 1 + 2 * g, 3))
    Bf[g:g + n + 1, g:g + n + 1, 0] = B[0]
    Bf[g:g + n + 1, g:g + n + 1, 1] = B[1]
    Bf[g:g + n + 1, g:g + n + 1, 2] = B[2]
    return w, Bf, dx


def riemann_1d(n, left, right, ghosts=2, x0=0.5):
    """1D two-state problem on [0,1] with (rho, u, p) per side."""
    return sod_1d(n, ghosts=ghosts, x0=x0, left=left, right=right)


def diagonal_advection(dim, n, ghosts=2, rho0=1.0, rho1=0.1, p=1.0):
    """Smooth density wave advected along the diagonal of the periodic unit
    square / cube (Examples/Diagonal/Problem2D.cpp:16-37, Problem3D.cpp:24-36):
    rho = rho0 + rho1 sin(2 pi (x + y [+ z])), p = 1, v = (1, 1[, 1]), cells
    n per side, dx = 1/n, centres at (i + 1/2) dx."""
    d = 1.0 / n
    c = (np.arange(n) + 0.5) * d
    g = ghosts
    w = np.zeros((n + 2 * g,) * dim + (5,))
    sl = (slice(g, g + n),) * dim
    s = sum(np.meshgrid(*([c] * dim), indexing="ij"))
    w[sl + (0,)] = rho0 + rho1 * np.sin(2 * math.pi * s)
    w[sl + (1,)] = p
    for a in range(dim):
        w[sl + (2 + a,)] = 1.0
    return w, d


def diagonal_errors(w, n, t, ghosts, rho0=1.0, rho1=0.1):
    """L1, L2 and max error of the density against the advected wave at time t
    (Examples/Diagonal/Problem2D.cpp:72-99): the exact density at a centre is
    rho0 + rho1 sin(2 pi (x + y - 2 t)) in 2D, (x + y + z - 3 t) in 3D; L1 and
    L2 are means over the n^dim cells."""
    dim = w.ndim - 1
    c = (np.arange(n) + 0.5) / n
    s = sum(np.meshgrid(*([c] * dim), indexing="ij"))
    exact = rho0 + rho1 * np.sin(2.0 * math.pi * (s - dim * t))
    err = np.abs(w[(slice(ghosts, ghosts + n),) * dim + (0,)] - exact)
    cells = float(n ** dim)
    return float(err.sum() / cells), float(math.sqrt((err * err).sum() / cells)), float(err.max())


def loop_potential(nx, ny, d, gaussian=False, B0=1e-6, centre=(1.0, 0.5)):
    """Vector potential A_z of the field loop at the grid nodes (i dx, j dy),
    i <= nx, j <= ny (Examples/LoopAdvection/Problem2D.cpp:54-60,
    Problem3D.cpp:53-58; independent of z): B0 max(r0 - r, 0) with r0 = 0.2
    (uniform |B| inside the loop), or B0 exp(-r^2 / (2 r0^2)) with r0 = 0.1."""
    r0 = 0.1 if gaussian else 0.2
    X, Y = np.meshgrid(np.arange(nx + 1) * d - centre[0], np.arange(ny + 1) * d - centre[1], indexing="ij")
    r = np.sqrt(X * X + Y * Y)
    if gaussian:
        return B0 * np.exp(-0.5 * (r / r0) ** 2)
    return B0 * np.maximum(r0 - r, 0.0)


def faces_from_potential(Az, d, ghosts, nz=None):
    """Face-centred B of A = (0, 0, A_z(x, y)) by CT::Faraday(A, B, -1/dx,
    -1/dy[, -1/dz], 0) on a zero field (MHD/B_fields.cpp:21-66): x faces (i, j)
    take (A[i, j+1] - A[i, j]) / dy, y faces (i, j) take -(A[i+1, j] - A[i, j]) /
    dx, z faces zero, each evaluated as the reference does (0 - diff * (-1/d));
    with nz the same values on every z layer of a 3D face array. Ghost faces
    stay zero for the boundary fill."""
    nx, ny = Az.shape[0] - 1, Az.shape[1] - 1
    g = ghosts
    inv = -1.0 / d
    bx = 0.0 - (Az[:, 1:] - Az[:, :-1]) * inv
    by = 0.0 - (-(Az[1:, :] - Az[:-1, :]) * inv)
    if nz is None:
        B = np.zeros((nx + 1 + 2 * g, ny + 1 + 2 * g, 3))
        B[g:g + nx + 1, g:g + ny, 0] = bx
        B[g:g + nx, g:g + ny + 1, 1] = by
        return B
    B = np.zeros((nx + 1 + 2 * g, ny + 1 + 2 * g, nz + 1 + 2 * g, 3))
    B[g:g + nx + 1, g:g + ny, g:g + nz, 0] = bx[:, :, None]
    B[g:g + nx, g:g + ny + 1, g:g + nz, 1] = by[:, :, None]
    return B


def field_loop(dim, n, ghosts=3, gaussian=False, rho=1.0, p=5.0, B0=1e-6):
    """Field-loop advection on the periodic [0,2] x [0,1] (x [0,1]) box with
    n x n/2 (x n/2) cells of width 2/n (Examples/LoopAdvection/Problem2D.cpp:
    17-52, Problem3D.cpp:17-51): rho = 1, p = 5, v = (2, 0.5) in 2D and (2, 1,
    1) in 3D, B from the loop's potential (loop_potential). Returns the cell
    array (cell B left zero: initialize_B_fields fills it), the face array and
    dx."""
    ns = (n, n // 2) if dim == 2 else (n, n // 2, n // 2)
    v = (2.0, 0.5) if dim == 2 else (2.0, 1.0, 1.0)
    d = 2.0 / n
    g = ghosts
    w = np.zeros(tuple(x + 2 * g for x in ns) + (8,))
    sl = tuple(slice(g, g + x) for x in ns)
    w[sl + (0,)] = rho
    w[sl + (1,)] = p
    for a in range(dim):
        w[sl + (2 + a,)] = v[a]
    Az = loop_potential(ns[0], ns[1], d, gaussian, B0)
    B = faces_from_potential(Az, d, g, nz=None if dim == 2 else ns[2])
    return w, B, d


def loop_errors(w, w0, n, ghosts, B0=1e-6):
    """L1, L2 and max of | |B|^2 - |B_0|^2 | / B0^2 over the cells against the
    initial cell field w0 (Examples/LoopAdvection/Problem2D.cpp:87-117,
    Problem3D.cpp:71-95; at the final time the loop is back where it
    started). L1 and L2 divide by n^dim, as the reference's problemComplete
    does, although the box holds n^dim / 2^(dim-1) cells."""
    g = ghosts
    dim = w.ndim - 1
    sl = tuple(slice(g, g + x) for x in ((n, n // 2) if dim == 2 else (n, n // 2, n // 2)))
    b2 = (w[sl + (slice(5, 8),)] ** 2).sum(axis=-1)
    b2e = (w0[sl + (slice(5, 8),)] ** 2).sum(axis=-1)
    err = np.abs(b2 - b2e) / (B0 * B0)
    cells = float(n ** dim)
    return float(err.sum() / cells), float(math.sqrt((err * err).sum() / cells)), float(err.max())


def batch_instances(n1d=2048, n2d=256, seed=5, sizes_1d=(64, 4096), sizes_2d=(64, 128, 256)):
    """The batched uneven-instance workload: n1d 1D hydro Riemann problems with
    N log-uniform in sizes_1d and per-side rho log-uniform in [0.01, 10], p
    log-uniform in [0.01, 100], u uniform in [-2, 2]; and n2d 2D MHD blasts
    (rho = 1, p = 0.1, p = 10 inside r < 0.1, B = (1/sqrt2, 1/sqrt2, 0),
    periodic) at sizes drawn uniformly from sizes_2d. Returns two lists of
    dicts with the arrays each grid needs."""
    rng = np.random.default_rng(seed)
    one = []
    for _ in range(n1d):
        n = int(np.exp(rng.uniform(np.log(sizes_1d[0]), np.log(sizes_1d[1] + 1))))
        n = min(max(n, sizes_1d[0]), sizes_1d[1])
        st = []
        for _side in range(2):
            rho = float(np.exp(rng.uniform(np.log(0.01), np.log(10.0))))
            p = float(np.exp(rng.uniform(np.log(0.01), np.log(100.0))))
            u = float(rng.uniform(-2.0, 2.0))
            st.append((rho, u, p))
        w, dx = riemann_1d(n, st[0], st[1])
        one.append({"n": n, "w": w, "dx": dx})
    two = []
    for _ in range(n2d):
        n = int(sizes_2d[rng.integers(len(sizes_2d))])
        w, Bf, dx = blast_2d_mhd(n, ghosts=3)
        two.append({"n": n, "w": w, "B": Bf, "dx": dx})
    return one, two


def rel_l1(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Relative L1 difference per field over the last axis: sum|a-b| / sum|b|."""
    ax = tuple(range(a.ndim - 1))
    num = np.abs(a - b).sum(axis=ax)
    den = np.abs(b).sum(axis=ax)
    return num / np.where(den > 0, den, 1.0)
