"""CPU restatement of DRAGONHOARD's file contents: which datasets
writeToFile writes and what they hold (DRAGONHOARD/HDF5Output.cpp:103-528),
and the state loadFromFile restores (HDF5Restart.cpp:61-377).

Test infrastructure: the checker the device snapshot and restart tests compare
against. It works on the host mirror of a grid (the padded primitive array in
the reference's cell order, fields rho, p, vx, vy, vz[, Bx, By, Bz], and face B
with three components), with numpy float64 arithmetic in the reference's
operand order, so E and the momenta match the reference bit for bit.

Parity pin: HDF5 is not installed here, so the reference's writer cannot run;
the dataset selection follows the macros of HDF5Output.cpp:21-30 and the
flattening of HDF5Output.cpp:174, 308, 445 (x fastest) line by line, and the
restart round trips of the reference's own tests (Testing/Core/IO_Tests.cpp)
pin the pair of them.
"""
from __future__ import annotations

import numpy as np

GAMMA = 5.0 / 3.0
GM1 = GAMMA - 1.0
K1_8PI = 0.125 / np.pi


def _energy(w, mhd):
    # PrimitiveState::energy (FluidElement.cpp:53-59)
    rho, p, vx, vy, vz = (w[..., i] for i in range(5))
    E = p / GM1 + (rho / 2.0) * (vx * vx + vy * vy + vz * vz)
    if mhd:
        bx, by, bz = w[..., 5], w[..., 6], w[..., 7]
        E = E + (bx * bx + by * by + bz * bz) * K1_8PI
    return E


def _pressure(rho, mx, my, mz, E, B, mhd):
    # ConservativeState::pressure (FluidElement.cpp:60-66)
    eth = E - (mx * mx + my * my + mz * mz) / (2.0 * rho)
    if mhd:
        eth = eth - (B[0] * B[0] + B[1] * B[1] + B[2] * B[2]) * K1_8PI
    return GM1 * eth


def _flat(a, dim):
    """Reference order (x slowest) -> file order (x fastest): dims {nz, ny, nx}."""
    return np.ascontiguousarray(np.transpose(a, tuple(range(dim))[::-1]))


def selection(write_option, redundant):
    """HDF5Output.cpp:21-30."""
    prims = bool(write_option & 1)
    consv = bool(write_option & 4)
    redundants = redundant != 0
    write_e = bool(write_option & 2) and (consv or redundants)
    return prims, consv, redundants, write_e


def expected_datasets(w, B, dim, mhd, ghosts, g, write_option=3, redundant=1):
    """The datasets writeToFile writes for a grid whose padded host arrays are
    w (cells x fields) and B (faces x 3, MHD 2D / 3D), with dtypes."""
    prims, consv, redundants, write_e = selection(write_option, redundant)
    sl = tuple(slice(None) if ghosts else slice(g, -g) for _ in range(dim))
    c = w[sl]
    out = {"/fluid/rho": _flat(c[..., 0], dim)}
    if prims:
        out["/fluid/v/x"] = _flat(c[..., 2], dim)
        out["/fluid/v/y"] = _flat(c[..., 3], dim)
        out["/fluid/v/z"] = _flat(c[..., 4], dim)
        out["/fluid/p"] = _flat(c[..., 1], dim)
    if write_e:
        E = _flat(_energy(c, mhd), dim)
        out["/fluid/E"] = E if (consv or redundant == 2) else E.astype(np.float32)
        if consv:
            for k, name in enumerate("xyz"):
                out[f"/fluid/momentum/{name}"] = _flat(c[..., 2 + k] * c[..., 0], dim)
    if mhd:
        if dim == 1:
            for k, name in enumerate("xyz"):
                out[f"/fluid/B/{name}"] = _flat(c[..., 5 + k], dim)
        else:
            if redundants:
                for k, name in enumerate("xyz"):
                    b = _flat(c[..., 5 + k], dim)
                    out[f"/fluid/B/{name}"] = b if redundant == 2 else b.astype(np.float32)
            fsl = tuple(slice(None) if ghosts else slice(g, -g) for _ in range(dim))
            f = B[fsl]
            for k, name in enumerate("xyz"):
                out[f"/fluid/Bf/{name}"] = _flat(f[..., k], dim)
    return out


def expected_attrs(dim, mhd, n, d, ghosts, g, t, cycle, write_option=3):
    """HDF5Output.cpp:129-146 (and the 2D / 3D twins)."""
    a = {"format_version": 1, "write_option": write_option, "dim": dim, "MHD": int(mhd), "ng": g if ghosts else 0}
    for k, name in enumerate(("nx", "ny", "nz")[:dim]):
        a[name] = n[k]
    for k, name in enumerate(("dx", "dy", "dz")[:dim]):
        a[name] = d[k]
    a["cycle"] = cycle
    a["time"] = t
    return a


def restored_state(w0, B0, files, dim, mhd, file_mhd, g, ng_file, write_option):
    """The host arrays loadFromFile leaves on a grid whose arrays were (w0,
    B0), given the file's datasets ({key: x-fastest array}); ng_file is the
    file's ng attribute (clamped to the grid's ghosts as the reference does)."""
    w = w0.copy()
    B = None if B0 is None else B0.copy()
    ng = min(ng_file, g)
    lo = g - ng
    sl = tuple(slice(lo, w.shape[a] - lo) for a in range(dim))

    def cell(key):
        a = np.asarray(files[key], dtype=np.float64).reshape(-1)
        ext = tuple(w[sl].shape[:dim])
        n = int(np.prod(ext))
        # the reference indexes the file array with the clamped ng
        return np.transpose(a[:n].reshape(ext[::-1]), tuple(range(dim))[::-1])

    c = w[sl]
    c[..., 0] = cell("/fluid/rho")
    if mhd:
        if file_mhd:
            for k, name in enumerate("xyz"):
                key = f"/fluid/B/{name}"
                c[..., 5 + k] = cell(key) if (key in files or dim == 1) else 0.0
        else:
            c[..., 5:8] = 0.0
    if write_option & 1:
        c[..., 1] = cell("/fluid/p")
        c[..., 2] = cell("/fluid/v/x")
        c[..., 3] = cell("/fluid/v/y")
        c[..., 4] = cell("/fluid/v/z")
    else:
        rho = c[..., 0]
        mx, my, mz = cell("/fluid/momentum/x"), cell("/fluid/momentum/y"), cell("/fluid/momentum/z")
        E = cell("/fluid/E")
        Bc = (c[..., 5], c[..., 6], c[..., 7]) if mhd else None
        # PrimitiveState(ConservativeState) (FluidElement.cpp:44-51)
        c[..., 2] = mx / rho
        c[..., 3] = my / rho
        c[..., 4] = mz / rho
        c[..., 1] = _pressure(rho, mx, my, mz, E, Bc, mhd)
    if B is not None and dim > 1:
        fsl = tuple(slice(lo, B.shape[a] - lo) for a in range(dim))
        f = B[fsl]
        ext = tuple(f.shape[:dim])
        n = int(np.prod(ext))
        for k, name in enumerate("xyz"):
            key = f"/fluid/Bf/{name}"
            if file_mhd and key in files:
                a = np.asarray(files[key], dtype=np.float64).reshape(-1)[:n]
                f[..., k] = np.transpose(a.reshape(ext[::-1]), tuple(range(dim))[::-1])
            else:
                f[..., k] = 0.0
    return w, B
