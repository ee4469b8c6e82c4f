"""Output and restart from device buffers: DRAGONHOARD's interface
(DRAGONHOARD/DragonHoard.hpp:16-33) over the C ABI's dragon_gpu_hoard_*.

``write_to_file`` snapshots a grid's device state into the reference's file
layout (HDF5, the keys of HDF5_Attrs.hpp:14-59, x-fastest datasets) without a
round trip of the padded state through Python: the device packs the datasets,
a copy stream downloads them and a host thread writes and compresses the file.
With ``wait=False`` it returns once the snapshot is taken, and the grid can
keep stepping while the file is written (two snapshots can be in flight; a
third waits for the oldest). ``load_from_file`` is the restart
(HDF5Restart.cpp:61-377).

Module-level settings mirror DRAGONHOARD_Config.h: ``output_dir``,
``output_base_name`` and ``options`` (write option, redundant-value
precision, compression level, ghosts).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

from . import _lib

# DRAGONHOARD_Config.h:16-35
output_base_name = "frame"
output_dir = ""
FILE_EXT = ".h5"
HDF5_WRITE_PRIMITIVE = 1
HDF5_WRITE_CONSERVATIVE = 6
HDF5_WRITE_PRIMITIVE_AND_ENERGY = 3
HDF5_WRITE_PRIMITIVE_AND_CONSERVATIVE = 7
HDF5_WRITE_OMIT = 0
HDF5_WRITE_FLOAT = 1
HDF5_WRITE_DOUBLE = 2


@dataclass
class Options:
    """The compile-time switches of DRAGONHOARD_Config.h, as run-time options."""

    write_option: int = HDF5_WRITE_PRIMITIVE_AND_ENERGY   # HDF5_WRITE_OPTION
    redundant_vals: int = HDF5_WRITE_FLOAT                 # HDF5_REDUNDANT_VALS_OPTION
    compression_level: int = 4                             # HDF5_COMPRESSION_LEVEL (<= 0: contiguous)
    write_ghosts: bool = False                             # WRITE_GHOSTS_TO_FILE
    threads: int = 0                                       # host threads compressing chunks (0: all cores)

    def to_c(self) -> _lib.HoardOpts:
        o = _lib.HoardOpts()
        o.write_option = int(self.write_option)
        o.redundant = int(self.redundant_vals)
        o.compression = int(self.compression_level)
        o.ghosts = int(bool(self.write_ghosts))
        o.threads = int(self.threads)
        return o


options = Options()


def cycle_string(n: int) -> str:
    """Frame number padded with zeros to five digits (HDF5Output.cpp:33-36)."""
    zeros = "0000" if n < 10 else "000" if n < 100 else "00" if n < 1000 else "0" if n < 10000 else ""
    return zeros + str(n)


def _path(filename: str) -> str:
    return output_dir + "/" + filename


def _with_ext(filename: str) -> str:
    # HDF5Restart.cpp:52-56 (checkExtension)
    if len(filename) > len(FILE_EXT) and filename.endswith(FILE_EXT):
        return filename
    return filename + FILE_EXT


def verify_output_directory() -> None:
    """Creates output_dir, or raises if it exists and is not a directory (OutputDir.cpp:18-27)."""
    if os.path.exists(output_dir):
        if not os.path.isdir(output_dir):
            raise RuntimeError(output_dir + " exists but is not a directory")
    else:
        os.makedirs(output_dir)


def restart_file_name(restart_frame: int = 0) -> str:
    """The file a restart loads (OutputDir.cpp:29-72): frame number
    ``restart_frame`` of output_dir's ``[NAME]_#####.h5`` files, or the
    highest-numbered one when restart_frame < 0; "" if there is none."""
    best, best_n = "", -1
    for name in sorted(os.listdir(output_dir)):
        if not os.path.isfile(os.path.join(output_dir, name)):
            continue
        dot = name.rfind(".")
        if (name[dot:] if dot >= 0 else "") != FILE_EXT:
            continue
        end = name.find(".")
        pos = name.rfind("_", 0, end)
        digits = name[pos + 1:end] if pos >= 0 else ""
        if not digits.isdigit():
            continue
        n = int(digits)
        if restart_frame >= 0:
            if n == restart_frame:
                return name
        elif n > best_n:
            best, best_n = name, n
    return best


def _is_dist(grid) -> bool:
    from . import dist
    return isinstance(grid, dist._DistBase)


def write_to_file(grid, t: float, cycle: int, filename: str, wait: bool = True, opts: Options | None = None) -> None:
    """DRAGONHOARD::writeToFile(grid, t, cycle, filename): writes
    ``output_dir + "/" + filename + ".h5"`` from the grid's device state.

    For a distributed grid (dragon_b200.dist) every rank calls it: the slabs
    are gathered, rank 0 writes the file of the whole grid, and the call
    returns on every rank once the file is complete (``wait`` is ignored)."""
    if _is_dist(grid):
        _write_dist(grid, t, cycle, _path(filename) + FILE_EXT, opts or options)
        return
    lib = grid._lib
    grid._to_device()
    o = (opts or options).to_c()
    path = (_path(filename) + FILE_EXT).encode()
    fn = lib.dragon_gpu_hoard_write if wait else lib.dragon_gpu_hoard_write_async
    _lib.check(fn(grid._h, float(t), int(cycle), path, ctypes.byref(o)))


def wait(grid) -> None:
    """Waits for every file of ``grid`` still being written."""
    _lib.check(grid._lib.dragon_gpu_hoard_wait(grid._h))


def load_from_file(grid, filename: str) -> tuple[float, int]:
    """DRAGONHOARD::loadFromFile(grid, t, cycle, filename): restarts ``grid``
    from ``output_dir + "/" + filename`` (".h5" appended when missing); returns
    (t, cycle). The grid's spacing becomes the file's.

    A distributed grid restarts on every rank from the same file (each rank
    reads it); its spacing must equal the file's."""
    if _is_dist(grid):
        return _load_dist(grid, _path(_with_ext(filename)))
    lib = grid._lib
    grid._to_device()
    path = (_path(_with_ext(filename))).encode()
    t = ctypes.c_double()
    cyc = ctypes.c_int()
    _lib.check(lib.dragon_gpu_hoard_load(grid._h, path, ctypes.byref(t), ctypes.byref(cyc)))
    grid._device_ran()
    for a, k in enumerate(("dx", "dy", "dz")[:grid.dim]):
        v = ctypes.c_double()
        _lib.check(lib.dragon_h5_read_attr(path, k.encode(), ctypes.byref(v)))
        setattr(grid, k, v.value)
    return t.value, cyc.value


def write_arrays(path: str, dim: int, mhd: bool, n, ghosts: int, d, t: float, cycle: int, w: np.ndarray,
                 B: np.ndarray | None = None, opts: Options | None = None) -> None:
    """The file writeToFile writes, from host arrays of a grid (w: the padded
    cell array, fields last; B: the padded face array of an MHD 2D / 3D grid)."""
    lib = _lib.load()
    n3 = (ctypes.c_int * 3)(*(list(n) + [1] * (3 - len(n))))
    d3 = (ctypes.c_double * 3)(*(list(d) + [0.0] * (3 - len(d))))
    wa = np.ascontiguousarray(w, dtype=np.float64)
    Ba = None if B is None else np.ascontiguousarray(B, dtype=np.float64)
    o = (opts or options).to_c()
    _lib.check(lib.dragon_hoard_write_host(path.encode(), int(dim), int(bool(mhd)), n3, int(ghosts), d3, float(t),
                                           int(cycle), wa.ctypes.data_as(_lib.c_double_p),
                                           None if Ba is None else Ba.ctypes.data_as(_lib.c_double_p), ctypes.byref(o)))


def load_arrays(path: str, dim: int, mhd: bool, n, ghosts: int, w: np.ndarray, B: np.ndarray | None = None):
    """loadFromFile into host arrays of a grid (modified in place: C-contiguous
    float64); returns (t, cycle, spacing)."""
    lib = _lib.load()
    n3 = (ctypes.c_int * 3)(*(list(n) + [1] * (3 - len(n))))
    for a in (w, B):
        if a is not None and (a.dtype != np.float64 or not a.flags.c_contiguous):
            raise ValueError("arrays must be C-contiguous float64")
    t = ctypes.c_double()
    cyc = ctypes.c_int()
    d3 = (ctypes.c_double * 3)()
    _lib.check(lib.dragon_hoard_load_host(path.encode(), int(dim), int(bool(mhd)), n3, int(ghosts),
                                          w.ctypes.data_as(_lib.c_double_p),
                                          None if B is None else B.ctypes.data_as(_lib.c_double_p), ctypes.byref(t),
                                          ctypes.byref(cyc), d3))
    return t.value, cyc.value, tuple(d3[a] for a in range(dim))


def _write_dist(grid, t, cycle, path, opts):
    import torch.distributed as tdist
    out = grid.gather()
    w, B = out if isinstance(out, tuple) else (out, None)
    if grid.rank == 0:
        write_arrays(path, grid.dim, grid.config.mhd, grid.N, grid.ghosts, grid.d, t, cycle, w, B, opts)
    tdist.barrier(group=grid.group)


def _load_dist(grid, path):
    out = grid.gather()
    w, B = out if isinstance(out, tuple) else (out, None)
    w = np.ascontiguousarray(w)
    B = None if B is None else np.ascontiguousarray(B)
    t, cycle, d = load_arrays(path, grid.dim, grid.config.mhd, grid.N, grid.ghosts, w, B)
    if tuple(d) != tuple(grid.d):
        raise ValueError(f"the file's spacing {d} differs from the distributed grid's {tuple(grid.d)}")
    grid.scatter(w, B)
    return t, cycle


writeToFile = write_to_file
loadFromFile = load_from_file
cycleString = cycle_string
restartFileName = restart_file_name
verifyOutputDirectory = verify_output_directory


# ---- the file format on host arrays -------------------------------------------
_TYPES = {np.dtype(np.float64): 0, np.dtype(np.float32): 1}


def write_h5(path: str, attrs: dict, datasets: dict, level: int = 4, threads: int = 0) -> None:
    """Writes an HDF5 file of scalar attributes ({name: int | float}) on the
    root group and float / double datasets ({"/a/b": array}, rank 1 to 3)."""
    lib = _lib.load()
    A = (_lib.H5Attr * max(1, len(attrs)))()
    keep = []
    for i, (k, v) in enumerate(attrs.items()):
        kb = k.encode()
        keep.append(kb)
        A[i].name = kb
        if isinstance(v, (int, np.integer)) and not isinstance(v, bool):
            A[i].type, A[i].ivalue = 2, int(v)
        else:
            A[i].type, A[i].dvalue = 0, float(v)
    D = (_lib.H5Dataset * max(1, len(datasets)))()
    for i, (k, arr) in enumerate(datasets.items()):
        a = np.ascontiguousarray(arr)
        if a.dtype not in _TYPES:
            a = np.ascontiguousarray(a, dtype=np.float64)
        keep.append(a)
        kb = k.encode()
        keep.append(kb)
        D[i].path = kb
        D[i].rank = a.ndim
        for r in range(a.ndim):
            D[i].dims[r] = a.shape[r]
        D[i].type = _TYPES[a.dtype]
        D[i].data = a.ctypes.data
    _lib.check(lib.dragon_h5_write(path.encode(), A, len(attrs), D, len(datasets), int(level), int(threads)))


def read_h5_attr(path: str, name: str) -> float:
    lib = _lib.load()
    v = ctypes.c_double()
    _lib.check(lib.dragon_h5_read_attr(path.encode(), name.encode(), ctypes.byref(v)))
    return v.value


def read_h5(path: str, key: str) -> np.ndarray:
    """A dataset of an HDF5 file, converted to double, in its own shape."""
    lib = _lib.load()
    rank = ctypes.c_int()
    dims = (ctypes.c_longlong * 3)()
    _lib.check(lib.dragon_h5_dataset_shape(path.encode(), key.encode(), ctypes.byref(rank), dims))
    shape = tuple(dims[i] for i in range(rank.value))
    out = np.zeros(int(np.prod(shape)) if shape else 1)
    _lib.check(lib.dragon_h5_read(path.encode(), key.encode(), out.ctypes.data_as(_lib.c_double_p), out.size))
    return out.reshape(shape)
