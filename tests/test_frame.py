"""The ghost-frame enumeration of the 2D MHD step (dragon_b200/csrc/frame.cuh),
compiled for the host (tests/hostcheck): every point of each padded array
that the step's update does not write is enumerated exactly once, in bounds,
and nothing else. The step copies those points from its input buffers, so
the committed arrays keep the ghosts the reference keeps (it commits the
interior only, Unsplit.cpp:104-107)."""
import ctypes

import pytest

from conftest import build_hostcheck


@pytest.fixture(scope="module")
def H():
    L = ctypes.CDLL(build_hostcheck("mhd"))
    L.hc_frame_point.restype = ctypes.c_int
    L.hc_frame_point.argtypes = [ctypes.c_longlong, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                 ctypes.POINTER(ctypes.c_int)]
    L.hc_frame_count.restype = ctypes.c_longlong
    L.hc_frame_count.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    L.hc_mhd2d_frame_points.restype = ctypes.c_longlong
    L.hc_mhd2d_frame_points.argtypes = [ctypes.c_longlong] * 3
    return L


def arrays(nx, ny, g):
    """(range, box written by the update) of the cells and the three face-B
    components: cells [0, nx) x [0, ny); x faces [0, nx] x [0, ny); y faces
    [0, nx) x [0, ny]; the cell-centred Bz on the face grid [0, nx) x [0, ny)."""
    cells = ((-g, nx + g, -g, ny + g), (0, nx, 0, ny))
    fr = (-g, nx + 1 + g, -g, ny + 1 + g)
    return [cells, (fr, (0, nx + 1, 0, ny)), (fr, (0, nx, 0, ny + 1)), (fr, (0, nx, 0, ny))]


@pytest.mark.parametrize("nx,ny,g", [(1, 1, 1), (16, 16, 3), (17, 5, 3), (40, 40, 3), (64, 33, 2), (3, 100, 4)])
def test_frame_is_the_complement_of_the_update(H, nx, ny, g):
    total = 0
    for r, b in arrays(nx, ny, g):
        R = (ctypes.c_int * 4)(*r)
        Bx = (ctypes.c_int * 4)(*b)
        n = H.hc_frame_count(R, Bx)
        ij = (ctypes.c_int * 2)()
        got = []
        for k in range(n):
            assert H.hc_frame_point(k, R, Bx, ij) == 1
            got.append((ij[0], ij[1]))
        assert H.hc_frame_point(n, R, Bx, ij) == 0  # one past the last point
        want = {(i, j) for i in range(r[0], r[1]) for j in range(r[2], r[3])
                if not (b[0] <= i < b[1] and b[2] <= j < b[3])}
        assert len(got) == len(set(got)) and set(got) == want
        total += n
    assert H.hc_mhd2d_frame_points(nx, ny, g) == total
