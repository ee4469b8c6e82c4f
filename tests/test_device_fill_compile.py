"""User ghost fills compiled for the device: the NVRTC side needs no GPU, so
the compile, its error path and the Python element run on the CPU here; the
fills themselves are checked on the GPU in test_gpu_device_fill.py."""
import ctypes

import pytest

import dragon_b200 as dg
from dragon_b200 import _lib
from dragon_b200.boundary import USER

FIXED_X = """
__device__ void fixed_x(const dragon_fill_ctx& c, int i, int j, int k) {
    for (int f = 0; f < c.nf; f++) c.set(f, i, j, k, c.params[f]);
}
"""


def test_compile_and_log():
    L = _lib.load()
    out = ctypes.c_void_p()
    assert L.dragon_gpu_user_fill_create(FIXED_X.encode(), b"fixed_x", ctypes.byref(out)) == 0
    assert out.value
    assert L.dragon_gpu_user_fill_log(out) == b""
    assert L.dragon_gpu_user_fill_destroy(out) == 0


def test_compile_error_carries_the_nvrtc_log():
    L = _lib.load()
    out = ctypes.c_void_p()
    src = b"__device__ void f(const dragon_fill_ctx& c, int i, int j, int k) { c.set(0, i, j, k, nope); }"
    assert L.dragon_gpu_user_fill_create(src, b"f", ctypes.byref(out)) == 1
    assert not out.value
    msg = L.dragon_gpu_last_error().decode()
    assert "did not compile" in msg and "nope" in msg


@pytest.mark.parametrize("name", [b"", b"1abc", b"a-b", b"x y"])
def test_function_name_must_be_an_identifier(name):
    L = _lib.load()
    out = ctypes.c_void_p()
    assert L.dragon_gpu_user_fill_create(FIXED_X.encode(), name, ctypes.byref(out)) == 1


def test_missing_function_is_a_compile_error():
    L = _lib.load()
    out = ctypes.c_void_p()
    assert L.dragon_gpu_user_fill_create(FIXED_X.encode(), b"not_there", ctypes.byref(out)) == 1


def test_python_element():
    e = dg.DeviceGhostFill(FIXED_X, "fixed_x", faces="X-", params=[1, 2, 3, 4, 5])
    assert e.kind == USER and not e.is_custom
    assert e.faces == dg.X_negative and e.fill_faces == dg.X_negative
    again = dg.DeviceGhostFill(FIXED_X, "fixed_x", faces=0, fill_faces="X+")
    assert again._fill is e._fill  # compiled once per source and function
    assert again.faces == 0 and again.fill_faces == dg.X_positive
    bl = dg.Periodic("Y") + e
    assert not bl.has_custom()
