"""Host side of the ghost-slab path for user GhostFill elements: the layout
the Python grid gives a slab of its host mirror matches the halo buffer order
of dragon_gpu_halo_pack / _unpack (include/dragon_gpu.h: field, layer, then
the transverse axes, last fastest; corners: the padded transverse extent),
written out here element by element; and the slabs chosen for an element's
faces."""
import itertools

import numpy as np
import pytest

from dragon_b200.grid import buffer_to_slab, slab_to_buffer


def halo_order(arr, dim, axis, first, layers, g):
    """dragon_gpu_halo_pack's buffer, element by element."""
    nf = arr.shape[-1]
    trans = [b for b in range(dim) if b != axis]
    out = []
    for f in range(nf):
        for layer in range(layers):
            for t in itertools.product(*[range(arr.shape[b]) for b in trans]):
                idx = [0] * dim
                idx[axis] = first + g + layer
                for b, v in zip(trans, t):
                    idx[b] = v
                out.append(arr[tuple(idx) + (f,)])
    return np.array(out)


@pytest.mark.parametrize("dim,axis,first,layers", [(2, 0, -2, 4), (2, 0, 5, 4), (2, 1, -2, 3), (2, 1, 6, 4),
                                                   (3, 0, -2, 4), (3, 1, 3, 3), (3, 2, -2, 4)])
def test_slab_buffer_order_and_round_trip(dim, axis, first, layers):
    g, nf = 2, 5
    shape = tuple([9, 8, 7][:dim])
    rng = np.random.default_rng(dim * 10 + axis)
    arr = rng.normal(size=tuple(n + 2 * g for n in shape) + (nf,))
    buf = slab_to_buffer(arr, dim, axis, first, layers, g)
    np.testing.assert_array_equal(buf.ravel(), halo_order(arr, dim, axis, first, layers, g))
    other = np.zeros_like(arr)
    buffer_to_slab(buf, other, dim, axis, first, layers, g)
    sl = [slice(None)] * dim
    sl[axis] = slice(first + g, first + g + layers)
    np.testing.assert_array_equal(other[tuple(sl)], arr[tuple(sl)])
    assert np.count_nonzero(other) == np.count_nonzero(arr[tuple(sl)])


def test_custom_slabs_per_face():
    from dragon_b200.grid import custom_slabs
    X_neg, X_pos, Y_neg, Y_pos = 1, 2, 4, 8
    assert custom_slabs((64, 32), 2, X_neg) == [(0, -2, 4)]
    assert custom_slabs((64, 32), 2, X_neg | X_pos) == [(0, -2, 4), (0, 62, 4)]
    assert custom_slabs((64, 32), 3, Y_pos, reach=1) == [(1, 31, 4)]
    assert custom_slabs((64, 32, 16), 2, X_neg | Y_neg | 32) == [(0, -2, 4), (1, -2, 4), (2, 14, 4)]
    # slabs covering an axis end to end: the full round trip instead
    assert custom_slabs((4, 32), 2, X_neg | X_pos) is None
    assert custom_slabs((64, 32), 2, X_neg, reach=100) is None
