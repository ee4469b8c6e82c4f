"""The HDF5 subset behind the output / restart path, on the CPU.

* The test-side reader (tests/h5subset.py) and the library's C++ reader both
  read a file written by the HDF5 library itself (scipy's MATLAB 7.3 test
  file: a 1 x 9 double array of k * pi / 4) to the bit: the format pin.
* Files from the library's writer (dragon_h5_write) read back to the bit
  through both readers: ranks 1 to 3, float and double, edge chunks, one- to
  three-level chunk B-trees, contiguous and deflated layouts, nested groups,
  int and double attributes.
* The writer's structures meet what the HDF5 library checks when it reads
  them: superblock fields and end-of-file address, full-size B-tree and symbol
  table nodes, sorted names, lexicographically ordered chunk keys whose right
  key bounds the node, a local heap with an empty free list.
"""
import os
import struct

import numpy as np
import pytest

import h5subset

from dragon_b200 import hoard

MATLAB_H5 = os.path.join(os.path.dirname(np.__file__), "..", "scipy", "io", "matlab", "tests", "data",
                         "testhdf5_7.4_GLNX86.mat")


def _matlab_file():
    p = os.path.abspath(MATLAB_H5)
    if not os.path.exists(p):
        pytest.skip("scipy's HDF5 test file is not installed")
    return p


def test_reader_pinned_on_a_file_the_hdf5_library_wrote():
    f = h5subset.File(_matlab_file())
    assert f.superblock["version"] == 0
    ds = f["testdouble"]
    assert ds.attrs["MATLAB_class"] == b"double"
    v = ds.read()
    assert v.dtype == np.float64 and v.shape == (9, 1)
    np.testing.assert_array_equal(v.ravel(), np.pi / 4 * np.arange(9))


def test_library_reader_pinned_on_a_file_the_hdf5_library_wrote():
    v = hoard.read_h5(_matlab_file(), "/testdouble")
    np.testing.assert_array_equal(v.ravel(), np.pi / 4 * np.arange(9))
    with pytest.raises(Exception):
        hoard.read_h5(_matlab_file(), "/nothing")


CASES = {
    "/fluid/rho": ((37, 70), np.float64),
    "/fluid/v/x": ((37, 70), np.float64),
    "/fluid/E": ((37, 70), np.float32),
    "/fluid/Bf/x": ((5, 40, 33), np.float64),
    "/fluid/B/y": ((17, 16, 15), np.float32),
    "/line": ((2049,), np.float64),
    "/one": ((1,), np.float64),
}


@pytest.mark.parametrize("level", [0, 1, 4, 9])
def test_writer_round_trip_both_readers(tmp_path, level):
    rng = np.random.default_rng(level)
    data = {k: rng.standard_normal(s).astype(t) for k, (s, t) in CASES.items()}
    attrs = {"format_version": 1, "dim": 2, "cycle": -3, "dx": 0.1, "time": 1e-300}
    p = str(tmp_path / "f.h5")
    hoard.write_h5(p, attrs, data, level=level, threads=3)
    f = h5subset.File(p)
    assert sorted(f.keys()) == ["fluid", "line", "one"]
    assert sorted(f["fluid"].keys()) == ["B", "Bf", "E", "rho", "v"]
    for k, v in data.items():
        got = f[k].read()
        assert got.dtype == v.dtype and got.shape == v.shape
        np.testing.assert_array_equal(got, v)
        np.testing.assert_array_equal(hoard.read_h5(p, k), v.astype(np.float64))
        assert (f[k].filters != []) == (level > 0)
    for k, v in attrs.items():
        assert f.attrs[k] == v and type(f.attrs[k]).__name__ == ("int32" if isinstance(v, int) else "float64")
        assert hoard.read_h5_attr(p, k) == v


def test_deep_chunk_trees(tmp_path):
    """4883 chunks of 1024 elements: a three-level chunk B-tree (64 entries a node)."""
    a = np.arange(5_000_001, dtype=np.float64) * 0.5
    b = np.random.default_rng(3).standard_normal((130, 150, 170))
    p = str(tmp_path / "deep.h5")
    hoard.write_h5(p, {}, {"/a": a, "/g/b": b}, level=1)
    f = h5subset.File(p)
    d = f.buf.d
    root = struct.unpack_from("<Q", d, f["/a"].layout + 3)[0]
    assert d[root + 5] == 2  # level of the root node
    np.testing.assert_array_equal(f["/a"].read(), a)
    np.testing.assert_array_equal(hoard.read_h5(p, "/a"), a)
    np.testing.assert_array_equal(f["/g/b"].read(), b)


def _check_structures(path):
    """What the HDF5 library verifies when it opens and reads these files."""
    d = open(path, "rb").read()
    assert d[:8] == h5subset.SIG and d[8:16] == bytes([0, 0, 0, 0, 0, 8, 8, 0])
    leaf_k, node_k = struct.unpack_from("<HH", d, 16)
    base, free, eof, drv = struct.unpack_from("<QQQQ", d, 24)
    assert (leaf_k, node_k, base, free, drv) == (4, 16, 0, h5subset.UNDEF, h5subset.UNDEF)
    assert eof == len(d)
    f = h5subset.File(path)

    def check_group(g):
        for body in g.msgs[0x11]:
            btree, heap = struct.unpack_from("<QQ", d, body)
            assert d[heap:heap + 4] == b"HEAP" and d[heap + 4] == 0
            size, free_head, data = struct.unpack_from("<QQQ", d, heap + 8)
            assert free_head == 1 and size % 8 == 0 and data == heap + 32 and data + size <= len(d)
            names = d[data:data + size]
            assert names[:8] == bytes(8)
            assert d[btree:btree + 4] == b"TREE" and d[btree + 4] == 0
            assert btree + 24 + 32 * 8 + 33 * 8 <= len(d)  # full-size node (internal K 16)
            used = struct.unpack_from("<H", d, btree + 6)[0]
            prev = b""
            for e in range(used):
                snod = struct.unpack_from("<Q", d, btree + 32 + 16 * e)[0]
                rkey = struct.unpack_from("<Q", d, btree + 40 + 16 * e)[0]
                assert d[snod:snod + 4] == b"SNOD" and snod + 8 + 8 * 40 <= len(d)
                n = struct.unpack_from("<H", d, snod + 6)[0]
                ent = [names[struct.unpack_from("<Q", d, snod + 8 + 40 * k)[0]:].split(b"\0")[0] for k in range(n)]
                assert ent == sorted(ent) and all(x > prev for x in ent)
                assert names[rkey:].split(b"\0")[0] == ent[-1]
                prev = ent[-1]
        for name in g.keys():
            obj = g[name]
            if isinstance(obj, h5subset.Group):
                check_group(obj)
            else:
                check_dataset(obj)

    def check_dataset(ds):
        assert 0x05 in ds.msgs  # fill value message (required of datasets)
        lay = ds.layout
        if d[lay + 1] != 2:
            return
        rank1 = d[lay + 2]
        root = struct.unpack_from("<Q", d, lay + 3)[0]
        ks = 8 + 8 * rank1
        keys = []

        def walk(addr, level):
            assert d[addr:addr + 4] == b"TREE" and d[addr + 4] == 1 and d[addr + 5] == level
            assert addr + 24 + 64 * 8 + 65 * ks <= len(d)  # full-size node (chunk K 32)
            used = struct.unpack_from("<H", d, addr + 6)[0]
            assert 1 <= used <= 64
            node_keys = [struct.unpack_from("<%dQ" % rank1, d, addr + 24 + e * (ks + 8) + 8) for e in range(used + 1)]
            assert node_keys == sorted(node_keys) and len(set(node_keys)) == len(node_keys)
            for e in range(used):
                child = struct.unpack_from("<Q", d, addr + 24 + e * (ks + 8) + ks)[0]
                if level:
                    sub = walk(child, level - 1)
                    assert sub[0] == node_keys[e] and sub[1] == node_keys[e + 1]
                else:
                    keys.append(node_keys[e])
            return node_keys[0], node_keys[-1]

        walk(root, d[root + 5])
        assert keys == sorted(keys) and all(k[-1] == 0 for k in keys)

    check_group(f)


@pytest.mark.parametrize("level", [0, 4])
def test_writer_structures(tmp_path, level):
    rng = np.random.default_rng(7)
    data = {k: rng.standard_normal(s).astype(t) for k, (s, t) in CASES.items()}
    data["/z/a/b/c"] = rng.standard_normal((300, 300))
    data.update({f"/many/n{k:02d}": rng.standard_normal(3) for k in range(20)})  # three symbol table nodes
    p = str(tmp_path / "s.h5")
    hoard.write_h5(p, {"ng": 2}, data, level=level)
    _check_structures(p)
    f = h5subset.File(p)
    assert sorted(f["many"].keys()) == [f"n{k:02d}" for k in range(20)]
    np.testing.assert_array_equal(f["/many/n13"].read(), data["/many/n13"])


def test_writer_rejects_bad_input(tmp_path):
    p = str(tmp_path / "bad.h5")
    with pytest.raises(Exception):
        hoard.write_h5(p, {}, {"relative": np.zeros(3)})
    with pytest.raises(Exception):
        hoard.write_h5(p, {}, {"/a": np.zeros(3), "/a/b": np.zeros(3)})
    with pytest.raises(Exception):
        hoard.write_h5(p, {}, {"/a": np.zeros((2, 2, 2, 2))})
    with pytest.raises(Exception):
        hoard.write_h5(p, {}, {"/a": np.zeros((0, 3))})
    with pytest.raises(Exception):
        hoard.write_h5(str(tmp_path / "no" / "dir.h5"), {}, {"/a": np.zeros(3)})


def test_reader_rejects_non_hdf5(tmp_path):
    p = tmp_path / "x.h5"
    p.write_bytes(b"not an hdf5 file" * 64)
    with pytest.raises(Exception):
        hoard.read_h5(str(p), "/a")
    with pytest.raises(h5subset.H5FormatError):
        h5subset.File(str(p))


def test_cycle_string_and_restart_file_name(tmp_path, monkeypatch):
    assert [hoard.cycle_string(n) for n in (0, 7, 42, 999, 1234, 56789, 123456)] == [
        "00000", "00007", "00042", "00999", "01234", "56789", "123456"]
    monkeypatch.setattr(hoard, "output_dir", str(tmp_path))
    for name in ("frame_00003.h5", "frame_00011.h5", "frame_x.h5", "other_00020.txt", "frame_00007.h5"):
        (tmp_path / name).write_bytes(b"")
    assert hoard.restart_file_name(7) == "frame_00007.h5"
    assert hoard.restart_file_name(-1) == "frame_00011.h5"
    assert hoard.restart_file_name(5) == ""
    (tmp_path / "sub").mkdir()
    monkeypatch.setattr(hoard, "output_dir", str(tmp_path / "sub" / "deeper"))
    hoard.verify_output_directory()
    assert os.path.isdir(tmp_path / "sub" / "deeper")
    monkeypatch.setattr(hoard, "output_dir", str(tmp_path / "frame_00003.h5"))
    with pytest.raises(RuntimeError):
        hoard.verify_output_directory()


# ---- the host writer and loader against the oracle's restatement ----------------

def _random_grid(dim, mhd, g, seed):
    rng = np.random.default_rng(seed)
    n = (7, 5, 4)[:dim]
    nf = 8 if mhd else 5
    w = rng.uniform(-1, 1, tuple(x + 2 * g for x in n) + (nf,))
    w[..., 0] = rng.uniform(0.5, 2.0, w.shape[:-1])
    w[..., 1] = rng.uniform(0.1, 3.0, w.shape[:-1])
    B = rng.uniform(-1, 1, tuple(x + 1 + 2 * g for x in n) + (3,)) if (mhd and dim > 1) else None
    return n, w, B


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("mhd", [False, True])
@pytest.mark.parametrize("opt,red,ghosts,level", [(3, 1, False, 4), (7, 2, True, 0), (6, 0, False, 1),
                                                  (1, 1, True, 4), (3, 0, True, 0)])
def test_host_writer_matches_oracle(tmp_path, dim, mhd, opt, red, ghosts, level):
    """dragon_hoard_write_host: the datasets and attributes the oracle's
    restatement of writeToFile gives, bit for bit (the same plan and values the
    device pack uses)."""
    from oracle import hoard_port
    g = 3 if mhd else 2
    n, w, B = _random_grid(dim, mhd, g, seed=dim * 100 + opt * 10 + red)
    d = (0.1, 0.2, 0.3)[:dim]
    p = str(tmp_path / "h.h5")
    hoard.write_arrays(p, dim, mhd, n, g, d, 0.25, 12, w, B,
                       hoard.Options(write_option=opt, redundant_vals=red, compression_level=level, write_ghosts=ghosts))
    f = h5subset.File(p)
    want = hoard_port.expected_datasets(w, B, dim, mhd, ghosts, g, opt, red)
    got = {}

    def walk(grp, prefix):
        for k in grp.keys():
            o = grp[k]
            if isinstance(o, h5subset.Group):
                walk(o, prefix + "/" + k)
            else:
                got[prefix + "/" + k] = o.read()
    walk(f, "")
    assert sorted(got) == sorted(want)
    for k, v in want.items():
        assert got[k].dtype == v.dtype and got[k].shape == v.shape, k
        np.testing.assert_array_equal(got[k], v, err_msg=k)
    assert {k: f.attrs[k] for k in f.attrs} == hoard_port.expected_attrs(dim, mhd, n, d, ghosts, g, 0.25, 12, opt)


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("mhd", [False, True])
@pytest.mark.parametrize("opt,red,ghosts", [(6, 1, False), (7, 0, True), (3, 0, False), (1, 2, True)])
def test_host_loader_matches_oracle(tmp_path, dim, mhd, opt, red, ghosts):
    """dragon_hoard_load_host: the state the oracle's restatement of
    loadFromFile restores (conservative restarts, omitted cell B, cells
    outside the file's range untouched), bit for bit."""
    from oracle import hoard_port
    g = 3 if mhd else 2
    n, w, B = _random_grid(dim, mhd, g, seed=7 + dim + opt)
    d = (0.1, 0.2, 0.3)[:dim]
    p = str(tmp_path / "r.h5")
    hoard.write_arrays(p, dim, mhd, n, g, d, 1.5, 9, w, B,
                       hoard.Options(write_option=opt, redundant_vals=red, write_ghosts=ghosts))
    _, w0, B0 = _random_grid(dim, mhd, g, seed=99)
    w1 = w0.copy()
    B1 = None if B0 is None else B0.copy()
    t, cycle, dd = hoard.load_arrays(p, dim, mhd, n, g, w1, B1)
    assert (t, cycle, dd) == (1.5, 9, d)
    f = h5subset.File(p)
    files = {}

    def walk(grp, prefix):
        for k in grp.keys():
            o = grp[k]
            if isinstance(o, h5subset.Group):
                walk(o, prefix + "/" + k)
            else:
                files[prefix + "/" + k] = o.read()
    walk(f, "")
    ww, BB = hoard_port.restored_state(w0, B0, files, dim, mhd, mhd, g, g if ghosts else 0, opt)
    np.testing.assert_array_equal(w1, ww)
    if BB is not None:
        np.testing.assert_array_equal(B1, BB)


def test_host_writer_rejects_bad_options(tmp_path):
    n, w, _ = _random_grid(2, False, 2, 3)
    p = str(tmp_path / "o.h5")
    for o in (hoard.Options(write_option=2), hoard.Options(write_option=0), hoard.Options(redundant_vals=3),
              hoard.Options(compression_level=10)):
        with pytest.raises(Exception):
            hoard.write_arrays(p, 2, False, n, 2, (0.1, 0.2), 0.0, 0, w, None, o)


def test_host_loader_checks(tmp_path):
    """HDF5Restart.cpp's checks on host arrays: dimension, extents, physics."""
    n, w, _ = _random_grid(2, False, 2, 1)
    p = str(tmp_path / "c.h5")
    hoard.write_arrays(p, 2, False, n, 2, (0.1, 0.2), 0.0, 0, w)
    with pytest.raises(Exception, match="Expected 3 dimensions but got 2"):
        hoard.load_arrays(p, 3, False, n + (4,), 2, np.zeros((11, 9, 8, 5)))
    with pytest.raises(Exception, match="File size does not match"):
        hoard.load_arrays(p, 2, False, (7, 6), 2, np.zeros((11, 10, 5)))
    nm, wm, Bm = _random_grid(2, True, 3, 2)
    pm = str(tmp_path / "m.h5")
    hoard.write_arrays(pm, 2, True, nm, 3, (0.1, 0.2), 0.0, 0, wm, Bm)
    with pytest.raises(Exception, match="MHD"):
        hoard.load_arrays(pm, 2, False, nm, 3, np.zeros((13, 11, 5)))
