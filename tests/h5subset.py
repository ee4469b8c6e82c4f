"""A pure-numpy reader for the subset of the HDF5 file format that DRAGONHOARD
files use. Test infrastructure: it checks, independently of the library's own
C++ reader, what the device snapshot writer puts on disk.

HDF5 is not installed on these machines (no libhdf5, no h5py), so both sides of
the format are restated here from the public HDF5 File Format Specification
(version 3.0): superblock versions 0 and 1, version-1 object headers with
continuation blocks, symbol-table groups (version-1 B-tree of type 0, local
heap, symbol-table nodes), dataspace / datatype / fill value / layout (compact,
contiguous, chunked with a version-1 B-tree of type 1; layout messages of
versions 1 to 3) / filter pipeline (deflate, shuffle) / attribute messages,
IEEE float and two's-complement integer types, little- or big-endian. The
reader is pinned by a file the HDF5 library wrote (scipy's MATLAB 7.3 test
file, ``tests/test_hoard_format.py``).
"""
import struct
import zlib

import numpy as np

SIG = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


class H5FormatError(ValueError):
    pass


class _Buf:
    def __init__(self, data, base):
        self.d = data
        self.base = base

    def u(self, off, n):
        return int.from_bytes(self.d[off:off + n], "little")

    def at(self, addr):
        return self.base + addr


class Dataset:
    def __init__(self, f, msgs):
        self.f = f
        self.msgs = msgs
        self.attrs = f._attrs(msgs)
        self.shape = f._dataspace(msgs[0x01][0])
        self.dtype, self.type_desc = f._datatype(msgs[0x03][0])
        self.layout = msgs[0x08][0]
        self.filters = f._filters(msgs[0x0B][0]) if 0x0B in msgs else []

    def read(self):
        return self.f._read_data(self)


class Group:
    def __init__(self, f, msgs):
        self.f = f
        self.msgs = msgs
        self.attrs = f._attrs(msgs)
        self.links = f._links(msgs)

    def keys(self):
        return list(self.links)

    def __contains__(self, name):
        return name in self.links

    def __getitem__(self, path):
        node = self
        for part in [p for p in path.split("/") if p]:
            if not isinstance(node, Group) or part not in node.links:
                raise KeyError(path)
            node = node.f._object(node.links[part])
        return node


class File(Group):
    """Open an HDF5 file (from a path or bytes) and expose its root group."""

    def __init__(self, src):
        data = src if isinstance(src, (bytes, bytearray)) else open(src, "rb").read()
        sb = -1
        for off in [0] + [512 << k for k in range(20)]:
            if off + 8 > len(data):
                break
            if data[off:off + 8] == SIG:
                sb = off
                break
        if sb < 0:
            raise H5FormatError("no HDF5 signature")
        ver = data[sb + 8]
        if ver not in (0, 1):
            raise H5FormatError(f"superblock version {ver} is outside the supported subset")
        if data[sb + 13] != 8 or data[sb + 14] != 8:
            raise H5FormatError("only 8-byte offsets and lengths are supported")
        p = sb + 24 if ver == 0 else sb + 28
        base, _fs, eof, _drv = struct.unpack_from("<QQQQ", data, p)
        self.buf = _Buf(data, sb if base == 0 else base)
        self.superblock = dict(version=ver, leaf_k=struct.unpack_from("<H", data, sb + 16)[0],
                               internal_k=struct.unpack_from("<H", data, sb + 18)[0], eof=eof)
        ent = p + 32
        root = struct.unpack_from("<Q", data, ent + 8)[0]
        self.root_addr = root
        Group.__init__(self, self, self._header(root))

    # -- object headers -------------------------------------------------------
    def _header(self, addr):
        b = self.buf
        a = b.at(addr)
        if b.d[a:a + 4] == b"OHDR":
            raise H5FormatError("version-2 object headers are outside the supported subset")
        if b.d[a] != 1:
            raise H5FormatError(f"object header version {b.d[a]} at {addr}")
        nmsg = b.u(a + 2, 2)
        size = b.u(a + 8, 4)
        blocks = [(a + 16, size)]
        msgs = {}
        seen = 0
        while blocks and seen < nmsg:
            start, length = blocks.pop(0)
            q = start
            while q + 8 <= start + length and seen < nmsg:
                mtype, msize, mflags = b.u(q, 2), b.u(q + 2, 2), b.d[q + 4]
                body = q + 8
                if mflags & 0x02:
                    raise H5FormatError("shared messages are outside the supported subset")
                if mtype == 0x10:
                    caddr, clen = struct.unpack_from("<QQ", b.d, body)
                    blocks.append((b.at(caddr), clen))
                elif mtype != 0x00:
                    msgs.setdefault(mtype, []).append(body)
                seen += 1
                q = body + msize
        return msgs

    def _object(self, addr):
        msgs = self._header(addr)
        if 0x11 in msgs or 0x02 in msgs or 0x06 in msgs:
            return Group(self, msgs)
        if 0x08 in msgs:
            return Dataset(self, msgs)
        raise H5FormatError(f"object at {addr} is neither a group nor a dataset")

    # -- groups -------------------------------------------------------------
    def _links(self, msgs):
        b = self.buf
        out = {}
        for body in msgs.get(0x11, []):
            btree, heap = struct.unpack_from("<QQ", b.d, body)
            names = self._heap(heap)
            self._walk_group_btree(btree, names, out)
        for body in msgs.get(0x06, []):
            name, addr = self._link_message(body)
            if addr is not None:
                out[name] = addr
        return out

    def _heap(self, addr):
        b = self.buf
        a = b.at(addr)
        if b.d[a:a + 4] != b"HEAP":
            raise H5FormatError(f"bad local heap at {addr}")
        size = b.u(a + 8, 8)
        data_addr = b.u(a + 24, 8)
        return b.d[b.at(data_addr):b.at(data_addr) + size]

    @staticmethod
    def _cstr(blob, off):
        end = blob.index(b"\0", off)
        return blob[off:end].decode()

    def _walk_group_btree(self, addr, names, out):
        b = self.buf
        a = b.at(addr)
        if b.d[a:a + 4] != b"TREE":
            raise H5FormatError(f"bad B-tree node at {addr}")
        ntype, level, used = b.d[a + 4], b.d[a + 5], b.u(a + 6, 2)
        if ntype != 0:
            raise H5FormatError("group B-tree of the wrong type")
        q = a + 24 + 8  # past the header and key 0
        for _ in range(used):
            child = b.u(q, 8)
            q += 16
            if level > 0:
                self._walk_group_btree(child, names, out)
            else:
                self._snod(child, names, out)

    def _snod(self, addr, names, out):
        b = self.buf
        a = b.at(addr)
        if b.d[a:a + 4] != b"SNOD":
            raise H5FormatError(f"bad symbol table node at {addr}")
        n = b.u(a + 6, 2)
        for k in range(n):
            e = a + 8 + 40 * k
            name_off, hdr = struct.unpack_from("<QQ", b.d, e)
            out[self._cstr(names, name_off)] = hdr

    def _link_message(self, body):
        d = self.buf.d
        flags = d[body + 1]
        q = body + 2
        ltype = 0
        if flags & 0x08:
            ltype = d[q]
            q += 1
        if flags & 0x04:
            q += 8
        if flags & 0x10:
            q += 1
        nlen_size = 1 << (flags & 0x03)
        nlen = int.from_bytes(d[q:q + nlen_size], "little")
        q += nlen_size
        name = d[q:q + nlen].decode()
        q += nlen
        if ltype != 0:
            return name, None
        return name, struct.unpack_from("<Q", d, q)[0]

    # -- messages -------------------------------------------------------------
    def _dataspace(self, body):
        d = self.buf.d
        ver, rank = d[body], d[body + 1]
        if ver == 1:
            q = body + 8
        elif ver == 2:
            if d[body + 3] == 0:  # scalar
                return ()
            q = body + 4
        else:
            raise H5FormatError(f"dataspace version {ver}")
        return tuple(struct.unpack_from("<%dQ" % rank, d, q)) if rank else ()

    def _datatype(self, body):
        d = self.buf.d
        cv = d[body]
        cls, ver = cv & 0x0F, cv >> 4
        bits = d[body + 1] | (d[body + 2] << 8) | (d[body + 3] << 16)
        size = struct.unpack_from("<I", d, body + 4)[0]
        order = ">" if bits & 1 else "<"
        if cls == 0:
            signed = bool(bits & 0x08)
            dt = np.dtype(f"{order}{'i' if signed else 'u'}{size}")
            return dt, dict(cls="int", size=size, signed=signed, order=order)
        if cls == 1:
            if size not in (4, 8):
                raise H5FormatError(f"float of {size} bytes")
            off, prec, eloc, esize, mloc, msize, bias = struct.unpack_from("<HHBBBBI", d, body + 8)
            ieee = (4, 32, 23, 8, 0, 23, 127) if size == 4 else (8, 64, 52, 11, 0, 52, 1023)
            if (size, prec, eloc, esize, mloc, msize, bias) != ieee or off != 0:
                raise H5FormatError("non-IEEE float layout")
            if ((bits >> 8) & 0xFF) != size * 8 - 1 or ((bits >> 4) & 0x3) != 2:
                raise H5FormatError("non-IEEE float sign / normalisation")
            return np.dtype(f"{order}f{size}"), dict(cls="float", size=size, order=order, version=ver)
        if cls == 3:
            return np.dtype(f"S{size}"), dict(cls="string", size=size)
        raise H5FormatError(f"datatype class {cls} is outside the supported subset")

    def _filters(self, body):
        d = self.buf.d
        ver, n = d[body], d[body + 1]
        q = body + (8 if ver == 1 else 2)
        out = []
        for _ in range(n):
            fid = struct.unpack_from("<H", d, q)[0]
            if ver == 1 or fid >= 256:
                nlen, flags, ncd = struct.unpack_from("<HHH", d, q + 2)
                q += 8
                if ver == 1:
                    q += (nlen + 7) // 8 * 8
                else:
                    q += nlen
            else:
                flags, ncd = struct.unpack_from("<HH", d, q + 2)
                q += 6
            cd = list(struct.unpack_from("<%dI" % ncd, d, q))
            q += 4 * ncd
            if ver == 1 and ncd % 2:
                q += 4
            out.append((fid, flags, cd))
        return out

    def _attrs(self, msgs):
        d = self.buf.d
        out = {}
        for body in msgs.get(0x0C, []):
            ver = d[body]
            if ver == 1:
                nsz, tsz, ssz = struct.unpack_from("<HHH", d, body + 2)
                q = body + 8
                pad = lambda n: (n + 7) // 8 * 8  # noqa: E731
                name = d[q:q + nsz].split(b"\0")[0].decode()
                q += pad(nsz)
                tq = q
                q += pad(tsz)
                sq = q
                q += pad(ssz)
            elif ver in (2, 3):
                nsz, tsz, ssz = struct.unpack_from("<HHH", d, body + 2)
                q = body + 8 + (1 if ver == 3 else 0)
                name = d[q:q + nsz].split(b"\0")[0].decode()
                q += nsz
                tq = q
                q += tsz
                sq = q
                q += ssz
            else:
                raise H5FormatError(f"attribute message version {ver}")
            dt, desc = self._datatype(tq)
            shape = self._dataspace(sq)
            n = int(np.prod(shape)) if shape else 1
            val = np.frombuffer(d, dtype=dt, count=n, offset=q)
            out[name] = val.reshape(shape) if shape else val[0]
        return out

    # -- raw data ---------------------------------------------------------------
    def _read_data(self, ds):
        b = self.buf
        d = b.d
        body = ds.layout
        ver = d[body]
        n = int(np.prod(ds.shape)) if ds.shape else 1
        esize = ds.dtype.itemsize
        if ver in (1, 2):  # the older layout message: rank+1 sizes, then class-specific fields
            rank1, cls = d[body + 1], d[body + 2]
            q = body + 8
            if cls == 1:
                addr = struct.unpack_from("<Q", d, q)[0]
                if addr == UNDEF:
                    return np.zeros(ds.shape, ds.dtype)
                return np.frombuffer(d, dtype=ds.dtype, count=n, offset=b.at(addr)).reshape(ds.shape)
            if cls == 2:
                btree = struct.unpack_from("<Q", d, q)[0]
                cdims = struct.unpack_from("<%dI" % rank1, d, q + 8)
                out = np.zeros(ds.shape, ds.dtype)
                if btree != UNDEF:
                    self._walk_chunk_btree(btree, rank1, tuple(cdims[:-1]), ds, out)
                return out
            raise H5FormatError(f"layout class {cls} in a version-{ver} layout message")
        if ver != 3:
            raise H5FormatError(f"layout message version {ver}")
        cls = d[body + 1]
        if cls == 0:
            size = struct.unpack_from("<H", d, body + 2)[0]
            raw = d[body + 4:body + 4 + size]
            return np.frombuffer(raw, dtype=ds.dtype, count=n).reshape(ds.shape)
        if cls == 1:
            addr = struct.unpack_from("<Q", d, body + 2)[0]
            if addr == UNDEF:
                return np.zeros(ds.shape, ds.dtype)
            return np.frombuffer(d, dtype=ds.dtype, count=n, offset=b.at(addr)).reshape(ds.shape)
        if cls != 2:
            raise H5FormatError(f"layout class {cls}")
        rank1 = d[body + 2]
        btree = struct.unpack_from("<Q", d, body + 3)[0]
        cdims = struct.unpack_from("<%dI" % rank1, d, body + 11)
        chunk = tuple(cdims[:-1])
        if cdims[-1] != esize:
            raise H5FormatError("chunk element size does not match the datatype")
        out = np.zeros(ds.shape, ds.dtype)
        if btree != UNDEF:
            self._walk_chunk_btree(btree, rank1, chunk, ds, out)
        return out

    def _walk_chunk_btree(self, addr, rank1, chunk, ds, out):
        b = self.buf
        d = b.d
        a = b.at(addr)
        if d[a:a + 4] != b"TREE" or d[a + 4] != 1:
            raise H5FormatError(f"bad chunk B-tree node at {addr}")
        level, used = d[a + 5], b.u(a + 6, 2)
        ksize = 8 + 8 * rank1
        q = a + 24
        for _ in range(used):
            csize, fmask = struct.unpack_from("<II", d, q)
            offs = struct.unpack_from("<%dQ" % rank1, d, q + 8)
            child = struct.unpack_from("<Q", d, q + ksize)[0]
            q += ksize + 8
            if level > 0:
                self._walk_chunk_btree(child, rank1, chunk, ds, out)
                continue
            raw = d[b.at(child):b.at(child) + csize]
            for k, (fid, _flags, cd) in reversed(list(enumerate(ds.filters))):
                if fmask & (1 << k):
                    continue
                if fid == 1:
                    raw = zlib.decompress(raw)
                elif fid == 2:
                    es = cd[0] if cd else ds.dtype.itemsize
                    arr = np.frombuffer(raw, np.uint8).reshape(es, -1)
                    raw = arr.T.copy().tobytes()
                elif fid == 3:
                    raw = raw[:-4]
                else:
                    raise H5FormatError(f"filter {fid} is outside the supported subset")
            blk = np.frombuffer(raw, dtype=ds.dtype, count=int(np.prod(chunk))).reshape(chunk)
            sl = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs[:-1], chunk, ds.shape))
            out[sl] = blk[tuple(slice(0, s.stop - s.start) for s in sl)]
