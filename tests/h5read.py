"""Minimal, strict HDF5 reader (test infrastructure only).

There is no libhdf5 and no h5py in this image, so the tests read the
library's snapshot files (coolbubble_b200/csrc/cb_h5.cpp) with this reader.
It follows the published HDF5 File Format Specification for the structures
that libhdf5 writes with its default ("earliest") format bounds:

  superblock version 0 (optionally behind a user block: 512, 1024, ... bytes)
  version-1 object headers (with continuation blocks)
  groups as symbol tables: version-1 B-tree of type 0, symbol-table nodes,
    local heap
  dataspace (versions 1, 2), datatype (fixed point, IEEE float, string),
  layout (versions 1-3: compact, contiguous, chunked with a version-1
  B-tree of type 1), filter pipeline (versions 1, 2: deflate, shuffle),
  attribute messages (versions 1-3)

and checks what a conforming reader relies on: signatures and versions,
8-byte message alignment, message counts, whole B-tree nodes inside the
file, node levels, key order, chunk offsets on the chunk grid, decoded chunk
sizes, and that no two structures overlap.

Before it is trusted on this library's files, tests/test_h5.py checks it on
a file written by libhdf5 itself: scipy's test file testhdf5_7.4_GLNX86.mat
(MATLAB 7.3 format = HDF5 behind a 512-byte user block).
"""
import struct
import zlib

import numpy as np

SIG = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF
CHUNK_K = 32          # B-tree K of chunk indexes for version-0 superblocks


class H5Error(Exception):
    pass


def _need(cond, msg):
    if not cond:
        raise H5Error(msg)


def _pad8(x):
    return (x + 7) & ~7


class _Type:
    def __init__(self, body):
        cls, ver = body[0] & 0x0F, body[0] >> 4
        _need(ver in (1, 2, 3), "datatype version %d" % ver)
        bits = body[1] | body[2] << 8 | body[3] << 16
        (self.size,) = struct.unpack_from("<I", body, 4)
        self.cls = cls
        if cls == 0:                                    # fixed point
            signed = bool(bits & 0x08)
            _need(not bits & 0x01, "big-endian integer")
            self.dtype = np.dtype(("<i%d" if signed else "<u%d") % self.size)
        elif cls == 1:                                  # floating point
            _need(not bits & 0x01, "big-endian float")
            off, prec, eloc, esz, mloc, msz, bias = struct.unpack_from("<HHBBBBI", body, 8)
            std = {4: (0, 32, 23, 8, 0, 23, 127, 31), 8: (0, 64, 52, 11, 0, 52, 1023, 63)}
            _need(self.size in std, "float of %d bytes" % self.size)
            _need((off, prec, eloc, esz, mloc, msz, bias, body[2]) == std[self.size], "non-IEEE float layout")
            _need((bits >> 4) & 3 == 2, "float mantissa normalisation")
            self.dtype = np.dtype("<f%d" % self.size)
        elif cls == 3:                                  # string
            self.dtype = np.dtype("S%d" % self.size)
        else:
            raise H5Error("datatype class %d not supported" % cls)
        self.raw_size = 8 + {0: 4, 1: 12, 3: 0}[cls]


def _dataspace(body):
    ver = body[0]
    if ver == 1:
        rank, flags = body[1], body[2]
        p = 8
    elif ver == 2:
        rank, flags, kind = body[1], body[2], body[3]
        p = 4
        _need(kind in (0, 1), "null dataspace")
    else:
        raise H5Error("dataspace version %d" % ver)
    dims = struct.unpack_from("<%dQ" % rank, body, p)
    p += 8 * rank
    maxd = None
    if flags & 1:
        maxd = struct.unpack_from("<%dQ" % rank, body, p)
        p += 8 * rank
        _need(all(m == UNDEF or m >= d for m, d in zip(maxd, dims)), "maximum below dimension")
    return tuple(int(d) for d in dims), p


def _pipeline(body):
    ver, n = body[0], body[1]
    _need(ver in (1, 2), "filter pipeline version %d" % ver)
    p = 8 if ver == 1 else 2
    out = []
    for _ in range(n):
        (fid,) = struct.unpack_from("<H", body, p)
        p += 2
        nlen = 0
        if ver == 1 or fid >= 256:
            (nlen,) = struct.unpack_from("<H", body, p)
            p += 2
        flags, ncd = struct.unpack_from("<HH", body, p)
        p += 4
        name = body[p:p + nlen].split(b"\0")[0].decode()
        if ver == 1:
            _need(nlen % 8 == 0, "filter name not padded to 8")
        p += nlen
        cd = list(struct.unpack_from("<%dI" % ncd, body, p))
        p += 4 * ncd
        if ver == 1 and ncd % 2:
            p += 4
        out.append({"id": fid, "name": name, "flags": flags, "cd": cd})
    return out


class Dataset:
    def __init__(self, f, addr, msgs):
        self.file, self.addr = f, addr
        self.attrs = {}
        self.filters = []
        self.layout = None
        for mtype, _flags, body in msgs:
            if mtype == 0x1:
                self.shape, _ = _dataspace(body)
            elif mtype == 0x3:
                self.type = _Type(body)
            elif mtype == 0x8:
                self.layout = body
            elif mtype == 0xB:
                self.filters = _pipeline(body)
            elif mtype == 0xC:
                k, v = f._attribute(body)
                self.attrs[k] = v
        _need(self.layout is not None, "dataset without layout message")
        self.dtype = self.type.dtype
        self._parse_layout()

    def _parse_layout(self):
        b = self.layout
        ver = b[0]
        self.chunks = None
        if ver in (1, 2):
            ndims, cls = b[1], b[2]
            p = 8
            addr = None
            if cls != 0:
                (addr,) = struct.unpack_from("<Q", b, p)
                p += 8
            dims = struct.unpack_from("<%dI" % ndims, b, p)
            p += 4 * ndims
            if cls == 1:
                self.kind, self.data_addr = "contiguous", addr
                self.data_size = int(np.prod(dims[:-1])) * dims[-1] if dims else 0
                _need(dims[-1] == self.type.size, "contiguous element size")
                _need(tuple(dims[:-1]) == self.shape, "contiguous dims differ from the dataspace")
            elif cls == 2:
                raise H5Error("version 1/2 chunked layout not supported")
            else:
                raise H5Error("compact layout version %d not supported" % ver)
        elif ver == 3:
            cls = b[1]
            if cls == 0:
                (size,) = struct.unpack_from("<H", b, 2)
                self.kind, self.compact = "compact", bytes(b[4:4 + size])
            elif cls == 1:
                self.kind = "contiguous"
                self.data_addr, self.data_size = struct.unpack_from("<QQ", b, 2)
            elif cls == 2:
                ndims = b[2]
                (self.btree,) = struct.unpack_from("<Q", b, 3)
                dims = struct.unpack_from("<%dI" % ndims, b, 11)
                _need(ndims == len(self.shape) + 1, "chunk rank")
                _need(dims[-1] == self.type.size, "chunk element size %d" % dims[-1])
                self.kind, self.chunks = "chunked", tuple(int(d) for d in dims[:-1])
                _need(all(1 <= c for c in self.chunks), "empty chunk")
            else:
                raise H5Error("layout class %d" % cls)
        else:
            raise H5Error("layout version %d" % ver)

    def read(self):
        n = int(np.prod(self.shape)) if self.shape else 1
        es = self.type.size
        if self.kind == "contiguous":
            if self.data_addr == UNDEF:
                return np.zeros(self.shape, self.dtype)
            _need(self.data_size == n * es, "contiguous size")
            raw = self.file._take(self.data_addr, self.data_size, "data")
            self.file.check_overlaps()
            return np.frombuffer(raw, self.dtype).reshape(self.shape).copy()
        if self.kind == "compact":
            return np.frombuffer(self.compact, self.dtype)[:n].reshape(self.shape).copy()
        out = np.zeros(self.shape, self.dtype)
        self.chunk_count = 0
        self.chunk_bytes = 0
        self.chunk_masks = []
        if self.btree == UNDEF:
            return out
        rank = len(self.shape)
        seen = set()
        leaves = []
        self.file._chunk_tree(self.btree, rank + 1, None, leaves)
        prev = None
        for key, addr in leaves:
            size, mask, off = key
            _need(off[-1] == 0, "element dimension offset")
            off = off[:-1]
            _need(all(o % c == 0 for o, c in zip(off, self.chunks)), "chunk offset off the grid")
            _need(all(o < d for o, d in zip(off, self.shape)), "chunk outside the dataset")
            _need(prev is None or off > prev, "chunk keys not in increasing order")
            _need(off not in seen, "chunk stored twice")
            seen.add(off)
            prev = off
            raw = self.file._take(addr, size, "chunk")
            data = self._unfilter(raw, mask)
            m = int(np.prod(self.chunks))
            _need(len(data) == m * es, "decoded chunk of %d bytes, expected %d" % (len(data), m * es))
            block = np.frombuffer(data, self.dtype).reshape(self.chunks)
            sl = tuple(slice(o, min(o + c, d)) for o, c, d in zip(off, self.chunks, self.shape))
            out[sl] = block[tuple(slice(0, s.stop - s.start) for s in sl)]
            self.chunk_count += 1
            self.chunk_bytes += size
            self.chunk_masks.append(mask)
        self.file.check_overlaps()
        return out

    def _unfilter(self, raw, mask):
        data = raw
        for i in reversed(range(len(self.filters))):
            if mask >> i & 1:
                continue
            flt = self.filters[i]
            if flt["id"] == 1:
                data = zlib.decompress(data)
            elif flt["id"] == 2:
                es = flt["cd"][0] if flt["cd"] else self.type.size
                _need(len(data) % es == 0, "shuffled size")
                data = np.frombuffer(data, np.uint8).reshape(es, -1).T.copy().tobytes()
            else:
                raise H5Error("filter %d not supported" % flt["id"])
        return data

    def __getitem__(self, key):
        return self.read()[key]


class File:
    def __init__(self, path):
        self.buf = open(path, "rb").read()
        self.regions = []
        base = None
        for off in [0] + [512 << k for k in range(16)]:
            if off + 8 <= len(self.buf) and self.buf[off:off + 8] == SIG:
                base = off
                break
        _need(base is not None, "no HDF5 signature")
        sb = self.buf[base:base + 96]
        _need(len(sb) == 96, "truncated superblock")
        _need(sb[8] == 0, "superblock version %d (only 0 is read)" % sb[8])
        _need(sb[9] == 0 and sb[10] == 0 and sb[12] == 0, "superblock sub-versions")
        _need(sb[13] == 8 and sb[14] == 8, "offset/length sizes")
        self.leaf_k, self.internal_k = struct.unpack_from("<HH", sb, 16)
        _need(self.leaf_k > 0 and self.internal_k > 0, "group K")
        base_addr, fs_addr, eof, drv = struct.unpack_from("<4Q", sb, 24)
        _need(base_addr == base, "base address %d, signature at %d" % (base_addr, base))
        _need(drv == UNDEF, "driver information block")
        # the end-of-file address is absolute; every other address is relative to the base
        _need(base < eof <= len(self.buf), "file shorter than its end-of-file address")
        self.base, self.eof = base, eof - base
        self._mark(0, 96, "superblock")
        name_off, oh, cache = struct.unpack_from("<QQI", sb, 56)
        btree, heap = struct.unpack_from("<QQ", sb, 80)
        msgs = self._object_header(oh)
        stab = [b for t, _, b in msgs if t == 0x11]
        _need(len(stab) == 1, "root group without a symbol-table message")
        bt2, hp2 = struct.unpack_from("<QQ", stab[0], 0)
        if cache == 1:
            _need((btree, heap) == (bt2, hp2), "root entry scratch pad differs from the symbol-table message")
        self.attrs = {}
        for t, _, b in msgs:
            if t == 0xC:
                k, v = self._attribute(b)
                self.attrs[k] = v
        self.links = self._group(bt2, hp2)
        self.datasets = {}
        for name, addr in self.links.items():
            self.datasets[name] = Dataset(self, addr, self._object_header(addr))
        self.check_overlaps()

    # -- raw access ------------------------------------------------------
    def _mark(self, addr, size, what):
        _need(addr != UNDEF and addr + size <= self.eof, "%s at %d+%d beyond the end of file %d"
              % (what, addr, size, self.eof))
        self.regions.append((addr, size, what))

    def check_overlaps(self):
        """No two structures read so far share a byte (the same structure read twice is fine)."""
        self.regions = sorted(set(self.regions))
        for (a, s, w), (b, t, v) in zip(self.regions, self.regions[1:]):
            _need(a + s <= b, "%s at %d+%d overlaps %s at %d+%d" % (w, a, s, v, b, t))

    def _take(self, addr, size, what):
        self._mark(addr, size, what)
        return self.buf[self.base + addr:self.base + addr + size]

    def _peek(self, addr, size):
        _need(addr + size <= self.eof, "read beyond the end of file")
        return self.buf[self.base + addr:self.base + addr + size]

    # -- structures --------------------------------------------------------
    def _object_header(self, addr):
        pre = self._take(addr, 16, "object header")
        ver, _, nmsg, _ref, size = struct.unpack_from("<BBHII", pre, 0)
        _need(ver == 1, "object header version %d" % ver)
        blocks = [(addr + 16, size)]
        msgs = []
        while blocks:
            a, size = blocks.pop(0)
            data = self._take(a, size, "object header messages")
            p = 0
            while p < size:
                _need(p + 8 <= size, "message header past the block")
                mtype, msize, mflags = struct.unpack_from("<HHB", data, p)
                _need(msize % 8 == 0, "message %#x of %d bytes (not 8-aligned)" % (mtype, msize))
                _need(p + 8 + msize <= size, "message %#x past the block" % mtype)
                body = data[p + 8:p + 8 + msize]
                if mtype == 0x10:
                    blocks.append(struct.unpack_from("<QQ", body, 0))
                msgs.append((mtype, mflags, body))
                p += 8 + msize
        _need(len(msgs) == nmsg, "object header says %d messages, holds %d" % (nmsg, len(msgs)))
        return msgs

    def _attribute(self, body):
        ver = body[0]
        _need(ver in (1, 2, 3), "attribute version %d" % ver)
        nsz, tsz, ssz = struct.unpack_from("<HHH", body, 2)
        p = 8 + (1 if ver == 3 else 0)
        pad = _pad8 if ver == 1 else (lambda x: x)
        name = bytes(body[p:p + nsz]).split(b"\0")[0].decode()
        _need(body[p + nsz - 1] == 0, "attribute name not terminated")
        p += pad(nsz)
        t = _Type(body[p:p + tsz])
        p += pad(tsz)
        dims, _ = _dataspace(body[p:p + ssz])
        p += pad(ssz)
        n = int(np.prod(dims)) if dims else 1
        _need(p + n * t.size <= len(body), "attribute data past the message")
        v = np.frombuffer(bytes(body[p:p + n * t.size]), t.dtype)
        return name, (v[0] if not dims else v.reshape(dims))

    def _heap(self, addr):
        h = self._take(addr, 32, "local heap")
        _need(h[:4] == b"HEAP" and h[4] == 0, "local heap signature/version")
        size, free, data = struct.unpack_from("<QQQ", h, 8)
        _need(free == 1 or free < size, "local heap free list")
        return self._take(data, size, "local heap data")

    def _group(self, btree, heap):
        names = self._heap(heap)

        def name_at(off):
            end = names.index(b"\0", off)
            return names[off:end].decode()

        links = {}
        order = []

        def node(addr, level_expected):
            nsz = 24 + (2 * self.internal_k + 1) * 8 + 2 * self.internal_k * 8
            b = self._take(addr, nsz, "group B-tree node")
            _need(b[:4] == b"TREE" and b[4] == 0, "group B-tree signature/type")
            level, n = b[5], struct.unpack_from("<H", b, 6)[0]
            _need(level_expected is None or level == level_expected, "B-tree level")
            _need(1 <= n <= 2 * self.internal_k, "group B-tree entries %d" % n)
            for i in range(n):
                (child,) = struct.unpack_from("<Q", b, 24 + 8 + 16 * i)
                if level > 0:
                    node(child, level - 1)
                else:
                    snod(child)

        def snod(addr):
            sz = 8 + 2 * self.leaf_k * 40
            b = self._take(addr, sz, "symbol-table node")
            _need(b[:4] == b"SNOD" and b[4] == 1, "symbol-table node signature/version")
            (n,) = struct.unpack_from("<H", b, 6)
            _need(n <= 2 * self.leaf_k, "symbol-table node with %d entries" % n)
            for i in range(n):
                off, oh, cache = struct.unpack_from("<QQI", b, 8 + 40 * i)
                nm = name_at(off)
                order.append(nm)
                links[nm] = oh

        node(btree, None)
        enc = [o.encode() for o in order]
        _need(enc == sorted(enc), "links not in name order")
        return links

    def _chunk_tree(self, addr, ndims, level_expected, out):
        ksz = 8 + 8 * ndims
        nsz = 24 + (2 * CHUNK_K + 1) * ksz + 2 * CHUNK_K * 8
        b = self._take(addr, nsz, "chunk B-tree node")
        _need(b[:4] == b"TREE" and b[4] == 1, "chunk B-tree signature/type")
        level, n = b[5], struct.unpack_from("<H", b, 6)[0]
        _need(level_expected is None or level == level_expected, "chunk B-tree level")
        _need(1 <= n <= 2 * CHUNK_K, "chunk B-tree entries %d" % n)
        p = 24
        keys, kids = [], []
        for i in range(n + 1):
            size, mask = struct.unpack_from("<II", b, p)
            off = tuple(struct.unpack_from("<%dQ" % ndims, b, p + 8))
            keys.append((size, mask, off))
            p += ksz
            if i < n:
                kids.append(struct.unpack_from("<Q", b, p)[0])
                p += 8
        for i in range(n):
            _need(keys[i][2] < keys[i + 1][2], "chunk B-tree keys out of order")
        for i in range(n):
            if level > 0:
                first = len(out)
                self._chunk_tree(kids[i], ndims, level - 1, out)
                _need(out[first][0][2] == keys[i][2], "internal key differs from the child's first key")
            else:
                out.append((keys[i], kids[i]))

    # -- mapping interface -------------------------------------------------
    def keys(self):
        return list(self.links)

    def __contains__(self, name):
        return name in self.datasets

    def __getitem__(self, name):
        return self.datasets[name]
