"""HDF5 files without the HDF5 library: the subset an Athena++ snapshot (.athdf) needs.

The reference reads and writes its snapshots through h5wasm, the HDF5 library compiled to
WebAssembly (src/io/athdf.ts:15-60). That library is not part of this project's image, so this
module restates the published on-disk format (the HDF5 File Format Specification, version 3.0)
for the structures such a file holds.

Writer: a version 0 superblock, version 1 object headers, the root group as a symbol table (a
version 1 B-tree of symbol-table nodes over a local heap), attributes in the root's header, and
datasets of fixed-point, floating-point and fixed-length string data, stored contiguously or in
gzip-compressed chunks indexed by a version 1 B-tree. These are the structures the HDF5 library
itself writes with its default (earliest) format settings, which every HDF5 reader takes.

Reader: superblocks of versions 0-3 (with a user block in front), object headers of versions 1
and 2 with continuation blocks, groups as symbol tables or as compact link messages, attribute
messages of versions 1-3, fixed-point, floating-point, fixed-length and variable-length string
types, compact, contiguous and version 1 B-tree chunked layouts, and the deflate, shuffle and
Fletcher-32 filters. Checksums of version 2 structures are not verified. Dense (fractal-heap)
link and attribute storage is refused with a clear error.
"""
from __future__ import annotations

import mmap
import os
import struct
import zlib

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF
# Fan-outs this writer declares in its superblock: symbol-table nodes of up to 2 x 4 entries and
# group B-tree nodes of up to 2 x 16 children (the library's defaults). Chunk B-tree nodes hold up
# to 2 x K children, K = 32 in a version 0 superblock; a file with chunked datasets gets a version 1
# superblock whose K fits its largest dataset in one node (up to MAX_CHUNK_K), so that a small
# file's index is small.
LEAF_K, GROUP_K, CHUNK_K, MAX_CHUNK_K = 4, 16, 32, 4096


class H5Error(ValueError):
    """A file this module cannot read, or an object it cannot write."""


def _pad8(n: int) -> int:
    return (n + 7) & ~7


# ---------------------------------------------------------------------------------------------
# Datatypes and dataspaces (the datatype message 0x0003 and the dataspace message 0x0001)
# ---------------------------------------------------------------------------------------------

def _datatype(dt: np.dtype, utf8: bool = False) -> bytes:
    """Encoded datatype message for a little-endian number or a fixed-length byte string."""
    dt = np.dtype(dt)
    if dt.kind in "iu":
        bits = 0x08 if dt.kind == "i" else 0x00  # bit 3: signed; bit 0 = 0: little-endian
        return struct.pack("<B3sI", 0x10 | 0, bytes([bits, 0, 0]), dt.itemsize) + struct.pack("<HH", 0, 8 * dt.itemsize)
    if dt.kind == "f":
        if dt.itemsize == 4:
            sign, eloc, esize, msize, bias = 31, 23, 8, 23, 127
        elif dt.itemsize == 8:
            sign, eloc, esize, msize, bias = 63, 52, 11, 52, 1023
        else:
            raise H5Error(f"no float type of {dt.itemsize} bytes is written")
        # bit field: little-endian, zero padding, mantissa normalised with an implied msb (2 << 4)
        return (struct.pack("<B3sI", 0x10 | 1, bytes([0x20, sign, 0]), dt.itemsize)
                + struct.pack("<HHBBBBI", 0, 8 * dt.itemsize, eloc, esize, 0, msize, bias))
    if dt.kind == "S":
        # null-padded fixed-length string, ASCII (charset 0) or UTF-8 (charset 1)
        return struct.pack("<B3sI", 0x10 | 3, bytes([0x01 | ((1 if utf8 else 0) << 4), 0, 0]), max(1, dt.itemsize))
    raise H5Error(f"no HDF5 type is written for {dt}")


def _dataspace(shape, maxshape=None) -> bytes:
    """Version 1 dataspace: rank 0 is a scalar."""
    rank = len(shape)
    flags = 1 if maxshape is not None else 0
    out = struct.pack("<BBBB4x", 1, rank, flags, 0)
    out += b"".join(struct.pack("<Q", int(d)) for d in shape)
    if maxshape is not None:
        out += b"".join(struct.pack("<Q", UNDEF if m is None else int(m)) for m in maxshape)
    return out


def _message(mtype: int, data: bytes, flags: int = 0) -> bytes:
    """A version 1 object-header message: its 8-byte header and its data padded to 8 bytes."""
    if len(data) > 0xFFFF:
        raise H5Error(f"an object-header message of {len(data)} bytes is larger than HDF5 allows (65535)")
    body = data + b"\0" * (_pad8(len(data)) - len(data))
    return struct.pack("<HHB3x", mtype, len(body), flags) + body


def _object_header(messages: list[bytes]) -> bytes:
    size = sum(len(m) for m in messages)
    return struct.pack("<BBHII4x", 1, 0, len(messages), 1, size) + b"".join(messages)


# ---------------------------------------------------------------------------------------------
# Writer
# ---------------------------------------------------------------------------------------------

class _Dataset:
    def __init__(self, name, data, chunks, gzip, maxshape):
        self.name = name
        self.data = np.ascontiguousarray(data)
        if self.data.dtype.byteorder == ">":
            self.data = self.data.astype(self.data.dtype.newbyteorder("<"))
        self.chunks = tuple(int(c) for c in chunks) if chunks is not None else None
        self.gzip = int(gzip)
        self.maxshape = maxshape
        self.dtype_msg = _datatype(self.data.dtype)


def _chunk_grid(shape, chunks):
    counts = [max(1, -(-int(s) // int(c))) for s, c in zip(shape, chunks)]
    for flat in range(int(np.prod(counts))):
        idx = []
        r = flat
        for c in reversed(counts):
            idx.append(r % c)
            r //= c
        yield tuple(reversed(idx))


class H5Writer:
    """Collects root attributes and root datasets, then writes one HDF5 file.

    ``attr(name, value, dtype)`` takes a number, a sequence of numbers or a string (or a list of
    strings with an ``S<n>`` dtype); ``dataset(name, array, chunks=, gzip=, maxshape=)`` takes a
    numpy array of numbers. With ``gzip`` > 0 the dataset is stored in chunks (``chunks``, or the
    whole array as one chunk), each compressed with HDF5's deflate filter at that level.
    """

    def __init__(self):
        self.attrs: list[tuple[str, bytes]] = []
        self.sets: list[_Dataset] = []

    def attr(self, name: str, value, dtype=None) -> None:
        if isinstance(value, str) or (dtype is not None and np.dtype(dtype).kind == "S" and not isinstance(value, (list, tuple))):
            raw = value.encode("utf-8") if isinstance(value, str) else bytes(value)
            size = np.dtype(dtype).itemsize if dtype is not None else max(1, len(raw))
            if len(raw) > size:
                raise H5Error(f"attribute {name!r}: {len(raw)} bytes do not fit a string of {size}")
            arr, shape = raw.ljust(size, b"\0"), ()
            dt = np.dtype(f"S{size}")
            utf8 = not raw.isascii()
        elif dtype is not None and np.dtype(dtype).kind == "S":
            dt = np.dtype(dtype)
            items = [v.encode("utf-8") if isinstance(v, str) else bytes(v) for v in value]
            if any(len(v) > dt.itemsize for v in items):
                raise H5Error(f"attribute {name!r}: a string is longer than {dt.itemsize} bytes")
            arr, shape = b"".join(v.ljust(dt.itemsize, b"\0") for v in items), (len(items),)
            utf8 = not all(v.isascii() for v in items)
        else:
            a = np.asarray(value, dtype=dtype)
            dt = a.dtype.newbyteorder("<") if a.dtype.byteorder == ">" else a.dtype
            arr, shape = a.astype(dt).tobytes(), a.shape
            utf8 = False
        nm = name.encode("utf-8") + b"\0"
        dtm, dsm = _datatype(dt, utf8), _dataspace(shape)
        body = (struct.pack("<BBHHH", 1, 0, len(nm), len(dtm), len(dsm)) + nm.ljust(_pad8(len(nm)), b"\0")
                + dtm.ljust(_pad8(len(dtm)), b"\0") + dsm.ljust(_pad8(len(dsm)), b"\0") + arr)
        self.attrs.append((name, _message(0x000C, body)))

    def dataset(self, name: str, data, chunks=None, gzip: int = 0, maxshape=None) -> None:
        if "/" in name or not name:
            raise H5Error(f"dataset names are plain names in the root group: {name!r}")
        if any(d.name == name for d in self.sets):
            raise H5Error(f"dataset {name!r} is written twice")
        data = np.asarray(data)
        if gzip and chunks is None:
            chunks = data.shape
        if chunks is not None and (len(chunks) != data.ndim or any(int(c) < 1 for c in chunks)):
            raise H5Error(f"dataset {name!r}: chunks {chunks} do not fit shape {data.shape}")
        self.sets.append(_Dataset(name, data, chunks, gzip, maxshape))

    # -- layout ---------------------------------------------------------------------------------
    def write(self, path=None) -> bytes | None:
        """Write the file to ``path`` (a file name or a binary file object), or return its bytes."""
        sets = sorted(self.sets, key=lambda d: d.name.encode("utf-8"))
        if len(sets) > 2 * LEAF_K * 2 * GROUP_K:
            raise H5Error("too many datasets for one symbol-table B-tree node")
        # local heap: "" at offset 0, then each name null-terminated and padded to 8
        heap = bytearray(8)
        name_off = []
        for d in sets:
            name_off.append(len(heap))
            nm = d.name.encode("utf-8") + b"\0"
            heap += nm + b"\0" * (_pad8(len(nm)) - len(nm))
        groups = [list(range(i, min(i + 2 * LEAF_K, len(sets)))) for i in range(0, len(sets), 2 * LEAF_K)]

        # raw data first in memory: chunked sets are compressed here so their sizes are known
        raw_parts = []  # (dataset index, chunk offset tuple or None, bytes or ndarray)
        for si, d in enumerate(sets):
            if d.chunks is None:
                raw_parts.append((si, None, d.data))
                continue
            for ci in _chunk_grid(d.data.shape, d.chunks):
                lo = [c * k for c, k in zip(ci, d.chunks)]
                block = np.zeros(d.chunks, d.data.dtype)
                sl = tuple(slice(l, min(l + k, s)) for l, k, s in zip(lo, d.chunks, d.data.shape))
                block[tuple(slice(0, s.stop - s.start) for s in sl)] = d.data[sl]
                b = block.tobytes()
                raw_parts.append((si, tuple(lo), zlib.compress(b, d.gzip) if d.gzip else b))

        # chunk-index fan-out, and with it the superblock's version and size
        nchunks = [sum(1 for si2, off, _ in raw_parts if si2 == si and off is not None) for si in range(len(sets))]
        ck = CHUNK_K
        if any(nchunks):
            ck = min(MAX_CHUNK_K, max(1, -(-max(nchunks) // 2)))
        sb_version = 1 if ck != CHUNK_K else 0
        SB = 96 if sb_version == 0 else 104
        root_msgs_len = [len(_message(0x0011, b"\0" * 16))] + [len(m) for _, m in self.attrs]
        root_oh = 16 + sum(root_msgs_len)
        heap_hdr = 32
        btree = 24 + (2 * GROUP_K + 1) * 8 + 2 * GROUP_K * 8
        snod = 8 + 2 * LEAF_K * 40
        addr = SB
        a_root = addr; addr = _pad8(addr + root_oh)
        a_heap = addr; addr = _pad8(addr + heap_hdr)
        a_heapdata = addr; addr = _pad8(addr + len(heap))
        a_btree = addr; addr += btree
        a_snod = []
        for _ in groups:
            a_snod.append(addr); addr += snod
        # dataset headers: their sizes do not depend on addresses
        oh_size, chunk_nodes = [], []
        for d in sets:
            oh_size.append(len(self._dataset_header(d, 0, 0)))
        a_oh = []
        for s in oh_size:
            a_oh.append(addr); addr = _pad8(addr + s)
        # chunk B-trees (one or more levels of nodes of up to 2 x CHUNK_K entries)
        chunk_keys = {si: [] for si in range(len(sets))}
        for si, off, b in raw_parts:
            if off is not None:
                chunk_keys[si].append([off, b])
        node_size = lambda rank: 24 + (2 * ck + 1) * (8 + 8 * (rank + 1)) + 2 * ck * 8
        tree_plan = {}
        for si, keys in chunk_keys.items():
            if not keys:
                continue
            levels = []
            count = len(keys)
            while True:
                nodes = -(-count // (2 * ck))
                levels.append(nodes)
                if nodes == 1:
                    break
                count = nodes
            rank = sets[si].data.ndim
            addrs = []
            for nodes in levels:
                row = []
                for _ in range(nodes):
                    row.append(addr); addr += node_size(rank)
                addrs.append(row)
            tree_plan[si] = addrs  # addrs[0]: leaves; addrs[-1]: the root (one node)
        # raw data
        raw_addr = []
        for si, off, b in raw_parts:
            addr = _pad8(addr)
            raw_addr.append(addr)
            addr += b.nbytes if isinstance(b, np.ndarray) else len(b)
        eof = addr

        # encode
        out = bytearray()
        out += SIGNATURE + struct.pack("<BBBBBBBB", sb_version, 0, 0, 0, 0, 8, 8, 0) + struct.pack("<HHI", LEAF_K, GROUP_K, 0)
        if sb_version == 1:
            out += struct.pack("<HH", ck, 0)  # indexed-storage internal node K, reserved
        out += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
        out += struct.pack("<QQII", 0, a_root, 1, 0) + struct.pack("<QQ", a_btree, a_heap)
        out += b"\0" * (SB - len(out))
        assert len(out) == SB

        def put(at, b):
            if len(out) < at:
                out.extend(b"\0" * (at - len(out)))
            assert len(out) == at, (at, len(out))
            out.extend(b)

        root_msgs = [_message(0x0011, struct.pack("<QQ", a_btree, a_heap), flags=1)] + [m for _, m in self.attrs]
        put(a_root, _object_header(root_msgs))
        # H5HL: no free block is offset 1 (an offset no 8-aligned block can have)
        put(a_heap, b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap), 1, a_heapdata))
        put(a_heapdata, bytes(heap))
        # group B-tree: key 0 is "", key i + 1 the largest name in child i
        bt = b"TREE" + struct.pack("<BBHQQ", 0, 0, len(groups), UNDEF, UNDEF)
        keys = [0] + [name_off[g[-1]] for g in groups]
        body = b""
        for i in range(2 * GROUP_K + 1):
            body += struct.pack("<Q", keys[i] if i < len(keys) else 0)
            if i < 2 * GROUP_K:
                body += struct.pack("<Q", a_snod[i] if i < len(a_snod) else 0)
        put(a_btree, bt + body)
        for g, a in zip(groups, a_snod):
            ent = b"".join(struct.pack("<QQII16x", name_off[i], a_oh[i], 0, 0) for i in g)
            put(a, b"SNOD" + struct.pack("<BBH", 1, 0, len(g)) + ent.ljust(2 * LEAF_K * 40, b"\0"))
        # dataset headers
        part_of = {}
        for k, (si, off, b) in enumerate(raw_parts):
            part_of.setdefault(si, []).append(k)
        for si, d in enumerate(sets):
            if d.chunks is None:
                k = part_of[si][0]
                put(a_oh[si], self._dataset_header(d, raw_addr[k], d.data.nbytes))
            else:
                put(a_oh[si], self._dataset_header(d, tree_plan[si][-1][0], 0))
        # chunk B-tree nodes
        for si, addrs in tree_plan.items():
            d = sets[si]
            rank = d.data.ndim
            items = [(raw_parts[k][1], len(raw_parts[k][2]), raw_addr[k]) for k in part_of[si]]
            end = tuple(o + c for o, c in zip(items[-1][0], d.chunks))
            level_items = items
            for lev, row in enumerate(addrs):
                nxt = []
                for n, a in enumerate(row):
                    sub = level_items[n * 2 * ck:(n + 1) * 2 * ck]
                    hi = level_items[(n + 1) * 2 * ck][0] if (n + 1) * 2 * ck < len(level_items) else end
                    node = b"TREE" + struct.pack("<BBHQQ", 1, lev, len(sub),
                                                 row[n - 1] if n > 0 else UNDEF, row[n + 1] if n + 1 < len(row) else UNDEF)
                    for i in range(2 * ck + 1):
                        if i < len(sub):
                            off, nb, ca = sub[i]
                            node += struct.pack("<II", nb, 0) + b"".join(struct.pack("<Q", o) for o in off) + struct.pack("<Q", 0)
                            node += struct.pack("<Q", ca)
                        elif i == len(sub):
                            node += struct.pack("<II", 0, 0) + b"".join(struct.pack("<Q", o) for o in hi) + struct.pack("<Q", 0)
                            if i < 2 * ck:
                                node += struct.pack("<Q", 0)
                        else:
                            node += b"\0" * (8 + 8 * (rank + 1))
                            if i < 2 * ck:
                                node += struct.pack("<Q", 0)
                    put(a, node)
                    nxt.append((sub[0][0], sub[0][1], a))
                level_items = nxt

        # raw data: uncompressed arrays go out as views of themselves, never copied
        pieces = [out]
        at = len(out)
        for k, (si, off, b) in enumerate(raw_parts):
            if raw_addr[k] > at:
                pieces.append(b"\0" * (raw_addr[k] - at))
                at = raw_addr[k]
            mv = memoryview(b.reshape(-1)).cast("B") if isinstance(b, np.ndarray) else b
            pieces.append(mv)
            at += len(mv)
        assert at == eof
        if path is None:
            return b"".join(bytes(p) for p in pieces)
        return self._emit(path, pieces)

    @staticmethod
    def _emit(path, pieces):
        if hasattr(path, "write"):
            for p in pieces:
                path.write(p)
            return None
        with open(path, "wb") as f:
            for p in pieces:
                f.write(p)
        return None

    @staticmethod
    def _dataset_header(d: _Dataset, data_addr: int, nbytes: int) -> bytes:
        rank = d.data.ndim
        msgs = [_message(0x0001, _dataspace(d.data.shape, d.maxshape)),
                _message(0x0003, d.dtype_msg, flags=1),
                # fill value, version 2: allocated early, written if set, none defined
                _message(0x0005, struct.pack("<BBBB", 2, 1 if d.chunks is None else 3, 2, 0), flags=1)]
        if d.chunks is None:
            msgs.append(_message(0x0008, struct.pack("<BBQQ", 3, 1, data_addr, nbytes)))
        else:
            lay = struct.pack("<BBBQ", 3, 2, rank + 1, data_addr)
            lay += b"".join(struct.pack("<I", int(c)) for c in d.chunks) + struct.pack("<I", d.data.dtype.itemsize)
            msgs.append(_message(0x0008, lay))
            if d.gzip:
                # deflate (id 1), optional, one client value (the level), padded to 8 bytes
                msgs.append(_message(0x000B, struct.pack("<BB6xHHHHI4x", 1, 1, 1, 0, 1, 1, d.gzip)))
        return _object_header(msgs)


# ---------------------------------------------------------------------------------------------
# Reader
# ---------------------------------------------------------------------------------------------

class _Type:
    """A decoded datatype: a numpy dtype, or a variable-length string."""

    def __init__(self, dtype=None, vlen_str=False, size=0, charset=0):
        self.dtype = dtype
        self.vlen_str = vlen_str
        self.size = size if dtype is None else dtype.itemsize
        self.charset = charset


class Dataset:
    """A dataset of an open :class:`H5File`: ``shape``, ``dtype``, ``attrs``, ``read()`` and
    numpy-style slicing (``d[1:2, 5:9]``)."""

    def __init__(self, file, name, space, dtype, layout, filters, attrs):
        self.file, self.name = file, name
        self.shape, self.maxshape = space
        self._type = dtype
        self.dtype = dtype.dtype
        self._layout = layout
        self._filters = filters
        self.attrs = attrs
        self._whole = None

    def read(self) -> np.ndarray:
        return self.file._read_data(self)

    def __getitem__(self, key):
        lay = self._layout
        if lay[0] == "contiguous" and self._type.dtype is not None:
            # contiguous storage: the slice is copied out of the mapped file, nothing else read
            return np.array(self.file._contiguous_view(self)[key]).astype(self.dtype.newbyteorder("="), copy=False)
        # other layouts are decoded whole once, then sliced
        if self._whole is None:
            self._whole = self.read()
        return self._whole[key]


class H5File:
    """Read-only view of an HDF5 file (a path, or the file's bytes).

    ``attrs`` holds the root group's attributes; ``keys()``, ``f[name]`` and ``get(name)``
    give the root group's datasets (``a/b`` paths walk subgroups).
    """

    def __init__(self, src):
        self._mm = None
        if isinstance(src, (bytes, bytearray, memoryview)):
            self.buf = memoryview(bytes(src))
        else:
            fh = open(os.fspath(src), "rb")
            try:
                size = os.fstat(fh.fileno()).st_size
                self._mm = mmap.mmap(fh.fileno(), 0, access=mmap.ACCESS_READ) if size else None
            finally:
                fh.close()
            self.buf = memoryview(self._mm) if self._mm is not None else memoryview(b"")
        self._find_superblock()
        self._ghc = {}
        self.attrs, self._root = self._group_at(self._root_addr)

    def close(self):
        if self._mm is not None:
            try:
                self.buf.release()
                self._mm.close()
            except BufferError:
                pass  # arrays still view the mapping: it closes when they are gone
            self._mm = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- low level ------------------------------------------------------------------------------
    def _u(self, at, n):
        if at < 0 or at + n > len(self.buf):
            raise H5Error("the file ends inside an HDF5 structure (truncated or not HDF5)")
        return int.from_bytes(self.buf[at:at + n], "little")

    def _bytes(self, at, n) -> bytes:
        if at < 0 or at + n > len(self.buf):
            raise H5Error("the file ends inside an HDF5 structure (truncated or not HDF5)")
        return bytes(self.buf[at:at + n])

    def _abs(self, a):
        return self.base + a

    def _find_superblock(self):
        at = 0
        while at + 8 <= len(self.buf):
            if bytes(self.buf[at:at + 8]) == SIGNATURE:
                break
            at = 512 if at == 0 else at * 2
        else:
            raise H5Error("this is not an HDF5 file")
        v = self._u(at + 8, 1)
        # addresses count from the superblock, wherever a user block puts it (the library
        # replaces a stored base address that differs by the superblock's own offset)
        self.base = at
        if v in (0, 1):
            self.so, self.sl = self._u(at + 13, 1), self._u(at + 14, 1)
            p = at + 24 + (4 if v == 1 else 0)
            p += 4 * self.so
            # root group symbol-table entry: name offset, header address, cache type, scratch
            self._root_addr = self._u(p + self.so, self.so)
        elif v in (2, 3):
            self.so, self.sl = self._u(at + 9, 1), self._u(at + 10, 1)
            self._root_addr = self._u(at + 12 + 3 * self.so, self.so)
        else:
            raise H5Error(f"HDF5 superblock version {v} is not read")
        if self.so != 8 or self.sl != 8:
            raise H5Error("only files with 8-byte offsets and lengths are read")

    def _undef(self, a):
        return a == (1 << (8 * self.so)) - 1

    # -- object headers -------------------------------------------------------------------------
    def _messages(self, addr):
        """[(type, data bytes)] of the object header at ``addr`` (file-relative)."""
        at = self._abs(addr)
        out = []
        if self._bytes(at, 4) == b"OHDR":
            ver, flags = self._u(at + 4, 1), self._u(at + 5, 1)
            if ver != 2:
                raise H5Error(f"object header version {ver} is not read")
            p = at + 6
            if flags & 0x20:
                p += 16
            if flags & 0x10:
                p += 4
            nsz = 1 << (flags & 3)
            size = self._u(p, nsz)
            p += nsz
            blocks = [(p, size)]
            track = bool(flags & 0x04)
            while blocks:
                p, size = blocks.pop(0)
                end = p + size
                while p + 4 <= end:
                    mt, ms, mf = self._u(p, 1), self._u(p + 1, 2), self._u(p + 3, 1)
                    p += 4 + (2 if track else 0)
                    data = self._bytes(p, ms)
                    p += ms
                    if mt == 0x10:
                        ca, cl = struct.unpack_from("<QQ", data)
                        cat = self._abs(ca)
                        if self._bytes(cat, 4) != b"OCHK":
                            raise H5Error("bad object header continuation block")
                        blocks.append((cat + 4, cl - 8))
                    elif mt != 0:
                        out.append((mt, data, mf))
            return out
        ver = self._u(at, 1)
        if ver != 1:
            raise H5Error(f"object header version {ver} is not read")
        nmsg, size = self._u(at + 2, 2), self._u(at + 8, 4)
        blocks = [(at + 16, size)]
        seen = 0
        while blocks and seen < nmsg:
            p, size = blocks.pop(0)
            end = p + size
            while p + 8 <= end and seen < nmsg:
                mt, ms, mf = self._u(p, 2), self._u(p + 2, 2), self._u(p + 4, 1)
                data = self._bytes(p + 8, ms)
                p += 8 + ms
                seen += 1
                if mt == 0x10:
                    ca, cl = struct.unpack_from("<QQ", data)
                    blocks.append((self._abs(ca), cl))
                elif mt != 0:
                    out.append((mt, data, mf))
        return out

    # -- types ----------------------------------------------------------------------------------
    def _parse_type(self, d: bytes, o: int = 0) -> tuple[_Type, int]:
        cv = d[o]
        cls, bits = cv & 0x0F, d[o + 1] | (d[o + 2] << 8) | (d[o + 3] << 16)
        size = struct.unpack_from("<I", d, o + 4)[0]
        p = o + 8
        if cls == 0:
            order = ">" if bits & 1 else "<"
            kind = "i" if bits & 0x08 else "u"
            return _Type(np.dtype(f"{order}{kind}{size}")), p + 4
        if cls == 1:
            order = ">" if bits & 1 else "<"
            if size not in (2, 4, 8):
                raise H5Error(f"a float of {size} bytes is not read")
            return _Type(np.dtype(f"{order}f{size}")), p + 12
        if cls == 3:
            return _Type(np.dtype(f"S{size}"), charset=(bits >> 4) & 0x0F), p
        if cls == 9:
            base, p2 = self._parse_type(d, p)
            if bits & 0x0F == 1:
                return _Type(None, vlen_str=True, size=size, charset=(bits >> 8) & 0x0F), p2
            raise H5Error("variable-length sequences are not read")
        if cls == 8:  # enumeration: read as its base integer type
            base, p2 = self._parse_type(d, p)
            return base, len(d)
        raise H5Error(f"HDF5 datatype class {cls} is not read")

    def _parse_space(self, d: bytes, o: int = 0):
        ver, rank, flags = d[o], d[o + 1], d[o + 2]
        if ver == 1:
            p = o + 8
        elif ver == 2:
            if d[o + 3] == 2:  # null dataspace
                return (), ()
            p = o + 4
        else:
            raise H5Error(f"dataspace version {ver} is not read")
        dims = struct.unpack_from(f"<{rank}Q", d, p)
        p += 8 * rank
        maxd = None
        if flags & 1:
            maxd = tuple(None if self._undef(m) else m for m in struct.unpack_from(f"<{rank}Q", d, p))
            p += 8 * rank
        return tuple(int(x) for x in dims), maxd, p

    def _values(self, typ: _Type, shape, raw: bytes):
        n = int(np.prod(shape)) if shape else 1
        if typ.vlen_str:
            items = []
            for i in range(n):
                ln, ga, gi = struct.unpack_from("<IQI", raw, i * 16)
                items.append(self._global(ga, gi)[:ln].decode("utf-8", "replace") if ga else "")
            return items[0] if not shape else np.array(items, dtype=object).reshape(shape)
        a = np.frombuffer(raw[: n * typ.dtype.itemsize], dtype=typ.dtype)
        if typ.dtype.kind == "S":
            strs = [bytes(x).rstrip(b"\0").decode("utf-8", "replace") for x in a]
            return strs[0] if not shape else strs
        a = a.astype(typ.dtype.newbyteorder("=")) if typ.dtype.byteorder not in ("=", "|") else a.copy()
        return a.reshape(shape) if shape else a[0]

    def _global(self, coll, index) -> bytes:
        if coll not in self._ghc:
            at = self._abs(coll)
            if self._bytes(at, 4) != b"GCOL":
                raise H5Error("bad global heap collection")
            size = self._u(at + 8, 8)
            objs, p, end = {}, at + 16, at + size
            while p + 16 <= end:
                idx, osz = self._u(p, 2), self._u(p + 8, 8)
                if idx == 0:
                    break
                objs[idx] = self._bytes(p + 16, osz)
                p += 16 + _pad8(osz)
            self._ghc[coll] = objs
        return self._ghc[coll].get(index, b"")

    def _attribute(self, d: bytes):
        ver = d[0]
        nlen, tlen, slen = struct.unpack_from("<HHH", d, 2)
        if ver == 1:
            p = 8
            name = d[p:p + nlen].rstrip(b"\0").decode("utf-8")
            p += _pad8(nlen)
            typ, _ = self._parse_type(d, p)
            p += _pad8(tlen)
            space = self._parse_space(d, p)
            p += _pad8(slen)
        elif ver in (2, 3):
            p = 8 if ver == 2 else 9
            name = d[p:p + nlen].rstrip(b"\0").decode("utf-8")
            p += nlen
            typ, _ = self._parse_type(d, p)
            p += tlen
            space = self._parse_space(d, p)
            p += slen
        else:
            raise H5Error(f"attribute message version {ver} is not read")
        shape = space[0]
        if typ.vlen_str:
            return name, self._values(typ, shape, d[p:])
        return name, self._values(typ, shape, d[p:])

    # -- groups ---------------------------------------------------------------------------------
    def _group_at(self, addr):
        """(attributes, {name: object header address}) of the group whose header is at addr."""
        attrs, links = {}, {}
        for mt, d, _ in self._messages(addr):
            if mt == 0x000C:
                k, v = self._attribute(d)
                attrs[k] = v
            elif mt == 0x0011:
                bt, hp = struct.unpack_from("<QQ", d)
                links.update(self._symbol_table(bt, hp))
            elif mt == 0x0006:
                k, a = self._link(d)
                if a is not None:
                    links[k] = a
            elif mt == 0x0002:
                if not self._undef(struct.unpack_from("<Q", d, 2 + (8 if d[1] & 1 else 0))[0]):
                    raise H5Error("groups with dense (fractal heap) link storage are not read")
            elif mt == 0x0015:
                fh = struct.unpack_from("<Q", d, 2 + (2 if d[1] & 1 else 0))[0]
                if not self._undef(fh):
                    raise H5Error("dense (fractal heap) attribute storage is not read")
        return attrs, links

    def _link(self, d: bytes):
        flags = d[1]
        p = 2
        ltype = 0
        if flags & 0x08:
            ltype = d[p]; p += 1
        if flags & 0x04:
            p += 8
        if flags & 0x10:
            p += 1
        ln_size = 1 << (flags & 3)
        ln = int.from_bytes(d[p:p + ln_size], "little"); p += ln_size
        name = d[p:p + ln].decode("utf-8"); p += ln
        if ltype == 0:
            return name, struct.unpack_from("<Q", d, p)[0]
        return name, None  # soft and external links are not followed

    def _symbol_table(self, btree, heap):
        hat = self._abs(heap)
        if self._bytes(hat, 4) != b"HEAP":
            raise H5Error("bad local heap")
        seg = self._abs(self._u(hat + 24, 8))

        def name_at(off):
            p = seg + off
            end = p
            while self._u(end, 1):
                end += 1
            return self._bytes(p, end - p).decode("utf-8")

        links = {}
        stack = [btree]
        while stack:
            at = self._abs(stack.pop())
            if self._bytes(at, 4) != b"TREE" or self._u(at + 4, 1) != 0:
                raise H5Error("bad group B-tree node")
            level, used = self._u(at + 5, 1), self._u(at + 6, 2)
            p = at + 24
            for i in range(used):
                child = self._u(p + 8, 8)
                p += 16
                if level > 0:
                    stack.append(child)
                    continue
                sat = self._abs(child)
                if self._bytes(sat, 4) != b"SNOD":
                    raise H5Error("bad symbol table node")
                ns = self._u(sat + 6, 2)
                for e in range(ns):
                    q = sat + 8 + 40 * e
                    links[name_at(self._u(q, 8))] = self._u(q + 8, 8)
        return links

    # -- objects --------------------------------------------------------------------------------
    def keys(self):
        return list(self._root.keys())

    def __contains__(self, name):
        return self.get(name) is not None

    def __getitem__(self, name):
        obj = self.get(name)
        if obj is None:
            raise KeyError(name)
        return obj

    def get(self, name):
        links = self._root
        parts = [p for p in name.split("/") if p]
        for i, part in enumerate(parts):
            if part not in links:
                return None
            addr = links[part]
            msgs = self._messages(addr)
            if any(mt in (0x0011, 0x0006, 0x0002) for mt, _, _ in msgs) and not any(mt == 0x0008 for mt, _, _ in msgs):
                if i == len(parts) - 1:
                    return _Group(self, addr)
                links = self._group_at(addr)[1]
                continue
            if i != len(parts) - 1:
                return None
            return self._dataset(part, msgs)
        return None

    def _dataset(self, name, msgs):
        space = typ = layout = None
        filters, attrs = [], {}
        for mt, d, _ in msgs:
            if mt == 0x0001:
                s = self._parse_space(d)
                space = (s[0], s[1])
            elif mt == 0x0003:
                typ, _ = self._parse_type(d)
            elif mt == 0x0008:
                layout = self._parse_layout(d)
            elif mt == 0x000B:
                filters = self._parse_filters(d)
            elif mt == 0x000C:
                k, v = self._attribute(d)
                attrs[k] = v
        if space is None or typ is None or layout is None:
            raise H5Error(f"{name!r} is not a dataset this reader understands")
        return Dataset(self, name, space, typ, layout, filters, attrs)

    def _parse_layout(self, d: bytes):
        ver = d[0]
        if ver in (1, 2):
            rank, cls = d[1], d[2]
            p = 8
            if cls == 0:
                dims = struct.unpack_from(f"<{rank}I", d, p); p += 4 * rank
                size = struct.unpack_from("<I", d, p)[0]
                return ("compact", bytes(d[p + 4:p + 4 + size]))
            a = struct.unpack_from("<Q", d, p)[0]; p += 8
            dims = struct.unpack_from(f"<{rank}I", d, p)
            if cls == 1:
                return ("contiguous", a, None)
            return ("chunked", a, tuple(dims))
        if ver in (3, 4):
            cls = d[1]
            if cls == 0:
                size = struct.unpack_from("<H", d, 2)[0]
                return ("compact", bytes(d[4:4 + size]))
            if cls == 1:
                a, size = struct.unpack_from("<QQ", d, 2)
                return ("contiguous", a, size)
            if cls == 2 and ver == 3:
                rank = d[2]
                a = struct.unpack_from("<Q", d, 3)[0]
                dims = struct.unpack_from(f"<{rank}I", d, 11)
                return ("chunked", a, tuple(dims))
            raise H5Error("version 4 chunk indexes are not read (only version 1 B-trees)")
        raise H5Error(f"data layout version {ver} is not read")

    def _parse_filters(self, d: bytes):
        ver, n = d[0], d[1]
        p = 8 if ver == 1 else 2
        out = []
        for _ in range(n):
            fid = struct.unpack_from("<H", d, p)[0]; p += 2
            nlen = 0
            if ver == 1 or fid >= 256:
                nlen = struct.unpack_from("<H", d, p)[0]; p += 2
            flags, nv = struct.unpack_from("<HH", d, p); p += 4
            if nlen:
                p += _pad8(nlen) if ver == 1 else nlen
            vals = struct.unpack_from(f"<{nv}I", d, p); p += 4 * nv
            if ver == 1 and nv % 2:
                p += 4
            out.append((fid, vals))
        return out

    # -- data -----------------------------------------------------------------------------------
    def _contiguous_view(self, ds: Dataset) -> np.ndarray:
        _, a, size = ds._layout
        n = int(np.prod(ds.shape)) if ds.shape else 1
        nbytes = n * ds._type.size
        if self._undef(a):
            return np.zeros(ds.shape, ds.dtype)
        at = self._abs(a)
        if at + nbytes > len(self.buf):
            raise H5Error(f"dataset {ds.name!r} runs past the end of the file")
        return np.frombuffer(self.buf, dtype=ds.dtype, count=n, offset=at).reshape(ds.shape)

    def _read_data(self, ds: Dataset):
        lay = ds._layout
        n = int(np.prod(ds.shape)) if ds.shape else 1
        if lay[0] == "compact":
            raw = lay[1]
        elif lay[0] == "contiguous":
            if ds._type.dtype is not None:
                return self._contiguous_view(ds).astype(ds.dtype.newbyteorder("="), copy=True)
            raw = b"" if self._undef(lay[1]) else self._bytes(self._abs(lay[1]), n * ds._type.size)
        else:
            return self._read_chunked(ds)
        return self._values(ds._type, ds.shape, raw)

    def _read_chunked(self, ds: Dataset):
        _, root, cdims = ds._layout
        rank = len(ds.shape)
        chunk = cdims[:rank]
        esize = ds._type.size
        if ds._type.dtype is None:
            raise H5Error("chunked variable-length data is not read")
        out = np.zeros(ds.shape, ds.dtype)
        if self._undef(root):
            return out
        nd = len(cdims)
        stack = [root]
        while stack:
            at = self._abs(stack.pop())
            if self._bytes(at, 4) != b"TREE" or self._u(at + 4, 1) != 1:
                raise H5Error("bad chunk B-tree node")
            level, used = self._u(at + 5, 1), self._u(at + 6, 2)
            p = at + 24
            ksize = 8 + 8 * nd
            for i in range(used):
                csize, mask = self._u(p, 4), self._u(p + 4, 4)
                off = [self._u(p + 8 + 8 * k, 8) for k in range(rank)]
                child = self._u(p + ksize, 8)
                p += ksize + 8
                if level > 0:
                    stack.append(child)
                    continue
                raw = self._bytes(self._abs(child), csize)
                for j in range(len(ds._filters) - 1, -1, -1):
                    if mask & (1 << j):
                        continue
                    fid, vals = ds._filters[j]
                    if fid == 1:
                        raw = zlib.decompress(raw)
                    elif fid == 2:
                        cnt = len(raw) // esize
                        raw = np.frombuffer(raw[: cnt * esize], np.uint8).reshape(esize, cnt).T.tobytes() + raw[cnt * esize:]
                    elif fid == 3:
                        raw = raw[:-4]
                    else:
                        raise H5Error(f"HDF5 filter {fid} is not read")
                blk = np.frombuffer(raw[: int(np.prod(chunk)) * esize], dtype=ds.dtype).reshape(chunk)
                dst = tuple(slice(o, min(o + c, s)) for o, c, s in zip(off, chunk, ds.shape))
                src = tuple(slice(0, s.stop - s.start) for s in dst)
                out[dst] = blk[src]
        return out.astype(ds.dtype.newbyteorder("="), copy=False)


class _Group:
    def __init__(self, f: H5File, addr):
        self.file = f
        self.attrs, self._links = f._group_at(addr)

    def keys(self):
        return list(self._links.keys())
