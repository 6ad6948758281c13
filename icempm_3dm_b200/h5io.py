"""HDF5 files in the classic layout the reference's snapshots and raw point
clouds use, read and written from the published HDF5 File Format
Specification (version 2.0) without the HDF5 library.

Scope (what the reference's HDF5 C++ calls produce with default file
properties, simulation/snapshotmanager.cpp:20-45 and :299-405):

- superblock version 0 (or 1), 8-byte offsets and lengths;
- the root group as a symbol table (version 1 B-tree of type 0, local heap,
  symbol table nodes), datasets directly under it;
- version 1 object headers, with continuation blocks;
- dataspace (versions 1, 2), datatype (fixed-point and IEEE float, little-
  or big-endian; compounds of them, as the animation frames' records use),
  fill value (version 2), data layout (version 3:
  compact, contiguous, chunked; versions 1 and 2 read), filter pipeline
  (versions 1, 2: deflate, shuffle, Fletcher-32), attributes (versions 1-3);
- chunk indexes as version 1 B-trees of type 1, any depth.

Anything outside that raises H5Error naming the structure. The writer emits
the same structures the HDF5 library writes for H5File(..., H5F_ACC_TRUNC) +
createDataSet/createAttribute with native types: the message versions,
flags and field values of the reference's own 3d_200k.h5 (checked byte for
byte by the tests), a 544-byte group B-tree node (K = 16), 328-byte symbol
table nodes (K = 4), 2096-byte chunk B-tree nodes (K = 32) and the chunk
index's right-most key carrying the element size in its last coordinate.
"""
import mmap
import os
import struct
import zlib
from concurrent.futures import ThreadPoolExecutor

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
_SIG = b"\x89HDF\r\n\x1a\n"
_GROUP_K = 16        # group internal node K (B-tree of type 0)
_LEAF_K = 4          # group leaf node K (symbol table node entries / 2)
_CHUNK_K = 32        # indexed storage internal node K (B-tree of type 1)

FILTER_DEFLATE, FILTER_SHUFFLE, FILTER_FLETCHER32 = 1, 2, 3


class H5Error(Exception):
    pass


def _pad8(n):
    return (n + 7) & ~7


# ------------------------------------------------------------------ reading

class H5File:
    """Read-only view of an HDF5 file: dataset names, attributes, data."""

    def __init__(self, path):
        self.path = os.fspath(path)
        self._f = open(self.path, "rb")
        size = os.fstat(self._f.fileno()).st_size
        if size < 96:
            raise H5Error(f"{self.path}: too short for an HDF5 superblock")
        self._mm = mmap.mmap(self._f.fileno(), 0, access=mmap.ACCESS_READ)
        self._b = memoryview(self._mm)
        self._base = self._find_superblock()
        self._datasets = {}
        self._read_superblock()

    # -- helpers
    def _u(self, off, n):
        return int.from_bytes(self._b[off:off + n], "little")

    def _find_superblock(self):
        off = 0
        while off + 8 <= len(self._b):
            if bytes(self._b[off:off + 8]) == _SIG:
                return off
            off = 512 if off == 0 else off * 2
        raise H5Error(f"{self.path}: no HDF5 signature")

    def close(self):
        if self._mm is not None:
            self._b.release()
            self._mm.close()
            self._f.close()
            self._mm = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- superblock and root group
    def _read_superblock(self):
        s = self._base
        ver = self._b[s + 8]
        if ver not in (0, 1):
            raise H5Error(f"superblock version {ver} (only 0 and 1 are read)")
        if self._b[s + 13] != 8 or self._b[s + 14] != 8:
            raise H5Error("only 8-byte offsets and lengths are read")
        self._addr_base = self._u(s + 24, 8)
        entry = s + 56 + (4 if ver == 1 else 0)
        ohdr = self._u(entry + 8, 8)
        cache = self._u(entry + 16, 4)
        if cache == 1:
            btree, heap = self._u(entry + 24, 8), self._u(entry + 32, 8)
        else:
            msgs = self._messages(ohdr)
            st = [d for t, f, d in msgs if t == 0x11]
            if not st:
                raise H5Error("root group is not a symbol-table group")
            btree = int.from_bytes(st[0][0:8], "little")
            heap = int.from_bytes(st[0][8:16], "little")
        self._read_group(btree, heap)

    def _a(self, addr):
        return self._addr_base + addr

    def _heap(self, addr):
        a = self._a(addr)
        if bytes(self._b[a:a + 4]) != b"HEAP":
            raise H5Error(f"local heap signature missing at {addr}")
        return self._a(self._u(a + 24, 8)), self._u(a + 8, 8)

    def _heap_name(self, data, size, off):
        if off >= size:
            raise H5Error("name offset outside the local heap")
        end = bytes(self._b[data + off:data + size]).index(b"\0")
        return bytes(self._b[data + off:data + off + end]).decode()

    def _check(self, a, n):
        if a < 0 or a + n > len(self._b):
            raise H5Error(f"structure at {a} runs past the end of the file")

    def _read_group(self, btree, heap):
        data, size = self._heap(heap)
        self._check(data, size)
        stack, seen = [btree], set()
        while stack:
            addr = stack.pop()
            if addr in seen:
                raise H5Error("group B-tree revisits a node")
            seen.add(addr)
            a = self._a(addr)
            self._check(a, 24)
            if bytes(self._b[a:a + 4]) != b"TREE" or self._b[a + 4] != 0:
                raise H5Error("group B-tree node expected")
            level, used = self._b[a + 5], self._u(a + 6, 2)
            p = a + 24
            for i in range(used):
                child = self._u(p + 8, 8)
                p += 16
                if level > 0:
                    stack.append(child)
                else:
                    self._read_snod(child, data, size)

    def _read_snod(self, addr, data, size):
        a = self._a(addr)
        self._check(a, 8)
        if bytes(self._b[a:a + 4]) != b"SNOD":
            raise H5Error("symbol table node signature missing")
        nsym = self._u(a + 6, 2)
        self._check(a + 8, 40 * nsym)
        for k in range(nsym):
            e = a + 8 + 40 * k
            name = self._heap_name(data, size, self._u(e, 8))
            self._datasets[name] = self._u(e + 8, 8)

    # -- object headers
    def _messages(self, addr):
        a = self._a(addr)
        self._check(a, 16)
        if bytes(self._b[a:a + 4]) == b"OHDR":
            raise H5Error("version 2 object headers are not read")
        if self._b[a] != 1:
            raise H5Error(f"object header version {self._b[a]}")
        blocks = [(a + 16, self._u(a + 8, 4))]
        seen = set()
        out = []
        while blocks:
            p, n = blocks.pop(0)
            if p in seen:
                raise H5Error("object header continuation revisits a block")
            seen.add(p)
            self._check(p, n)
            end = p + n
            while p + 8 <= end:
                t, sz, fl = self._u(p, 2), self._u(p + 2, 2), self._b[p + 4]
                if p + 8 + sz > end:
                    raise H5Error("header message runs past its block")
                d = bytes(self._b[p + 8:p + 8 + sz])
                if t == 0x10:
                    blocks.append((self._a(int.from_bytes(d[0:8], "little")), int.from_bytes(d[8:16], "little")))
                elif t != 0:
                    out.append((t, fl, d))
                p += 8 + sz
        return out

    # -- public API
    def keys(self):
        return sorted(self._datasets)

    def __contains__(self, name):
        return name in self._datasets

    def _info(self, name):
        if name not in self._datasets:
            raise KeyError(name)
        info = {"filters": [], "attrs": {}}
        for t, fl, d in self._messages(self._datasets[name]):
            if t == 0x01:
                info["shape"] = _parse_dataspace(d)[0]
            elif t == 0x03:
                info["dtype"] = _parse_datatype(d)[0]
            elif t == 0x08:
                info["layout"] = _parse_layout(d)
            elif t == 0x0B:
                info["filters"] = _parse_filters(d)
            elif t == 0x0C:
                nm, val = self._parse_attribute(d)
                info["attrs"][nm] = val
        for k in ("shape", "dtype", "layout"):
            if k not in info:
                raise H5Error(f"{name}: object header without a {k} message")
        return info

    def attrs(self, name):
        return self._info(name)["attrs"]

    def shape(self, name):
        return self._info(name)["shape"]

    def read(self, name):
        info = self._info(name)
        shape, dt, lay = info["shape"], info["dtype"], info["layout"]
        count = int(np.prod(shape, dtype=object)) if shape else 1
        if count * dt.itemsize > 1 << 40:
            raise H5Error(f"{name}: dataspace {shape} of {dt} is beyond 1 TiB")
        if lay[0] == "compact":
            return np.frombuffer(lay[1], dtype=dt, count=count).reshape(shape).copy()
        if lay[0] == "contiguous":
            addr, size = lay[1], lay[2]
            if addr == UNDEF:
                return np.zeros(shape, dtype=dt)
            if size < count * dt.itemsize:
                raise H5Error(f"{name}: contiguous storage smaller than the dataspace")
            a = self._a(addr)
            self._check(a, count * dt.itemsize)
            return np.frombuffer(self._b[a:a + count * dt.itemsize], dtype=dt).reshape(shape).copy()
        return self._read_chunked(name, shape, dt, lay[1], lay[2], info["filters"])

    def _read_chunked(self, name, shape, dt, btree, cdims, filters):
        rank = len(shape)
        if len(cdims) != rank + 1 or cdims[-1] != dt.itemsize:
            raise H5Error(f"{name}: chunk dimensions {cdims} do not match the dataspace")
        cshape = tuple(cdims[:rank])
        out = np.zeros(shape, dtype=dt)
        cbytes = int(np.prod(cshape)) * dt.itemsize
        chunks = []
        for off, size, mask, addr in self._chunks(btree, rank):
            a = self._a(addr)
            self._check(a, size)
            if any(o >= s for o, s in zip(off, shape)):
                raise H5Error(f"{name}: chunk offset {off} outside the dataspace {shape}")
            chunks.append((off, a, size, mask))

        def decode(item):
            off, a, size, mask = item
            raw = _unfilter(bytes(self._b[a:a + size]), filters, mask, dt.itemsize)
            if len(raw) != cbytes:
                raise H5Error(f"{name}: chunk at {off} decodes to {len(raw)} bytes, expected {cbytes}")
            chunk = np.frombuffer(raw, dtype=dt).reshape(cshape)
            dst = tuple(slice(o, min(o + c, s)) for o, c, s in zip(off, cshape, shape))
            src = tuple(slice(0, d.stop - d.start) for d in dst)
            out[dst] = chunk[src]

        # filtered chunks decode on a pool of threads (zlib releases the GIL);
        # each writes its own part of out
        workers = min(len(chunks), os.cpu_count() or 1, 32) if filters else 1
        if workers > 1:
            with ThreadPoolExecutor(workers) as ex:
                list(ex.map(decode, chunks))
        else:
            for item in chunks:
                decode(item)
        return out

    def _chunks(self, btree, rank):
        ks = 8 + 8 * (rank + 1)
        stack, seen = [btree], set()
        while stack:
            addr = stack.pop()
            if addr in seen:
                raise H5Error("chunk B-tree revisits a node")
            seen.add(addr)
            a = self._a(addr)
            self._check(a, 24)
            if bytes(self._b[a:a + 4]) != b"TREE" or self._b[a + 4] != 1:
                raise H5Error("chunk B-tree node expected")
            level, used = self._b[a + 5], self._u(a + 6, 2)
            self._check(a + 24, used * (ks + 8) + ks)
            p = a + 24
            for i in range(used):
                size, mask = self._u(p, 4), self._u(p + 4, 4)
                off = tuple(self._u(p + 8 + 8 * d, 8) for d in range(rank))
                child = self._u(p + ks, 8)
                p += ks + 8
                if level > 0:
                    stack.append(child)
                else:
                    yield off, size, mask, child

    def _parse_attribute(self, d):
        ver = d[0]
        if ver == 1:
            nsz, tsz, ssz = struct.unpack_from("<HHH", d, 2)
            p = 8
            name = d[p:p + nsz].split(b"\0")[0].decode()
            p += _pad8(nsz)
            dt = _parse_datatype(d[p:p + tsz])[0]
            p += _pad8(tsz)
            shape = _parse_dataspace(d[p:p + ssz])[0]
            p += _pad8(ssz)
        elif ver in (2, 3):
            nsz, tsz, ssz = struct.unpack_from("<HHH", d, 2)
            p = 8 if ver == 2 else 9
            name = d[p:p + nsz].split(b"\0")[0].decode()
            p += nsz
            dt = _parse_datatype(d[p:p + tsz])[0]
            p += tsz
            shape = _parse_dataspace(d[p:p + ssz])[0]
            p += ssz
        else:
            raise H5Error(f"attribute message version {ver}")
        count = int(np.prod(shape)) if shape else 1
        val = np.frombuffer(d[p:p + count * dt.itemsize], dtype=dt, count=count)
        return name, (val[0] if count == 1 else val.reshape(shape).copy())


def _parse_dataspace(d):
    ver, rank, flags = d[0], d[1], d[2]
    if ver == 1:
        p = 8
    elif ver == 2:
        p = 4
        if d[3] == 2:       # null dataspace
            return (0,), None
    else:
        raise H5Error(f"dataspace version {ver}")
    dims = tuple(int.from_bytes(d[p + 8 * i:p + 8 * i + 8], "little") for i in range(rank))
    maxd = None
    if flags & 1:
        q = p + 8 * rank
        maxd = tuple(int.from_bytes(d[q + 8 * i:q + 8 * i + 8], "little") for i in range(rank))
    return dims, maxd


def _parse_datatype(d):
    """(numpy dtype, bytes used) of a datatype message."""
    cls, ver = d[0] & 0x0F, d[0] >> 4
    bits = d[1] | (d[2] << 8) | (d[3] << 16)
    size = int.from_bytes(d[4:8], "little")
    if ver not in (1, 2, 3):
        raise H5Error(f"datatype version {ver}")
    order = ">" if bits & 1 else "<"
    if cls == 0:
        kind = "i" if bits & 0x08 else "u"
        if size not in (1, 2, 4, 8):
            raise H5Error(f"fixed-point size {size}")
        return np.dtype(f"{order}{kind}{size}"), 12
    if cls == 1:
        if size not in (4, 8):
            raise H5Error(f"floating-point size {size}")
        return np.dtype(f"{order}f{size}"), 20
    if cls == 6:
        names, formats, offsets = [], [], []
        p = 8
        for _ in range(bits & 0xFFFF):
            end = d.index(b"\0", p)
            names.append(d[p:end].decode())
            p = p + _pad8(end - p + 1) if ver < 3 else end + 1
            if ver < 3:
                off, p = int.from_bytes(d[p:p + 4], "little"), p + 4
            else:
                w = 1 if size < 1 << 8 else 2 if size < 1 << 16 else 3 if size < 1 << 24 else 4
                off, p = int.from_bytes(d[p:p + w], "little"), p + w
            if ver == 1:
                if d[p] != 0:
                    raise H5Error("compound members with array dimensions are not read")
                p += 28
            sub, used = _parse_datatype(d[p:])
            p += used
            formats.append(sub)
            offsets.append(off)
        return np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": size}), p
    raise H5Error(f"datatype class {cls} is not read")


def _parse_layout(d):
    ver = d[0]
    if ver == 3:
        cls = d[1]
        if cls == 0:
            n = int.from_bytes(d[2:4], "little")
            return ("compact", d[4:4 + n])
        if cls == 1:
            return ("contiguous", int.from_bytes(d[2:10], "little"), int.from_bytes(d[10:18], "little"))
        if cls == 2:
            nd = d[2]
            addr = int.from_bytes(d[3:11], "little")
            dims = tuple(int.from_bytes(d[11 + 4 * i:15 + 4 * i], "little") for i in range(nd))
            return ("chunked", addr, dims)
        raise H5Error(f"layout class {cls}")
    if ver in (1, 2):
        nd, cls = d[1], d[2]
        p = 8
        addr = UNDEF
        if cls != 0:
            addr = int.from_bytes(d[p:p + 8], "little")
            p += 8
        dims = tuple(int.from_bytes(d[p + 4 * i:p + 4 * i + 4], "little") for i in range(nd))
        p += 4 * nd
        if cls == 0:
            n = int.from_bytes(d[p:p + 4], "little")
            return ("compact", d[p + 4:p + 4 + n])
        if cls == 1:
            return ("contiguous", addr, int(np.prod(dims)))
        return ("chunked", addr, dims)
    raise H5Error(f"layout version {ver}")


def _parse_filters(d):
    ver, n = d[0], d[1]
    p = 8 if ver == 1 else 2
    out = []
    for _ in range(n):
        fid = int.from_bytes(d[p:p + 2], "little")
        if ver == 1 or fid >= 256:
            nlen = int.from_bytes(d[p + 2:p + 4], "little")
            p += 4
        else:
            nlen = 0
            p += 2
        flags, ncd = struct.unpack_from("<HH", d, p)
        p += 4
        p += _pad8(nlen) if ver == 1 else nlen
        cd = struct.unpack_from(f"<{ncd}I", d, p)
        p += 4 * ncd
        if ver == 1 and ncd % 2:
            p += 4
        out.append((fid, flags, cd))
    return out


def _unfilter(raw, filters, mask, elem):
    for i in reversed(range(len(filters))):
        if mask & (1 << i):
            continue
        fid = filters[i][0]
        if fid == FILTER_DEFLATE:
            try:
                raw = zlib.decompress(raw)   # zlib stream; Adler-32 checked
            except zlib.error as e:
                raise H5Error(f"deflate stream: {e}") from None
        elif fid == FILTER_SHUFFLE:
            es = filters[i][2][0] if filters[i][2] else elem
            n = len(raw) // es
            body = np.frombuffer(raw[:n * es], dtype=np.uint8).reshape(es, n).T.reshape(-1)
            raw = body.tobytes() + raw[n * es:]
        elif fid == FILTER_FLETCHER32:
            raw = raw[:-4]
        else:
            raise H5Error(f"filter {fid} is not decoded")
    return raw


# ------------------------------------------------------------------ writing

def _datatype_bytes(dt):
    """Version-1 datatype message (unpadded) for a native numeric type, or a
    compound of them (class 6: per member the name padded to 8 bytes, the
    byte offset, the version-1 dimension fields, all zero, and the member's
    datatype)."""
    dt = np.dtype(dt)
    if dt.names is not None:
        body = b""
        for name in dt.names:
            sub, off = dt.fields[name][:2]
            if sub.names is not None or sub.shape:
                raise H5Error("nested or array compound members are not written")
            nm = name.encode() + b"\0"
            body += nm + b"\0" * (_pad8(len(nm)) - len(nm))
            body += struct.pack("<I", off) + b"\0" * 28 + _datatype_bytes(sub)
        n = len(dt.names)
        return bytes([0x16, n & 0xFF, n >> 8, 0]) + struct.pack("<I", dt.itemsize) + body
    if dt.byteorder == ">":
        raise H5Error("big-endian data is not written")
    if dt.kind in "iu":
        bits = 0x08 if dt.kind == "i" else 0x00
        return bytes([0x10, bits, 0, 0]) + struct.pack("<IHH", dt.itemsize, 0, 8 * dt.itemsize)
    if dt.kind == "f" and dt.itemsize == 8:
        return bytes([0x11, 0x20, 63, 0]) + struct.pack("<IHHBBBBI", 8, 0, 64, 52, 11, 0, 52, 1023)
    if dt.kind == "f" and dt.itemsize == 4:
        return bytes([0x11, 0x20, 31, 0]) + struct.pack("<IHHBBBBI", 4, 0, 32, 23, 8, 0, 23, 127)
    raise H5Error(f"dtype {dt} is not written")


def _dataspace_bytes(shape):
    """Version-1 simple dataspace with maximum dimensions equal to the dims."""
    rank = len(shape)
    return bytes([1, rank, 1, 0, 0, 0, 0, 0]) + struct.pack(f"<{2 * rank}Q", *shape, *shape)


def _msg(t, data, flags=0):
    data = data + b"\0" * (_pad8(len(data)) - len(data))
    return struct.pack("<HHB3x", t, len(data), flags) + data


def _attribute_msg(name, value):
    arr = np.asarray(value)
    if arr.ndim == 0:
        arr = arr.reshape(1)
    nm = name.encode() + b"\0"
    dtb = _datatype_bytes(arr.dtype)
    dsb = _dataspace_bytes(arr.shape)
    body = struct.pack("<BBHHH", 1, 0, len(nm), len(dtb), len(dsb))
    for part in (nm, dtb, dsb):
        body += part + b"\0" * (_pad8(len(part)) - len(part))
    body += np.ascontiguousarray(arr, dtype=arr.dtype.newbyteorder("<")).tobytes()
    return _msg(0x0C, body)


def _object_header(msgs):
    body = b"".join(msgs)
    return struct.pack("<BBHII4x", 1, 0, len(msgs), 1, len(body)) + body


class H5Writer:
    """Writes datasets with attributes under the root group of a new file.

    create_dataset(name, data, chunks=None, deflate=None, attrs=None):
      data    numpy array (native numeric dtype), any rank >= 1;
      chunks  chunk shape (tuple) for chunked storage, None for contiguous;
      deflate zlib level 0-9 on chunked storage (the HDF5 deflate filter);
      attrs   {name: scalar or array}; dtypes are kept (np.int32 for
              NATIVE_INT, np.uint32 for NATIVE_UINT, np.float64 for
              NATIVE_DOUBLE, ...), written in the given order.
    Data is streamed to the file as datasets are created; the metadata is
    written by close().
    """

    def __init__(self, path):
        self.path = os.fspath(path)
        self._f = open(self.path, "wb")
        self._f.write(b"\0" * 96)        # superblock, written last
        self._sets = []

    def _tell(self):
        return self._f.tell()

    def create_dataset(self, name, data, chunks=None, deflate=None, attrs=None):
        if any(s[0] == name for s in self._sets):
            raise H5Error(f"dataset {name} exists")
        if not name or "/" in name or "\0" in name:
            raise H5Error(f"dataset name {name!r}: datasets are written under the root group only")
        data = np.asarray(data)
        if data.ndim == 0:
            data = data.reshape(1)
        data = np.ascontiguousarray(data, dtype=data.dtype.newbyteorder("<"))
        shape = data.shape
        if chunks is None:
            addr = self._tell()
            self._f.write(memoryview(data).cast("B"))
            layout = ("contiguous", addr, data.nbytes)
        else:
            chunks = tuple(int(c) for c in chunks)
            if len(chunks) != data.ndim or min(chunks) < 1:
                raise H5Error("chunk shape must have the dataset's rank")
            entries = []
            grid = [range(0, s, c) for s, c in zip(shape, chunks)]
            offs = [tuple(g[i] for g, i in zip(grid, off)) for off in np.ndindex(*[len(g) for g in grid])]

            def encode(o):
                block = np.zeros(chunks, dtype=data.dtype)
                src = tuple(slice(a, min(a + c, s)) for a, c, s in zip(o, chunks, shape))
                block[tuple(slice(0, x.stop - x.start) for x in src)] = data[src]
                raw = block.tobytes()
                return zlib.compress(raw, int(deflate)) if deflate is not None else raw

            # zlib releases the GIL: deflated chunks are compressed on a pool
            # of threads, a window at a time, and written in chunk order (the
            # file's bytes do not depend on the number of threads)
            workers = min(len(offs), os.cpu_count() or 1, 32) if deflate is not None else 1
            if workers > 1:
                with ThreadPoolExecutor(workers) as ex:
                    for i in range(0, len(offs), 2 * workers):
                        window = offs[i:i + 2 * workers]
                        for o, raw in zip(window, ex.map(encode, window)):
                            entries.append((o, len(raw), self._tell()))
                            self._f.write(raw)
            else:
                for o in offs:
                    raw = encode(o)
                    entries.append((o, len(raw), self._tell()))
                    self._f.write(raw)
            layout = ("chunked", entries, chunks)
        self._sets.append((name, shape, data.dtype, layout, deflate, list((attrs or {}).items())))

    def _chunk_btree(self, entries, rank, elem):
        """Writes the chunk index bottom-up; returns the root address."""
        ks = 8 + 8 * (rank + 1)
        node_size = 24 + 2 * _CHUNK_K * 8 + (2 * _CHUNK_K + 1) * ks

        def key(size, off, last):
            return struct.pack(f"<II{rank + 1}Q", size, 0, *off, last)

        # level 0 items: (first key, final key, child address)
        items = [(key(sz, off, 0), key(0, off, elem), addr) for off, sz, addr in entries]
        level = 0
        while True:
            groups = [items[i:i + 2 * _CHUNK_K] for i in range(0, len(items), 2 * _CHUNK_K)]
            addrs = [self._tell() + g * node_size for g in range(len(groups))]
            nxt = []
            for gi, g in enumerate(groups):
                left = addrs[gi - 1] if gi > 0 else UNDEF
                right = addrs[gi + 1] if gi + 1 < len(groups) else UNDEF
                body = b"TREE" + struct.pack("<BBHQQ", 1, level, len(g), left, right)
                for first, _, child in g:
                    body += first + struct.pack("<Q", child)
                body += g[-1][1]
                body += b"\0" * (node_size - len(body))
                self._f.write(body)
                nxt.append((g[0][0], g[-1][1], addrs[gi]))
            if len(nxt) == 1:
                return nxt[0][2]
            items, level = nxt, level + 1

    def close(self):
        if self._f is None:
            return
        f = self._f
        ohdrs = {}
        for name, shape, dt, layout, deflate, attrs in self._sets:
            msgs = [_msg(0x01, _dataspace_bytes(shape)), _msg(0x03, _datatype_bytes(dt), flags=1)]
            if layout[0] == "contiguous":
                msgs.append(_msg(0x05, bytes([2, 2, 2, 1, 0, 0, 0, 0]), flags=1))
                lay = struct.pack("<BBQQ", 3, 1, layout[1], layout[2])
            else:
                msgs.append(_msg(0x05, bytes([2, 3, 2, 1, 0, 0, 0, 0]), flags=1))
                if deflate is not None:
                    pl = struct.pack("<BB6x", 1, 1) + struct.pack("<HHHH", FILTER_DEFLATE, 8, 1, 1) \
                        + b"deflate\0" + struct.pack("<I4x", int(deflate))
                    msgs.append(_msg(0x0B, pl, flags=1))
                root = self._chunk_btree(layout[1], len(shape), dt.itemsize)
                lay = struct.pack("<BBBQ", 3, 2, len(shape) + 1, root) + \
                    struct.pack(f"<{len(shape) + 1}I", *layout[2], dt.itemsize)
            msgs.append(_msg(0x08, lay))
            for an, av in attrs:
                msgs.append(_attribute_msg(an, av))
            ohdrs[name] = f.tell()
            f.write(_object_header(msgs))
        # local heap: "" then the names, each padded to 8 bytes
        names = sorted(ohdrs, key=lambda s: s.encode())
        heap_data = b"\0" * 8
        offs = {}
        for nm in names:
            offs[nm] = len(heap_data)
            e = nm.encode() + b"\0"
            heap_data += e + b"\0" * (_pad8(len(e)) - len(e))
        # symbol table nodes (2 * _LEAF_K entries each), group B-tree, heap, root header
        snod_size = 8 + 2 * _LEAF_K * 40
        groups = [names[i:i + 2 * _LEAF_K] for i in range(0, len(names), 2 * _LEAF_K)] or [[]]
        if len(groups) > 2 * _GROUP_K:
            raise H5Error("more datasets than one group B-tree node holds")
        snod_addr = []
        for g in groups:
            snod_addr.append(f.tell())
            body = b"SNOD" + struct.pack("<BBH", 1, 0, len(g))
            for nm in g:
                body += struct.pack("<QQII16x", offs[nm], ohdrs[nm], 0, 0)
            f.write(body + b"\0" * (snod_size - len(body)))
        btree = f.tell()
        node_size = 24 + 2 * _GROUP_K * 8 + (2 * _GROUP_K + 1) * 8
        body = b"TREE" + struct.pack("<BBHQQ", 0, 0, len(groups), UNDEF, UNDEF) + struct.pack("<Q", 0)
        for g, a in zip(groups, snod_addr):
            body += struct.pack("<QQ", a, offs[g[-1]] if g else 0)
        f.write(body + b"\0" * (node_size - len(body)))
        heap = f.tell()
        # free-list head 1: the HDF5 library's marker for "no free block"
        f.write(b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap_data), 1, heap + 32))
        f.write(heap_data)
        root = f.tell()
        f.write(_object_header([_msg(0x11, struct.pack("<QQ", btree, heap))]))
        eof = f.tell()
        sb = _SIG + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", _LEAF_K, _GROUP_K, 0)
        sb += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
        sb += struct.pack("<QQII", 0, root, 1, 0) + struct.pack("<QQ", btree, heap)
        f.seek(0)
        f.write(sb)
        f.close()
        self._f = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
