"""A small reader and writer for the subset of HDF5 that forcepho's stores use.

forcepho keeps pixel data, PSF mixtures and Sersic amplitude tables in HDF5
files written by h5py with its default ("earliest") format
(forcepho/patches/storage.py:62-300, 525-578; forcepho/sources.py:623-645).
h5py is not a dependency of this package, so this module reads and writes
those files directly, following the published HDF5 File Format Specification
(version 2.0 structures that "earliest" files use):

* superblock version 0, 8-byte offsets and lengths;
* groups as symbol tables: a version-1 B-tree of group nodes whose leaves are
  symbol-table nodes (``SNOD``), names in a local heap (``HEAP``);
* object headers version 1 (with continuation blocks);
* datasets with contiguous or compact layout (layout message version 3);
* datatypes: fixed-point integers, IEEE floats, fixed-length strings,
  variable-length strings (global heap, read only), compound types and array
  members (what ``PSFStore`` parameter tables hold);
* attributes (message version 1, 2 or 3) of those types.

Chunked or compressed datasets, dense attribute storage and the "latest"
link-message groups are not supported; opening such an object raises
``NotImplementedError``.  The reader is checked on forcepho's own data files
(Sersic tables, PSF store); the writer follows the same structures and is
checked by round trips through the reader, not against libhdf5, which is not
available here.  Contiguous datasets are returned as read-only
``numpy.memmap`` views, so slicing a large pixel store reads only what is
used.
"""

import os
import struct

import numpy as np

__all__ = ["File", "Group", "Dataset", "write"]

_SIG = b"\x89HDF\r\n\x1a\n"
_UNDEF = 0xFFFFFFFFFFFFFFFF


# ------------------------------------------------------------------ reading
class _Reader:
    def __init__(self, path):
        self.path = path
        self.f = open(path, "rb")
        sb = self.read(0, 96)
        if sb[:8] != _SIG:
            raise ValueError(f"{path}: not an HDF5 file")
        if sb[8] != 0:
            raise NotImplementedError(f"{path}: superblock version {sb[8]} (only 0)")
        if sb[13] != 8 or sb[14] != 8:
            raise NotImplementedError(f"{path}: offsets/lengths of {sb[13]}/{sb[14]} bytes")
        self.root_addr = struct.unpack("<Q", sb[64:72])[0]

    def read(self, off, n):
        self.f.seek(off)
        b = self.f.read(n)
        if len(b) != n:
            raise ValueError(f"{self.path}: truncated file (read {n} bytes at {off})")
        return b

    def close(self):
        self.f.close()

    # -- object headers
    def messages(self, addr):
        head = self.read(addr, 16)
        version, _, _, _, hsize = struct.unpack("<BBHII", head[:12])
        if version != 1:
            raise NotImplementedError(f"object header version {version} (only 1)")
        blocks, out = [(addr + 16, hsize)], []
        while blocks:
            a, n = blocks.pop(0)
            b = self.read(a, n)
            q = 0
            while q + 8 <= n:
                mtype, msize = struct.unpack("<HH", b[q:q + 4])
                out.append((mtype, b[q + 8:q + 8 + msize]))
                if mtype == 0x10:
                    blocks.append(struct.unpack("<QQ", b[q + 8:q + 24]))
                q += 8 + msize
        return out

    # -- groups
    def group_entries(self, addr):
        """{name: object header address} of the group whose header is at addr."""
        btree = heap = None
        for mtype, data in self.messages(addr):
            if mtype == 0x11:
                btree, heap = struct.unpack("<QQ", data[:16])
            elif mtype in (0x02, 0x06, 0x0A):
                raise NotImplementedError("link-message (new-style) groups are not supported")
        if btree is None:
            raise ValueError("object is not a group")
        h = self.read(heap, 32)
        if h[:4] != b"HEAP":
            raise ValueError("bad local heap")
        hsize, _, haddr = struct.unpack("<QQQ", h[8:32])
        names = self.read(haddr, hsize)
        out = {}
        self._walk_btree(btree, names, out)
        return out

    def _walk_btree(self, addr, names, out):
        t = self.read(addr, 24)
        if t[:4] != b"TREE" or t[4] != 0:
            raise ValueError("bad group B-tree node")
        level, used = t[5], struct.unpack("<H", t[6:8])[0]
        body = self.read(addr + 24, 8 + 16 * used)
        for i in range(used):
            child = struct.unpack("<Q", body[8 + 16 * i:16 + 16 * i])[0]
            if level > 0:
                self._walk_btree(child, names, out)
            else:
                self._read_snod(child, names, out)

    def _read_snod(self, addr, names, out):
        s = self.read(addr, 8)
        if s[:4] != b"SNOD":
            raise ValueError("bad symbol table node")
        n = struct.unpack("<H", s[6:8])[0]
        ents = self.read(addr + 8, 40 * n)
        for i in range(n):
            lno, oh = struct.unpack("<QQ", ents[40 * i:40 * i + 16])
            out[names[lno:names.index(b"\0", lno)].decode()] = oh

    def is_group(self, addr):
        return any(m == 0x11 for m, _ in self.messages(addr))

    # -- global heap (variable-length strings)
    def global_object(self, coll, index):
        h = self.read(coll, 16)
        if h[:4] != b"GCOL":
            raise ValueError("bad global heap collection")
        size = struct.unpack("<Q", h[8:16])[0]
        b = self.read(coll, size)
        q = 16
        while q + 16 <= size:
            idx, _, _, osize = struct.unpack("<HHIQ", b[q:q + 16])
            if idx == 0:
                break
            if idx == index:
                return b[q + 16:q + 16 + osize]
            q += 16 + ((osize + 7) & ~7)
        raise ValueError("global heap object not found")


def _parse_dataspace(data):
    version, nd, flags = data[0], data[1], data[2]
    if version == 1:
        off = 8
    elif version == 2:
        if data[3] == 0:     # scalar
            return ()
        if data[3] == 2:     # null
            return None
        off = 4
    else:
        raise NotImplementedError(f"dataspace version {version}")
    return tuple(struct.unpack("<%dQ" % nd, data[off:off + 8 * nd]))


def _parse_datatype(data):
    """(numpy dtype, bytes consumed, kind) for a datatype message; kind is
    'vlen_str' for variable-length strings, else None."""
    cls, version = data[0] & 0x0F, data[0] >> 4
    bits = data[1] | (data[2] << 8) | (data[3] << 16)
    size = struct.unpack("<I", data[4:8])[0]
    order = ">" if bits & 1 else "<"
    if cls == 0:
        props = 4
        return np.dtype(f"{order}{'i' if bits & 8 else 'u'}{size}"), 8 + props, None
    if cls == 1:
        return np.dtype(f"{order}f{size}"), 8 + 12, None
    if cls == 3:
        return np.dtype(f"S{size}"), 8, None
    if cls == 6:
        nmem = bits & 0xFFFF
        q, fields = 8, []
        for _ in range(nmem):
            end = data.index(b"\0", q)
            name = data[q:end].decode()
            if version < 3:
                q = q + ((end - q + 1 + 7) & ~7)
                off = struct.unpack("<I", data[q:q + 4])[0]
                q += 4
                if version == 1:
                    nd = data[q]
                    dims = struct.unpack("<4I", data[q + 12:q + 28])[:nd]
                    q += 28
                else:
                    dims = ()
            else:
                q = end + 1
                nb = 1 if size < 256 else 2 if size < 65536 else 4 if size < 2 ** 32 else 8
                off = int.from_bytes(data[q:q + nb], "little")
                q += nb
                dims = ()
            mdt, used, _ = _parse_datatype(data[q:])
            q += used
            if dims:
                mdt = np.dtype((mdt, dims))
            fields.append((name, mdt, off))
        dt = np.dtype({"names": [f[0] for f in fields], "formats": [f[1] for f in fields],
                       "offsets": [f[2] for f in fields], "itemsize": size})
        return dt, q, None
    if cls == 9:
        base, used, _ = _parse_datatype(data[8:])
        if (bits & 0xF) == 1:   # string
            return np.dtype(object), 8 + used, "vlen_str"
        raise NotImplementedError("variable-length sequences are not supported")
    if cls == 10:
        nd = data[8]
        if version == 2:
            dims = struct.unpack("<%dI" % nd, data[12:12 + 4 * nd])
            q = 12 + 8 * nd
        else:
            dims = struct.unpack("<%dI" % nd, data[9:9 + 4 * nd])
            q = 9 + 4 * nd
        base, used, _ = _parse_datatype(data[q:])
        return np.dtype((base, tuple(dims))), q + used, None
    raise NotImplementedError(f"datatype class {cls}")


def _decode(r, raw, dtype, kind, shape):
    if kind == "vlen_str":
        n = int(np.prod(shape)) if shape else 1
        out = []
        for i in range(n):
            ln, coll, idx = struct.unpack("<IQI", raw[16 * i:16 * i + 16])
            out.append(r.global_object(coll, idx)[:ln].decode() if ln else "")
        return out[0] if not shape else np.array(out, dtype=object).reshape(shape)
    a = np.frombuffer(raw, dtype=dtype, count=int(np.prod(shape)) if shape else 1)
    a = a.reshape(shape) if shape else a[0]
    if isinstance(a, np.ndarray) and a.dtype.names is None and a.dtype.byteorder == ">":
        a = a.astype(a.dtype.newbyteorder("="))
    if isinstance(a, bytes):
        return a.rstrip(b"\0").decode()
    return a


def _parse_attribute(r, data):
    version = data[0]
    nsize, tsize, ssize = struct.unpack("<HHH", data[2:8])
    q = 8 if version < 3 else 9
    pad = (lambda n: (n + 7) & ~7) if version == 1 else (lambda n: n)
    name = data[q:q + nsize].rstrip(b"\0").decode()
    q += pad(nsize)
    dtype, _, kind = _parse_datatype(data[q:q + tsize])
    q += pad(tsize)
    shape = _parse_dataspace(data[q:q + ssize])
    q += pad(ssize)
    if shape is None:
        return name, None
    n = int(np.prod(shape)) if shape else 1
    nbytes = n * (16 if kind == "vlen_str" else dtype.itemsize)
    return name, _decode(r, data[q:q + nbytes], dtype, kind, shape)


class _Node:
    def __init__(self, r, addr, name):
        self._r, self._addr, self.name = r, addr, name
        self._attrs = None

    @property
    def attrs(self):
        if self._attrs is None:
            self._attrs = {}
            for mtype, data in self._r.messages(self._addr):
                if mtype == 0x0C:
                    k, v = _parse_attribute(self._r, data)
                    self._attrs[k] = v
                elif mtype == 0x15:
                    raise NotImplementedError("dense attribute storage is not supported")
        return self._attrs


class Dataset(_Node):
    """A dataset: ``shape``, ``dtype``, ``attrs``; index it (``ds[...]``,
    ``ds[:]``) to read."""

    def __init__(self, r, addr, name):
        super().__init__(r, addr, name)
        self.shape, self.dtype, self._kind, self._layout = (), None, None, None
        for mtype, data in r.messages(addr):
            if mtype == 0x01:
                self.shape = _parse_dataspace(data)
            elif mtype == 0x03:
                self.dtype, _, self._kind = _parse_datatype(data)
            elif mtype == 0x08:
                if data[0] != 3:
                    raise NotImplementedError(f"layout message version {data[0]}")
                if data[1] == 1:
                    self._layout = ("contiguous",) + struct.unpack("<QQ", data[2:18])
                elif data[1] == 0:
                    n = struct.unpack("<H", data[2:4])[0]
                    self._layout = ("compact", bytes(data[4:4 + n]))
                else:
                    raise NotImplementedError("chunked datasets are not supported")

    @property
    def size(self):
        return int(np.prod(self.shape)) if self.shape else 1

    def array(self):
        """The whole dataset: a read-only ``numpy.memmap`` when it is stored
        contiguously (nothing is read until indexed), else an ndarray."""
        if self._kind == "vlen_str":
            raw = self._read_raw(16 * self.size)
            return _decode(self._r, raw, self.dtype, self._kind, self.shape)
        if self._layout[0] == "contiguous" and self._layout[1] != _UNDEF and self.size > 0:
            return np.memmap(self._r.path, dtype=self.dtype, mode="r", offset=self._layout[1],
                             shape=self.shape if self.shape else (1,))
        raw = self._read_raw(self.size * self.dtype.itemsize)
        a = np.frombuffer(raw, dtype=self.dtype, count=self.size)
        return a.reshape(self.shape) if self.shape else a

    def _read_raw(self, n):
        if self._layout[0] == "compact":
            return self._layout[1][:n]
        if self._layout[1] == _UNDEF:
            return bytes(n)
        return self._r.read(self._layout[1], n)

    def __getitem__(self, key):
        a = self.array()
        if not self.shape and key in ((), Ellipsis, slice(None)):
            return a[0]
        out = a[key]
        return np.array(out) if isinstance(out, np.ndarray) else out

    def __len__(self):
        return self.shape[0]


class Group(_Node):
    """A group: mapping of names to groups and datasets; ``"a/b"`` paths work."""

    def __init__(self, r, addr, name):
        super().__init__(r, addr, name)
        self._entries = None

    def _ents(self):
        if self._entries is None:
            self._entries = self._r.group_entries(self._addr)
        return self._entries

    def keys(self):
        return list(self._ents().keys())

    def __iter__(self):
        return iter(self.keys())

    def __contains__(self, path):
        try:
            self[path]
            return True
        except KeyError:
            return False

    def items(self):
        return [(k, self[k]) for k in self.keys()]

    def __getitem__(self, path):
        node = self
        for part in [p for p in path.split("/") if p]:
            if not isinstance(node, Group):
                raise KeyError(path)
            ents = node._ents()
            if part not in ents:
                raise KeyError(path)
            addr = ents[part]
            full = (node.name.rstrip("/") + "/" + part)
            node = (Group(self._r, addr, full) if self._r.is_group(addr)
                    else Dataset(self._r, addr, full))
        return node


class File(Group):
    """Open an HDF5 file for reading: ``File(path)["band/exp/data"][:]``."""

    def __init__(self, path, mode="r"):
        if mode != "r":
            raise ValueError("h5lite.File is read-only; use h5lite.write")
        r = _Reader(path)
        super().__init__(r, r.root_addr, "/")

    def close(self):
        self._r.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def read_tree(path, memmap=False):
    """{path: array} of every dataset and {path: attrs} of every object.
    With `memmap`, contiguous datasets come back as read-only memory maps
    (nothing is read until used)."""
    data, attrs = {}, {}
    with File(path) as f:
        def walk(g, prefix):
            attrs[prefix or "/"] = dict(g.attrs)
            for k in g.keys():
                node = g[k]
                p = f"{prefix}/{k}" if prefix else k
                if isinstance(node, Group):
                    walk(node, p)
                else:
                    if not node.shape:
                        data[p] = node[...]
                    elif memmap:
                        data[p] = node.array()
                    else:
                        data[p] = np.array(node[:])
                    attrs[p] = dict(node.attrs)
        walk(f, "")
    return data, attrs


# ------------------------------------------------------------------ writing
_LEAF_K, _NODE_K = 4, 16


def _dt_message(dt):
    """Datatype message bytes for a numpy dtype (not padded: member types of
    a compound follow one another unpadded)."""
    dt = np.dtype(dt)
    if dt.subdtype is not None:
        base, dims = dt.subdtype
        body = struct.pack("<B3x", len(dims)) + struct.pack("<%dI" % len(dims), *dims)
        body += struct.pack("<%dI" % len(dims), *range(len(dims)))
        return (struct.pack("<B3sI", 0x2A, b"\0\0\0", dt.itemsize) + body
                + _dt_message(base))
    if dt.names is not None:
        body = b""
        for name in dt.names:
            mdt, off = dt.fields[name][:2]
            nm = name.encode() + b"\0"
            body += nm + b"\0" * (((len(nm) + 7) & ~7) - len(nm)) + struct.pack("<I", off)
            body += _dt_message(mdt)
        n = len(dt.names)
        return (struct.pack("<B", 0x26) + struct.pack("<I", n)[:3]
                + struct.pack("<I", dt.itemsize) + body)
    if dt.kind in "iu":
        bits = 8 if dt.kind == "i" else 0
        if dt.byteorder == ">":
            bits |= 1
        return struct.pack("<BBBBIHH", 0x10, bits, 0, 0, dt.itemsize, 0, 8 * dt.itemsize)
    if dt.kind == "f":
        bits = 0x20 if dt.byteorder != ">" else 0x21
        if dt.itemsize == 4:
            props = struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
        elif dt.itemsize == 8:
            props = struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
        else:
            raise NotImplementedError(f"float of {dt.itemsize} bytes")
        return (struct.pack("<BBBBI", 0x11, bits, 0x1F if dt.itemsize == 4 else 0x3F, 0,
                            dt.itemsize) + props)
    if dt.kind == "S":
        return struct.pack("<BBBBI", 0x13, 0, 0, 0, dt.itemsize)
    raise NotImplementedError(f"dtype {dt} cannot be written")


def _pad(b):
    return b + b"\0" * ((-len(b)) % 8)


def _space_message(shape):
    if shape == ():
        return struct.pack("<BBBB4x", 1, 0, 0, 0)
    return struct.pack("<BBBB4x", 1, len(shape), 0, 0) + struct.pack("<%dQ" % len(shape), *shape)


def _attr_value(v):
    if isinstance(v, str):
        v = np.bytes_(v.encode())
    if isinstance(v, bytes):
        v = np.bytes_(v)
    a = np.asarray(v)
    if a.dtype.kind == "U":
        a = a.astype("S")
    if a.dtype.kind == "b":
        a = a.astype(np.uint8)
    if a.dtype.kind == "S" and a.dtype.itemsize == 0:
        a = a.astype("S1")
    return a if a.flags.c_contiguous else a.copy()


def _attr_message(name, value):
    a = _attr_value(value)
    nm = name.encode() + b"\0"
    t, s = _dt_message(a.dtype), _space_message(a.shape)
    head = struct.pack("<BBHHH", 1, 0, len(nm), len(t), len(s))
    return _pad(head + _pad(nm) + _pad(t) + _pad(s) + a.tobytes())


class _Out:
    """The file being laid out: structures are kept as (address, bytes);
    dataset contents as (address, array) and streamed to the file at the
    end, so writing a large store needs memory for its structures only."""

    def __init__(self):
        self.end = 96                 # the superblock comes first
        self.chunks = {}
        self.raw = []

    def alloc(self, n, align=8):
        self.end += (-self.end) % align
        addr = self.end
        self.end += n
        return addr

    def put(self, addr, b):
        self.chunks[addr] = bytes(b)

    def put_array(self, addr, a):
        self.raw.append((addr, a))

    def get(self, addr, n):
        return self.chunks[addr][:n]

    def save(self, f, block=1 << 26):
        f.truncate(self.end)
        for addr, b in self.chunks.items():
            f.seek(addr)
            f.write(b)
        for addr, a in self.raw:
            flat = a.reshape(-1)
            step = max(1, block // max(a.itemsize, 1))
            f.seek(addr)
            for i in range(0, flat.size, step):
                f.write(np.ascontiguousarray(flat[i:i + step]).tobytes())


def _header(out, msgs):
    body, n = b"", len(msgs)
    for mtype, data in msgs:
        data = _pad(data)
        body += struct.pack("<HHB3x", mtype, len(data), 0) + data
    if len(body) < 24:   # pad small headers with a NIL message
        body += struct.pack("<HHB3x", 0, 16 - len(body), 0) + b"\0" * (16 - len(body))
        n += 1
    addr = out.alloc(16 + len(body))
    out.put(addr, struct.pack("<BBHII4x", 1, 0, n, 1, len(body)) + body)
    return addr


def _write_group(out, tree):
    """tree: {"attrs": {}, "children": {name: tree-or-dataset}}; returns the
    address of the group's object header."""
    names = sorted(tree["children"])
    child_addr = {}
    for n in names:
        c = tree["children"][n]
        child_addr[n] = _write_group(out, c) if "children" in c else _write_dataset(out, c)
    # local heap: "" at 0, then the names
    heap = bytearray(b"\0" * 8)
    offs = {}
    for n in names:
        offs[n] = len(heap)
        heap += _pad(n.encode() + b"\0")
    heap += b"\0" * max(16, (-len(heap)) % 8)     # a free block, as libraries leave one
    free_off = len(heap) - 16
    heap[free_off:free_off + 16] = struct.pack("<QQ", 1, 16)
    hdata = out.alloc(len(heap))
    out.put(hdata, bytes(heap))
    hhead = out.alloc(32)
    out.put(hhead, b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap), free_off, hdata))
    # symbol nodes of at most 2*LEAF_K entries each, under B-tree nodes
    per = 2 * _LEAF_K
    snods = []
    for i in range(0, max(len(names), 1), per):
        chunk = names[i:i + per]
        addr = out.alloc(8 + 40 * per)
        b = b"SNOD" + struct.pack("<BBH", 1, 0, len(chunk))
        for n in chunk:
            b += struct.pack("<QQII16x", offs[n], child_addr[n], 0, 0)
        out.put(addr, b)
        snods.append((addr, offs[chunk[-1]] if chunk else 0))
    btree = _write_btree(out, snods, level=0)
    msgs = [(0x11, struct.pack("<QQ", btree, hhead))]
    msgs += [(0x0C, _attr_message(k, v)) for k, v in tree["attrs"].items()]
    return _header(out, msgs)


def _write_btree(out, children, level):
    """children: [(address, key)] with key = heap offset of the child's last
    name; builds as many levels as needed (2*NODE_K children per node)."""
    per = 2 * _NODE_K
    nodes = []
    for i in range(0, len(children), per):
        chunk = children[i:i + per]
        size = 24 + 8 * (2 * _NODE_K + 1) + 8 * 2 * _NODE_K
        addr = out.alloc(size)
        b = b"TREE" + struct.pack("<BBHQQ", 0, level, len(chunk), _UNDEF, _UNDEF)
        b += struct.pack("<Q", 0)
        for a, key in chunk:
            b += struct.pack("<QQ", a, key)
        out.put(addr, b)
        nodes.append((addr, chunk[-1][1]))
    if len(nodes) == 1:
        return nodes[0][0]
    return _write_btree(out, nodes, level + 1)


def _write_dataset(out, ds):
    a = np.asarray(ds["data"])
    a = a if a.flags.c_contiguous else a.copy()    # (ascontiguousarray makes 0-d 1-d)
    if a.dtype.byteorder == ">":
        a = a.astype(a.dtype.newbyteorder("<"))
    raw = out.alloc(a.nbytes)
    out.put_array(raw, a)
    msgs = [(0x01, _space_message(a.shape)),
            (0x03, _dt_message(a.dtype)),
            (0x05, struct.pack("<BBBB", 2, 2, 2, 0)),   # fill value: never written
            (0x08, struct.pack("<BBQQ", 3, 1, raw, a.nbytes))]
    msgs += [(0x0C, _attr_message(k, v)) for k, v in ds["attrs"].items()]
    return _header(out, msgs)


def write(path, datasets, attrs=None):
    """Write a new HDF5 file.

    Parameters
    ----------
    datasets : {path: ndarray}, e.g. ``{"F200W/exp1/data": a}``; intermediate
        groups are created.
    attrs : {path: {name: value}}; ``"/"`` is the root group.  Values are
        numbers, numpy arrays or strings (stored as fixed-length strings).
    """
    attrs = attrs or {}
    root = {"attrs": dict(attrs.get("/", {})), "children": {}}

    def group(p):
        g = root
        for part in [x for x in p.split("/") if x]:
            g = g["children"].setdefault(part, {"attrs": {}, "children": {}})
        return g

    for p, a in datasets.items():
        parent, _, leaf = p.strip("/").rpartition("/")
        group(parent)["children"][leaf] = {"data": np.asarray(a),
                                           "attrs": dict(attrs.get(p, {}))}
    for p, av in attrs.items():
        if p != "/" and p not in datasets:
            group(p)["attrs"].update(av)

    out = _Out()
    root_addr = _write_group(out, root)
    sb = _SIG + struct.pack("<BBBBBBBBHHI", 0, 0, 0, 0, 0, 8, 8, 0, _LEAF_K, _NODE_K, 0)
    sb += struct.pack("<QQQQ", 0, _UNDEF, out.end, _UNDEF)
    # root symbol table entry, caching the root's B-tree and heap
    msgs = dict(_messages_in_header(out, root_addr))
    btree, heap = struct.unpack("<QQ", msgs[0x11][:16])
    sb += struct.pack("<QQII", 0, root_addr, 1, 0) + struct.pack("<QQ", btree, heap)
    out.put(0, sb)
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        out.save(f)
    os.replace(tmp, path)


def _messages_in_header(out, addr):
    b = out.chunks[addr]
    version, _, n, _, hsize = struct.unpack("<BBHII", b[:12])
    q, end, msgs = 16, 16 + hsize, []
    while q + 8 <= end:
        mtype, msize = struct.unpack("<HH", b[q:q + 4])
        msgs.append((mtype, b[q + 8:q + 8 + msize]))
        q += 8 + msize
    return msgs
