"""Extract a Sersic mixture amplitude table from a forcepho spline-data file.

forcepho ships its Sersic Gaussian-mixture amplitude tables as HDF5 files
(``sersic_splinedata*.h5``: datasets ``nsersic``, ``rh``, ``amplitudes`` of
shape (n_grid, n_radii) and ``radii``), read by ``Galaxy.initialize_splines``
(forcepho/sources.py:623-645).  h5py is not available to this package, so this
script reads those four contiguous datasets with a minimal HDF5 reader (format
superblock version 0, object header version 1, symbol-table root group,
contiguous layout: the only features those files use) and writes
``sersic_splinedata_large.npz`` next to itself:

    ngrid (n_n,), rgrid (n_r,), amplitudes (n_n, n_r, n_radii), radii (n_radii,)

Usage: python -m forcepho_b200.data.make_sersic_table <path/to/sersic_splinedata_large.h5>
"""

import os
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "sersic_splinedata_large.npz")


def _read(f, off, n):
    f.seek(off)
    return f.read(n)


def _object_messages(f, addr):
    head = _read(f, addr, 16)
    version, _, nmsg, _, hsize = struct.unpack("<BBHII", head[:12])
    if version != 1:
        raise ValueError(f"object header version {version} not supported")
    blocks, msgs = [(addr + 16, hsize)], []
    while blocks:
        a, n = blocks.pop(0)
        b = _read(f, a, n)
        q = 0
        while q + 8 <= n:
            mtype, msize = struct.unpack("<HH", b[q:q + 4])
            data = b[q + 8:q + 8 + msize]
            q += 8 + msize
            msgs.append((mtype, data))
            if mtype == 0x10:  # continuation
                blocks.append(struct.unpack("<QQ", data[:16]))
    return msgs


def _dataset(f, addr):
    shape = dtype = layout = None
    for mtype, data in _object_messages(f, addr):
        if mtype == 0x1:  # dataspace
            nd = data[1]
            off = 8 if data[0] == 1 else 4
            shape = struct.unpack("<%dQ" % nd, data[off:off + 8 * nd])
        elif mtype == 0x3:  # datatype
            cls, bits = data[0] & 0xF, data[1]
            size = struct.unpack("<I", data[4:8])[0]
            order = ">" if bits & 1 else "<"
            if cls == 1:
                dtype = np.dtype(f"{order}f{size}")
            elif cls == 0:
                dtype = np.dtype(f"{order}{'i' if (bits >> 3) & 1 else 'u'}{size}")
            else:
                raise ValueError(f"datatype class {cls} not supported")
        elif mtype == 0x8:  # layout
            if data[0] != 3 or data[1] != 1:
                raise ValueError("only contiguous layout (version 3) is supported")
            layout = struct.unpack("<QQ", data[2:18])
    n = int(np.prod(shape)) if shape else 1
    raw = _read(f, layout[0], n * dtype.itemsize)
    return np.frombuffer(raw, dtype=dtype).reshape(shape).astype(dtype.newbyteorder("="))


def read_h5_datasets(path):
    """Return {name: ndarray} for the datasets of the root group."""
    with open(path, "rb") as f:
        sb = _read(f, 0, 128)
        if sb[:8] != b"\x89HDF\r\n\x1a\n":
            raise ValueError("not an HDF5 file")
        if sb[8] != 0 or sb[13] != 8 or sb[14] != 8:
            raise ValueError("only superblock version 0 with 8-byte offsets is supported")
        p = 24 + 32  # fixed fields + 4 addresses
        _, _, _, _ = struct.unpack("<QQII", sb[p:p + 24])
        btree, heap = struct.unpack("<QQ", sb[p + 24:p + 40])
        h = _read(f, heap, 32)
        hsize, _, haddr = struct.unpack("<QQQ", h[8:32])
        heapdata = _read(f, haddr, hsize)
        t = _read(f, btree, 8 + 16 + 16 * 64)
        if t[:4] != b"TREE" or t[5] != 0:
            raise ValueError("unexpected root group b-tree")
        used = struct.unpack("<H", t[6:8])[0]
        children = [struct.unpack("<Q", t[24 + 16 * i + 8:24 + 16 * i + 16])[0]
                    for i in range(used)]
        out = {}
        for c in children:
            s = _read(f, c, 8 + 40 * 64)
            if s[:4] != b"SNOD":
                raise ValueError("unexpected symbol node")
            for i in range(struct.unpack("<H", s[6:8])[0]):
                lno, oh = struct.unpack("<QQ", s[8 + 40 * i:24 + 40 * i])
                name = heapdata[lno:heapdata.index(b"\0", lno)].decode()
                out[name] = _dataset(f, oh)
    return out


def table_from_h5(path):
    d = read_h5_datasets(path)
    n, r, A = d["nsersic"].astype(np.float64), d["rh"].astype(np.float64), d["amplitudes"]
    ngrid, rgrid = np.unique(n), np.unique(r)
    # forcepho reshapes amplitudes[:, i] to (n_n, n_r) (sources.py:637-640)
    amps = np.stack([A[:, i].reshape(len(ngrid), len(rgrid)) for i in range(A.shape[1])], -1)
    return dict(ngrid=ngrid, rgrid=rgrid, amplitudes=amps, radii=d["radii"].astype(np.float64))


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else None
    if not src:
        sys.exit(__doc__)
    tab = table_from_h5(src)
    np.savez_compressed(OUT, **tab)
    print(OUT, {k: v.shape for k, v in tab.items()})
