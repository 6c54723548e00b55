"""Reading FITS files: headers, image HDUs and binary tables.

forcepho reads its images, uncertainty maps and source catalogs with
``astropy.io.fits`` (forcepho/patches/pixel_patch.py:380-470,
forcepho/patches/storage.py:413-425, tests/cswap_test.py:27-28).  astropy is
not a dependency of this package; this module reads the parts of the FITS
standard (version 4.0) those files use: 2880-byte blocks of 80-character
header cards, primary and IMAGE extensions with BITPIX 8/16/32/64/-32/-64
(with BSCALE/BZERO), and BINTABLE extensions with scalar or fixed-repeat
columns of types L, B, I, J, K, E, D and A.  Data are big-endian in the file
and returned in native byte order; image arrays keep FITS axis order reversed
as numpy does (``NAXIS2`` rows of ``NAXIS1`` columns).
"""

import numpy as np

__all__ = ["Header", "read_hdus", "getdata", "getheader"]

_BLOCK = 2880


class Header(dict):
    """Header keywords in card order (a dict; values are parsed to bool,
    int, float or str).  ``Header.fromstring`` parses concatenated 80-character
    cards, the form ``astropy.io.fits.Header.tostring`` writes (and forcepho's
    MetaStore stores as JSON, forcepho/patches/storage.py:375-425)."""

    @classmethod
    def fromstring(cls, s):
        h = cls()
        if isinstance(s, bytes):
            s = s.decode("ascii")
        for i in range(0, len(s), 80):
            card = s[i:i + 80]
            key = card[:8].strip()
            if key == "END":
                break
            if not key or key in ("COMMENT", "HISTORY") or card[8:10] != "= ":
                continue
            h[key] = _parse_value(card[10:])
        return h

    def tostring(self):
        cards = []
        for k, v in self.items():
            if isinstance(v, bool):
                val = "T" if v else "F"
                cards.append(f"{k:<8}= {val:>20}")
            elif isinstance(v, (int, np.integer)):
                cards.append(f"{k:<8}= {int(v):>20d}")
            elif isinstance(v, (float, np.floating)):
                cards.append(f"{k:<8}= {_fmt_float(float(v)):>20}")
            else:
                sv = str(v).replace("'", "''")
                cards.append(f"{k:<8}= '{sv:<8}'")
        cards.append("END")
        return "".join(c[:80].ljust(80) for c in cards)


def _fmt_float(v):
    s = repr(v)
    if "e" in s:
        m, e = s.split("e")
        s = f"{m}E{e}"
    elif "." not in s and "inf" not in s and "nan" not in s:
        s += ".0"
    return s


def _parse_value(v):
    v = v.strip()
    if v.startswith("'"):
        out, i = [], 1
        while i < len(v):
            if v[i] == "'":
                if i + 1 < len(v) and v[i + 1] == "'":
                    out.append("'")
                    i += 2
                    continue
                break
            out.append(v[i])
            i += 1
        return "".join(out).rstrip()
    v = v.split("/")[0].strip()
    if v == "T":
        return True
    if v == "F":
        return False
    if v == "":
        return None
    try:
        return int(v)
    except ValueError:
        pass
    try:
        return float(v.replace("D", "E"))
    except ValueError:
        return v


_IMG = {8: ">u1", 16: ">i2", 32: ">i4", 64: ">i8", -32: ">f4", -64: ">f8"}
_COL = {"L": ("?", 1), "B": (">u1", 1), "I": (">i2", 2), "J": (">i4", 4), "K": (">i8", 8),
        "E": (">f4", 4), "D": (">f8", 8), "A": ("S", 1)}


def _read_header(b, off):
    cards = []
    while True:
        if off + _BLOCK > len(b):
            raise ValueError("truncated FITS header")
        blk = b[off:off + _BLOCK].decode("ascii")
        off += _BLOCK
        done = False
        for i in range(0, _BLOCK, 80):
            cards.append(blk[i:i + 80])
            if blk[i:i + 8].strip() == "END" and blk[i:i + 8].rstrip() == "END":
                done = True
                break
        if done:
            return Header.fromstring("".join(cards)), off


def _table(h, raw):
    nrow, rowlen, nf = h["NAXIS2"], h["NAXIS1"], h["TFIELDS"]
    names, formats, offsets, off = [], [], [], 0
    for i in range(1, nf + 1):
        form = str(h[f"TFORM{i}"]).strip()
        j = 0
        while j < len(form) and form[j].isdigit():
            j += 1
        rep = int(form[:j]) if j else 1
        code = form[j]
        if code not in _COL:
            raise NotImplementedError(f"BINTABLE column type {code!r}")
        base, size = _COL[code]
        if code == "A":
            fmt = f"S{rep}"
        else:
            fmt = base if rep == 1 else (base, (rep,))
        names.append(str(h.get(f"TTYPE{i}", f"col{i}")).strip())
        formats.append(fmt)
        offsets.append(off)
        off += rep * size
    dt = np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": rowlen})
    rec = np.frombuffer(raw, dtype=dt, count=nrow)
    out = np.zeros(nrow, dtype=[(n, np.dtype(f).newbyteorder("=") if not isinstance(f, tuple)
                                 else (np.dtype(f[0]).newbyteorder("="), f[1]))
                                for n, f in zip(names, formats)])
    for n in names:
        out[n] = rec[n]
    return out


def read_hdus(path):
    """[(Header, data)] of every HDU; data is an ndarray (image), a
    structured array (table) or None."""
    with open(path, "rb") as f:
        b = f.read()
    off, out = 0, []
    while off < len(b):
        if not b[off:off + 8].strip(b" \0"):
            break
        h, off = _read_header(b, off)
        bitpix, naxis = h["BITPIX"], h.get("NAXIS", 0)
        dims = [h[f"NAXIS{i}"] for i in range(1, naxis + 1)]
        n = int(np.prod(dims)) if naxis else 0
        nbytes = abs(bitpix) // 8 * h.get("GCOUNT", 1) * (h.get("PCOUNT", 0) + n)
        raw = b[off:off + nbytes]
        off += (nbytes + _BLOCK - 1) // _BLOCK * _BLOCK
        data = None
        if h.get("XTENSION", "").strip() == "BINTABLE":
            data = _table(h, raw)
        elif n:
            data = np.frombuffer(raw, dtype=_IMG[bitpix], count=n).reshape(dims[::-1])
            data = data.astype(data.dtype.newbyteorder("="))
            if "BSCALE" in h or "BZERO" in h:
                data = data * h.get("BSCALE", 1.0) + h.get("BZERO", 0.0)
        out.append((h, data))
    return out


def _select(hdus, ext):
    if isinstance(ext, int):
        return hdus[ext]
    for h, d in hdus:
        if str(h.get("EXTNAME", "")).strip().upper() == str(ext).upper():
            return h, d
    raise KeyError(f"no extension {ext!r}")


def getdata(path, ext=0):
    """Data of one HDU (by index, negative allowed, or EXTNAME)."""
    return _select(read_hdus(path), ext)[1]


def getheader(path, ext=0):
    return _select(read_hdus(path), ext)[0]
