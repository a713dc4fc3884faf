"""A minimal FITS reader: headers, images and binary tables.

The reference reads its exposures with ``astropy.io.fits``
(forcepho/patches/pixel_patch.py:379-486: ``fits.getheader``, ``fits.getdata``
of the science and uncertainty extensions, and the source catalog table of
the last extension, tests/cswap_test.py:30-31).  astropy is not installed
here, so this module reads what those calls read, from the FITS standard
(version 4.0): 2880-byte records of 80-character header cards, then the data
unit, big-endian.

* images: BITPIX 8, 16, 32, 64, -32, -64, with BSCALE/BZERO applied when
  present (as astropy does); the array has numpy axis order (NAXISn ...
  NAXIS1);
* binary tables (XTENSION = 'BINTABLE'): fields of TFORM L, B, I, J, K, E, D
  and A with repeat counts, returned as a numpy structured array with native
  byte order.
"""

import numpy as np

__all__ = ["HDU", "read_fits", "getheader", "getdata", "write_fits"]

BLOCK = 2880
CARD = 80

_BITPIX = {8: ">u1", 16: ">i2", 32: ">i4", 64: ">i8", -32: ">f4", -64: ">f8"}
_TFORM = {"L": "?", "B": "u1", "I": ">i2", "J": ">i4", "K": ">i8", "E": ">f4", "D": ">f8", "A": "S"}


def _value(text):
    """Value of a header card's value field (string, bool, int or float)."""
    t = text.strip()
    if t.startswith("'"):
        # quoted string: '' is an escaped quote; trailing blanks are insignificant
        out, i = [], 1
        while i < len(t):
            if t[i] == "'":
                if i + 1 < len(t) and t[i + 1] == "'":
                    out.append("'")
                    i += 2
                    continue
                break
            out.append(t[i])
            i += 1
        return "".join(out).rstrip()
    v = t.split("/", 1)[0].strip()
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


class HDU:
    """One header-data unit: ``header`` (dict, keys in card order) and ``data``
    (numpy array, structured array for tables, or None)."""

    def __init__(self, header, data):
        self.header = header
        self.data = data

    def __repr__(self):
        kind = self.header.get("XTENSION", "PRIMARY")
        shape = None if self.data is None else self.data.shape
        return "HDU(%s, %s)" % (kind, shape)


def _read_header(buf, pos):
    header = {}
    while True:
        if pos + BLOCK > len(buf):
            raise ValueError("truncated FITS header")
        block = buf[pos:pos + BLOCK].decode("ascii", errors="replace")
        pos += BLOCK
        end = False
        for j in range(0, BLOCK, CARD):
            card = block[j:j + CARD]
            key = card[:8].strip()
            if key == "END":
                end = True
                break
            if card[8:10] == "= " and key:
                header[key] = _value(card[10:])
        if end:
            return header, pos


def _data_size(h):
    naxis = int(h.get("NAXIS", 0))
    if naxis == 0:
        return 0
    n = 1
    for a in range(1, naxis + 1):
        n *= int(h["NAXIS%d" % a])
    # |BITPIX| / 8 x GCOUNT x (PCOUNT + NAXIS1 x ... x NAXISn)
    return abs(int(h["BITPIX"])) // 8 * int(h.get("GCOUNT", 1)) * (int(h.get("PCOUNT", 0)) + n)


def _table(h, raw):
    nrow = int(h["NAXIS2"])
    fields = []
    for k in range(1, int(h["TFIELDS"]) + 1):
        form = str(h["TFORM%d" % k]).strip()
        i = 0
        while i < len(form) and form[i].isdigit():
            i += 1
        rep = int(form[:i]) if i else 1
        code = form[i]
        if code not in _TFORM:
            raise ValueError("unsupported TFORM %r" % form)
        name = str(h.get("TTYPE%d" % k, "col%d" % k)).strip()
        if code == "A":
            fields.append((name, "S%d" % rep))
        elif rep == 1:
            fields.append((name, _TFORM[code]))
        else:
            fields.append((name, _TFORM[code], (rep,)))
    dt = np.dtype(fields)
    if dt.itemsize != int(h["NAXIS1"]):
        raise ValueError("table row of %d bytes, NAXIS1 says %d" % (dt.itemsize, int(h["NAXIS1"])))
    arr = np.frombuffer(raw, dtype=dt, count=nrow)
    return arr.astype(dt.newbyteorder("="))


def read_fits(path):
    """Every HDU of a FITS file, in order."""
    with open(path, "rb") as f:
        buf = f.read()
    hdus, pos = [], 0
    while pos + BLOCK <= len(buf):
        if not buf[pos:pos + 8].strip(b" \0"):
            break                                   # trailing padding
        header, pos = _read_header(buf, pos)
        size = _data_size(header)
        raw = buf[pos:pos + size]
        pos += (size + BLOCK - 1) // BLOCK * BLOCK
        data = None
        if header.get("XTENSION") == "BINTABLE":
            data = _table(header, raw)
        elif int(header.get("NAXIS", 0)) > 0:
            naxis = int(header["NAXIS"])
            shape = tuple(int(header["NAXIS%d" % a]) for a in range(naxis, 0, -1))
            data = np.frombuffer(raw, dtype=_BITPIX[int(header["BITPIX"])],
                                 count=int(np.prod(shape))).reshape(shape)
            scale, zero = header.get("BSCALE", 1), header.get("BZERO", 0)
            if scale != 1 or zero != 0:
                data = data * scale + zero
            else:
                data = data.astype(data.dtype.newbyteorder("="))
        hdus.append(HDU(header, data))
    return hdus


def getheader(path, ext=0):
    return read_fits(path)[ext].header


def getdata(path, ext=0):
    return read_fits(path)[ext].data


def _card(key, value):
    if isinstance(value, bool):
        v = ("T" if value else "F").rjust(20)
    elif isinstance(value, (int, np.integer)):
        v = str(int(value)).rjust(20)
    elif isinstance(value, (float, np.floating)):
        v = ("%.16G" % float(value)).rjust(20)
    else:
        v = "'" + str(value).replace("'", "''").ljust(8) + "'"
    return ("%-8s= %s" % (key, v)).ljust(CARD)[:CARD]


def write_fits(path, hdus):
    """Write a list of (header dict, array) pairs: images (float32/float64/
    int arrays) or structured arrays as binary tables.  The header dicts add
    their own keywords after the mandatory ones."""
    out = bytearray()
    for k, (hdr, data) in enumerate(hdus):
        cards = []
        if data is not None and data.dtype.names:
            rev = {"?": "L", "u1": "B", "i2": "I", "i4": "J", "i8": "K", "f4": "E", "f8": "D"}
            forms, be = [], []
            for name in data.dtype.names:
                base, shape = data.dtype[name].base, data.dtype[name].shape
                rep = int(np.prod(shape)) if shape else 1
                if base.kind == "S":
                    forms.append((name, "%dA" % base.itemsize))
                    be.append((name, base))
                else:
                    code = rev[base.str[1:]]
                    forms.append((name, ("%d%s" % (rep, code)) if rep > 1 else code))
                    be.append((name, base.newbyteorder(">"), shape) if shape else (name, base.newbyteorder(">")))
            arr = data.astype(np.dtype(be))
            cards += [_card("XTENSION", "BINTABLE"), _card("BITPIX", 8), _card("NAXIS", 2),
                      _card("NAXIS1", arr.dtype.itemsize), _card("NAXIS2", len(arr)), _card("PCOUNT", 0),
                      _card("GCOUNT", 1), _card("TFIELDS", len(forms))]
            for i, (name, form) in enumerate(forms, 1):
                cards += [_card("TTYPE%d" % i, name), _card("TFORM%d" % i, form)]
            raw = arr.tobytes()
        else:
            arr = np.asarray(data) if data is not None else None
            bitpix = {np.dtype("uint8"): 8, np.dtype("int16"): 16, np.dtype("int32"): 32,
                      np.dtype("int64"): 64, np.dtype("float32"): -32, np.dtype("float64"): -64}
            if k == 0:
                cards.append(_card("SIMPLE", True))
            else:
                cards.append(_card("XTENSION", "IMAGE"))
            if arr is None:
                cards += [_card("BITPIX", 8), _card("NAXIS", 0)]
                raw = b""
            else:
                cards += [_card("BITPIX", bitpix[arr.dtype]), _card("NAXIS", arr.ndim)]
                for a in range(arr.ndim):
                    cards.append(_card("NAXIS%d" % (a + 1), arr.shape[arr.ndim - 1 - a]))
                raw = arr.astype(arr.dtype.newbyteorder(">")).tobytes()
            if k == 0:
                cards.append(_card("EXTEND", True))
            else:
                cards += [_card("PCOUNT", 0), _card("GCOUNT", 1)]
        for key, v in hdr.items():
            cards.append(_card(key, v))
        cards.append("END".ljust(CARD))
        head = "".join(cards).encode("ascii")
        out += head + b" " * (-len(head) % BLOCK)
        out += raw + b"\0" * (-len(raw) % BLOCK)
    with open(path, "wb") as f:
        f.write(bytes(out))
