"""Convert forcepho's Sersic Gaussian-mixture amplitude table (HDF5) to ``.npz``.

The reference ships ``tests/data/sersic_splinedata_large.h5`` (identical copy at
``demo/data/sersic_splinedata_large.h5``) with four datasets:

* ``amplitudes``  f64 [n_grid, n_radii]  mixture amplitude per (sersic, rh) node
* ``nsersic``     f32 [n_grid]           Sersic index of each node
* ``rh``          f64 [n_grid]           half-light radius (arcsec) of each node
* ``radii``       f64 [n_radii]          fixed Gaussian radii (arcsec)

The reference reads it with h5py in ``forcepho/sources.py:623-639``
(``Galaxy.initialize_splines``).  h5py is not installed in this image, so this
script carries a minimal reader for the subset of the HDF5 format the file
uses (superblock v0, v1 group B-tree + local heap, v1 object headers,
contiguous little-endian numeric datasets).  Run once; the ``.npz`` it writes
is committed next to it and is what the package loads at run time.

Usage::

    python forcepho_b200/data/convert_splinedata.py <path/to/sersic_splinedata_large.h5>
"""

import os
import sys

import numpy as np


class _H5:
    """Just enough of HDF5 to list the root group and read contiguous datasets."""

    SIG = b"\x89HDF\r\n\x1a\n"

    def __init__(self, path):
        with open(path, "rb") as fp:
            self.buf = fp.read()
        if self.buf[:8] != self.SIG:
            raise ValueError("not an HDF5 file (bad signature)")
        if self.buf[8] != 0:
            raise ValueError("only superblock version 0 is supported")
        self.so = self.buf[13]  # size of offsets
        self.sl = self.buf[14]  # size of lengths
        # superblock v0: 24 fixed bytes, then 4 addresses, then root symbol entry
        p = 24 + 4 * self.so
        _, root_ohdr, cache_type, scratch = self._symbol_entry(p)
        if cache_type != 1:
            raise ValueError("root group entry has no cached symbol table")
        self.btree_addr = self._uint(scratch, self.so)
        self.heap_addr = self._uint(scratch + self.so, self.so)

    # --- primitive readers ---
    def _uint(self, pos, n):
        return int.from_bytes(self.buf[pos:pos + n], "little")

    def _symbol_entry(self, pos):
        name_off = self._uint(pos, self.so)
        ohdr = self._uint(pos + self.so, self.so)
        cache_type = self._uint(pos + 2 * self.so, 4)
        scratch = pos + 2 * self.so + 8
        return name_off, ohdr, cache_type, scratch

    def _heap_data(self):
        p = self.heap_addr
        if self.buf[p:p + 4] != b"HEAP":
            raise ValueError("bad local heap signature")
        p += 8 + 2 * self.sl
        return self._uint(p, self.so)

    def _heap_name(self, off):
        start = self._heap_data() + off
        end = self.buf.index(b"\x00", start)
        return self.buf[start:end].decode()

    # --- group listing ---
    def members(self):
        out = {}
        self._walk_btree(self.btree_addr, out)
        return out

    def _walk_btree(self, addr, out):
        if self.buf[addr:addr + 4] != b"TREE":
            raise ValueError("bad B-tree signature")
        level = self.buf[addr + 5]
        used = self._uint(addr + 6, 2)
        p = addr + 8 + 2 * self.so          # skip siblings
        p += self.sl                          # key 0
        for _ in range(used):
            child = self._uint(p, self.so)
            p += self.so + self.sl
            if level > 0:
                self._walk_btree(child, out)
            else:
                self._read_snod(child, out)

    def _read_snod(self, addr, out):
        if self.buf[addr:addr + 4] != b"SNOD":
            raise ValueError("bad symbol node signature")
        nsym = self._uint(addr + 6, 2)
        p = addr + 8
        esize = 2 * self.so + 24
        for i in range(nsym):
            name_off, ohdr, _, _ = self._symbol_entry(p + i * esize)
            out[self._heap_name(name_off)] = ohdr

    # --- object header messages ---
    def _messages(self, addr):
        if self.buf[addr] != 1:
            raise ValueError("only v1 object headers are supported")
        nmsg = self._uint(addr + 2, 2)
        hsize = self._uint(addr + 8, 4)
        blocks = [(addr + 16, hsize)]
        msgs = []
        while blocks and len(msgs) < nmsg:
            start, size = blocks.pop(0)
            p = start
            while p + 8 <= start + size and len(msgs) < nmsg:
                mtype = self._uint(p, 2)
                msize = self._uint(p + 2, 2)
                body = p + 8
                if mtype == 0x10:  # continuation
                    blocks.append((self._uint(body, self.so),
                                   self._uint(body + self.so, self.sl)))
                msgs.append((mtype, body, msize))
                p = body + msize
        return msgs

    def read(self, name):
        ohdr = self.members()[name]
        shape = dtype = addr = None
        for mtype, body, _ in self._messages(ohdr):
            if mtype == 0x01:   # dataspace
                ver, ndim, flags = self.buf[body], self.buf[body + 1], self.buf[body + 2]
                p = body + (8 if ver == 1 else 4)
                shape = tuple(self._uint(p + i * self.sl, self.sl) for i in range(ndim))
            elif mtype == 0x03:  # datatype
                cls = self.buf[body] & 0x0F
                bits0 = self.buf[body + 1]
                size = self._uint(body + 4, 4)
                if bits0 & 1:
                    raise ValueError("big-endian data not supported")
                if cls == 1:
                    dtype = np.dtype("<f%d" % size)
                elif cls == 0:
                    dtype = np.dtype(("<i%d" if bits0 & 0x08 else "<u%d") % size)
                else:
                    raise ValueError("unsupported datatype class %d" % cls)
            elif mtype == 0x08:  # data layout
                ver = self.buf[body]
                if ver == 3:
                    if self.buf[body + 1] != 1:
                        raise ValueError("only contiguous layout supported")
                    addr = self._uint(body + 2, self.so)
                else:
                    if self.buf[body + 2] != 1:
                        raise ValueError("only contiguous layout supported")
                    addr = self._uint(body + 8, self.so)
        if shape is None or dtype is None or addr is None:
            raise ValueError("dataset %s is missing a required message" % name)
        count = int(np.prod(shape)) if shape else 1
        arr = np.frombuffer(self.buf, dtype=dtype, count=count, offset=addr)
        return arr.reshape(shape).copy()


def read_splinedata_h5(path):
    """Return the four spline-table arrays from an HDF5 file."""
    h5 = _H5(path)
    return {k: h5.read(k) for k in ("amplitudes", "nsersic", "rh", "radii")}


def main(argv):
    if len(argv) != 2:
        print(__doc__)
        return 2
    tables = read_splinedata_h5(argv[1])
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                       "sersic_splinedata_large.npz")
    np.savez_compressed(out, **tables)
    for k, v in tables.items():
        print(k, v.dtype, v.shape, float(v.min()), float(v.max()))
    print("wrote", out)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
