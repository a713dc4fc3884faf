"""A small HDF5 reader for forcepho's stores (no h5py).

The reference keeps its PSF mixtures, pixel and metadata stores and Sersic
amplitude tables in HDF5 files read with h5py
(forcepho/patches/storage.py:43-489).  h5py is not installed here.  This
module reads the subset of the format (HDF5 file format specification,
version 0 superblock) that those files use:

* superblock v0; groups as v1 B-trees with symbol nodes and a local heap
  (root group and nested groups, found through each group's symbol-table
  message);
* v1 object headers with continuation blocks;
* attributes (message 0x000C, versions 1 and 3);
* datatypes: fixed point, floating point, fixed-length strings, compound
  (versions 1-3) and arrays, little- or big-endian;
* dataspaces v1/v2 and data layouts v1-v3, contiguous or compact.

Chunked or compressed datasets raise ``ValueError``.

    f = H5File(path)
    grp = f["CLEAR"]                    # Group
    grp.attrs["n_psf_per_source"]
    grp["parameters"][...]              # numpy (structured) array
"""

import numpy as np

__all__ = ["H5File", "Group", "Dataset"]

SIG = b"\x89HDF\r\n\x1a\n"


class _Buf:
    def __init__(self, buf):
        self.b = buf
        if buf[:8] != SIG:
            raise ValueError("not an HDF5 file (bad signature)")
        if buf[8] != 0:
            raise ValueError("only superblock version 0 is supported")
        self.so = buf[13]
        self.sl = buf[14]

    def u(self, pos, n):
        return int.from_bytes(self.b[pos:pos + n], "little")

    # --- object headers ---
    def messages(self, addr):
        if self.b[addr] != 1:
            raise ValueError("only v1 object headers are supported")
        nmsg = self.u(addr + 2, 2)
        hsize = self.u(addr + 8, 4)
        blocks = [(addr + 16, hsize)]
        msgs = []
        while blocks and len(msgs) < nmsg:
            start, size = blocks.pop(0)
            p = start
            while p + 8 <= start + size and len(msgs) < nmsg:
                mtype = self.u(p, 2)
                msize = self.u(p + 2, 2)
                body = p + 8
                if mtype == 0x10:
                    blocks.append((self.u(body, self.so), self.u(body + self.so, self.sl)))
                msgs.append((mtype, body, msize))
                p = body + msize
        return msgs

    # --- groups ---
    def group_members(self, btree, heap):
        out = {}
        if self.b[heap:heap + 4] != b"HEAP":
            raise ValueError("bad local heap signature")
        heap_data = self.u(heap + 8 + 2 * self.sl, self.so)
        self._walk(btree, heap_data, out)
        return out

    def _walk(self, addr, heap_data, out):
        if self.b[addr:addr + 4] != b"TREE":
            raise ValueError("bad B-tree signature")
        level = self.b[addr + 5]
        used = self.u(addr + 6, 2)
        p = addr + 8 + 2 * self.so + self.sl
        for _ in range(used):
            child = self.u(p, self.so)
            p += self.so + self.sl
            if level > 0:
                self._walk(child, heap_data, out)
            else:
                self._snod(child, heap_data, out)

    def _snod(self, addr, heap_data, out):
        if self.b[addr:addr + 4] != b"SNOD":
            raise ValueError("bad symbol node signature")
        nsym = self.u(addr + 6, 2)
        esize = 2 * self.so + 24
        for i in range(nsym):
            e = addr + 8 + i * esize
            name_off = self.u(e, self.so)
            ohdr = self.u(e + self.so, self.so)
            start = heap_data + name_off
            name = self.b[start:self.b.index(b"\x00", start)].decode()
            out[name] = ohdr

    # --- datatypes and dataspaces ---
    def dtype(self, pos):
        """(numpy dtype, size in bytes of the datatype message) at pos."""
        cv = self.b[pos]
        cls, ver = cv & 0x0F, cv >> 4
        f0, f1 = self.b[pos + 1], self.b[pos + 2]
        size = self.u(pos + 4, 4)
        props = pos + 8
        if cls in (0, 1):
            endian = ">" if f0 & 1 else "<"
            if cls == 0:
                kind = "i" if f0 & 0x08 else "u"
                return np.dtype("%s%s%d" % (endian, kind, size)), 8 + 4
            return np.dtype("%sf%d" % (endian, size)), 8 + 12
        if cls == 3:
            return np.dtype("S%d" % size), 8
        if cls == 6:
            nmemb = f0 | (f1 << 8)
            names, formats, offsets = [], [], []
            p = props
            for _ in range(nmemb):
                end = self.b.index(b"\x00", p)
                name = self.b[p:end].decode()
                if ver < 3:
                    p = p + ((end - p) // 8 + 1) * 8          # name padded to a multiple of 8
                else:
                    p = end + 1
                if ver == 1:
                    off = self.u(p, 4)
                    dims = self.b[p + 4]
                    shape = tuple(self.u(p + 16 + 4 * k, 4) for k in range(dims))
                    p += 16 + 16
                    sub, sz = self.dtype(p)
                    if shape:
                        sub = np.dtype((sub, shape))
                elif ver == 2:
                    off = self.u(p, 4)
                    p += 4
                    sub, sz = self.dtype(p)
                else:
                    nb = max(1, (size.bit_length() + 7) // 8)
                    off = self.u(p, nb)
                    p += nb
                    sub, sz = self.dtype(p)
                names.append(name)
                formats.append(sub)
                offsets.append(off)
                p += sz
            return np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": size}), p - pos
        if cls == 10:
            dims = self.b[props]
            if ver < 3:
                shape = tuple(self.u(props + 4 + 4 * k, 4) for k in range(dims))
                p = props + 4 + 4 * dims + 4 * dims
            else:
                shape = tuple(self.u(props + 1 + 4 * k, 4) for k in range(dims))
                p = props + 1 + 4 * dims
            base, sz = self.dtype(p)
            return np.dtype((base, shape)), p + sz - pos
        raise ValueError("unsupported HDF5 datatype class %d" % cls)

    def dataspace(self, pos):
        ver, ndim = self.b[pos], self.b[pos + 1]
        p = pos + (8 if ver == 1 else 4)
        if ver == 2 and self.b[pos + 3] == 0:
            return ()                                   # scalar
        return tuple(self.u(p + i * self.sl, self.sl) for i in range(ndim))

    def layout(self, pos):
        """('contiguous', address) or ('compact', (offset, size))."""
        ver = self.b[pos]
        if ver == 3:
            cls = self.b[pos + 1]
            if cls == 1:
                return "contiguous", self.u(pos + 2, self.so)
            if cls == 0:
                n = self.u(pos + 2, 2)
                return "compact", (pos + 4, n)
            raise ValueError("chunked datasets are not supported")
        ndim, cls = self.b[pos + 1], self.b[pos + 2]
        if cls == 1:
            return "contiguous", self.u(pos + 8, self.so)
        if cls == 0:
            p = pos + 8 + 4 * ndim
            n = self.u(p, 4)
            return "compact", (p + 4, n)
        raise ValueError("chunked datasets are not supported")

    def attributes(self, addr):
        out = {}
        for mtype, body, _ in self.messages(addr):
            if mtype != 0x0C:
                continue
            ver = self.b[body]
            nlen, tlen, slen = self.u(body + 2, 2), self.u(body + 4, 2), self.u(body + 6, 2)
            p = body + 8
            name = self.b[p:p + nlen].rstrip(b"\x00").decode()
            pad = (lambda n: (n + 7) // 8 * 8) if ver == 1 else (lambda n: n)
            if ver == 3:
                p += 1
                p = body + 9
            p += pad(nlen)
            dt, _ = self.dtype(p)
            p += pad(tlen)
            shape = self.dataspace(p)
            p += pad(slen)
            count = int(np.prod(shape)) if shape else 1
            val = np.frombuffer(self.b, dtype=dt, count=count, offset=p).copy()
            out[name] = val.reshape(shape) if shape else val[0]
        return out


class Dataset:
    def __init__(self, f, addr, name):
        self._f, self._addr, self.name = f, addr, name
        self.shape = self.dtype = self._where = None
        for mtype, body, _ in f.messages(addr):
            if mtype == 0x01:
                self.shape = f.dataspace(body)
            elif mtype == 0x03:
                self.dtype, _ = f.dtype(body)
            elif mtype == 0x08:
                self._where = f.layout(body)
        if self.dtype is None or self._where is None or self.shape is None:
            raise ValueError("%s is not a dataset" % name)

    @property
    def attrs(self):
        return self._f.attributes(self._addr)

    def __getitem__(self, key):
        return self.read()[key]

    def read(self):
        count = int(np.prod(self.shape)) if self.shape else 1
        kind, where = self._where
        off = where if kind == "contiguous" else where[0]
        arr = np.frombuffer(self._f.b, dtype=self.dtype, count=count, offset=off).copy()
        return arr.reshape(self.shape) if self.shape else arr[0]


class Group:
    def __init__(self, f, addr, name="/"):
        self._f, self._addr, self.name = f, addr, name
        self._members = None
        for mtype, body, _ in f.messages(addr):
            if mtype == 0x11:                           # symbol table
                self._members = f.group_members(f.u(body, f.so), f.u(body + f.so, f.so))
        if self._members is None:
            raise ValueError("%s is not a group" % name)

    def keys(self):
        return list(self._members)

    def __contains__(self, k):
        return k.split("/", 1)[0] in self._members

    @property
    def attrs(self):
        return self._f.attributes(self._addr)

    def __getitem__(self, path):
        head, _, rest = path.strip("/").partition("/")
        addr = self._members[head]
        name = self.name.rstrip("/") + "/" + head
        is_group = any(m == 0x11 for m, _, _ in self._f.messages(addr))
        obj = Group(self._f, addr, name) if is_group else Dataset(self._f, addr, name)
        return obj[rest] if rest else obj


class H5File(Group):
    """The root group of an HDF5 file."""

    def __init__(self, path):
        with open(path, "rb") as fp:
            f = _Buf(fp.read())
        root_entry = 24 + 4 * f.so
        root_ohdr = f.u(root_entry + f.so, f.so)
        super().__init__(f, root_ohdr, "/")
