"""Minimal reader of HDF5 files with a version-0 superblock (test
infrastructure: it reads the reference's result fixtures when the golden
vectors are regenerated; no HDF5 library or h5py exists in this image).

Supported, which is what the reference's writer (src/io/mod_hdf5_io.f90,
HDF5 default file creation properties) produces for its result files:
superblock v0 with 8-byte offsets and lengths; version-1 object headers with
continuation blocks; groups stored as symbol tables (version-1 B-tree of
group nodes + local heap); datasets with simple dataspaces, fixed-point,
floating-point and fixed-length string datatypes, contiguous or compact
layout (version 3); attributes (message 0x000C, versions 1 and 2).

Arrays come back in the file's row-major order: a Fortran array a(3, n)
written by the reference has the dataspace (n, 3) and reads as shape (n, 3).
"""
import numpy as np


class H5Error(RuntimeError):
    pass


def _u(b, off, n):
    return int.from_bytes(b[off:off + n], "little")


class _Node:
    def __init__(self, f, addr):
        self.f = f
        self.addr = addr
        self.msgs = f._messages(addr)


class Group(_Node):
    def __init__(self, f, addr, stab=None):
        super().__init__(f, addr)
        if stab is None:
            for mt, data in self.msgs:
                if mt == 0x0011:
                    stab = (_u(data, 0, 8), _u(data, 8, 8))
        if stab is None:
            raise H5Error("group without a symbol table message at %#x" % addr)
        self.btree, self.heap = stab
        self._links = None

    def links(self):
        """name -> (object header address, scratch of the symbol table entry)."""
        if self._links is None:
            heap_data = self.f._local_heap(self.heap)
            out = {}
            for ent in self.f._btree_group_entries(self.btree):
                name_off, oh, cache, scratch = ent
                end = heap_data.index(b"\0", name_off)
                out[heap_data[name_off:end].decode()] = (oh, cache, scratch)
            self._links = out
        return self._links

    def keys(self):
        return list(self.links().keys())

    def __contains__(self, name):
        return name in self.links()

    def __getitem__(self, path):
        node = self
        for part in [p for p in path.split("/") if p]:
            if not isinstance(node, Group):
                raise KeyError(path)
            oh, cache, scratch = node.links()[part]
            node = node.f._open(oh, cache, scratch)
        return node

    def attrs(self):
        return self.f._attributes(self.msgs)


class Dataset(_Node):
    def __init__(self, f, addr):
        super().__init__(f, addr)
        self.shape = None
        self.dtype = None
        self.layout = None
        for mt, data in self.msgs:
            if mt == 0x0001:
                self.shape = self.f._dataspace(data)
            elif mt == 0x0003:
                self.dtype = self.f._datatype(data)
            elif mt == 0x0008:
                self.layout = data
        if self.shape is None or self.dtype is None or self.layout is None:
            raise H5Error("incomplete dataset header at %#x" % addr)

    def attrs(self):
        return self.f._attributes(self.msgs)

    def read(self):
        lay = self.layout
        ver = lay[0]
        if ver != 3:
            raise H5Error("data layout version %d not supported" % ver)
        cls = lay[1]
        count = int(np.prod(self.shape)) if self.shape else 1
        nbytes = count * self.dtype.itemsize
        if cls == 1:  # contiguous
            addr, size = _u(lay, 2, 8), _u(lay, 10, 8)
            if addr == 0xFFFFFFFFFFFFFFFF:
                raw = bytes(nbytes)
            else:
                raw = self.f.b[addr:addr + min(size, nbytes)]
        elif cls == 0:  # compact
            size = _u(lay, 2, 2)
            raw = lay[4:4 + size]
        else:
            raise H5Error("chunked layout not supported")
        a = np.frombuffer(raw[:nbytes], dtype=self.dtype, count=count)
        if self.dtype.kind == "S":
            a = np.array([s.rstrip(b"\0 ").decode() for s in a])
        return a.reshape(self.shape) if self.shape else a.reshape(())


class File(Group):
    def __init__(self, path):
        with open(path, "rb") as fh:
            self.b = fh.read()
        b = self.b
        if b[:8] != b"\x89HDF\r\n\x1a\n":
            raise H5Error("not an HDF5 file")
        if b[8] != 0:
            raise H5Error("superblock version %d not supported" % b[8])
        if b[13] != 8 or b[14] != 8:
            raise H5Error("only 8-byte offsets and lengths are supported")
        # root group symbol table entry after the 4 addresses (base, free
        # space, end of file, driver info)
        ent = 24 + 4 * 8
        oh = _u(b, ent + 8, 8)
        cache = _u(b, ent + 16, 4)
        scratch = b[ent + 24:ent + 40]
        self.f = self
        stab = (_u(scratch, 0, 8), _u(scratch, 8, 8)) if cache == 1 else None
        Group.__init__(self, self, oh, stab)

    # ------------------------------------------------------------ plumbing
    def _open(self, oh, cache, scratch):
        if cache == 1:
            return Group(self, oh, (_u(scratch, 0, 8), _u(scratch, 8, 8)))
        msgs = self._messages(oh)
        if any(mt == 0x0011 for mt, _ in msgs):
            return Group(self, oh)
        return Dataset(self, oh)

    def _messages(self, addr):
        b = self.b
        if b[addr] != 1:
            raise H5Error("object header version %d at %#x not supported" % (b[addr], addr))
        nmsg = _u(b, addr + 2, 2)
        size = _u(b, addr + 8, 4)
        blocks = [(addr + 16, size)]  # messages start after the 12-byte prefix + 4 pad
        out = []
        while blocks and len(out) < nmsg:
            start, length = blocks.pop(0)
            off = start
            while off + 8 <= start + length and len(out) < nmsg:
                mt = _u(b, off, 2)
                ms = _u(b, off + 2, 2)
                data = b[off + 8:off + 8 + ms]
                if mt == 0x0010:  # continuation
                    blocks.append((_u(data, 0, 8), _u(data, 8, 8)))
                out.append((mt, data))
                off += 8 + ms
        return out

    def _local_heap(self, addr):
        b = self.b
        if b[addr:addr + 4] != b"HEAP":
            raise H5Error("bad local heap at %#x" % addr)
        size = _u(b, addr + 8, 8)
        data_addr = _u(b, addr + 24, 8)
        return b[data_addr:data_addr + size]

    def _btree_group_entries(self, addr):
        b = self.b
        if b[addr:addr + 4] != b"TREE":
            raise H5Error("bad B-tree node at %#x" % addr)
        ntype, level, used = b[addr + 4], b[addr + 5], _u(b, addr + 6, 2)
        if ntype != 0:
            raise H5Error("B-tree node type %d is not a group node" % ntype)
        off = addr + 8 + 16  # left and right sibling addresses
        children = []
        off += 8  # key 0 (heap offset)
        for _ in range(used):
            children.append(_u(b, off, 8))
            off += 16  # child address + next key
        out = []
        for c in children:
            if level > 0:
                out.extend(self._btree_group_entries(c))
            else:
                out.extend(self._snod(c))
        return out

    def _snod(self, addr):
        b = self.b
        if b[addr:addr + 4] != b"SNOD":
            raise H5Error("bad symbol table node at %#x" % addr)
        n = _u(b, addr + 6, 2)
        out = []
        off = addr + 8
        for _ in range(n):
            out.append((_u(b, off, 8), _u(b, off + 8, 8), _u(b, off + 16, 4),
                        b[off + 24:off + 40]))
            off += 40
        return out

    @staticmethod
    def _dataspace(data):
        ver = data[0]
        rank = data[1]
        if ver == 1:
            off = 8
        elif ver == 2:
            off = 4
        else:
            raise H5Error("dataspace version %d not supported" % ver)
        return tuple(_u(data, off + 8 * i, 8) for i in range(rank))

    @staticmethod
    def _datatype(data):
        cls = data[0] & 0x0F
        bits0 = data[1]
        size = _u(data, 4, 4)
        order = ">" if (bits0 & 1) else "<"
        if cls == 0:  # fixed point
            signed = bool(bits0 & 0x08)
            return np.dtype("%s%s%d" % (order, "i" if signed else "u", size))
        if cls == 1:  # floating point
            return np.dtype("%sf%d" % (order, size))
        if cls == 3:  # string
            return np.dtype("S%d" % size)
        raise H5Error("datatype class %d not supported" % cls)

    def _attributes(self, msgs):
        out = {}
        for mt, data in msgs:
            if mt != 0x000C:
                continue
            ver = data[0]
            nlen, dtlen, dslen = _u(data, 2, 2), _u(data, 4, 2), _u(data, 6, 2)
            pad = (lambda n: (n + 7) & ~7) if ver == 1 else (lambda n: n)
            off = 8
            name = data[off:off + nlen].rstrip(b"\0").decode()
            off += pad(nlen)
            dt = self._datatype(data[off:off + dtlen])
            off += pad(dtlen)
            shape = self._dataspace(data[off:off + dslen])
            off += pad(dslen)
            count = int(np.prod(shape)) if shape else 1
            a = np.frombuffer(data[off:off + count * dt.itemsize], dtype=dt, count=count)
            if dt.kind == "S":
                a = np.array([s.rstrip(b"\0 ").decode() for s in a])
            out[name] = a.reshape(shape) if shape else a.reshape(())
        return out


def walk(g, prefix=""):
    """(path, Dataset or Group) for every object below g."""
    for k in g.keys():
        node = g[k]
        yield prefix + k, node
        if isinstance(node, Group):
            yield from walk(node, prefix + k + "/")
