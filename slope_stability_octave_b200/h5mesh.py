"""HDF5 mesh ingestion (+MESH/load_mesh_P2.m:25-57) with a reader of its own.

No HDF5 library is available here, so ``H5File`` reads the subset of the HDF5 file format
(version 0/1 structures, as written by HDF5's default "earliest" format) that the
reference's mesh files use, following the published HDF5 File Format Specification:

  superblock version 0 or 1             root group symbol-table entry
  object headers version 1              messages: dataspace (0x0001), datatype (0x0003),
                                        data layout (0x0008), filter pipeline (0x000B),
                                        symbol table (0x0011), continuation (0x0010)
  groups                                B-tree version 1 (type 0) -> symbol-table nodes
                                        (SNOD) -> names in the local heap (HEAP), or compact
                                        groups of link messages (0x0006)
  datasets                              contiguous, compact or chunked (B-tree version 1,
                                        type 1) storage; deflate (zlib) and shuffle filters;
                                        little- and big-endian integers and IEEE floats

Arrays come back in the file's (C) order; MATLAB/Octave's h5read returns the reversed
dimensions, which ``load_mesh_P2`` undoes with a transpose as the reference's callers see it.
"""
from __future__ import annotations

import zlib

import numpy as np


class H5Error(ValueError):
    pass


class H5File:
    SIGNATURE = b"\x89HDF\r\n\x1a\n"

    def __init__(self, path):
        with open(path, "rb") as fh:
            self.buf = fh.read()
        base = self.buf.find(self.SIGNATURE)
        # the superblock sits at 0, 512, 1024, ... (a user block may precede it)
        if base < 0 or base % 512:
            raise H5Error(f"{path}: no HDF5 superblock")
        self.base = base
        b = self.buf
        ver = b[base + 8]
        if ver not in (0, 1):
            raise H5Error(f"superblock version {ver} is not supported (0 or 1 expected)")
        self.so, self.sl = b[base + 13], b[base + 14]        # sizes of offsets and lengths
        if self.so != 8 or self.sl != 8:
            raise H5Error("only 8-byte offsets and lengths are supported")
        p = base + 24 + (4 if ver == 1 else 0)
        # base address, free-space address, end of file, driver information
        self.base_addr = self._u(p, 8)
        p += 4 * 8
        self.root = self._symbol_entry(p)

    # ------------------------------------------------------------------ primitives
    def _u(self, p, n):
        return int.from_bytes(self.buf[p:p + n], "little")

    def _addr(self, a):
        return self.base_addr + a

    def _symbol_entry(self, p):
        return dict(name_off=self._u(p, 8), header=self._u(p + 8, 8), cache=self._u(p + 16, 4),
                    btree=self._u(p + 24, 8), heap=self._u(p + 32, 8))

    # ------------------------------------------------------------------ object headers
    def _messages(self, addr):
        """(type, data offset, size) of every message of a version-1 object header."""
        p = self._addr(addr)
        if self.buf[p] != 1:
            raise H5Error(f"object header version {self.buf[p]} is not supported")
        nmsg = self._u(p + 2, 2)
        hsize = self._u(p + 8, 4)
        blocks = [(p + 16, hsize)]
        out = []
        while blocks and len(out) < nmsg:
            q, size = blocks.pop(0)
            end = q + size
            while q + 8 <= end and len(out) < nmsg:
                mtype, msize = self._u(q, 2), self._u(q + 2, 2)
                data = q + 8
                if mtype == 0x0010:      # continuation: more messages elsewhere
                    blocks.append((self._addr(self._u(data, 8)), self._u(data + 8, 8)))
                out.append((mtype, data, msize))
                q = data + msize
        return out

    # ------------------------------------------------------------------ groups
    def _heap_data(self, addr):
        p = self._addr(addr)
        if self.buf[p:p + 4] != b"HEAP":
            raise H5Error("local heap signature missing")
        return self._addr(self._u(p + 24, 8))

    def _name(self, heap_data, off):
        q = heap_data + off
        e = self.buf.index(b"\0", q)
        return self.buf[q:e].decode()

    def _group_entries(self, btree, heap):
        hd = self._heap_data(heap)
        out = {}
        stack = [btree]
        while stack:
            p = self._addr(stack.pop())
            if self.buf[p:p + 4] != b"TREE" or self.buf[p + 4] != 0:
                raise H5Error("group B-tree node expected")
            level, used = self.buf[p + 5], self._u(p + 6, 2)
            q = p + 24 + 8                           # past the first key
            for _ in range(used):
                child = self._u(q, 8)
                q += 16                              # child address + next key
                if level > 0:
                    stack.append(child)
                    continue
                s = self._addr(child)
                if self.buf[s:s + 4] != b"SNOD":
                    raise H5Error("symbol-table node expected")
                for k in range(self._u(s + 6, 2)):
                    e = self._symbol_entry(s + 8 + 40 * k)
                    out[self._name(hd, e["name_off"])] = e
        return out

    def _link(self, p):
        """(name, object header address) of a hard link message (0x0006)."""
        flags = self.buf[p + 1]
        q = p + 2
        ltype = 0
        if flags & 0x08:
            ltype = self.buf[q]
            q += 1
        if flags & 0x04:
            q += 8                                   # creation order
        if flags & 0x10:
            q += 1                                   # name character set
        nlen_size = 1 << (flags & 0x03)
        nlen = self._u(q, nlen_size)
        q += nlen_size
        name = self.buf[q:q + nlen].decode()
        if ltype != 0:
            raise H5Error(f"link {name!r}: only hard links are supported")
        return name, self._u(q + nlen, 8)

    def _children(self, header_addr, entry=None):
        if entry is not None and entry.get("cache") == 1:
            return self._group_entries(entry["btree"], entry["heap"])
        links = {}
        for mtype, data, _ in self._messages(header_addr):
            if mtype == 0x0011:                      # symbol table (old-style group)
                return self._group_entries(self._u(data, 8), self._u(data + 8, 8))
            if mtype == 0x0006:                      # link (compact new-style group)
                name, addr = self._link(data)
                links[name] = dict(header=addr, cache=0)
            if mtype == 0x0002 and self._u(data + 2 + (8 if self.buf[data + 1] & 1 else 0), 8) != (1 << 64) - 1:
                raise H5Error("groups with dense link storage are not supported")
        if links:
            return links
        raise H5Error("not a group")

    def keys(self, group="/"):
        return sorted(self._lookup(group)[1].keys())

    def _lookup(self, path):
        entry = self.root
        kids = self._children(entry["header"], entry)
        parts = [x for x in path.split("/") if x]
        for i, name in enumerate(parts):
            if name not in kids:
                raise KeyError(path)
            entry = kids[name]
            if i + 1 < len(parts):
                kids = self._children(entry["header"], entry)
        return entry, (kids if not parts else None)

    # ------------------------------------------------------------------ datasets
    def _dtype(self, p):
        cls, ver = self.buf[p] & 0x0F, self.buf[p] >> 4
        bits = self._u(p + 1, 3)
        size = self._u(p + 4, 4)
        order = ">" if bits & 1 else "<"
        if cls == 0:
            return np.dtype(f"{order}{'i' if bits & 8 else 'u'}{size}")
        if cls == 1:
            if size not in (4, 8):
                raise H5Error(f"float of {size} bytes")
            return np.dtype(f"{order}f{size}")
        raise H5Error(f"datatype class {cls} (version {ver}) is not supported")

    def _dataspace(self, p):
        ver, ndim, flags = self.buf[p], self.buf[p + 1], self.buf[p + 2]
        q = p + (8 if ver == 1 else 4)
        return tuple(self._u(q + 8 * i, 8) for i in range(ndim))

    def _filters(self, p):
        ver, nf = self.buf[p], self.buf[p + 1]
        q = p + (8 if ver == 1 else 2)
        out = []
        for _ in range(nf):
            fid = self._u(q, 2)
            if ver == 1 or fid >= 256:
                nlen = self._u(q + 2, 2)
                ncd = self._u(q + 6, 2)
                q += 8 + ((nlen + 7) // 8) * 8 if ver == 1 else 8 + nlen
            else:
                ncd = self._u(q + 4, 2)
                q += 6
            cd = [self._u(q + 4 * i, 4) for i in range(ncd)]
            q += 4 * ncd + (4 if ver == 1 and ncd % 2 else 0)
            out.append((fid, cd))
        return out

    def _unfilter(self, raw, filters, mask, itemsize):
        for i, (fid, cd) in reversed(list(enumerate(filters))):
            if mask & (1 << i):
                continue
            if fid == 1:
                raw = zlib.decompress(raw)
            elif fid == 2:
                a = np.frombuffer(raw, np.uint8).reshape(itemsize, -1)
                raw = a.T.tobytes()
            else:
                raise H5Error(f"filter {fid} is not supported")
        return raw

    def read(self, path):
        entry, _ = self._lookup(path)
        shape = dtype = layout = None
        filters = []
        for mtype, data, _ in self._messages(entry["header"]):
            if mtype == 0x0001:
                shape = self._dataspace(data)
            elif mtype == 0x0003:
                dtype = self._dtype(data)
            elif mtype == 0x0008:
                layout = data
            elif mtype == 0x000B:
                filters = self._filters(data)
        if shape is None or dtype is None or layout is None:
            raise H5Error(f"{path} is not a dataset")
        n = int(np.prod(shape)) if shape else 1
        ver = self.buf[layout]
        if ver == 3:
            cls = self.buf[layout + 1]
            q = layout + 2
            if cls == 0:
                size = self._u(q, 2)
                raw = self.buf[q + 2:q + 2 + size]
                return np.frombuffer(raw, dtype, n).reshape(shape).astype(dtype.newbyteorder("="))
            if cls == 1:
                a = self._addr(self._u(q, 8))
                return np.frombuffer(self.buf, dtype, n, a).reshape(shape).astype(dtype.newbyteorder("="))
            if cls != 2:
                raise H5Error(f"layout class {cls}")
            ndim = self.buf[q] - 1
            btree = self._u(q + 1, 8)
            cdims = [self._u(q + 9 + 4 * i, 4) for i in range(ndim)]
        elif ver in (1, 2):
            ndim, cls = self.buf[layout + 1], self.buf[layout + 2]
            q = layout + 8
            if cls == 1:
                a = self._addr(self._u(q, 8))
                return np.frombuffer(self.buf, dtype, n, a).reshape(shape).astype(dtype.newbyteorder("="))
            if cls != 2:
                raise H5Error(f"layout class {cls}")
            btree = self._u(q, 8)
            ndim -= 1
            cdims = [self._u(q + 8 + 4 * i, 4) for i in range(ndim)]
        else:
            raise H5Error(f"data layout version {ver}")
        out = np.zeros(shape, dtype.newbyteorder("="))
        stack = [btree]
        while stack:
            p = self._addr(stack.pop())
            if self.buf[p:p + 4] != b"TREE" or self.buf[p + 4] != 1:
                raise H5Error("chunk B-tree node expected")
            level, used = self.buf[p + 5], self._u(p + 6, 2)
            ksize = 8 + 8 * (ndim + 1)
            q = p + 24
            for _ in range(used):
                csize, mask = self._u(q, 4), self._u(q + 4, 4)
                off = [self._u(q + 8 + 8 * i, 8) for i in range(ndim)]
                child = self._u(q + ksize, 8)
                q += ksize + 8
                if level > 0:
                    stack.append(child)
                    continue
                a = self._addr(child)
                raw = self._unfilter(self.buf[a:a + csize], filters, mask, dtype.itemsize)
                chunk = np.frombuffer(raw, dtype, int(np.prod(cdims))).reshape(cdims)
                sl = tuple(slice(o, min(o + c, s)) for o, c, s in zip(off, cdims, shape))
                out[sl] = chunk[tuple(slice(0, x.stop - x.start) for x in sl)]
        return out


def load_mesh_P2(file_path, boundary_type=0):
    """(coord 3 x n_n, elem 10 x n_e (0-based), surf 6 x n_f (0-based), Q 3 x n_n bool,
    material n_e, boundary n_f) as +MESH/load_mesh_P2.m:25-57 returns them (indices 0-based
    here): faces with boundary labels 1/2 fix the first coordinate, 3/4 the second, 5 the
    third (every component with ``boundary_type``), then coordinates and Q are reordered
    [x; z; y]."""
    f = H5File(file_path)
    # h5read gives MATLAB the reversed (Fortran) dimensions: transpose the C-order arrays
    boundary = f.read("/boundary").ravel()
    elem = f.read("/elem").T.astype(np.int64)
    face = f.read("/face").T.astype(np.int64)
    material = f.read("/material").ravel()
    node = f.read("/node").T.astype(np.float64)
    if node.shape[0] != 3:
        raise H5Error(f"/node has shape {node.shape[::-1]} in the file; 3 coordinates per node expected")
    Q = np.ones(node.shape, bool)
    for labels, comp in (((1, 2), 0), ((3, 4), 1)):
        Q[comp, np.unique(face[:, np.isin(boundary, labels)])] = False
    bottom = np.unique(face[:, boundary == 5])
    if boundary_type:
        Q[:, bottom] = False
    else:
        Q[2, bottom] = False
    order = [0, 2, 1]
    return node[order], elem, face, Q[order], material, boundary
