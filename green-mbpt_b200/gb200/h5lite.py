"""Minimal read-only HDF5 reader (pure Python + numpy + zlib).

It covers what green-mbpt's input, integral and result files use:
- superblocks v0/v1 and v2/v3;
- version-1 object headers, and version-2 ones ("OHDR" with "OCHK" continuation chunks);
- old-style groups (symbol-table message -> v1 group B-tree -> SNOD nodes + local heap), and new-style groups with their links stored compactly in the object header;
- contiguous and compact layouts;
- chunked layouts indexed by a v1 B-tree, by a single chunk or implicitly;
- the deflate and shuffle filters;
- fixed-point, floating-point, string, compound and variable-length datatypes, and attributes.  There is no h5py or libhdf5 in this environment; gb200.inputs
reads the solver's input files with it.

The format facts used here follow the public HDF5 File Format Specification
(version 3.0), sections II (superblock), III.A/B (B-trees, symbol table
nodes), III.D (local heap), IV.A (object headers) and IV.A.2 (messages:
link info, link and data layout among them).
"""
from __future__ import annotations

import mmap
import os
import zlib

import numpy as np

_SIG = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


class H5Error(RuntimeError):
    pass


class _Dtype:
    def __init__(self, np_dtype, kind):
        self.np = np_dtype
        self.kind = kind  # "num" | "str"


class H5File:
    def __init__(self, path: str):
        # mapped, not read: integral files run to gigabytes and only the touched pages are loaded
        with open(path, "rb") as fh:
            if os.fstat(fh.fileno()).st_size == 0:
                raise H5Error(f"{path}: empty file")
            self.buf = mmap.mmap(fh.fileno(), 0, access=mmap.ACCESS_READ)
        self.path = path
        b = self.buf
        if b[:8] != _SIG:
            raise H5Error(f"{path}: not an HDF5 file")
        ver = b[8]
        self._cache = {}
        if ver in (2, 3):
            # signature, version, offset/length sizes, flags, base, extension, eof, root header, checksum
            self.so, self.sl = b[9], b[10]
            if self.so != 8 or self.sl != 8:
                raise H5Error("only 8-byte offsets/lengths supported")
            self.base = self._u(12, 8)
            self.root_addr = self._u(36, 8)
            return
        if ver not in (0, 1):
            raise H5Error(f"{path}: superblock version {ver} not supported")
        self.so = b[13]
        self.sl = b[14]
        if self.so != 8 or self.sl != 8:
            raise H5Error("only 8-byte offsets/lengths supported")
        p = 24 if ver == 0 else 28
        self.base = self._u(p, 8)
        p += 4 * 8  # base, free-space, eof, driver
        # root symbol table entry
        self.root_addr = self._u(p + 8, 8)

    # -- primitive readers -------------------------------------------------
    def _u(self, off, n):
        return int.from_bytes(self.buf[off:off + n], "little")

    # -- object headers ----------------------------------------------------
    def _messages(self, addr):
        if addr in self._cache:
            return self._cache[addr]
        b = self.buf
        if b[addr:addr + 4] == b"OHDR":
            msgs = self._messages_v2(addr)
            self._cache[addr] = msgs
            return msgs
        if b[addr] != 1:
            raise H5Error(f"object header version {b[addr]} at {addr:#x}")
        nmsg = self._u(addr + 2, 2)
        hsize = self._u(addr + 8, 4)
        blocks = [(addr + 16, hsize)]
        msgs = []
        while blocks and len(msgs) < nmsg:
            start, size = blocks.pop(0)
            p = start
            end = start + size
            while p + 8 <= end and len(msgs) < nmsg:
                mtype = self._u(p, 2)
                msize = self._u(p + 2, 2)
                data = b[p + 8:p + 8 + msize]
                p += 8 + msize
                if mtype == 0x10:  # continuation
                    blocks.append((int.from_bytes(data[0:8], "little"), int.from_bytes(data[8:16], "little")))
                msgs.append((mtype, data))
        self._cache[addr] = msgs
        return msgs

    def _messages_v2(self, addr):
        """Messages of a version-2 object header: chunk 0 after the prefix, more chunks ("OCHK")
        named by continuation messages; each chunk ends with a 4-byte checksum."""
        b = self.buf
        if b[addr + 4] != 2:
            raise H5Error(f"object header version {b[addr + 4]} at {addr:#x}")
        flags = b[addr + 5]
        p = addr + 6
        if flags & 0x20:
            p += 16  # access, modification, change, birth times
        if flags & 0x10:
            p += 4  # attribute phase-change values
        nb = 1 << (flags & 3)
        size0 = self._u(p, nb)
        p += nb
        order = 2 if flags & 0x04 else 0  # creation order field in every message header
        blocks = [(p, p + size0)]
        msgs = []
        while blocks:
            start, end = blocks.pop(0)
            q = start
            while q + 4 + order <= end:
                mtype = b[q]
                msize = self._u(q + 1, 2)
                q += 4 + order
                data = b[q:q + msize]
                q += msize
                if mtype == 0x10:  # continuation: address and length of an OCHK block
                    ca = int.from_bytes(data[0:8], "little")
                    cl = int.from_bytes(data[8:16], "little")
                    if b[ca:ca + 4] != b"OCHK":
                        raise H5Error("bad object header continuation signature")
                    blocks.append((ca + 4, ca + cl - 4))
                msgs.append((mtype, data))
        return msgs

    # -- groups ------------------------------------------------------------
    def _local_heap_data(self, addr):
        b = self.buf
        if b[addr:addr + 4] != b"HEAP":
            raise H5Error("bad local heap signature")
        return self._u(addr + 24, 8)

    def _heap_str(self, heap_data, off):
        b = self.buf
        s = heap_data + off
        e = b.find(b"\x00", s)
        if e < 0:
            raise H5Error("unterminated local heap string")
        return b[s:e].decode()

    def _group_entries(self, btree, heap):
        hd = self._local_heap_data(heap)
        out = {}
        stack = [btree]
        while stack:
            node = stack.pop()
            b = self.buf
            if b[node:node + 4] != b"TREE":
                raise H5Error("bad v1 B-tree signature")
            ntype = b[node + 4]
            level = b[node + 5]
            used = self._u(node + 6, 2)
            if ntype != 0:
                raise H5Error("expected group B-tree")
            p = node + 8 + 16 + 8  # header + siblings + key0
            for _ in range(used):
                child = self._u(p, 8)
                p += 16  # child + next key
                if level > 0:
                    stack.append(child)
                else:
                    if b[child:child + 4] != b"SNOD":
                        raise H5Error("bad SNOD signature")
                    nsym = self._u(child + 6, 2)
                    q = child + 8
                    for _ in range(nsym):
                        name_off = self._u(q, 8)
                        oh = self._u(q + 8, 8)
                        out[self._heap_str(hd, name_off)] = oh
                        q += 40
        return out

    @staticmethod
    def _link(data):
        """(name, object header address) of a hard link message; None for soft/external links."""
        flags = data[1]
        p = 2
        ltype = 0
        if flags & 0x08:
            ltype = data[p]
            p += 1
        if flags & 0x04:
            p += 8  # creation order
        if flags & 0x10:
            p += 1  # name character set
        nb = 1 << (flags & 3)
        n = int.from_bytes(data[p:p + nb], "little")
        p += nb
        name = data[p:p + n].decode()
        p += n
        if ltype != 0:
            return None
        return name, int.from_bytes(data[p:p + 8], "little")

    def _children(self, addr):
        msgs = self._messages(addr)
        for mtype, data in msgs:
            if mtype == 0x11:
                bt = int.from_bytes(data[0:8], "little")
                hp = int.from_bytes(data[8:16], "little")
                return self._group_entries(bt, hp)
        if not any(m in (0x02, 0x06, 0x0A) for m, _ in msgs):
            return None
        for mtype, data in msgs:
            if mtype == 0x02:  # link info: links in a fractal heap when its address is defined
                p = 2 + (8 if data[1] & 0x01 else 0)
                if int.from_bytes(data[p:p + 8], "little") != UNDEF:
                    raise H5Error("groups with densely stored links are not supported")
        out = {}
        for mtype, data in msgs:
            if mtype == 0x06:
                ln = self._link(data)
                if ln is not None:
                    out[ln[0]] = ln[1]
        return out

    def _resolve(self, path):
        addr = self.root_addr
        for part in [p for p in path.split("/") if p]:
            ch = self._children(addr)
            if ch is None or part not in ch:
                raise KeyError(f"{self.path}: no object '{path}'")
            addr = ch[part]
        return addr

    def keys(self, path="/"):
        ch = self._children(self._resolve(path))
        return sorted(ch) if ch is not None else []

    def is_group(self, path):
        return self._children(self._resolve(path)) is not None

    def walk(self, path="/"):
        """Yield every dataset path under `path`."""
        for k in self.keys(path):
            full = (path.rstrip("/") + "/" + k)
            if self.is_group(full):
                yield from self.walk(full)
            else:
                yield full

    # -- datatypes / dataspaces -------------------------------------------
    @staticmethod
    def _dtype(data):
        cls = data[0] & 0x0F
        bits = data[1] | (data[2] << 8) | (data[3] << 16)
        size = int.from_bytes(data[4:8], "little")
        order = ">" if (bits & 1) else "<"
        if cls == 0:
            signed = bool(bits & 0x08)
            return _Dtype(np.dtype(f"{order}{'i' if signed else 'u'}{size}"), "num")
        if cls == 1:
            return _Dtype(np.dtype(f"{order}f{size}"), "num")
        if cls == 3:
            return _Dtype(np.dtype(f"S{size}"), "str")
        if cls == 9:
            # variable-length sequence/string: (length u32, heap address u64, index u32)
            return _Dtype(np.dtype([("len", "<u4"), ("addr", "<u8"), ("idx", "<u4")]), "vlen")
        if cls == 6:
            # compound: only the {r, i} double/float pair is needed
            nmemb = bits & 0xFFFF
            ver = data[0] >> 4
            p = 8
            fields = []
            for _ in range(nmemb):
                e = data.index(b"\x00", p)
                name = data[p:e].decode()
                if ver < 3:
                    nlen = e - p + 1
                    p += (nlen + 7) // 8 * 8
                    off = int.from_bytes(data[p:p + 4], "little")
                    p += 4 + 1 + 3 + 4 + 4 + 16  # offset, dim, reserved, perm, reserved, dims
                else:
                    p = e + 1
                    nb = max(1, (size.bit_length() + 7) // 8)
                    off = int.from_bytes(data[p:p + nb], "little")
                    p += nb
                sub = H5File._dtype(data[p:])
                fields.append((name, sub.np, off))
                p += 8 + H5File._dtype_props_len(data[p:])
            return _Dtype(np.dtype({"names": [f[0] for f in fields], "formats": [f[1] for f in fields],
                                    "offsets": [f[2] for f in fields], "itemsize": size}), "num")
        raise H5Error(f"datatype class {cls} not supported")

    @staticmethod
    def _dtype_props_len(data):
        cls = data[0] & 0x0F
        return {0: 4, 1: 12, 3: 0}.get(cls, 0)

    def _dataspace(self, data):
        ver = data[0]
        ndim = data[1]
        if ver == 1:
            p = 8
        elif ver == 2:
            p = 4
            if data[3] == 0:  # scalar
                return ()
        else:
            raise H5Error(f"dataspace version {ver}")
        return tuple(int.from_bytes(data[p + 8 * i:p + 8 * i + 8], "little") for i in range(ndim))

    # -- datasets -----------------------------------------------------------
    def read(self, path):
        addr = self._resolve(path)
        msgs = self._messages(addr)
        shape = dtype = layout = None
        filters = []
        for mtype, data in msgs:
            if mtype == 0x01:
                shape = self._dataspace(data)
            elif mtype == 0x03:
                dtype = self._dtype(data)
            elif mtype == 0x08:
                layout = data
            elif mtype == 0x0B:
                filters = self._filters(data)
        if shape is None or dtype is None or layout is None:
            raise H5Error(f"{path}: not a dataset")
        raw = self._layout_bytes(layout, shape, dtype.np.itemsize, filters)
        arr = np.frombuffer(raw, dtype=dtype.np, count=int(np.prod(shape)) if shape else 1)
        arr = arr.reshape(shape) if shape else arr[0]
        return arr.copy() if isinstance(arr, np.ndarray) else arr

    def attr(self, path, name):
        addr = self._resolve(path)
        for mtype, data in self._messages(addr):
            if mtype != 0x0C:
                continue
            ver = data[0]
            nsz = int.from_bytes(data[2:4], "little")
            tsz = int.from_bytes(data[4:6], "little")
            ssz = int.from_bytes(data[6:8], "little")
            if ver == 1:
                pad = lambda n: (n + 7) // 8 * 8
                p = 8
                aname = data[p:p + nsz].rstrip(b"\x00").decode()
                p += pad(nsz)
                dt = self._dtype(data[p:p + tsz])
                p += pad(tsz)
                shp = self._dataspace(data[p:p + ssz])
                p += pad(ssz)
            else:
                p = 8 if ver == 2 else 9
                aname = data[p:p + nsz].rstrip(b"\x00").decode()
                p += nsz
                dt = self._dtype(data[p:p + tsz])
                p += tsz
                shp = self._dataspace(data[p:p + ssz])
                p += ssz
            if aname != name:
                continue
            n = int(np.prod(shp)) if shp else 1
            raw = data[p:p + n * dt.np.itemsize]
            val = np.frombuffer(raw, dtype=dt.np, count=n)
            if dt.kind == "str":
                return val[0].split(b"\x00")[0].decode()
            if dt.kind == "vlen":
                return self._global_heap_object(int(val[0]["addr"]), int(val[0]["idx"])).split(b"\x00")[0].decode()
            return val.reshape(shp) if shp else val[0]
        raise KeyError(f"{path}: no attribute '{name}'")

    def _global_heap_object(self, addr, index):
        b = self.buf
        if b[addr:addr + 4] != b"GCOL":
            raise H5Error("bad global heap signature")
        size = self._u(addr + 8, 8)
        p = addr + 16
        end = addr + size
        while p + 16 <= end:
            idx = self._u(p, 2)
            osz = self._u(p + 8, 8)
            if idx == 0:
                break
            if idx == index:
                return b[p + 16:p + 16 + osz]
            p += 16 + (osz + 7) // 8 * 8
        raise H5Error(f"global heap object {index} not found")

    def _filters(self, data):
        ver = data[0]
        n = data[1]
        out = []
        p = 8 if ver == 1 else 2
        for _ in range(n):
            fid = int.from_bytes(data[p:p + 2], "little")
            if ver == 1 or fid >= 256:
                nlen = int.from_bytes(data[p + 2:p + 4], "little")
                p += 4
            else:
                nlen = 0
                p += 2
            nval = int.from_bytes(data[p + 2:p + 4], "little")
            p += 4
            if ver == 1:
                p += (nlen + 7) // 8 * 8
            else:
                p += nlen
            vals = [int.from_bytes(data[p + 4 * i:p + 4 * i + 4], "little") for i in range(nval)]
            p += 4 * nval
            if ver == 1 and nval % 2:
                p += 4
            out.append((fid, vals))
        return out

    def _unfilter(self, chunk, filters, mask, itemsize):
        for i, (fid, vals) in reversed(list(enumerate(filters))):
            if mask & (1 << i):
                continue
            if fid == 1:
                chunk = zlib.decompress(chunk)
            elif fid == 2:
                a = np.frombuffer(chunk, dtype=np.uint8)
                n = a.size // itemsize
                chunk = a[: n * itemsize].reshape(itemsize, n).T.tobytes() + chunk[n * itemsize:]
            else:
                raise H5Error(f"filter {fid} not supported")
        return chunk

    def _layout_bytes(self, lay, shape, itemsize, filters):
        ver = lay[0]
        nelem = int(np.prod(shape)) if shape else 1
        total = nelem * itemsize
        if ver == 4 and lay[1] == 2:
            return self._chunked_v4(lay, shape, itemsize, filters)
        if ver in (3, 4):
            cls = lay[1]
            if cls == 0:
                size = int.from_bytes(lay[2:4], "little")
                return lay[4:4 + size]
            if cls == 1:
                addr = int.from_bytes(lay[2:10], "little")
                if addr == UNDEF:
                    return bytes(total)
                return self.buf[addr:addr + total]
            if cls == 2:
                nd = lay[2]
                bt = int.from_bytes(lay[3:11], "little")
                cdims = [int.from_bytes(lay[11 + 4 * i:15 + 4 * i], "little") for i in range(nd)]
                return self._chunked(bt, shape, cdims[:-1], itemsize, filters)
        elif ver in (1, 2):
            nd = lay[1]
            cls = lay[2]
            p = 8
            if cls == 0:
                dims = [int.from_bytes(lay[p + 4 * i:p + 4 * i + 4], "little") for i in range(nd)]
                p += 4 * nd
                size = int.from_bytes(lay[p:p + 4], "little")
                return lay[p + 4:p + 4 + size]
            addr = int.from_bytes(lay[p:p + 8], "little")
            p += 8
            dims = [int.from_bytes(lay[p + 4 * i:p + 4 * i + 4], "little") for i in range(nd)]
            if cls == 1:
                return self.buf[addr:addr + total]
            return self._chunked(addr, shape, dims[:-1], itemsize, filters)
        raise H5Error(f"layout version {ver} not supported")

    def _chunked_v4(self, lay, shape, itemsize, filters):
        """Version-4 chunked layout with a single-chunk (1) or implicit (2) index."""
        flags, nd, enc = lay[2], lay[3], lay[4]
        p = 5
        dims = [int.from_bytes(lay[p + enc * i:p + enc * (i + 1)], "little") for i in range(nd)]
        p += enc * nd
        cdims = dims[:-1]  # the last one is the element size
        itype = lay[p]
        p += 1
        nelem = int(np.prod(shape)) if shape else 1
        if itype == 1:
            csize = mask = None
            if flags & 0x02:  # filtered single chunk: its size and filter mask precede the address
                csize = int.from_bytes(lay[p:p + 8], "little")
                mask = int.from_bytes(lay[p + 8:p + 12], "little")
                p += 12
            addr = int.from_bytes(lay[p:p + 8], "little")
            if addr == UNDEF:
                return bytes(nelem * itemsize)
            if csize is None:
                return self.buf[addr:addr + nelem * itemsize]
            raw = self._unfilter(self.buf[addr:addr + csize], filters, mask, itemsize)
            return raw[:nelem * itemsize]
        if itype == 2:
            addr = int.from_bytes(lay[p:p + 8], "little")
            nd_ = len(shape)
            grid = [-(-s // c) for s, c in zip(shape, cdims)]
            csz = int(np.prod(cdims)) * itemsize
            out = np.zeros(tuple(shape) + (itemsize,), dtype=np.uint8)
            for i, idx in enumerate(np.ndindex(*grid)):
                c = np.frombuffer(self.buf[addr + i * csz:addr + (i + 1) * csz], dtype=np.uint8)
                c = c.reshape(tuple(cdims) + (itemsize,))
                sl_out = tuple(slice(k * d, min(k * d + d, s)) for k, d, s in zip(idx, cdims, shape))
                sl_in = tuple(slice(0, so.stop - so.start) for so in sl_out)
                out[sl_out] = c[sl_in]
            del nd_
            return out.tobytes()
        raise H5Error(f"chunk index type {itype} not supported")

    def _chunked(self, bt, shape, cdims, itemsize, filters):
        nd = len(shape)
        out = np.zeros(tuple(shape) + (itemsize,), dtype=np.uint8)
        stack = [bt]
        while stack:
            node = stack.pop()
            b = self.buf
            if b[node:node + 4] != b"TREE" or b[node + 4] != 1:
                raise H5Error("bad chunk B-tree")
            level = b[node + 5]
            used = self._u(node + 6, 2)
            ksz = 8 + 8 * (nd + 1)
            p = node + 24
            for _ in range(used):
                csize = self._u(p, 4)
                mask = self._u(p + 4, 4)
                offs = [self._u(p + 8 + 8 * i, 8) for i in range(nd)]
                child = self._u(p + ksz, 8)
                p += ksz + 8
                if level > 0:
                    stack.append(child)
                    continue
                raw = self._unfilter(b[child:child + csize], filters, mask, itemsize)
                c = np.frombuffer(raw, dtype=np.uint8)[: int(np.prod(cdims)) * itemsize]
                c = c.reshape(tuple(cdims) + (itemsize,))
                sl_out = tuple(slice(o, min(o + d, s)) for o, d, s in zip(offs, cdims, shape))
                sl_in = tuple(slice(0, so.stop - so.start) for so in sl_out)
                out[sl_out] = c[sl_in]
        return out.tobytes()
