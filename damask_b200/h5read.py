"""Minimal reader for HDF5 files: the result (DADF5) and restart files that DAMASK writes, and the
files of damask_b200.dadf5's writer (restart files of the Python host).

It covers the subset that libhdf5's defaults produce for these files: superblock
version 0, version-1 object headers (with continuation blocks), groups stored as
symbol tables (version-1 B-trees of symbol nodes + local heaps), and datasets of
fixed-point or IEEE floating-point elements in contiguous or chunked layout
(version-1 chunk B-trees) with the shuffle, deflate and Fletcher-32 filters.
Written from the public HDF5 file-format specification; no HDF5 library is needed.

    f = DADF5('result.hdf5')
    f.keys('increment_75/phase')            # group members
    P = f.read('increment_75/phase/<name>/mechanical/P')   # numpy array, C order
"""
from __future__ import annotations

import struct
import zlib

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF


class DADF5:
    def __init__(self, path):
        with open(path, 'rb') as fh:
            self.b = fh.read()
        b = self.b
        if b[:8] != b'\x89HDF\r\n\x1a\n':
            raise ValueError('not an HDF5 file')
        if b[8] != 0:
            raise ValueError(f'superblock version {b[8]} not supported')
        self.so, self.sl = b[13], b[14]
        if (self.so, self.sl) != (8, 8):
            raise ValueError('only 8-byte offsets and lengths are supported')
        # root group symbol table entry after the fixed fields (24 bytes) and 4 addresses
        root = 24 + 4 * 8
        self.root = self._entry(root)

    # ----------------------------------------------------------------- low level
    def _u(self, off, n):
        return int.from_bytes(self.b[off:off + n], 'little')

    def _entry(self, off):
        """Symbol table entry: (name offset, object header address, cache type, scratch)."""
        name_off = self._u(off, 8)
        header = self._u(off + 8, 8)
        cache = self._u(off + 16, 4)
        scratch = (self._u(off + 24, 8), self._u(off + 32, 8))
        return name_off, header, cache, scratch

    def _messages(self, addr):
        """Messages of a version-1 object header: list of (type, data offset, size)."""
        b = self.b
        if b[addr] != 1:
            raise ValueError(f'object header version {b[addr]} not supported')
        nmsg = self._u(addr + 2, 2)
        size = self._u(addr + 8, 4)
        blocks = [(addr + 16, size)]
        out = []
        while blocks and len(out) < nmsg:
            start, length = blocks.pop(0)
            off = start
            while off + 8 <= start + length and len(out) < nmsg:
                mtype = self._u(off, 2)
                msize = self._u(off + 2, 2)
                data = off + 8
                if mtype == 0x10:                                  # continuation
                    blocks.append((self._u(data, 8), self._u(data + 8, 8)))
                out.append((mtype, data, msize))
                off = data + msize
        return out

    def _heap_name(self, heap, name_off):
        if self.b[heap:heap + 4] != b'HEAP':
            raise ValueError('local heap signature')
        data = self._u(heap + 24, 8)
        s = data + name_off
        e = self.b.index(b'\x00', s)
        return self.b[s:e].decode()

    def _group_members(self, btree, heap):
        """Walk a group B-tree: {name: object header address}."""
        out = {}
        b = self.b
        if b[btree:btree + 4] != b'TREE':
            raise ValueError('group B-tree signature')
        level = b[btree + 5]
        used = self._u(btree + 6, 2)
        off = btree + 8 + 16                                       # after siblings
        children = []
        for _ in range(used):
            off += 8                                               # key (heap offset)
            children.append(self._u(off, 8))
            off += 8
        for ch in children:
            if level > 0:
                out.update(self._group_members(ch, heap))
                continue
            if b[ch:ch + 4] != b'SNOD':
                raise ValueError('symbol node signature')
            n = self._u(ch + 6, 2)
            for i in range(n):
                name_off, header, _, _ = self._entry(ch + 8 + 40 * i)
                out[self._heap_name(heap, name_off)] = header
        return out

    def _resolve(self, path):
        addr = self.root[1]
        for part in [p for p in path.strip('/').split('/') if p]:
            tab = self._symbol_table(addr)
            if tab is None:
                raise KeyError(path)
            members = self._group_members(*tab)
            if part not in members:
                raise KeyError(path)
            addr = members[part]
        return addr

    def _symbol_table(self, addr):
        for mtype, data, _ in self._messages(addr):
            if mtype == 0x11:
                return self._u(data, 8), self._u(data + 8, 8)
        return None

    # ---------------------------------------------------------------- public
    def keys(self, path=''):
        tab = self._symbol_table(self._resolve(path))
        if tab is None:
            raise KeyError(f'{path} is not a group')
        return sorted(self._group_members(*tab))

    def attrs(self, path=''):
        """Attributes of an object: {name: value} (strings decoded, numbers as numpy values)."""
        out = {}
        for mtype, d, _ in self._messages(self._resolve(path)):
            if mtype != 0x0C:
                continue
            ver = self.b[d]
            nlen, tlen, slen = self._u(d + 2, 2), self._u(d + 4, 2), self._u(d + 6, 2)
            pad = (lambda x: (x + 7) // 8 * 8) if ver == 1 else (lambda x: x)
            off = d + 8 + (1 if ver == 3 else 0)
            name = self.b[off:off + nlen].split(b'\x00')[0].decode()
            off += pad(nlen)
            vlen = self.b[off] & 0x0F == 9
            dt = np.dtype([('len', '<u4'), ('addr', '<u8'), ('idx', '<u4')]) if vlen else self._datatype(off)
            off += pad(tlen)
            shape = self._dataspace(off)
            off += pad(slen)
            n = int(np.prod(shape)) if shape else 1
            val = np.frombuffer(self.b, dt, n, off)
            if vlen:                                               # variable-length strings
                val = [self._global_heap(int(e['addr']), int(e['idx']))[:int(e['len'])].decode() for e in val]
                out[name] = val[0] if not shape else val
                continue
            if dt.kind == 'S':
                val = [v.split(b'\x00')[0].decode() for v in val]
                out[name] = val[0] if not shape else val
            else:
                out[name] = val[0] if not shape else val.reshape(shape).copy()
        return out

    def read(self, path):
        addr = self._resolve(path)
        shape = dtype = layout = None
        filters = []
        for mtype, data, size in self._messages(addr):
            if mtype == 0x01:
                shape = self._dataspace(data)
            elif mtype == 0x03:
                dtype = self._datatype(data)
            elif mtype == 0x08:
                layout = self._layout(data)
            elif mtype == 0x0B:
                filters = self._filters(data)
        if shape is None or dtype is None or layout is None:
            raise ValueError(f'{path} is not a dataset')
        n = int(np.prod(shape)) if shape else 1
        if layout[0] == 'contiguous':
            addr_d, size_d = layout[1], layout[2]
            if addr_d == UNDEF:
                return np.zeros(shape, dtype)
            return np.frombuffer(self.b, dtype, n, addr_d).reshape(shape).copy()
        if layout[0] == 'compact':
            return np.frombuffer(layout[1], dtype, n).reshape(shape).copy()
        _, btree, cdims = layout
        out = np.zeros(shape, dtype)
        es = dtype.itemsize
        for offs, mask, caddr, csize in self._chunks(btree, len(cdims)):
            raw = self.b[caddr:caddr + csize]
            for i in reversed(range(len(filters))):
                if mask >> i & 1:
                    continue
                fid, cd = filters[i]
                if fid == 1:
                    raw = zlib.decompress(raw)
                elif fid == 2:
                    m = len(raw) // es
                    raw = np.frombuffer(raw, np.uint8).reshape(es, m).T.tobytes()
                elif fid == 3:
                    raw = raw[:-4]
                else:
                    raise ValueError(f'filter {fid} not supported')
            chunk = np.frombuffer(raw, dtype, int(np.prod(cdims))).reshape(cdims)
            sl = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, cdims, shape))
            out[sl] = chunk[tuple(slice(0, x.stop - x.start) for x in sl)]
        return out

    # ---------------------------------------------------------------- messages
    def _dataspace(self, d):
        b = self.b
        ver, rank, flags = b[d], b[d + 1], b[d + 2]
        off = d + 8 if ver == 1 else d + 4
        return tuple(self._u(off + 8 * i, 8) for i in range(rank))

    def _datatype(self, d):
        b = self.b
        cls, bits0 = b[d] & 0x0F, b[d + 1]
        size = self._u(d + 4, 4)
        order = '>' if bits0 & 1 else '<'
        if cls == 1:
            return np.dtype(f'{order}f{size}')
        if cls == 0:
            return np.dtype(f'{order}{"i" if bits0 & 8 else "u"}{size}')
        if cls == 3:
            return np.dtype(f'S{size}')
        if cls == 6:                                               # compound, version 1 members
            nmem = self._u(d + 1, 2)
            off, fields = d + 8, []
            for _ in range(nmem):
                e = self.b.index(b'\x00', off)
                name = self.b[off:e].decode()
                off += (e - off + 1 + 7) // 8 * 8
                moff = self._u(off, 4)
                off += 4 + 1 + 3 + 4 + 4 + 16
                mt = self._datatype(off)
                fields.append((name, mt, moff))
                off += self._dtype_msg_size(off)
            return np.dtype({'names': [f[0] for f in fields], 'formats': [f[1] for f in fields],
                             'offsets': [f[2] for f in fields], 'itemsize': size})
        raise ValueError(f'datatype class {cls} not supported')

    def _global_heap(self, addr, index):
        """Object `index` of the global heap collection at `addr`."""
        if self.b[addr:addr + 4] != b'GCOL':
            raise ValueError('global heap signature')
        end = addr + self._u(addr + 8, 8)
        off = addr + 16
        while off + 16 <= end:
            idx, size = self._u(off, 2), self._u(off + 8, 8)
            if idx == index:
                return self.b[off + 16:off + 16 + size]
            if idx == 0:
                break
            off += 16 + (size + 7) // 8 * 8
        raise KeyError(f'global heap object {index}')

    def _dtype_msg_size(self, d):
        cls = self.b[d] & 0x0F
        return 8 + {0: 4, 1: 12, 3: 0}[cls]

    def _layout(self, d):
        b = self.b
        if b[d] != 3:
            raise ValueError(f'layout message version {b[d]} not supported')
        cls = b[d + 1]
        if cls == 0:
            size = self._u(d + 2, 2)
            return ('compact', self.b[d + 4:d + 4 + size])
        if cls == 1:
            return ('contiguous', self._u(d + 2, 8), self._u(d + 10, 8))
        if cls == 2:
            dim = b[d + 2]                                       # rank + 1 (element size last)
            btree = self._u(d + 3, 8)
            cdims = tuple(self._u(d + 11 + 4 * i, 4) for i in range(dim - 1))
            return ('chunked', btree, cdims)
        raise ValueError(f'layout class {cls} not supported')

    def _filters(self, d):
        b = self.b
        ver, nf = b[d], b[d + 1]
        off = d + 8 if ver == 1 else d + 2
        out = []
        for _ in range(nf):
            fid = self._u(off, 2)
            if ver == 1 or fid >= 256:
                nlen = self._u(off + 2, 2)
                flags, ncd = self._u(off + 4, 2), self._u(off + 6, 2)
                off += 8 + ((nlen + 7) // 8 * 8 if ver == 1 else nlen)
            else:
                flags, ncd = self._u(off + 2, 2), self._u(off + 4, 2)
                off += 6
            cd = [self._u(off + 4 * i, 4) for i in range(ncd)]
            off += 4 * ncd
            if ver == 1 and ncd % 2:
                off += 4
            out.append((fid, cd))
        return out

    def _chunks(self, btree, rank):
        """Raw-data B-tree: (chunk offsets, filter mask, address, stored size) per chunk."""
        b = self.b
        if b[btree:btree + 4] != b'TREE' or b[btree + 4] != 1:
            raise ValueError('chunk B-tree signature')
        level = b[btree + 5]
        used = self._u(btree + 6, 2)
        ksize = 8 + 8 * (rank + 1)
        off = btree + 24
        out = []
        for _ in range(used):
            csize = self._u(off, 4)
            mask = self._u(off + 4, 4)
            offs = tuple(self._u(off + 8 + 8 * i, 8) for i in range(rank))
            child = self._u(off + ksize, 8)
            if level > 0:
                out.extend(self._chunks(child, rank))
            else:
                out.append((offs, mask, child, csize))
            off += ksize + 8
        return out
