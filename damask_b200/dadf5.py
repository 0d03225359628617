"""Writer of DAMASK's result file (DADF5, an HDF5 file) for the grid solver's outputs.

The layout follows the reference's writer (src/result.f90:85-218 result_init /
result_addIncrement, :479-508 tensor datasets stored transposed, :534-846 the cell_to mappings,
:848-863 executionStamp; discretization.f90:81-96 displacements; discretization_grid.f90:228-240
geometry; phase_mechanical.f90:909-980 and phase_mechanical_plastic_phenopowerlaw.f90:405-439
phase outputs; homogenization_mechanical.f90:196-216):

    /                         DADF5_version_major/minor, creator, created, call, solver, job_name
    /geometry                 cells, size, origin (datasets with units; also as attributes)
    /cell_to/phase            (N, 1) {label, entry}; /cell_to/homogenization (N,) {label, entry}
    /setup/<file>             the input files' text
    /increment_<i>            attribute t/s
        geometry/u_p, u_n     displacements of cell centres and nodes
        phase/<name>/mechanical/<output>
        homogenization/<name>/mechanical/<output>

Every dataset carries the creator / created / description / unit attributes; slip outputs carry
their 'systems' labels.  String attributes are variable-length (global heap), as the reference's
are.  Differences in storage only: datasets are contiguous, without the reference's chunking,
shuffle/deflate and Fletcher-32 filters (readers see the same data), and the 'current' soft link
to the latest increment, which the reference uses while writing, is not stored.

The HDF5 subset written is what libhdf5 writes for these files with its default (earliest)
format: superblock version 0, version-1 object headers, groups as symbol tables (version-1
B-tree + local heap + symbol table nodes), attribute messages version 1, global heap collections
for variable-length strings.  It is written from the public HDF5 file-format specification.
"""
from __future__ import annotations

import struct
import time
from pathlib import Path

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
_SIG = b'\x89HDF\r\n\x1a\n'
_LEAF_K, _INTERNAL_K = 4, 16                  # group leaf / internal node K of the superblock
_SNOD_SIZE = 8 + 2 * _LEAF_K * 40
_BTREE_SIZE = 24 + (2 * _INTERNAL_K + 1) * 8 + 2 * _INTERNAL_K * 8
_HEAP_FREE_NULL = 1                           # end of a local heap's free list


def _pad8(b: bytes) -> bytes:
    return b + b'\0' * (-len(b) % 8)


# ------------------------------------------------------------------------------ messages
def _dt_float(size: int) -> bytes:
    if size == 8:
        return bytes([0x11, 0x20, 63, 0]) + struct.pack('<IHHBBBBI', 8, 0, 64, 52, 11, 0, 52, 1023)
    return bytes([0x11, 0x20, 31, 0]) + struct.pack('<IHHBBBBI', 4, 0, 32, 23, 8, 0, 23, 127)


def _dt_int(size: int, signed: bool) -> bytes:
    return bytes([0x10, 0x08 if signed else 0x00, 0, 0]) + struct.pack('<IHH', size, 0, 8 * size)


def _dt_fixed_string(size: int, space_pad: bool = False) -> bytes:
    return bytes([0x13, 0x02 if space_pad else 0x00, 0, 0]) + struct.pack('<I', size)


def _dt_vlen_string() -> bytes:
    return bytes([0x19, 0x01, 0, 0]) + struct.pack('<I', 16) + _dt_int(1, False)


def _dt_numpy(dt: np.dtype) -> bytes:
    dt = np.dtype(dt)
    if dt.names:                                            # compound, version-1 members
        body = b''
        for name in dt.names:
            ft, off = dt.fields[name][:2]
            # string members space-padded, as the reference's Fortran character labels
            mt = _dt_fixed_string(ft.itemsize, space_pad=True) if ft.kind == 'S' else _dt_numpy(ft)
            body += _pad8(name.encode() + b'\0') + struct.pack('<IB3xI4x16x', off, 0, 0) + mt
        return bytes([0x16, len(dt.names) & 0xFF, len(dt.names) >> 8, 0]) + struct.pack('<I', dt.itemsize) + body
    if dt.kind == 'f':
        return _dt_float(dt.itemsize)
    if dt.kind in 'iu':
        return _dt_int(dt.itemsize, dt.kind == 'i')
    if dt.kind == 'S':
        return _dt_fixed_string(dt.itemsize)
    raise TypeError(f'unsupported dtype {dt}')


def _dataspace(shape: tuple, with_max: bool = True) -> bytes:
    if not shape:
        return bytes([1, 0, 0, 0, 0, 0, 0, 0])
    flags = 1 if with_max else 0
    b = bytes([1, len(shape), flags, 0, 0, 0, 0, 0]) + b''.join(struct.pack('<Q', int(n)) for n in shape)
    if with_max:
        b += b''.join(struct.pack('<Q', int(n)) for n in shape)
    return b


def _message(mtype: int, data: bytes, flags: int = 0) -> bytes:
    data = _pad8(data)
    return struct.pack('<HHB3x', mtype, len(data), flags) + data


def _object_header(messages: list[bytes]) -> bytes:
    body = b''.join(messages)
    return struct.pack('<BBHII4x', 1, 0, len(messages), 1, len(body)) + body


# ------------------------------------------------------------------------------ tree
class _Node:
    def __init__(self):
        self.attrs: list[tuple[str, object]] = []
        self.addr = None

    def set_attr(self, name: str, value) -> None:
        self.attrs = [(n, v) for n, v in self.attrs if n != name] + [(name, value)]


class _Group(_Node):
    def __init__(self):
        super().__init__()
        self.children: dict[str, _Node] = {}


class _Dataset(_Node):
    def __init__(self, shape, dtype_msg, data_addr, nbytes):
        super().__init__()
        self.shape, self.dtype_msg, self.data_addr, self.nbytes = shape, dtype_msg, data_addr, nbytes


class H5Writer:
    """Minimal HDF5 writer: groups, contiguous datasets, attributes.  Dataset contents go to the
    file when they are added; the metadata (object headers, group indices, global heap) is
    written by close()."""

    def __init__(self, path):
        self.path = Path(path)
        self.fh = open(self.path, 'wb')
        self.fh.write(b'\0' * 96)                            # superblock, written by close()
        self.eof = 96
        self.root = _Group()

    def _node(self, path: str, create: bool = True) -> _Group:
        g = self.root
        for part in [p for p in path.strip('/').split('/') if p]:
            if part not in g.children:
                if not create:
                    raise KeyError(path)
                g.children[part] = _Group()
            g = g.children[part]
            if not isinstance(g, _Group):
                raise KeyError(f'{path} is not a group')
        return g

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        if not self.fh.closed:
            self.close()

    def group(self, path: str) -> _Group:
        return self._node(path)

    def dataset(self, path: str, data: np.ndarray, attrs: dict | None = None) -> None:
        parent, _, name = path.strip('/').rpartition('/')
        g = self._node(parent)
        a = np.ascontiguousarray(data)
        if a.dtype.byteorder == '>':
            a = a.astype(a.dtype.newbyteorder('<'))
        raw = a.tobytes()
        self.fh.write(raw)
        ds = _Dataset(a.shape, _dt_numpy(a.dtype), self.eof if raw else UNDEF, len(raw))
        self.eof += len(raw)
        for k, v in (attrs or {}).items():
            ds.set_attr(k, v)
        g.children[name] = ds

    def attrs(self, path: str, values: dict) -> None:
        node = self.root
        for part in [p for p in path.strip('/').split('/') if p]:
            node = node.children[part]
        for k, v in values.items():
            node.set_attr(k, v)

    # -------------------------------------------------------------- serialisation
    def close(self) -> None:
        strings: list[bytes] = []                             # global heap objects (vlen strings)

        def attr_message(name: str, value, refs: list) -> tuple[bytes, bytes]:
            if isinstance(value, str) or (isinstance(value, (list, tuple)) and value and isinstance(value[0], str)):
                vals = [value] if isinstance(value, str) else list(value)
                shape = () if isinstance(value, str) else (len(vals),)
                dt = _dt_vlen_string()
                data = b''
                for v in vals:
                    raw = v.encode()
                    strings.append(raw)
                    refs.append(len(data))                     # patched with the heap address later
                    data += struct.pack('<IQI', len(raw), 0, len(strings))
            else:
                # Python int/bool -> 32-bit integer, float -> double; numpy values keep their type
                if isinstance(value, (bool, int)):
                    a = np.asarray(int(value), '<i4')
                elif isinstance(value, float):
                    a = np.asarray(value, '<f8')
                else:
                    a = np.asarray(value)
                    a = a.astype(a.dtype.newbyteorder('<'))
                shape = a.shape
                dt = _dt_numpy(a.dtype)
                data = np.ascontiguousarray(a).tobytes()
            ds = _dataspace(shape)
            nm = name.encode() + b'\0'
            head = struct.pack('<BBHHH', 1, 0, len(nm), len(dt), len(ds))
            return head + _pad8(nm) + _pad8(dt) + _pad8(ds), data

        # pass 1: sizes and addresses of every metadata block
        blocks = []                                           # (node, kind, size)
        plans = {}

        def plan(node, name_heap=None):
            amsgs = []
            for n, v in node.attrs:
                refs = []
                head, data = attr_message(n, v, refs)
                amsgs.append((head, data, refs, len(strings)))
            if isinstance(node, _Group):
                names = sorted(node.children)
                heap = b'\0' * 8
                offsets = {}
                for n in names:
                    offsets[n] = len(heap)
                    heap += _pad8(n.encode() + b'\0')
                leaves = [names[i:i + 2 * _LEAF_K] for i in range(0, len(names), 2 * _LEAF_K)]
                # B-tree nodes per level (level 0 points at the symbol nodes); an empty group
                # has one node without entries
                levels = [max(1, (len(leaves) + 2 * _INTERNAL_K - 1) // (2 * _INTERNAL_K))]
                while levels[-1] > 1:
                    levels.append((levels[-1] + 2 * _INTERNAL_K - 1) // (2 * _INTERNAL_K))
                nbtree = sum(levels)
                plans[id(node)] = dict(attrs=amsgs, names=names, heap=heap, offsets=offsets, leaves=leaves,
                                       nbtree=nbtree)
                for n in names:
                    plan(node.children[n])
            else:
                plans[id(node)] = dict(attrs=amsgs)

        plan(self.root)
        # string references must be patched once the heap collections have addresses: lay the
        # collections out first (objects 1..n, split so that indices stay below 2^16)
        coll_objs = [strings[i:i + 60000] for i in range(0, len(strings), 60000)]
        coll_sizes = []
        for objs in coll_objs:
            size = 16 + sum(16 + (len(s) + 7) // 8 * 8 for s in objs) + 16
            coll_sizes.append(max(4096, (size + 7) // 8 * 8))
        addr = self.eof
        coll_addr = []
        for sz in coll_sizes:
            coll_addr.append(addr)
            addr += sz

        def header_bytes(node, addrs):
            p = plans[id(node)]
            msgs = []
            if isinstance(node, _Group):
                msgs.append(_message(0x11, struct.pack('<QQ', addrs['btree'], addrs['heap'])))
            else:
                msgs.append(_message(0x01, _dataspace(node.shape)))
                msgs.append(_message(0x03, node.dtype_msg, flags=1))
                msgs.append(_message(0x05, bytes([2, 2, 2, 0])))          # fill value: late, if set, undefined
                msgs.append(_message(0x08, bytes([3, 1]) + struct.pack('<QQ', node.data_addr, node.nbytes)))
            for head, data, refs, last in p['attrs']:
                data = bytearray(data)
                for k, off in enumerate(refs):
                    obj = last - len(refs) + k                          # 0-based global object number
                    ci, oi = divmod(obj, 60000)
                    struct.pack_into('<QI', data, off + 4, coll_addr[ci], oi + 1)
                msgs.append(_message(0x0C, head + bytes(data)))
            return _object_header(msgs)

        # pass 2: assign addresses (headers need only sizes, which do not depend on addresses)
        order = []

        def assign(node):
            nonlocal addr
            p = plans[id(node)]
            dummy = {'btree': 0, 'heap': 0}
            size = len(header_bytes(node, dummy))
            node.addr = addr
            addr += size
            if isinstance(node, _Group):
                p['heap_addr'] = addr
                addr += 32
                p['heap_data'] = addr
                addr += len(p['heap'])
                p['btree_addr'] = []
                for _ in range(p['nbtree']):
                    p['btree_addr'].append(addr)
                    addr += _BTREE_SIZE
                p['snod_addr'] = []
                for _ in p['leaves']:
                    p['snod_addr'].append(addr)
                    addr += _SNOD_SIZE
                for n in p['names']:
                    assign(node.children[n])
            order.append(node)

        assign(self.root)
        out = bytearray(addr - self.eof)

        def put(at, b):
            out[at - self.eof:at - self.eof + len(b)] = b

        # global heap collections
        k = 0
        for ci, objs in enumerate(coll_objs):
            b = b'GCOL' + bytes([1, 0, 0, 0]) + struct.pack('<Q', coll_sizes[ci])
            for oi, s in enumerate(objs):
                b += struct.pack('<HH4xQ', oi + 1, 0, len(s)) + _pad8(s)
                k += 1
            free = coll_sizes[ci] - len(b)
            b += struct.pack('<HH4xQ', 0, 0, free) + b'\0' * (free - 16)
            put(coll_addr[ci], b)

        def entry(name_off, node):
            if isinstance(node, _Group):
                p = plans[id(node)]
                return struct.pack('<QQII', name_off, node.addr, 1, 0) + struct.pack('<QQ', p['btree_addr'][-1],
                                                                                     p['heap_addr'])
            return struct.pack('<QQII', name_off, node.addr, 0, 0) + b'\0' * 16

        for node in order:
            p = plans[id(node)]
            if not isinstance(node, _Group):
                put(node.addr, header_bytes(node, {}))
                continue
            put(node.addr, header_bytes(node, {'btree': p['btree_addr'][-1], 'heap': p['heap_addr']}))
            put(p['heap_addr'], b'HEAP' + bytes([0, 0, 0, 0]) +
                struct.pack('<QQQ', len(p['heap']), _HEAP_FREE_NULL, p['heap_data']))
            put(p['heap_data'], p['heap'])
            # symbol table nodes
            for leaf, at in zip(p['leaves'], p['snod_addr']):
                b = b'SNOD' + bytes([1, 0]) + struct.pack('<H', len(leaf))
                for n in leaf:
                    b += entry(p['offsets'][n], node.children[n])
                put(at, b + b'\0' * (_SNOD_SIZE - len(b)))
            # B-tree: level 0 points at the symbol nodes; keys are heap offsets of the last name
            # of the preceding child (key 0: the empty name at offset 0)
            # of the preceding child (key 0: the empty name at offset 0).  Nodes are written level
            # by level; the last one is the root.
            children = [(at, p['offsets'][leaf[-1]]) for leaf, at in zip(p['leaves'], p['snod_addr'])]
            free_nodes = iter(p['btree_addr'])
            level = 0
            while True:
                groups = [children[i:i + 2 * _INTERNAL_K] for i in range(0, len(children), 2 * _INTERNAL_K)] or [[]]
                nxt = []
                for grp in groups:
                    at = next(free_nodes)
                    b = b'TREE' + bytes([0, level]) + struct.pack('<HQQ', len(grp), UNDEF, UNDEF)
                    b += struct.pack('<Q', 0)
                    for child, last in grp:
                        b += struct.pack('<QQ', child, last)
                    put(at, b + b'\0' * (_BTREE_SIZE - len(b)))
                    nxt.append((at, grp[-1][1] if grp else 0))
                if len(nxt) == 1:
                    break
                children = nxt
                level += 1
            if nxt[0][0] != p['btree_addr'][-1]:
                raise AssertionError('B-tree root placement')

        self.fh.write(bytes(out))
        # superblock version 0 with the root group's symbol table entry
        rp = plans[id(self.root)]
        sb = _SIG + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack('<HHI', _LEAF_K, _INTERNAL_K, 0)
        sb += struct.pack('<QQQQ', 0, UNDEF, addr, UNDEF)
        sb += struct.pack('<QQII', 0, self.root.addr, 1, 0) + struct.pack('<QQ', rp['btree_addr'][-1], rp['heap_addr'])
        self.fh.seek(0)
        self.fh.write(sb)
        self.fh.close()


# ------------------------------------------------------------------------------ DADF5
def now() -> str:
    """Date and time as the reference's now() (result.f90:869-880): YYYY-MM-DD HH:MM:SS+zzzz."""
    t = time.localtime()
    off = -time.altzone if t.tm_isdst > 0 else -time.timezone
    return time.strftime('%Y-%m-%d %H:%M:%S', t) + f'{"+" if off >= 0 else "-"}{abs(off) // 3600:02d}{abs(off) % 3600 // 60:02d}'


DESCRIPTIONS = {
    'F': ('deformation gradient', '1'), 'F_e': ('elastic deformation gradient', '1'),
    'F_p': ('plastic deformation gradient', '1'), 'F_i': ('inelastic deformation gradient', '1'),
    'L_p': ('plastic velocity gradient', '1/s'), 'L_i': ('inelastic velocity gradient', '1/s'),
    'P': ('first Piola-Kirchhoff stress', 'Pa'), 'S': ('second Piola-Kirchhoff stress', 'Pa'),
    'O': ('crystal orientation as quaternion q_0 (q_1 q_2 q_3)', '1'),
    'xi_sl': ('resistance against plastic slip', 'Pa'), 'gamma_sl': ('plastic shear', '1'),
}
TENSORS = ('F', 'F_e', 'F_p', 'F_i', 'L_p', 'L_i', 'P', 'S')


def slip_labels(directions: np.ndarray, planes: np.ndarray) -> list[str]:
    """crystal_labels_slip (crystal.f90:1642-1676, getlabels :2133-2181): '[d1 d2 d3](n1 n2 n3)',
    each index right-aligned in two characters."""
    def fmt(v):
        return ' '.join(f'{int(round(x)):2d}' for x in v)
    return [f'[{fmt(d)}]({fmt(n)})' for d, n in zip(directions, planes)]


class ResultFile:
    """DADF5 result file of a grid job with one phase and one homogenization (isostrain, one
    constituent per cell)."""

    def __init__(self, path, cells, size, phase_name: str, phase_lattice: str, homogenization_name: str = 'SX',
                 origin=(0.0, 0.0, 0.0), setup_files: dict | None = None, call: str = '',
                 creator: str = 'damask_b200', job_name: str = ''):
        self.w = H5Writer(path)
        self.cells = tuple(int(c) for c in cells)
        self.N = int(np.prod(self.cells))
        self.phase, self.lattice, self.homog = phase_name, phase_lattice, homogenization_name
        self.creator = creator
        w = self.w
        w.attrs('/', {'DADF5_version_major': 1, 'DADF5_version_minor': 4, 'creator': creator, 'created': now(),
                      'call': call, 'solver': 'grid', 'job_name': job_name or Path(path).stem})
        w.group('geometry')
        w.dataset('geometry/cells', np.asarray(self.cells, '<i4'), {'unit': '1'})
        w.dataset('geometry/size', np.asarray(size, '<f8'), {'unit': 'm³'})
        w.dataset('geometry/origin', np.asarray(origin, '<f8'), {'unit': 'm'})
        w.attrs('geometry', {'cells': np.asarray(self.cells, '<i4'), 'size': np.asarray(size, '<f8'),
                             'origin': np.asarray(origin, '<f8')})
        w.group('cell_to')
        w.attrs('cell_to', {'description': 'mappings to place data in space'})
        created = now()
        lp = max(len(phase_name), 1)
        ph = np.zeros((self.N, 1), np.dtype([('label', f'S{lp}'), ('entry', '<i8')]))
        ph['label'] = phase_name.encode()
        ph['entry'][:, 0] = np.arange(self.N)
        w.dataset('cell_to/phase', ph, self._stamp('cell ID and constituent ID to phase results', None, created))
        lh = max(len(homogenization_name), 1)
        ho = np.zeros(self.N, np.dtype([('label', f'S{lh}'), ('entry', '<i8')]))
        ho['label'] = homogenization_name.encode()
        ho['entry'] = np.arange(self.N)
        w.dataset('cell_to/homogenization', ho, self._stamp('cell ID to homogenization results', None, created))
        w.group('setup')
        w.attrs('setup', {'description': 'input data used to run the simulation'})
        for name, (text, description) in (setup_files or {}).items():
            raw = text.encode()
            w.dataset(f'setup/{name}', np.array([raw], f'S{max(len(raw), 1)}'),
                      self._stamp(description, None, created))

    def _stamp(self, description, unit, created=None):
        a = {'creator': f'{self.creator}', 'created': created or now(), 'description': description}
        if unit is not None:
            a['unit'] = unit
        return a

    def add_increment(self, inc: int, t: float, phase_outputs: dict, homogenization_outputs: dict | None = None,
                      u_p: np.ndarray | None = None, u_n: np.ndarray | None = None,
                      systems_sl: list[str] | None = None) -> None:
        """Outputs of increment `inc` at time t: per-voxel arrays (N, 9) for tensors in the solver's
        column-major component order, (N, 4) for O, (N, Ns) for xi_sl / gamma_sl."""
        w, g = self.w, f'increment_{inc}'
        w.group(g)
        w.attrs(g, {'t/s': float(t)})
        created = now()
        w.group(f'{g}/geometry')
        if u_n is not None:
            w.dataset(f'{g}/geometry/u_n', np.asarray(u_n, '<f8'), self._stamp('displacements of the nodes', 'm', created))
        if u_p is not None:
            w.dataset(f'{g}/geometry/u_p', np.asarray(u_p, '<f8'),
                      self._stamp('displacements of the materialpoints (cell centers)', 'm', created))
        base = f'{g}/phase/{self.phase}/mechanical'
        w.group(base)
        for label, data in phase_outputs.items():
            desc, unit = DESCRIPTIONS[label]
            attrs = self._stamp(desc, unit, created)
            a = np.asarray(data, '<f8')
            if label in TENSORS:
                # input: column-major components per voxel.  The reference stores each tensor
                # transposed from a (3,3,N) Fortran array, which reads as (N, 3, 3) with
                # [n, i, j] = T_ij.
                a = a.reshape(-1, 3, 3).transpose(0, 2, 1)
            if label == 'O':
                attrs['lattice'] = self.lattice
            if label in ('xi_sl', 'gamma_sl') and systems_sl is not None:
                attrs['systems'] = list(systems_sl)
            w.dataset(f'{base}/{label}', a, attrs)
        hbase = f'{g}/homogenization/{self.homog}/mechanical'
        w.group(hbase)
        for label, data in (homogenization_outputs or {}).items():
            desc, unit = DESCRIPTIONS[label]
            w.dataset(f'{hbase}/{label}', np.asarray(data, '<f8').reshape(-1, 3, 3).transpose(0, 2, 1),
                      self._stamp(desc, unit, created))

    def close(self) -> None:
        self.w.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        if not self.w.fh.closed:
            self.close()


def phase_systems(phase) -> list[str]:
    """'systems' labels of the slip outputs of a phase (config.Phase)."""
    import ctypes as C
    from . import _lib
    lib = _lib.load()
    out = (C.c_int * (6 * max(phase.n_slip, 1)))()
    ns = lib.dmk_phase_slip_systems(C.byref(phase.to_struct()), out)
    _lib.check(min(ns, 0))
    m = np.array(out[:6 * ns]).reshape(ns, 6)
    return slip_labels(m[:, :3], m[:, 3:])


PHASE_OUTPUTS = ('F', 'F_e', 'F_p', 'L_p', 'P', 'S', 'O', 'xi_sl', 'gamma_sl')


def write_increment(rf: ResultFile, solver, inc: int, t: float, phase_outputs=PHASE_OUTPUTS,
                    homogenization_outputs=('F', 'P'), systems_sl: list[str] | None = None) -> None:
    """materialpoint_result + discretization_result of one increment from a solver object
    (SpectralBasic, SpectralPolarization or the oracle): the requested phase outputs, the
    homogenization's F and P (isostrain with one constituent: the phase's) and u_p / u_n."""
    from .grid import displacements
    ip, nodes = solver.get_coords()
    u_p, u_n = displacements(solver.cells, solver.size, ip, nodes)
    ph = {k: solver.get_field(k) for k in phase_outputs}
    ho = {k: solver.get_field(k) for k in homogenization_outputs}
    rf.add_increment(inc, t, ph, ho, u_p=u_p, u_n=u_n, systems_sl=systems_sl)
