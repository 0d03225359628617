"""Reader of the grid geometry files (VTK ImageData, ``.vti``) that DAMASK_grid takes.

Follows the reference reader (src/grid/VTI.cpp:45-445): an ImageData in little-endian
byte order, optionally vtkZLibDataCompressor-compressed, with UInt32 or UInt64 block
headers; ``WholeExtent`` starts at 0 and gives the cells, ``Spacing`` times the cells
gives the physical size; ``Direction`` must be the identity; cell data arrays are
binary (base64).  Cell data come back in the file's order, x fastest, which is the
voxel order of the solver.
"""
from __future__ import annotations

import base64
import re
import xml.etree.ElementTree as ET
import zlib
from dataclasses import dataclass, field

import numpy as np

_VTK_TYPES = {'Int8': '<i1', 'UInt8': '<u1', 'Int16': '<i2', 'UInt16': '<u2', 'Int32': '<i4', 'UInt32': '<u4',
              'Int64': '<i8', 'UInt64': '<u8', 'Float32': '<f4', 'Float64': '<f8'}


class VTIError(ValueError):
    pass


@dataclass
class Geometry:
    cells: tuple
    size: tuple
    origin: tuple
    cell_data: dict = field(default_factory=dict)

    @property
    def material(self) -> np.ndarray:
        """0-based material index of every cell (the 'material' cell array)."""
        if 'material' not in self.cell_data:
            raise VTIError("no DataArray with Name='material' found")
        return self.cell_data['material'].astype(np.int32)


def _b64(text: str) -> bytes:
    # header and payload are base64-encoded separately and concatenated, padding included
    text = re.sub(r'\s+', '', text)
    return b''.join(base64.b64decode(seg) for seg in re.findall(r'[A-Za-z0-9+/]+={0,2}', text))


def _decode(text: str, compressed: bool, word: int) -> bytes:
    raw = _b64(text)
    fmt = '<u4' if word == 4 else '<u8'
    if compressed:
        if len(raw) < 3 * word:
            raise VTIError('header for compressed VTI too short')
        nblocks, bsize, last = (int(x) for x in np.frombuffer(raw[:3 * word], fmt))
        hsize = (3 + nblocks) * word
        if len(raw) < hsize:
            raise VTIError('missing header for compressed VTI')
        sizes = [int(x) for x in np.frombuffer(raw[3 * word:hsize], fmt)]
        out, off = [], hsize
        for i, cs in enumerate(sizes):
            if off + cs > len(raw):
                raise VTIError(f'invalid VTI, defined size overflowing for block {i}')
            want = last if (i + 1 == nblocks and last > 0) else bsize
            blk = zlib.decompress(raw[off:off + cs])
            if len(blk) != want:
                raise VTIError(f'zlib inflate failed on block {i}')
            out.append(blk)
            off += cs
        return b''.join(out)
    out, off = [], 0
    while off + word <= len(raw):
        n = int(np.frombuffer(raw[off:off + word], fmt)[0])
        off += word
        if n == 0:
            break
        if off + n > len(raw):
            raise VTIError('VTI uncompressed: data block exceeds payload')
        out.append(raw[off:off + n])
        off += n
    return b''.join(out)


def load_native(path, int_labels=('material',)) -> Geometry:
    """The same file through the library's C++ reader (dmk_vti_*, the counterpart of the
    reference's src/grid/VTI.cpp): arrays named in int_labels come back as int64, the others
    as float64."""
    import ctypes as C
    from . import _lib
    lib = _lib.load()
    h = C.c_void_p()
    rc = lib.dmk_vti_open(str(path).encode(), C.byref(h))
    if rc != 0:
        raise VTIError(lib.dmk_last_error().decode())
    try:
        cells = (C.c_int * 3)()
        size, origin = (C.c_double * 3)(), (C.c_double * 3)()
        lib.dmk_vti_geometry(h, cells, size, origin)
        geom = Geometry(tuple(cells), tuple(size), tuple(origin))
        buf = C.create_string_buffer(256)
        ncomp = C.c_int()
        n = lib.dmk_vti_label(h, 0, buf, 256, C.byref(ncomp))
        N = int(np.prod(geom.cells))
        for i in range(n):
            lib.dmk_vti_label(h, i, buf, 256, C.byref(ncomp))
            name, k = buf.value.decode(), ncomp.value
            if name in int_labels:
                out = np.empty(N * k, np.int64)
                rc = lib.dmk_vti_read_int(h, name.encode(), out.ctypes.data_as(C.POINTER(C.c_int64)), out.size)
            else:
                out = np.empty(N * k, np.float64)
                rc = lib.dmk_vti_read_real(h, name.encode(), out.ctypes.data_as(C.POINTER(C.c_double)), out.size)
            if rc != 0:
                raise VTIError(lib.dmk_last_error().decode())
            geom.cell_data[name] = out.reshape(N, k) if k > 1 else out
        return geom
    finally:
        lib.dmk_vti_close(h)


def load(path) -> Geometry:
    root = ET.parse(path).getroot()
    if root.tag != 'VTKFile':
        raise VTIError('missing <VTKFile> element')
    if root.get('type') != 'ImageData':
        raise VTIError(f"type is not ImageData (got '{root.get('type')}')")
    if root.get('byte_order') != 'LittleEndian':
        raise VTIError(f"byte_order must be 'LittleEndian' (got '{root.get('byte_order')}')")
    comp = root.get('compressor', '')
    if comp and comp != 'vtkZLibDataCompressor':
        raise VTIError(f"compressor is not vtkZLibDataCompressor (got '{comp}')")
    word = 8 if root.get('header_type', 'UInt32') == 'UInt64' else 4
    img = root.find('ImageData')
    if img is None:
        raise VTIError('missing ImageData element')
    d = img.get('Direction', '')
    if d and d.split() != '1 0 0 0 1 0 0 0 1'.split():
        raise VTIError(f"unsupported 'Direction' (got '{d}')")
    ext = [int(x) for x in img.get('WholeExtent', '').split()]
    if len(ext) != 6 or ext[0] != 0 or ext[2] != 0 or ext[4] != 0:
        raise VTIError(f"invalid 'WholeExtent' (got '{img.get('WholeExtent')}')")
    spacing = [float(x) for x in img.get('Spacing').split()]
    origin = tuple(float(x) for x in img.get('Origin', '0 0 0').split())
    cells = (ext[1], ext[3], ext[5])
    size = tuple(s * c for s, c in zip(spacing, cells))
    if min(size) <= 0:
        raise VTIError("one or more entries <= 0 for 'size'")
    if min(cells) < 1:
        raise VTIError("one or more entries < 1 for 'cells'")
    geom = Geometry(cells, size, origin)
    cd = img.find('Piece/CellData')
    if cd is not None:
        for arr in cd.findall('DataArray'):
            name = arr.get('Name')
            if name in geom.cell_data:
                raise VTIError(f"repeated label '{name}'")
            if arr.get('format') != 'binary':
                raise VTIError(f"DataArray '{name}' is not binary")
            t = arr.get('type')
            if t not in _VTK_TYPES:
                raise VTIError(f"unsupported type '{t}' for DataArray '{name}'")
            data = np.frombuffer(_decode(arr.text or '', bool(comp), word), _VTK_TYPES[t])
            ncomp = int(arr.get('NumberOfComponents', '1'))
            n = cells[0] * cells[1] * cells[2]
            if data.size != n * ncomp:
                raise VTIError(f"DataArray '{name}' has {data.size} values for {n} cells")
            geom.cell_data[name] = data.reshape(n, ncomp) if ncomp > 1 else data.copy()
    return geom
