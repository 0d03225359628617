"""The library's C++ .vti reader (dmk_vti_*, counterpart of the reference's src/grid/VTI.cpp)
against the known answers of the reference's VTI tests and against the Python reader."""
import base64
import json
import zlib
from pathlib import Path

import numpy as np
import pytest

from damask_b200 import vti

GOLD = Path(__file__).resolve().parent / 'golden' / 'golden_17grains_bcc.npz'


def vti_file(path, cells, arrays, header='UInt32', compressed=False):
    ext = ' '.join(f'0 {c}' for c in cells)
    comp = ' compressor="vtkZLibDataCompressor"' if compressed else ''
    body = ''.join(f'<DataArray type="{t}" Name="{n}" format="binary"{f" NumberOfComponents={chr(34)}{k}{chr(34)}" if k > 1 else ""}>'
                   f'{text}</DataArray>\n' for n, t, k, text in arrays)
    path.write_text(f'<?xml version="1.0"?>\n<VTKFile type="ImageData" version="0.1" byte_order="LittleEndian" '
                    f'header_type="{header}"{comp}>\n<ImageData WholeExtent="{ext}" Origin="0 0 0" Spacing="1e-6 2e-6 3e-6" '
                    f'Direction="1 0 0 0 1 0 0 0 1">\n<Piece Extent="{ext}"><CellData>\n{body}</CellData></Piece>'
                    f'</ImageData></VTKFile>\n')
    return path


def encode(raw: bytes, word: int, compressed: bool, block: int = 64) -> str:
    fmt = '<u4' if word == 4 else '<u8'
    if not compressed:
        return base64.b64encode(np.array([len(raw)], fmt).tobytes()).decode() + base64.b64encode(raw).decode()
    blocks = [zlib.compress(raw[i:i + block]) for i in range(0, len(raw), block)]
    head = np.array([len(blocks), block, len(raw) % block or block] + [len(b) for b in blocks], fmt).tobytes()
    return base64.b64encode(head).decode() + base64.b64encode(b''.join(blocks)).decode()


def test_known_answers_of_the_reference(tmp_path):
    known = json.loads(str(np.load(GOLD)['vti_known_json']))
    for key, (b64, word, compressed, expected) in known.items():
        p = vti_file(tmp_path / f'{key}.vti', (len(expected), 1, 1), [('data', 'UInt8', 1, b64)],
                     header='UInt64' if word == 8 else 'UInt32', compressed=compressed)
        g = vti.load_native(p, int_labels=('data',))
        assert list(g.cell_data['data']) == expected, key


@pytest.mark.parametrize('word,compressed', [(4, False), (8, False), (4, True), (8, True)])
def test_native_equals_python_reader(tmp_path, word, compressed):
    cells = (5, 4, 3)
    rng = np.random.default_rng(word + compressed)
    mat = rng.integers(0, 17, 60).astype('<i8')
    phi = rng.normal(size=(60, 3))
    arrays = [('material', 'Int64', 1, encode(mat.tobytes(), word, compressed)),
              ('phi', 'Float64', 3, encode(phi.tobytes(), word, compressed)),
              ('small', 'Int32', 1, encode(mat.astype('<i4').tobytes(), word, compressed))]
    p = vti_file(tmp_path / 'g.vti', cells, arrays, header='UInt64' if word == 8 else 'UInt32', compressed=compressed)
    a, b = vti.load(p), vti.load_native(p, int_labels=('material', 'small'))
    assert a.cells == b.cells == cells and np.allclose(b.size, (5e-6, 8e-6, 9e-6)) and a.origin == b.origin
    assert np.array_equal(b.cell_data['material'], mat) and np.array_equal(b.cell_data['phi'], phi)
    assert np.array_equal(b.cell_data['small'], mat)
    assert np.array_equal(a.material, b.material)


def test_native_errors(tmp_path):
    p = tmp_path / 'bad.vti'
    p.write_text('<VTKFile type="ImageData" byte_order="LittleEndian"><ImageData WholeExtent="0 1 0 1 0 1" '
                 'Spacing="1 1 1" Direction="0 1 0 1 0 0 0 0 1"/></VTKFile>')
    with pytest.raises(vti.VTIError, match='Direction'):
        vti.load_native(p)
    p.write_text('<VTKFile type="ImageData" byte_order="BigEndian"><ImageData WholeExtent="0 1 0 1 0 1" '
                 'Spacing="1 1 1"/></VTKFile>')
    with pytest.raises(vti.VTIError, match='LittleEndian'):
        vti.load_native(p)
    with pytest.raises(vti.VTIError, match='cannot open'):
        vti.load_native(tmp_path / 'missing.vti')


def test_native_rejects_malformed_attributes(tmp_path):
    """Malformed numbers in the XML come back as errors, not as exceptions across the C-ABI."""
    p = vti_file(tmp_path / 'g.vti', (2, 1, 1), [('material', 'Int64', 1, encode(np.zeros(2, '<i8').tobytes(), 4, False))])
    p.write_text(p.read_text().replace('Name="material"', 'Name="material" NumberOfComponents="many"'))
    with pytest.raises(vti.VTIError, match='invalid VTI'):
        vti.load_native(p)
