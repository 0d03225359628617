"""The HDF5 writer under the DADF5 result file (damask_b200/dadf5.py), read back with the
test-side reader that also reads the reference's own result file."""
import struct

import numpy as np

from damask_b200.dadf5 import H5Writer, ResultFile, slip_labels

from damask_b200.h5read import DADF5


def test_writer_roundtrip(tmp_path):
    p = tmp_path / 't.hdf5'
    w = H5Writer(p)
    w.attrs('/', {'i': 7, 'f': 2.5, 's': 'text', 'ls': ['a', 'bb'], 'arr': np.arange(3, dtype='<i4'),
                  'v': np.array([1.5, -2.0])})
    w.group('empty')
    for i in range(300):                                   # > 256 members: a two-level group B-tree
        w.dataset(f'many/d{i:03d}', np.full((2, 3), float(i)), {'unit': 'Pa', 'k': i})
    rec = np.zeros(5, np.dtype([('label', 'S4'), ('entry', '<i8')]))
    rec['label'], rec['entry'] = b'SX', np.arange(5)
    w.dataset('a/b/comp', rec)
    w.dataset('a/str', np.array([b'line 1\nline 2'], 'S13'))
    w.dataset('a/i4', np.arange(6, dtype='<i4').reshape(2, 3))
    w.close()
    raw = p.read_bytes()
    assert raw[:8] == b'\x89HDF\r\n\x1a\n' and raw[8] == 0 and raw[13:15] == bytes([8, 8])
    assert struct.unpack_from('<Q', raw, 40)[0] == len(raw)          # end-of-file address
    f = DADF5(p)
    assert f.keys() == ['a', 'empty', 'many'] and f.keys('empty') == []
    a = f.attrs()
    assert a['i'] == 7 and a['i'].dtype == np.int32 and a['f'] == 2.5 and a['s'] == 'text' and a['ls'] == ['a', 'bb']
    assert np.array_equal(a['arr'], [0, 1, 2]) and np.array_equal(a['v'], [1.5, -2.0])
    assert f.keys('many') == [f'd{i:03d}' for i in range(300)]
    assert np.array_equal(f.read('many/d217'), np.full((2, 3), 217.0))
    assert f.attrs('many/d299') == {'unit': 'Pa', 'k': 299}
    c = f.read('a/b/comp')
    assert list(c['entry']) == list(range(5)) and {x.strip() for x in c['label']} == {b'SX'}
    assert f.read('a/str')[0] == b'line 1\nline 2'
    assert np.array_equal(f.read('a/i4'), np.arange(6).reshape(2, 3))


def test_result_file_tensor_orientation(tmp_path):
    """Tensors are stored as (N, 3, 3) with [n, i, j] = T_ij, from the solver's column-major
    components, as the reference's transposed write (result.f90:479-508)."""
    p = tmp_path / 'r.hdf5'
    rf = ResultFile(p, (2, 1, 1), (1.0, 1.0, 1.0), 'Al', 'cF')
    T = np.array([[1.0, 2.0, 3.0], [4.0, 5.0, 6.0], [7.0, 8.0, 9.0]])
    col = np.tile(T.reshape(-1, order='F'), (2, 1))
    rf.add_increment(3, 1.5, {'P': col}, {'F': col})
    rf.close()
    f = DADF5(p)
    assert np.array_equal(f.read('increment_3/phase/Al/mechanical/P')[1], T)
    assert np.array_equal(f.read('increment_3/homogenization/SX/mechanical/F')[0], T)
    assert f.attrs('increment_3')['t/s'] == 1.5
    assert f.attrs('increment_3/phase/Al/mechanical/P')['unit'] == 'Pa'
    assert np.array_equal(f.read('geometry/cells'), [2, 1, 1])


def test_slip_labels_format():
    assert slip_labels([[1, -1, 1]], [[0, 1, 1]]) == ['[ 1 -1  1]( 0  1  1)']
