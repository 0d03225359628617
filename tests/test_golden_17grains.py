"""The reference's own regression result, pinned: 17 grains, bcc phenopowerlaw with
non-Schmid terms, tension along x with mixed boundary conditions, 150 increments
(reference tests/integration/test_plastic_detect_changes.py, model phenopowerlawbcc).

The fixture (tests/golden/golden_17grains_bcc.npz, made by make_golden_17grains.py from
the reference's resources) holds the inputs and the stored xi_sl / gamma_sl of
increments 0, 75 and 150.  The comparison uses the reference test's own tolerance:
|x - x_ref| <= atol + 0.025 |x_ref| with atol = max(1e-5 max|x_ref|, 1e-6).
"""
import base64
import json
import zlib
from pathlib import Path

import numpy as np
import pytest
import yaml

from damask_b200 import config, dadf5, vti
from damask_b200.grid import run_load_cases

from damask_b200.h5read import DADF5

GOLD = Path(__file__).resolve().parent / 'golden' / 'golden_17grains_bcc.npz'


@pytest.fixture(scope='module')
def gold():
    d = np.load(GOLD)
    return {k: d[k] for k in d.files}


def inputs(g):
    phase = config.Phase.from_dict(json.loads(str(g['phase_json'])))
    num = config.Numerics.from_dict(json.loads(str(g['numerics_json'])))
    lcs = config.parse_load(json.loads(str(g['load_json'])))
    return tuple(int(c) for c in g['cells']), tuple(float(s) for s in g['size']), g['material'], g['quaternions'], \
        phase, num, lcs


def run(solver, lcs):
    """Run all increments; xi_sl and gamma_sl at the stored increments 75 and 150."""
    out = {}

    def cb(rec):
        if rec.converged and rec.inc in (75, 150):
            out[rec.inc] = (solver.get_field('xi_sl').copy(), solver.get_field('gamma_sl').copy())

    stats = run_load_cases(solver, lcs, on_increment=cb)
    return out, stats


def within_reference_tolerance(x, ref):
    atol = max(np.abs(ref).max() * 1e-5, 1e-6)
    return np.abs(x - ref) <= atol + 0.025 * np.abs(ref)


def test_vti_known_answers(gold):
    """The VTI decoder against the known answers of the reference's VTI tests."""
    for key, (b64, word, compressed, expected) in json.loads(str(gold['vti_known_json'])).items():
        assert list(vti._decode(b64, compressed, word)) == expected, key


def test_vti_roundtrip_multiblock(tmp_path):
    """A compressed, multi-block Int64 material array with a UInt64 header reads back exactly."""
    cells = (5, 4, 3)
    mat = (np.arange(60, dtype=np.int64) * 7) % 11
    raw = mat.tobytes()
    bs = 128
    blocks = [zlib.compress(raw[i:i + bs]) for i in range(0, len(raw), bs)]
    header = np.array([len(blocks), bs, len(raw) % bs or bs] + [len(b) for b in blocks], '<u8').tobytes()
    text = base64.b64encode(header).decode() + base64.b64encode(b''.join(blocks)).decode()
    p = tmp_path / 'g.vti'
    p.write_text(f'''<?xml version="1.0"?>
<VTKFile type="ImageData" version="0.1" byte_order="LittleEndian" header_type="UInt64" compressor="vtkZLibDataCompressor">
  <ImageData WholeExtent="0 5 0 4 0 3" Origin="0 0 0" Spacing="2e-6 2e-6 2e-6" Direction="1 0 0 0 1 0 0 0 1">
  <Piece Extent="0 5 0 4 0 3"><CellData>
    <DataArray type="Int64" Name="material" format="binary">{text}</DataArray>
  </CellData></Piece></ImageData></VTKFile>''')
    g = vti.load(p)
    assert g.cells == cells and np.allclose(g.size, (1e-5, 8e-6, 6e-6))
    assert np.array_equal(g.material, mat)


def test_vti_rejects_bad_direction(tmp_path):
    p = tmp_path / 'bad.vti'
    p.write_text('<VTKFile type="ImageData" byte_order="LittleEndian"><ImageData WholeExtent="0 1 0 1 0 1" '
                 'Spacing="1 1 1" Direction="0 1 0 1 0 0 0 0 1"/></VTKFile>')
    with pytest.raises(vti.VTIError, match='Direction'):
        vti.load(p)


def test_inputs_parse(gold):
    cells, size, mat, q, phase, num, lcs = inputs(gold)
    assert cells == (10, 16, 12) and mat.max() == 16 and len(q) == 17
    assert phase.lattice == 'cI' and phase.n_slip == 12 and num.N_iter_min == 4
    assert len(lcs) == 1 and lcs[0].N == 150 and lcs[0].f_out == 75
    assert np.allclose(gold['xi_sl_0'], 405.8e6) and not gold['gamma_sl_0'].any()


@pytest.fixture(scope='module')
def oracle_run(gold, oracle_lib, tmp_path_factory):
    """The oracle over all 150 increments, writing its result file like the reference job
    (outputs xi_sl and gamma_sl of the phase, increments 0, 75, 150)."""
    cells, size, mat, q, phase, num, lcs = inputs(gold)
    o = oracle_lib.OracleSpectralBasic(cells, size, mat, q, phase, num)
    path = tmp_path_factory.mktemp('dadf5') / '17grains_tensionX.hdf5'
    rf = dadf5.ResultFile(path, cells, size, 'phenopowerlawbcc', 'cI', 'SX',
                          setup_files={n: ('', 'input file') for n in ('17grains.vti', 'material.yaml',
                                                                      'numerics.yaml', 'tensionX.yaml')})
    systems = dadf5.phase_systems(phase)
    outputs = ('xi_sl', 'gamma_sl')
    dadf5.write_increment(rf, o, 0, 0.0, outputs, (), systems)
    out = {}

    def cb(rec):
        if rec.converged and rec.inc % lcs[0].f_out == 0:
            out[rec.inc] = (o.get_field('xi_sl').copy(), o.get_field('gamma_sl').copy(), o.get_coords())
            dadf5.write_increment(rf, o, rec.inc, rec.t, outputs, (), systems)

    stats = run_load_cases(o, lcs, on_increment=cb)
    rf.close()
    o.close()
    return out, stats, path


def test_oracle_reproduces_reference_result(gold, oracle_run):
    """The oracle over all 150 increments against the reference's stored result."""
    out, stats, _ = oracle_run
    assert all(s.converged for s in stats) and len(stats) == 150
    for inc in (75, 150):
        xi, ga, _ = out[inc]
        assert within_reference_tolerance(xi, gold[f'xi_sl_{inc}']).all()
        assert within_reference_tolerance(ga, gold[f'gamma_sl_{inc}']).all()
        # much closer than the tolerance in the hardening variable
        assert np.abs(xi / gold[f'xi_sl_{inc}'] - 1).max() < 1e-3


def _tree(f: DADF5, path=''):
    out = {}
    for k in f.keys(path):
        p = f'{path}/{k}'.strip('/')
        try:
            out[k] = {'groups': _tree(f, p), 'attrs': f.attrs(p)}
        except KeyError:
            d = f.read(p)
            out[k] = {'shape': list(d.shape), 'dtype': str(d.dtype) if not d.dtype.names else list(d.dtype.names),
                      'attrs': f.attrs(p), 'data': d}
    return out


def _contains(mine: dict, ref: dict, where=''):
    """Every group, dataset (shape, dtype) and attribute of ref is in mine."""
    for k, r in ref.items():
        assert k in mine, f'{where}/{k} missing'
        m = mine[k]
        for name, v in r['attrs'].items():
            assert name in m['attrs'], f'{where}/{k}@{name} missing'
            if name == 't/s':
                assert abs(m['attrs'][name] - v) <= 1e-12 * max(1.0, abs(v))
            elif where.strip('/') != 'setup':
                assert np.array_equal(np.asarray(m['attrs'][name]), np.asarray(v)), f'{where}/{k}@{name}'
        if 'groups' in r:
            _contains(m['groups'], r['groups'], f'{where}/{k}')
        elif where.strip('/') != 'setup':
            assert m['shape'] == r['shape'] and m['dtype'] == r['dtype'], f'{where}/{k}'


def test_result_file_has_reference_layout(gold, oracle_run):
    """The DADF5 file written for the job holds every group, dataset and attribute of the
    reference's result file (restricted to the job's phase), with the reference's descriptions,
    units, slip-system labels and times, and its data within the reference test's tolerance."""
    out, _, path = oracle_run
    f = DADF5(path)
    ref = json.loads(str(gold['layout_json']))
    assert set(ref['root_attrs']) <= set(f.attrs())
    assert f.attrs()['DADF5_version_major'] == 1
    mine = _tree(f)
    _contains(mine, ref['tree'])
    ph = f.read('cell_to/phase')
    assert ph.shape == (1920, 1) and (ph['entry'][:, 0] == np.arange(1920)).all()
    assert {x.decode().strip() for x in ph['label'].ravel()} == {'phenopowerlawbcc'}
    for inc in (75, 150):
        g = f'increment_{inc}'
        xi = f.read(f'{g}/phase/phenopowerlawbcc/mechanical/xi_sl')
        assert np.array_equal(xi, out[inc][0])
        assert within_reference_tolerance(xi, gold[f'xi_sl_{inc}']).all()
        for name in ('u_p', 'u_n'):
            u = f.read(f'{g}/geometry/{name}')
            assert within_reference_tolerance(u, gold[f'{name}_{inc}']).all(), (inc, name)


@pytest.mark.gpu
def test_gpu_reproduces_reference_result(gold, gpu, oracle_lib):
    """The CUDA path over all 150 increments: the reference's stored result at its own
    tolerance, and the oracle at 1e-9 with equal fixed-point iteration counts."""
    from damask_b200.grid import SpectralBasic
    cells, size, mat, q, phase, num, lcs = inputs(gold)
    g = SpectralBasic(cells, size, mat, q, phase, num)
    out, stats = run(g, lcs)
    g.close()
    o = oracle_lib.OracleSpectralBasic(cells, size, mat, q, phase, num)
    out_o, stats_o = run(o, lcs)
    o.close()
    assert [s.iterations for s in stats] == [s.iterations for s in stats_o]
    for inc in (75, 150):
        xi, ga = out[inc]
        assert within_reference_tolerance(xi, gold[f'xi_sl_{inc}']).all()
        assert within_reference_tolerance(ga, gold[f'gamma_sl_{inc}']).all()
        assert np.abs(xi - out_o[inc][0]).max() / np.abs(out_o[inc][0]).max() < 1e-9
        assert np.abs(ga - out_o[inc][1]).max() / np.abs(out_o[inc][1]).max() < 1e-9
