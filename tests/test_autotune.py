"""The autotuner (dmk_autotune): it picks a stress-kernel variant and voxel-chunk count by timing the
constitutive evaluation at the current state, and leaves the solve's results unchanged."""
import numpy as np
import pytest

from damask_b200 import workloads
from damask_b200.grid import IncrementDriver, SpectralBasic

pytestmark = pytest.mark.gpu


def _run(tune_at, n=4):
    rve, phase, lcs, num = workloads.make_cut('grid256_bcc24_2000g', (32, 32, 32))
    s = SpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, num)
    drv = IncrementDriver(s, lcs)
    stats, tuning = [], None
    for i in range(n):
        gen = drv.step_requests()
        try:
            gen.send(None)                       # forward and materialpoint_forward done
            if i == tune_at:
                tuning = s.autotune(reps=1)
            while True:
                gen.send(s.solution())
        except StopIteration as stop:
            stats.extend(stop.value)
    return s, stats, tuning


def test_autotune_keeps_results(gpu):
    """Tuning between the forward and the solution of the third increment: every candidate is
    reported with a positive time, the chosen pair is one of them, and the run continues bit for bit
    as the untuned run (iteration counts, <P>, stress and state fields)."""
    a, sa, _ = _run(None)
    b, sb, tuning = _run(2)
    cands = tuning['candidates']
    assert len(cands) == 9 and all(ms > 0 for _, _, ms in cands)
    assert {c[0] for c in cands} == {2, 3, 4} and {c[1] for c in cands} == {1, 2, 4}
    assert tuning['chosen'] in [(c[0], c[1]) for c in cands]
    assert [r.iterations for r in sa] == [r.iterations for r in sb]
    for x, y in zip(sa, sb):
        assert np.array_equal(x.P_av, y.P_av)
    for name in ('P', 'F_p', 'L_p', 'xi_sl', 'gamma_sl'):
        assert np.array_equal(a.get_field(name), b.get_field(name)), name
    print('autotune candidates (blocks/SM, chunks, ms):', cands, 'chosen', tuning['chosen'])
    a.close()
    b.close()


def test_set_tuning_rejects_unknown_variants(gpu):
    rve, phase, lcs, num = workloads.make_cut('grid256_bcc24_2000g', (16, 16, 16))
    s = SpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, phase, num)
    assert s.tuning() == (3, 1)
    s.set_tuning(2, 1)
    assert s.tuning() == (2, 1)
    with pytest.raises(Exception):
        s.set_tuning(5, 1)
    with pytest.raises(Exception):
        s.set_tuning(3, 8)
    s.close()
