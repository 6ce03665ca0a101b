"""The plain 2D solve (solver2d.Solve2D) on its engines: the batched
kernels on one instance replayed as one CUDA graph ('batch') or run in one
persistent cooperative launch per snapshot period ('persistent'), the
temporally blocked step ('tb') and the single-grid engine ('step').  The snapshots and
the one-period CW phasor must agree (the single-grid engine is pinned to the
oracle by test_gpu_parity.py; all three to FP64 at full size by
test_fp64_fullsize.py).  The schedule itself is CPU-checked."""
import numpy as np
import pytest

from lens_sensor_b200.geometry import Bead2D, Spec2D, Stack
from lens_sensor_b200.solver2d import schedule_2d

TOL = 1e-5


def _spec(pol='s'):
    st = Stack(1.49, 1.0, [(0.6, 1.333), (0.3, 1.34)], 1.376)
    return Spec2D(pol, 312, 168, 25e-9, st, 2.4e-6, Bead2D(4.0, 0.6, 1.59), npml=12, ramp_periods=4.0)


def test_schedule_2d_windows_and_snapshots():
    sc = schedule_2d(_spec(), 400, periods=1, snap_every=80)
    assert sc['dft'] == (400 - sc['steps_per_T'], 400) and sc['n_acc'] == sc['steps_per_T']
    assert sc['snaps'] == [80, 160, 240, 320, 400]
    assert schedule_2d(_spec(), 40, periods=2, snap_every=0)['n_acc'] == 40


def _rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / max(np.linalg.norm(np.asarray(b).ravel()), 1e-300))


@pytest.mark.gpu
@pytest.mark.parametrize('pol', ['s', 'p'])
def test_engines_agree(pol):
    from lens_sensor_b200.solver2d import Solve2D
    sp = _spec(pol)
    out = {}
    geo = None
    for eng in ('step', 'batch', 'tb', 'persistent'):
        s = Solve2D(sp, 400, snap_every=80, engine=eng, geo=geo)
        geo = s.geo
        if eng in ('batch', 'tb'):
            s.capture()
        s.run()
        out[eng] = s.host_results()
    for eng in ('batch', 'tb', 'persistent'):
        assert _rel(out[eng][0], out['step'][0]) <= TOL, (eng, 'phasor')
        assert _rel(out[eng][1], out['step'][1]) <= TOL, (eng, 'snapshots')
    assert np.abs(out['step'][0]).max() > 0


@pytest.mark.gpu
def test_captured_graph_replays_once():
    from lens_sensor_b200.solver2d import Solve2D
    s = Solve2D(_spec(), 160, snap_every=80, engine='batch').capture()
    s.run()
    assert s.n == 160 and s.graph is None and s.launches > 0
