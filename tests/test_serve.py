"""Serving loop (lens_sensor_b200.serve): admission, continuous batching, and that
every result is the same alone and in the mix.

The mix holds 2D TE/TM requests of different lengths (so batch members finish
at different times and later requests join a running batch with their own step
origin), two 3D solves and one stitch job, under a budget and slot limits that
make requests wait.  Each request is then served alone.  Results must agree
within the stated tolerance: phasors and stitch amplitudes bit for bit (no
request reads another's arrays; the batched kernel updates each tile from its
own instance), scalar sums to 1e-9 relative (the detector box sums use atomic
adds, whose order may differ).
"""
import numpy as np
import pytest
import torch

from lens_sensor_b200 import workloads as W
from lens_sensor_b200.geometry import Bead2D, Spec2D, Spec3D, Sphere, Stack
from lens_sensor_b200.stitch3d import StitchPlan

TOL_SCALAR = 1e-9


def test_serving_stream_is_seeded_poisson_mix():
    a, b = W.serving_stream(seed=7, count=200), W.serving_stream(seed=7, count=200)
    assert [(k, s, t) for k, _, s, t in a] == [(k, s, t) for k, _, s, t in b]
    t = np.array([x[3] for x in a])
    assert np.all(np.diff(t) > 0)
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert 0.012 < gaps.mean() < 0.03                     # mean 1/50 s
    kinds = [x[0] for x in a]
    assert 0.6 < kinds.count('2d') / 200 < 0.8
    assert kinds.count('stitch') >= 1
    for k, sp, steps, _ in a:
        if k == '3d':
            assert 256 <= sp.nx <= 512 and 128 <= sp.ny <= 192 and 160 <= sp.nz <= 256
            assert 2000 <= steps <= 4000
        if k == 'stitch':
            assert 4 <= sp.n_win <= 10 and sp.O == 40


def test_footprint_orders_requests():
    from lens_sensor_b200.serve import Request, footprint
    st = Stack(1.49, 1.0, [(1.0, 1.333)], 1.376)
    small = Request(0, '2d', Spec2D('s', 200, 120, 50e-9, st, 2e-6, npml=10), 100)
    big = Request(1, '2d', Spec2D('s', 400, 240, 50e-9, st, 2e-6, npml=10), 100)
    cube = Request(2, '3d', Spec3D('p', 64, 48, 40, 100.0, st, 2.0), 100)
    assert 0 < footprint(small) < footprint(big)
    assert footprint(cube) > 64 * 48 * 64 * 4 * 36


def _mix():
    st = Stack(1.49, 0.8, [(0.6, complex(1.333, 0.002)), (0.3, 1.34)], 1.376)
    reqs = []
    for q in range(6):
        nx, ny = 180 + 24 * q, 96 + 8 * q
        sp = Spec2D('s' if q % 2 == 0 else 'p', nx, ny, 50e-9, st, 2.0e-6, Bead2D(nx * 0.05 * 0.6, 0.5, 1.59),
                    npml=10)
        reqs.append(('2d', sp, 300 + 100 * q, 0.002 * q))
    st3 = Stack(1.49, 1.0, [(1.0, complex(1.333, 0.002)), (0.5, 1.34)], 1.376)
    for q in range(2):
        sp = Spec3D('p' if q == 0 else 's', 60 + 8 * q, 44, 36, 100.0, st3, 2.0,
                    [Sphere(2.5, 0.5, 1.59, -0.25, 0.1)], npml=8, waist_um=1.0)
        reqs.append(('3d', sp, 260 + 40 * q, 0.003 + 0.004 * q))
    pl = StitchPlan(Stack(1.491, 1.0, [(1.0, 1.336), (0.5, 1.342)], 1.376), 2.0, 4.0, 4.0, 2.0, 100.0, 2.0, 1.2,
                    1.491, beads=[Sphere(2.0, 0.5, 1.59)], waist_um=1.0, waist_z_um=1.0, n_sponge=8)
    reqs.append(('stitch', pl, pl.steps_win, 0.005))
    return reqs


def _serve(items, **kw):
    from lens_sensor_b200.serve import Request, Server
    reqs = [Request(i, k, sp, n, t) for i, (k, sp, n, t) in enumerate(items)]
    return Server(**kw).run(reqs)


@pytest.mark.gpu
def test_each_result_same_alone_and_in_mix():
    from lens_sensor_b200.serve import footprint, Request, summary
    items = _mix()
    big = max(footprint(Request(0, k, sp, n)) for k, sp, n, _ in items)
    mixed = _serve(items, budget=2.2 * big, slots2d=3, slots3d=2, quantum2d=64, quantum3d=48)
    s = summary(mixed)
    assert s['requests'] == len(items) and s['p99_s'] >= s['p50_s'] > 0
    # requests really overlapped and some joined a running batch
    assert any(r.t_admit > 0 for r in mixed)
    for r in mixed:
        assert r.t_done is not None and r.t_start is not None and r.t_admit <= r.t_start <= r.t_done
    byid = {r.rid: r for r in mixed}
    for i, item in enumerate(items):
        alone = _serve([item[:3] + (0.0,)])[0]
        got = byid[i]
        if got.kind == '2d':
            assert torch.equal(got.result['phasor'], alone.result['phasor']), i
            assert got.result['K'] == alone.result['K']
        elif got.kind == '3d':
            assert torch.equal(got.result['phasor'], alone.result['phasor']), i
            for k in ('P_in', 'P_out', 'transmission', 'p_emit'):
                np.testing.assert_allclose(got.result[k], alone.result[k], rtol=TOL_SCALAR, err_msg=k)
        else:
            assert np.array_equal(got.result['Efull'], alone.result['Efull'])
            assert np.array_equal(got.result['Iavg'], alone.result['Iavg'])
            np.testing.assert_allclose(got.result['transmission'], alone.result['transmission'], rtol=TOL_SCALAR)


@pytest.mark.gpu
def test_batch_members_match_the_plain_batch():
    """A 2D request served through the loop (joining with n_start > 0) gives the
    phasor of the same instance run alone in a plain batched sweep."""
    from lens_sensor_b200 import batch2d as B
    items = [x for x in _mix() if x[0] == '2d']
    served = _serve(items, slots2d=2, quantum2d=50)
    for r in served:
        sw = B.Sweep([r.spec], r.steps)
        sw.run(graphs=False)
        torch.cuda.synchronize()
        ph = sw.insts[0].phasor().cpu()
        assert torch.equal(ph, r.result['phasor'])
