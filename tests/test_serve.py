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


def _req(rid, kind, fp, arrival=0.0):
    from types import SimpleNamespace
    return SimpleNamespace(rid=rid, kind=kind, footprint=fp, arrival=arrival)


def test_admission_first_fit_with_held_claim_and_slots():
    """CPU: first fit in arrival order; the oldest request that does not fit keeps
    its claim (a later small one only fits beside it); slot limits per kind;
    a request larger than the whole budget is rejected, not queued forever."""
    from lens_sensor_b200.serve import admission
    q = [_req(0, '2d', 40), _req(1, '3d', 70), _req(2, '2d', 30), _req(3, '2d', 10), _req(4, '3d', 500)]
    adm, rej = admission(q, used=0, budget=100, n2d=0, n3d=0, slots2d=8, slots3d=4)
    # 0 fits (40); 1 does not (40 + 70 > 100) and holds its 70; beside that claim
    # neither 2 (40 + 70 + 30) nor 3 (40 + 70 + 10) fits; 4 can never fit
    assert [r.rid for r in adm] == [0] and [r.rid for r in rej] == [4]
    adm, rej = admission(q[1:4], used=0, budget=100, n2d=0, n3d=0, slots2d=8, slots3d=4)
    assert [r.rid for r in adm] == [1, 2]          # 70 + 30 = 100 fits exactly
    adm, _ = admission(q[:4], used=0, budget=1000, n2d=0, n3d=0, slots2d=1, slots3d=4)
    assert [r.rid for r in adm] == [0, 1]          # one 2D slot: 2 and 3 wait for it
    adm, _ = admission(q[:4], used=0, budget=1000, n2d=0, n3d=4, slots2d=8, slots3d=4)
    assert [r.rid for r in adm] == [0, 2, 3]       # no 3D slot free


@pytest.mark.gpu
def test_rejected_cancelled_and_failed_requests_leave_the_rest_intact():
    """A request too large for the budget is rejected, one is cancelled while it
    runs, one fails in its host-side setup; every other request completes with
    the result it has when served alone, and the memory account returns to 0."""
    from lens_sensor_b200 import geometry as G
    from lens_sensor_b200.serve import Request, Server, footprint, summary
    items = [x for x in _mix() if x[0] != 'stitch']
    reqs = [Request(i, k, sp, n, t) for i, (k, sp, n, t) in enumerate(items)]
    budget = 2.2 * max(footprint(r) for r in reqs)
    st = Stack(1.49, 1.0, [(1.0, 1.333)], 1.376)
    huge = Request(100, '3d', Spec3D('p', 2048, 512, 1024, 30.0, st, 2.0), 100, 0.001)
    reqs.append(huge)
    reqs[1].cancel_at = 0.05                       # a 2D member, cancelled mid-run
    bad = reqs[2]
    srv = Server(budget=budget, slots2d=3, slots3d=2, quantum2d=32, quantum3d=32)

    def build2d(sp):
        if sp is bad.spec:
            raise RuntimeError('host setup failed')
        return G.build_2d(sp)
    srv.build2d = build2d
    out = srv.run(reqs)
    byid = {r.rid: r for r in out}
    assert byid[100].status == 'rejected' and 'exceeds the budget' in byid[100].error
    assert byid[2].status == 'failed' and 'host setup failed' in byid[2].error
    assert byid[1].status in ('cancelled', 'done')   # it may finish before the cancel lands
    assert srv.used == 0
    s = summary(out)
    assert s['statuses']['rejected'] == 1 and s['statuses']['failed'] == 1
    for r in out:
        if r.rid in (1, 2, 100) or r.status != 'done':
            continue
        alone = _serve([items[r.rid][:3] + (0.0,)])[0]
        assert torch.equal(r.result['phasor'], alone.result['phasor']), r.rid
