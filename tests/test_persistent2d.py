"""The persistent cooperative batched step (lens_batch2d_run: all steps of a
batch in one launch, grid barriers between phases) against the step-by-step
batched launches (lens_batch2d_step).  Both run the same tile functions in the
same per-thread order, so fields and DFT sums must be identical bit for bit:
TE and TM (with the TM node DFT phase), FP32 and FP16 storage, members that
join late (n_start), and a single full-size config-2 instance."""
from dataclasses import replace

import pytest


def _specs(count):
    from lens_sensor_b200.workloads import sweep2d
    specs, _ = sweep2d(count=count)
    return [replace(sp, nx=min(sp.nx, 170 + 37 * q), ny=min(sp.ny, 130 + 23 * q)) for q, sp in enumerate(specs)]


def _same(a, b):
    import torch
    for x, y in zip(a.insts, b.insts):
        for u, v in zip(x.f, y.f):
            assert torch.equal(u, v)
        assert torch.equal(x.dft, y.dft)


@pytest.mark.gpu
@pytest.mark.parametrize('storage', ['f32', 'f16'])
def test_persistent_matches_stepped(storage):
    import torch
    from lens_sensor_b200 import batch2d as B
    specs = _specs(6)
    a = B.Sweep(specs, 240, storage, by=4)
    b = B.Sweep(specs, 240, storage, by=4, geos=[q.geo for q in a.insts])
    a.run(graphs=False)
    assert b.run(persistent=True) == 1
    torch.cuda.synchronize()
    _same(a, b)


@pytest.mark.gpu
def test_persistent_in_pieces_and_late_members():
    """Two launches of 120 and 80 steps equal one of 200; a member that joins at
    batch step 40 (n_start) is advanced from its own step 0."""
    import torch
    from lens_sensor_b200 import batch2d as B
    specs = _specs(4)
    a = B.Sweep(specs, 200, 'f32', by=4)
    b = B.Sweep(specs, 200, 'f32', by=4, geos=[q.geo for q in a.insts])
    for sw in (a, b):
        sw.insts[3].s.n_start = 40
    ga, gb = a._groups(4, None)[0], b._groups(4, None)[0]
    ga.step(a.table, 40, 160)
    gb.step_persistent(b.table, 40, 100)
    gb.step_persistent(b.table, 140, 60)
    torch.cuda.synchronize()
    gb.check()
    _same(a, b)


@pytest.mark.gpu
def test_persistent_full_size_instance():
    import torch
    from lens_sensor_b200 import batch2d as B
    from lens_sensor_b200.workloads import sweep2d
    specs, _ = sweep2d(count=3)
    a = B.Sweep(specs[1:3], 300, 'f32', by=8)
    b = B.Sweep(specs[1:3], 300, 'f32', by=8, geos=[q.geo for q in a.insts])
    a.run(graphs=True)
    b.run(persistent=True)
    torch.cuda.synchronize()
    _same(a, b)


@pytest.mark.gpu
def test_persistent_refuses_missing_barrier_state():
    import ctypes
    from lens_sensor_b200 import _native as N
    from lens_sensor_b200 import batch2d as B
    sw = B.Sweep(_specs(1), 10, 'f32', by=4)
    g = sw.groups[0]
    lib = N.load()
    st = lib.lens_batch2d_run(g.host, ctypes.c_void_p(g.dev_desc.data_ptr()), ctypes.c_void_p(g.dev_blk.data_ptr()),
                              ctypes.c_void_p(g.dev_owner.data_ptr()), 1, N.F32, 4, ctypes.byref(sw.table.s), 0, 4,
                              None, None, None)
    assert st == -1
