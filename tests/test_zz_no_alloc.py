"""The allocation-free batched 2D step (lens_batch2d_step_noalloc).

For callers that cannot allocate device memory, the batched step keeps its
descriptor copy and block plan in a fixed device array inside the library.
This test drives it through the C ABI on a small uneven TE/TM batch and checks
that two calls in a row give the same fields and phasors as the regular
entry point (lens_batch2d_step, whose plan tables the caller allocates), and
that oversized requests are refused.  It lives in its own file, collected
last, so a stop-at-first-failure run has already run every other test.
"""
import ctypes
from dataclasses import replace

import pytest

# same tolerance as the other batched tests: identical arithmetic, identical order
TOL = 1e-6


@pytest.mark.gpu
def test_noalloc_matches_batched_step_twice():
    import torch
    from lens_sensor_b200 import _native as N
    from lens_sensor_b200 import batch2d as B
    from lens_sensor_b200.workloads import sweep2d
    lib = N.load()
    specs, _ = sweep2d(count=5)
    specs = [replace(sp, nx=min(sp.nx, 140 + 19 * q), ny=min(sp.ny, 260 - 9 * q)) for q, sp in enumerate(specs)]
    steps = 200
    ref = B.Sweep(specs, steps, 'f32', by=4)
    mine = B.Sweep(specs, steps, 'f32', by=4, geos=[q.geo for q in ref.insts])
    host = (N.Inst2D * len(mine.insts))(*[q.s for q in mine.insts])
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    g = ref.groups[0]
    for n0, k in ((0, 120), (120, 80)):          # two calls in a row, the second inside the DFT window
        g.step(ref.table, n0, k)
        st = lib.lens_batch2d_step_noalloc(host, len(host), N.F32, 4, ctypes.byref(mine.table.s), n0, k, stream)
        assert st == 0, lib.lens_status_string(st)
        torch.cuda.synchronize()
        for a, b in zip(ref.insts, mine.insts):
            for x, y in zip(a.f, b.f):
                assert float((x - y).norm()) <= TOL * max(float(x.norm()), 1e-30)
            pa, pb = a.phasor(), b.phasor()
            assert float((pa - pb).abs().norm()) <= TOL * max(float(pa.abs().norm()), 1e-30)


@pytest.mark.gpu
def test_noalloc_rejects_oversized_batches():
    import torch
    from lens_sensor_b200 import _native as N
    from lens_sensor_b200 import batch2d as B
    from lens_sensor_b200.workloads import sweep2d
    lib = N.load()
    specs, _ = sweep2d(count=1)
    sw = B.Sweep([replace(specs[0], nx=120, ny=100)], 10, 'f32')
    many = (N.Inst2D * 513)(*([sw.insts[0].s] * 513))              # more than 512 instances
    st = lib.lens_batch2d_step_noalloc(many, 513, N.F32, 4, ctypes.byref(sw.table.s), 0, 1, None)
    assert st == -3 and lib.lens_status_string(st) == b'size exceeds the supported maximum'
    torch.cuda.synchronize()
