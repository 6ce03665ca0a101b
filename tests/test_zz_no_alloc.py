"""The allocation-free batched 2D step (lens_batch2d_step_noalloc).

For callers that cannot allocate device memory, the batched step keeps its
descriptor copy and block plan in a fixed device array inside the library.
These tests drive it through the C ABI on a small uneven TE/TM batch and check
that two calls in a row give the same fields and phasors as the regular entry
point (lens_batch2d_step, whose plan tables the caller allocates), bit for bit,
that a capturing stream is refused before anything is enqueued, and that
oversized requests are refused.  The file is collected last, so a
stop-at-first-failure run has already run every other test.
"""
import ctypes
from dataclasses import replace

import pytest

from lens_sensor_b200 import _native as N


@pytest.mark.gpu
def test_noalloc_matches_batched_step_twice():
    import torch
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
        # same kernels, same plan, same arithmetic: identical bits
        for a, b in zip(ref.insts, mine.insts):
            for x, y in zip(a.f, b.f):
                assert torch.equal(x, y)
            assert torch.equal(a.dft, b.dft)


@pytest.mark.gpu
def test_noalloc_refuses_a_capturing_stream():
    import torch
    from lens_sensor_b200 import batch2d as B
    from lens_sensor_b200.workloads import sweep2d
    lib = N.load()
    specs, _ = sweep2d(count=1)
    sw = B.Sweep([replace(specs[0], nx=120, ny=100)], 10, 'f32')
    host = (N.Inst2D * 1)(sw.insts[0].s)
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        g.capture_begin()
        st = lib.lens_batch2d_step_noalloc(host, 1, N.F32, 4, ctypes.byref(sw.table.s), 0, 1,
                                           ctypes.c_void_p(s.cuda_stream))
        g.capture_end()
    assert st == -1
    torch.cuda.synchronize()
    # the stream still works and the entry point runs outside capture
    st = lib.lens_batch2d_step_noalloc(host, 1, N.F32, 4, ctypes.byref(sw.table.s), 0, 1, None)
    assert st == 0
    torch.cuda.synchronize()


@pytest.mark.gpu
def test_noalloc_rejects_oversized_batches():
    import torch
    from lens_sensor_b200 import batch2d as B
    from lens_sensor_b200.workloads import sweep2d
    lib = N.load()
    specs, _ = sweep2d(count=1)
    sw = B.Sweep([replace(specs[0], nx=120, ny=100)], 10, 'f32')
    many = (N.Inst2D * 513)(*([sw.insts[0].s] * 513))              # more than 512 instances
    st = lib.lens_batch2d_step_noalloc(many, 513, N.F32, 4, ctypes.byref(sw.table.s), 0, 1, None)
    assert st == -3 and lib.lens_status_string(st) == b'size exceeds the supported maximum'
    torch.cuda.synchronize()


def _fake_inst(nx, ny):
    """A descriptor that passes the host-side checks; its pointers are never
    dereferenced because the call refuses it before enqueuing anything."""
    fake = 0x1000
    s = N.Inst2D()
    s.pol, s.nx, s.ny, s.pitch = 0, nx, ny, ny
    for q in range(3):
        s.f[q] = fake
    for q in range(2):
        s.c[q] = fake
    for ax, n in ((s.ax, nx), (s.ay, ny)):
        for p, m in ((ax.e, n), (ax.h, n - 1)):
            p.b = p.c = p.ik = fake
            p.n, p.lo, p.hi = m, 0, 0
    s.src.ix = -1
    return s


def test_noalloc_tile_limit_is_refused_on_the_host():
    """2^21 tiles is the limit of the owner table: 64 instances of 8192 x 4096
    nodes make exactly 2^21 tiles of 128 x 8 (the plan arithmetic accepts them),
    65 make more and are refused with LENS_ERR_SIZE before any CUDA call (so this
    runs without a GPU)."""
    lib = N.load()
    inst = _fake_inst(8192, 4096)
    tab = N.StepTable(0x1000, 0x1000, None, None, 0, 10)
    exact = (N.Inst2D * 64)(*([inst] * 64))
    assert lib.lens_batch2d_plan(exact, 64, 4, (ctypes.c_int * 65)(), None) == 1 << 21
    over = (N.Inst2D * 65)(*([inst] * 65))
    assert lib.lens_batch2d_step_noalloc(over, 65, N.F32, 4, ctypes.byref(tab), 0, 1, None) == -3
