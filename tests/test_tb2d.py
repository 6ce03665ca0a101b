"""The temporally blocked 2D step (lens_tb2d_step, LENS_TB_K steps per launch)
against the single-step batched step it replaces (lens_batch2d_step), on uneven
TE and TM batches: fields, psi-carrying strips, source rows, beads, loss and the
node-field DFT.  The single-step batched fields are identical to the single-grid
engine's, which the oracle tests pin to the reference (test_batch2d.py,
test_gpu_parity.py); the FP64 comparison at full size is test_fp64_fullsize.py."""
from dataclasses import replace

import numpy as np
import pytest

TOL = 2e-6     # relative L2 per field: the same arithmetic, contracted (FMA) in places by the compiler


def _specs(count, shrink=True):
    from lens_sensor_b200.workloads import sweep2d
    specs, _ = sweep2d(count=count)
    if shrink:   # small uneven grids that still hold strips, source rows and the bead
        specs = [replace(sp, nx=min(sp.nx, 170 + 37 * q), ny=min(sp.ny, 130 + 23 * q)) for q, sp in enumerate(specs)]
    return specs


def _rel(a, b):
    import torch
    a, b = a.double(), b.double()
    return float(torch.linalg.norm(a - b) / max(float(torch.linalg.norm(b)), 1e-30))


def _compare(specs, steps, chunk, storage='f32', tol=TOL):
    import torch
    from lens_sensor_b200 import batch2d as B
    ref = B.Sweep(specs, steps, storage, by=4)
    tb = B.Sweep(specs, steps, storage, geos=[q.geo for q in ref.insts], tb=True, chunk=chunk)
    ref.run(graphs=False)
    tb.run(graphs=False)
    torch.cuda.synchronize()
    worst = 0.0
    for a, b in zip(ref.insts, tb.insts):
        for x, y in zip(a.f, b.f):
            e = _rel(y.float(), x.float())
            worst = max(worst, e)
            assert e <= tol, (a.spec.pol, a.spec.nx, a.spec.ny, e)
        e = _rel(torch.view_as_real(b.phasor()), torch.view_as_real(a.phasor()))
        assert e <= tol, ('phasor', a.spec.pol, e)
    return worst


@pytest.mark.gpu
@pytest.mark.parametrize('chunk', [8, 37, 64])
def test_tb_matches_single_step_batch(chunk):
    # 5 instances, TE and TM alternating, 160 steps with the last 8 periods in the DFT window
    _compare(_specs(5), 160, chunk)


@pytest.mark.gpu
def test_tb_lossy_tm_and_small_grids():
    from lens_sensor_b200.geometry import Bead2D, Spec2D, Stack
    st = Stack(1.49, 1.0, [(0.4, complex(1.333, 0.01)), (0.2, 1.34)], 1.376)
    specs = [Spec2D('p', 40, 33, 25e-9, st, 1.2e-6, Bead2D(0.6, 0.3, 1.59), npml=6),
             Spec2D('s', 29, 150, 25e-9, st, 1.2e-6, Bead2D(0.4, 0.3, 1.59), npml=6),
             Spec2D('p', 300, 250, 25e-9, st, 3.0e-6, Bead2D(4.0, 0.5, 1.59), npml=12)]
    _compare(specs, 96, 16)


@pytest.mark.gpu
@pytest.mark.parametrize('storage', ['f16', 'bf16'])
def test_tb_reduced_storage_is_no_less_accurate(storage):
    """Reduced storage rounds what is stored: the single-step path every step,
    the temporally blocked path every LENS_TB_K steps (its intermediate levels
    stay FP32 in registers).  Against the FP32 single-step fields, the blocked
    path's error must not exceed the single-step path's."""
    import torch
    from lens_sensor_b200 import batch2d as B
    specs = _specs(3)
    ref = B.Sweep(specs, 200, 'f32', by=4)
    geos = [q.geo for q in ref.insts]
    step = B.Sweep(specs, 200, storage, by=4, geos=geos)
    tb = B.Sweep(specs, 200, storage, geos=geos, tb=True, chunk=32)
    for sw in (ref, step, tb):
        sw.run(graphs=False)
    torch.cuda.synchronize()
    for r, a, b in zip(ref.insts, step.insts, tb.insts):
        for x, y, z in zip(r.f, a.f, b.f):
            e_step, e_tb = _rel(y.float(), x.float()), _rel(z.float(), x.float())
            assert e_tb <= 1.05 * e_step + 1e-6, (r.spec.pol, e_step, e_tb)


@pytest.mark.gpu
def test_tb_full_size_instance():
    # one full-size sweep instance (2283 x 552 TE) over 400 steps
    specs = _specs(3, shrink=False)[2:3]
    _compare(specs, 400, 64)


@pytest.mark.gpu
def test_tb_refuses_spans_off_the_launch_pair():
    import ctypes
    from lens_sensor_b200 import _native as N
    from lens_sensor_b200 import batch2d as B
    sw = B.Sweep(_specs(1), 16, 'f32', tb=True)
    g = sw.groups[0]
    lib = N.load()
    st = lib.lens_tb2d_step(g.host, ctypes.c_void_p(g.dev_desc.data_ptr()), ctypes.c_void_p(g.dev_first.data_ptr()),
                            1, g.chunk, N.F32, ctypes.byref(sw.table.s), 0, 4, None)
    assert st == -1
    with pytest.raises(ValueError):
        B.Sweep(_specs(1), 12, 'f32', tb=True)


def test_tb_plan_counts_units_on_the_host():
    """Units = column tiles of 120 owned columns x row chunks (no GPU needed:
    the plan reads host descriptors only)."""
    import ctypes
    from lens_sensor_b200 import _native as N
    fake = 0x1000
    t = N.TB2D()
    g = t.g
    g.pol, g.nx, g.ny, g.pitch = 0, 1000, 481, 512
    for q in range(3):
        g.f[q] = fake
        t.f1[q] = fake
    for q in range(2):
        g.c[q] = fake
    for ax, n in ((g.ax, 1000), (g.ay, 481)):
        for p, m in ((ax.e, n), (ax.h, n - 1)):
            p.b = p.c = p.ik = fake
            p.n, p.lo, p.hi = m, 0, 0
    g.src.ix = -1
    first = (ctypes.c_int * 3)()
    arr = (N.TB2D * 2)(t, t)
    assert N.load().lens_tb2d_plan(arr, 2, 64, first) == 2 * 5 * 16
    assert list(first) == [0, 80, 160]
