"""The resident 2D launch (lens_rs2d_run: every field value in registers for
the whole schedule, bands of x rows exchanging one row per half step through
L2) against the step-by-step batched launches (lens_batch2d_step), which run
the same per-cell arithmetic one launch per half step.

CPU: the plan refuses what does not fit on the chip before touching the GPU.
GPU: TE, lossless and lossy TM (with the TM node DFT), bands of one row and of
many, several instances per launch, a schedule run in pieces, members that
joined late (n_start), full-size sweep instances (narrow and wide launches),
and config 0 through Solve2D(engine='resident') with the snapshots the kernel
writes."""
import ctypes
from dataclasses import replace

import numpy as np
import pytest

from lens_sensor_b200 import _native as N

# fields and DFT sums of the resident launch against the batched launches, as
# a fraction of each array's largest value: the same FP32 expressions, but the
# two kernels may fuse a different product of an expression into an FMA (one
# rounding apart per update), which grows to about 2e-6 over 240 steps
TOL = 2e-5
ERR_ARG, ERR_SIZE = -1, -3      # LENS_ERR_ARG, LENS_ERR_SIZE


def _fake_inst(nx, ny, pol, wy=4):
    s = N.Inst2D()
    s.pol, s.nx, s.ny, s.pitch = pol, nx, ny, (ny + 31) // 32 * 32
    for q in range(3):
        s.f[q] = 16
    s.c[0] = s.c[1] = 16
    for ax, n, w in ((s.ax, nx, 4), (s.ay, ny, wy)):
        for tag, m in (('e', n), ('h', n - 1)):
            setattr(ax, tag, N.Profile(16, 16, 16, m, w // 2, w - w // 2))
    for q in range(4):
        s.psi[q] = 16
    s.src = N.Source(-1, None, None, None, 0, 0, 0)
    return s


def test_plan_refuses_what_does_not_fit():
    lib = N.load()
    r, c, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    plan = lambda arr: lib.lens_rs2d_plan(arr, len(arr), ctypes.byref(r), ctypes.byref(c), ctypes.byref(t))
    assert plan((N.Inst2D * 1)(_fake_inst(200, 577, 0))) == ERR_SIZE       # more than 18 warps of columns
    assert plan((N.Inst2D * 1)(_fake_inst(200, 300, 1, wy=66))) == ERR_SIZE  # y strips wider than 64
    assert plan((N.Inst2D * 33)(*[_fake_inst(40, 40, 0)] * 33)) == ERR_SIZE  # more than 32 instances
    assert plan((N.Inst2D * 1)(_fake_inst(2, 40, 0))) == ERR_ARG            # nx < 3
    bad = _fake_inst(100, 40, 0)
    bad.psi[2] = None                                                          # a strip without its psi
    assert plan((N.Inst2D * 1)(bad)) == ERR_ARG


def _specs(count, lossy_tm=False):
    from lens_sensor_b200.geometry import Stack
    from lens_sensor_b200.workloads import N_AQ, N_CORNEA, N_MUCIN, N_PMMA, sweep2d
    specs, _ = sweep2d(count=count)
    out = [replace(sp, nx=min(sp.nx, 170 + 37 * q), ny=min(sp.ny, 130 + 23 * q)) for q, sp in enumerate(specs)]
    if lossy_tm:   # an absorbing aqueous layer inside the (shortened) domain
        st = Stack(N_PMMA, 2.0, [(1.5, complex(N_AQ, 0.001)), (0.5, N_MUCIN)], N_CORNEA)
        out = [replace(sp, stack=st, tear_m=0.4 * sp.ny * sp.dx) if sp.pol == 'p' else sp for sp in out]
    return out


def _close(a, b, tol=TOL):
    """Every field and DFT array of sweep a within tol (relative to its largest
    value) of sweep b's; returns whether all were bit-identical."""
    import torch
    same = True
    for x, y in zip(a.insts, b.insts):
        for u, v in list(zip(x.f, y.f)) + [(x.dft, y.dft)]:
            scale = max(float(v.abs().max()), 1e-30)
            assert float((u - v).abs().max()) <= tol * scale, (x.spec.nx, x.spec.ny, x.spec.pol)
            same = same and torch.equal(u, v)
    return same


@pytest.mark.gpu
@pytest.mark.parametrize('lossy', [False, True])
def test_resident_matches_stepped(lossy):
    import torch
    from lens_sensor_b200 import batch2d as B
    specs = _specs(6, lossy_tm=lossy)
    a = B.Sweep(specs, 240, 'f32', by=4)
    b = B.Sweep(specs, 240, 'f32', geos=[q.geo for q in a.insts], resident=True)
    if lossy:
        assert any(q.geo.get('da_x') is not None for q in a.insts if q.spec.pol == 'p')
    a.run(graphs=False)
    assert b.run() == len(b.groups) == 1
    torch.cuda.synchronize()
    print('resident vs stepped, bit-identical:', _close(b, a))


@pytest.mark.gpu
def test_bands_of_one_row():
    """Instances short enough that the plan gives every band one row (every row
    then reads both halo rows)."""
    import torch
    from lens_sensor_b200 import batch2d as B
    specs = [replace(sp, nx=60 + 9 * q, ny=90 + 31 * q) for q, sp in enumerate(_specs(2))]
    a = B.Sweep(specs, 200, 'f32', by=4)
    b = B.Sweep(specs, 200, 'f32', geos=[q.geo for q in a.insts], resident=True)
    assert b.groups[0].rows == 1
    a.run(graphs=False)
    b.run()
    torch.cuda.synchronize()
    _close(b, a)


@pytest.mark.gpu
def test_resident_in_pieces_and_late_members():
    """Launches of 100 and 60 steps equal one of 160 bit for bit (the state goes
    back to HBM between them); a member joining at batch step 40 (n_start) is
    advanced from its own step 0 like the batched launches do."""
    import torch
    from lens_sensor_b200 import batch2d as B
    specs = _specs(4)
    a = B.Sweep(specs, 200, 'f32', by=4)
    b = B.Sweep(specs, 200, 'f32', geos=[q.geo for q in a.insts], resident=True)
    c = B.Sweep(specs, 200, 'f32', geos=[q.geo for q in a.insts], resident=True)
    for sw in (a, b, c):
        sw.insts[3].s.n_start = 40
    ga = a._groups(4, None)[0]
    gb, gc = B.ResidentGroup(b.insts, b.dev), B.ResidentGroup(c.insts, c.dev)
    ga.step(a.table, 40, 160)
    gb.step(b.table, 40, 100)
    gb.step(b.table, 140, 60)
    gc.step(c.table, 40, 160)
    torch.cuda.synchronize()
    gb.check()
    gc.check()
    for x, y in zip(b.insts, c.insts):
        for u, v in list(zip(x.f, y.f)) + [(x.dft, y.dft)]:
            assert torch.equal(u, v)
    _close(b, a)


@pytest.mark.gpu
def test_resident_full_size_sweep_instances():
    """Full-size config-2 instances, several per launch, including the widest
    (ny > 512: the 18-warp launches) and the longest (bands of 17 rows)."""
    import torch
    from lens_sensor_b200 import batch2d as B
    from lens_sensor_b200.workloads import sweep2d
    specs, _ = sweep2d()
    pick = sorted(range(len(specs)), key=lambda q: -specs[q].nx)[:3] + \
        sorted(range(len(specs)), key=lambda q: -specs[q].ny)[:2] + [5, 6]
    sel = [specs[q] for q in dict.fromkeys(pick)]
    a = B.Sweep(sel, 300, 'f32', by=8)
    b = B.Sweep(sel, 300, 'f32', geos=[q.geo for q in a.insts], resident=True)
    assert any(g.threads > 512 for g in b.groups)
    a.run(graphs=True)
    b.run()
    torch.cuda.synchronize()
    print('groups', [(g.rows, g.ctas, g.threads, len(g.insts)) for g in b.groups])
    _close(b, a)


@pytest.mark.gpu
def test_config0_resident_matches_batch_engine():
    """Config 0 (1600 x 480 TE, 6000 steps) in one resident launch: the snapshots
    the kernel writes and the (compensated) phasor against the graph-replayed
    batched engine."""
    import torch
    from lens_sensor_b200.solver2d import Solve2D
    from lens_sensor_b200.workloads import planar2d_te
    sp, steps = planar2d_te()
    a = Solve2D(sp, steps, engine='batch').capture()
    a.run()
    b = Solve2D(sp, steps, engine='resident', geo=a.geo)
    b.run()
    torch.cuda.synchronize()
    b.check()
    assert b.launches == 1
    pa, sa = a.host_results()
    pb, sb = b.host_results()
    assert sa.shape == sb.shape == (30, sp.nx, sp.ny)
    for q in range(len(sa)):
        assert np.abs(sb[q] - sa[q]).max() <= TOL * max(np.abs(sa[q]).max(), 1e-30), q
    e = np.linalg.norm(pb - pa) / np.linalg.norm(pa)
    assert e <= 1e-5, e


@pytest.mark.gpu
def test_solve2d_default_engine():
    """Solve2D picks the resident launch when the grid fits the chip and the
    batched launches when it does not (ny > 576 columns)."""
    from lens_sensor_b200.solver2d import Solve2D
    sp = _specs(1)[0]
    assert Solve2D(sp, 40).engine == 'resident'
    wide = replace(sp, ny=600)
    s = Solve2D(wide, 40)
    assert s.engine == 'batch'
    s.capture().run()


@pytest.mark.gpu
def test_watchdog_ends_the_launch():
    """A band that withholds one halo row (lens_rs2d_watchdog_test): its
    neighbour's bounded wait runs out, the error word is set, the launch ends,
    and the next launch on the same buffers runs clean."""
    import time
    import torch
    from lens_sensor_b200 import batch2d as B
    sw = B.Sweep(_specs(2), 60, 'f32', resident=True)
    g = sw.groups[0]
    assert g.ctas >= 2
    lib = N.load()
    t0 = time.perf_counter()
    st = lib.lens_rs2d_watchdog_test(g.host, ctypes.c_void_p(g.dev_desc.data_ptr()), len(g.insts),
                                     ctypes.byref(sw.table.s), 0, 20, ctypes.c_void_p(g.scratch.data_ptr()),
                                     g.scratch.numel(), ctypes.c_void_p(g.err.data_ptr()), None)
    assert st == 0
    torch.cuda.synchronize()
    assert time.perf_counter() - t0 < 30
    assert int(g.err.item()) != 0
    with pytest.raises(N.LensError):
        g.check()
    sw.reset()
    g.step(sw.table, 0, 20)
    torch.cuda.synchronize()
    g.check()


def _strip_inst(nx, ny, strip=12, src=30):
    """A descriptor with x CPML strips of `strip` rows at both ends and a source
    pair at rows src, src+1 (placeholder pointers: host logic only)."""
    s = _fake_inst(nx, ny, 0)
    s.ax.e = N.Profile(16, 16, 16, nx, strip, strip)
    s.ax.h = N.Profile(16, 16, 16, nx - 1, strip, strip)
    s.src = N.Source(src, 16, 16, 16, ny, 1, ny)
    return s


def test_band_partition_on_the_host():
    """lens_rs2d_bands (no device): every row in exactly one band, bands within
    the row limit and the CTA count, bands holding x-strip / source / face rows
    shorter than the others, each instance starting at its row 0."""
    lib = N.load()
    nx = 1600
    arr = (N.Inst2D * 2)(_strip_inst(nx, 480), _strip_inst(700, 300, strip=10, src=40))
    buf = (ctypes.c_short * 512)()
    n = lib.lens_rs2d_bands(arr, 2, 200, 16, buf, 512)
    assert 0 < n <= 200
    first = list(buf[:n])
    starts = [b for b in range(n) if first[b] == 0]
    assert starts == [0, starts[1]] and len(starts) == 2
    for (a, b), size in (((0, starts[1]), nx), ((starts[1], n), 700)):
        rows = first[a:b] + [size]
        lens = [rows[k + 1] - rows[k] for k in range(b - a)]
        assert min(lens) >= 1 and max(lens) <= 16 and sum(lens) == size
        if size == nx:   # rows of the x strips (H: i < 12 or i >= nx-13; E: i >= nx-12), faces, source
            sp_row = lambda i: i < 12 or i >= nx - 13 or i in (30, 31)
            special = lambda lo, hi: any(sp_row(i) for i in range(lo, hi))
            sp = [ln for lo, ln in zip(rows, lens) if special(lo, lo + ln)]
            lean = [ln for lo, ln in zip(rows, lens) if not special(lo, lo + ln)]
            assert 2 * max(sp) <= max(lean), (sp, lean)   # a special row costs 3.4 lean rows
    assert lib.lens_rs2d_bands(arr, 2, 20, 16, buf, 512) == ERR_SIZE        # 2300 rows in 20 bands of 16
    assert lib.lens_rs2d_bands(arr, 2, 200, 16, buf, 0) == ERR_ARG


@pytest.mark.gpu
def test_staged_host_results_equal_direct():
    """Solve2D.stage_host() (host buffers prepared while the device steps) gives
    the same phasor and snapshots as the direct read-back."""
    from lens_sensor_b200.solver2d import Solve2D
    sp = _specs(1)[0]
    a = Solve2D(sp, 400, snap_every=100)
    b = Solve2D(sp, 400, snap_every=100, geo=a.geo)
    a.run()
    b.stage_host().run()
    pa, sa = a.host_results()
    pb, sb = b.host_results()
    assert sa.shape == sb.shape == (4, sp.nx, sp.ny)
    assert np.array_equal(pa, pb) and np.array_equal(sa, sb)
