"""Batched 2D solves (lens_batch2d_plan / lens_batch2d_step, batch2d.Sweep).

CPU: the block plan of uneven instances (counts, owner table, argument errors).
GPU: a batch of uneven TE/TM instances against the single-grid engine (same
per-cell arithmetic: FP32 fields identical; the batch's plain complex64 DFT
against the single path's compensated one), graph replay against direct
stepping, and the FP16 / BF16 storage variants against FP32 within their
stated tolerances.
"""
import ctypes
from dataclasses import replace

import numpy as np
import pytest

from lens_sensor_b200 import _native as N

# stated phasor tolerances of the storage variants against FP32 storage (400 steps)
TOL_F16 = 2e-3
TOL_BF16 = 1e-2


def _fake_inst(nx, ny, pol):
    """A descriptor with valid sizes and non-null placeholder pointers (never dereferenced)."""
    s = N.Inst2D()
    s.pol, s.nx, s.ny, s.pitch = pol, nx, ny, (ny + 31) // 32 * 32
    for q in range(3):
        s.f[q] = 16
    s.c[0] = s.c[1] = 16
    for ax, n in ((s.ax, nx), (s.ay, ny)):
        for tag, m in (('e', n), ('h', n - 1)):
            setattr(ax, tag, N.Profile(16, 16, 16, m, 2, 2))
    for q in range(4):          # every profile has strips, so every psi array is needed
        s.psi[q] = 16
    s.src = N.Source(-1, None, None, None, 0, 0, 0)
    return s


def test_plan_of_uneven_instances():
    lib = N.load()
    sizes = [(130, 70, 0), (64, 33, 1), (300, 200, 0)]
    arr = (N.Inst2D * 3)(*[_fake_inst(*v) for v in sizes])
    blk = (ctypes.c_int * 4)()
    by = 4
    n = lib.lens_batch2d_plan(arr, 3, by, blk, None)
    per = [((ny + 127) // 128) * ((nx + 2 * by - 1) // (2 * by)) for nx, ny, _ in sizes]
    assert n == sum(per) and list(blk) == [0, per[0], per[0] + per[1], sum(per)]
    owner = (ctypes.c_int * n)()
    assert lib.lens_batch2d_plan(arr, 3, by, blk, owner) == n
    assert list(owner) == [0] * per[0] + [1] * per[1] + [2] * per[2]
    assert lib.lens_batch2d_plan(arr, 3, 9, blk, None) == -1       # 32 x 9 threads > 256
    bad = (N.Inst2D * 1)(_fake_inst(2, 40, 0))                      # nx < 3
    assert lib.lens_batch2d_plan(bad, 1, 4, blk, None) == -1


def test_row_types_are_exact_rows_of_the_coefficients():
    """The row form (LensInst2D.rtype / ctab) holds each typed row's bytes exactly
    and covers the layered rows of sweep2d instances (TE, lossless and lossy TM)."""
    from lens_sensor_b200 import batch2d as B
    from lens_sensor_b200 import engine as E
    from lens_sensor_b200.geometry import build_2d
    from lens_sensor_b200.workloads import sweep2d
    specs, _ = sweep2d(count=4)
    for sp in specs:
        g = build_2d(sp)
        cn = ['ce_e', 'ce_h'] if sp.pol == 's' else ['ca_x', 'ca_y'] + (['da_x', 'da_y'] if g.get('da_x') is not None else [])
        P = E.pitch_of(sp.ny)
        rt, tab = B.row_types([g[k] for k in cn], (sp.nx, P), 'cpu')
        full = np.zeros((sp.nx, len(cn), P), np.float32)
        for q, k in enumerate(cn):
            v = np.asarray(g[k], np.float32)
            full[:v.shape[0], q, :v.shape[1]] = v
        rt, tab = rt.numpy(), tab.numpy()
        assert tab.shape[0] <= B.MAX_RTYPE and (rt != 255).mean() > 0.9
        for i in range(sp.nx):
            if rt[i] != 255:
                assert full[i].tobytes() == tab[rt[i]].tobytes(), i
    flat = [np.arange(12, dtype=np.float32).reshape(3, 4)]       # three different rows: no type
    assert B.row_types(flat, (3, 32), 'cpu') == (None, None)


def _small_sweep():
    from lens_sensor_b200.workloads import sweep2d
    specs, _ = sweep2d(count=6)
    return [replace(sp, nx=min(sp.nx, 150 + 23 * q), ny=min(sp.ny, 300 - 11 * q)) for q, sp in enumerate(specs)]


@pytest.mark.gpu
def test_batch_matches_single_grid_engine():
    import torch
    from lens_sensor_b200 import batch2d as B
    from lens_sensor_b200 import engine as E
    specs, steps = _small_sweep(), 400
    sw = B.Sweep(specs, steps, 'f32', by=4)
    sw.run(graphs=False)
    torch.cuda.synchronize()
    res = sw.results()
    for q, sp in enumerate(specs):
        geo = sw.insts[q].geo
        coef = {k: geo[k] for k in ('ce_e', 'ce_h', 'ca_x', 'ca_y', 'da_x', 'da_y') if k in geo}
        g = E.Grid2D(sp.pol, sp.nx, sp.ny, sp.dx, sp.dt, coef, geo['cx'], geo['cy'], geo['src'])
        ep = E.Epi2D(g, dft=sw.insts[q].window)
        g.step(sw.table, 0, steps, ep)
        torch.cuda.synchronize()
        names = ('ez', 'hx', 'hy') if sp.pol == 's' else ('ex', 'ey', 'hz')
        for c, nm in enumerate(names):
            a = sw.insts[q].f[c][:sp.nx, :sp.ny]
            b = getattr(g, nm)[:sp.nx, :sp.ny]
            assert float((a - b).norm()) <= 1e-6 * max(float(b.norm()), 1e-30), (q, nm)
        ph = (2.0 / sw.insts[q].n_acc) * ep.phasor()
        assert float((res[q]['phasor'] - ph).abs().norm()) < 1e-5 * float(ph.abs().norm()), q


@pytest.mark.gpu
def test_graph_replay_and_storage_variants():
    import torch
    from lens_sensor_b200 import batch2d as B
    specs, steps = _small_sweep(), 400
    a = B.Sweep(specs, steps, 'f32', by=4)
    a.run(graphs=False)
    b = B.Sweep(specs, steps, 'f32', by=8, geos=[q.geo for q in a.insts])
    b.run(graphs=True)
    torch.cuda.synchronize()
    for p, q in zip(a.insts, b.insts):
        for x, y in zip(p.f, q.f):
            assert torch.equal(x, y)
    ref = [r['phasor'] for r in a.results()]
    for st, tol in (('f16', TOL_F16), ('bf16', TOL_BF16)):
        c = B.Sweep(specs, steps, st, geos=[q.geo for q in a.insts])
        c.run()
        torch.cuda.synchronize()
        for q, r in enumerate(c.results()):
            err = float((r['phasor'] - ref[q]).abs().norm() / ref[q].abs().norm())
            assert err < tol, (st, q, err)


def test_overlap_uses_the_analyzer_windows():
    """Instance.overlap against the reference analyzer's band sums written out
    (common/fdtd_analyzer.py:2737-2747 index rounding, :2880-2935 windows and
    bands; custom-stack tear band), on a seeded CW amplitude.  CPU tensors."""
    import torch
    from types import SimpleNamespace
    from lens_sensor_b200 import batch2d as B
    from lens_sensor_b200.workloads import sweep2d
    specs, _ = sweep2d(count=4)
    rng = np.random.default_rng(5)
    for sp in specs:
        ph = torch.from_numpy(rng.standard_normal((sp.nx, sp.ny)) + 1j * rng.standard_normal((sp.nx, sp.ny)))
        got = B.Instance.overlap(SimpleNamespace(spec=sp), ph)
        # the analyzer: display extents x in [0, L], y in [-tear_buffer, -tear_buffer + H] (um)
        I = 0.5 * np.abs(ph.numpy()) ** 2
        L, H = sp.nx * sp.dx * 1e6, sp.ny * sp.dx * 1e6
        y0, y1 = -sp.tear_m * 1e6, -sp.tear_m * 1e6 + H
        xi = lambda v: int(round(v / L * sp.nx))
        vi = lambda v: int(round((v - y0) / (y1 - y0) * sp.ny))
        c, w = 0.8 * L, 0.1 * L
        dl = max(0, xi(c - w / 2))
        dh = max(dl + 1, min(xi(c + w / 2), sp.nx))
        lo, hi = max(0, vi(0.0)), min(sp.ny, vi(sp.stack.t_wg_um))
        tear = sum(t for t, _ in sp.stack.layers)
        tl = max(0, vi(-tear))
        band = lambda a, b: float(np.mean(np.sum(I[dl:dh, a:b], axis=1))) if b > a else 0.0
        want = band(tl, lo) / band(lo, hi)
        assert got == pytest.approx(want, rel=1e-12), (sp.nx, sp.ny, got, want)


class _FakeSweep:
    """Stand-in for batch2d.Sweep: instance q's phasor is q + 1, and reduced
    storage adds a relative error of 1e-6 (TE) or 1e-3 (TM)."""
    runs = []

    def __init__(self, specs, steps, storage='f32', by=8, budget=None, device=None, geos=None, resident=False):
        self.specs, self.storage = specs, storage
        _FakeSweep.runs.append((storage, [sp.tag for sp in specs]))

    def run(self):
        return 0

    def results(self):
        import torch
        out = []
        for sp in self.specs:
            e = 0.0 if self.storage == 'f32' else (1e-6 if sp.pol == 's' else 1e-3)
            out.append(dict(phasor=torch.full((4,), complex(sp.tag + 1, 0) * (1 + e), dtype=torch.complex128)))
        return out


def test_fp16_gate_accepts_per_polarisation(monkeypatch):
    """The gate probes every 4th instance of each polarisation in both storages,
    keeps FP16 for the TE instances (probe error 1e-6 <= tol/2) and runs the TM
    instances in FP32 (1e-3 > tol/2); probes keep their FP32 results."""
    from types import SimpleNamespace
    from lens_sensor_b200 import batch2d as B
    monkeypatch.setattr(B, 'Sweep', _FakeSweep)
    _FakeSweep.runs = []
    specs = [SimpleNamespace(pol='s' if q % 2 == 0 else 'p', tag=q) for q in range(16)]
    res, rep = B.gated_sweep(specs, 10, 'f16', tol=1e-4, probe_every=4, geos=[None] * 16)
    assert rep['accepted'] == {'s': True, 'p': False}
    probes = [p['index'] for p in rep['probes']]
    assert probes == [0, 1, 8, 9]
    assert all(res[q]['storage'] == 'f32' for q in probes)
    assert all(res[q]['storage'] == ('f16' if q % 2 == 0 else 'f32') for q in range(16) if q not in probes)
    assert rep['n_reduced'] == 6 and rep['n_f32'] == 10
    assert all(float(r['phasor'][0].real) == pytest.approx(q + 1, rel=2e-6) for q, r in enumerate(res))
    # both storages of the probes, then the accepted and the refused rest
    assert [r[0] for r in _FakeSweep.runs] == ['f32', 'f16', 'f16', 'f32']
