"""The temporally blocked 3D step (lens_fdtd3d_step_tb: two steps per launch,
epilogues fused) against the fused single-step kernel it replaces
(lens_fdtd3d_step), whose fields the oracle tests pin to the reference
(test_gpu_parity.py) and to FP64 at full size (test_fp64_fullsize.py).

Cases: the golden TM lossy grid with a bead, a TE grid whose sizes are not
multiples of the 12 x 28 tile, odd chunk lengths, and steps inside the DFT,
convergence and flux windows with detector boxes, so every fused epilogue is
compared: fields, volume phasors, convergence planes, flux sums and box sums.
"""
import json
import os

import numpy as np
import pytest

from oracle import harness as H

CASES = json.load(open(os.path.join(os.path.dirname(__file__), 'golden', 'cases.json')))
TOL = 2e-6        # relative L2: the same arithmetic, contracted (FMA) differently in places
TOL_ACC = 1e-5    # box and flux sums, phasors


def _grid(c, tb, chunk=40):
    from lens_sensor_b200 import engine as E
    s = H.setup_3d(c)
    src = dict(ix=s['src'].ix, amp=s['src'].amp, ph1=s['src'].ph1, ph2=s['src'].ph2)
    comp = 1 if c['pol'] == 'p' else 2
    g = E.Grid3D(c['Nx'], c['Ny'], c['Nz'], s['dx'], s['dt'], (s['ce_x'], s['ce_y'], s['ce_z']), s['da'],
                 s['cpml'], src, src_comp=comp, fused=True, tb=tb, tb_chunk=chunk)
    return g, s, comp


def _run(c, tb, steps, chunk=40):
    import torch
    from lens_sensor_b200 import engine as E
    g, s, comp = _grid(c, tb, chunk)
    tab = E.StepTable(0, steps, s['dt'], s['src'].omega, 2 * np.pi * s['f0'], E.cw_envelope(s['f0']))
    nsp = s['n_sp']
    nd = steps // 3
    ep = E.Epi3D(g, boxes=[(10, c['Nx'] - 12, 5, 30, nsp, -nsp), (30, 40, 0, c['Ny'], 0, c['Nz'])],
                 dft=(steps - nd, steps), comps=(0, 1, 2),
                 planes={'in': 20, 'out': c['Nx'] - 15, 'up': s['src'].ix - 1},
                 conv=(c['Nz'] // 2, (steps - 2 * nd, steps - nd)))
    if tb:
        g.step_tb(tab, 0, steps, ep)
    else:
        g.step(tab, 0, steps, ep)
    torch.cuda.synchronize()
    g.check_flag()
    return g, ep


def _rel(a, b):
    import torch
    a, b = a.double(), b.double()
    return float(torch.linalg.norm(a - b) / max(float(torch.linalg.norm(b)), 1e-300))


def _compare(c, steps, chunk=40):
    ref, er = _run(c, False, steps)
    tb, et = _run(c, True, steps, chunk)
    out = {}
    for names in (('ex', 'ey', 'ez'), ('hx', 'hy', 'hz')):
        import torch
        tot = float(torch.sqrt(sum(torch.linalg.norm(ref.view(n).double()) ** 2 for n in names)))
        for n in names:
            out[n] = float(torch.linalg.norm(tb.view(n).double() - ref.view(n).double())) / max(tot, 1e-300)
    for q in range(3):
        out[f'dft{q}'] = _rel(et.dft[q], er.dft[q])
    out['conv_last'] = _rel(et.conv_last, er.conv_last)
    out['conv_prev'] = _rel(et.conv_prev, er.conv_prev)
    out['planes'] = _rel(et.plane_acc, er.plane_acc)
    out['boxes'] = _rel(et.box_acc, er.box_acc)
    # (the two paths hold the state in different buffers: one flip per launch)
    for n in ('ex', 'ey', 'ez', 'hx', 'hy', 'hz'):
        assert out[n] <= TOL, (n, out)
    for n in ('dft0', 'dft1', 'dft2', 'conv_last', 'conv_prev', 'planes', 'boxes'):
        assert out[n] <= TOL_ACC, (n, out)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize('chunk', [40, 7])
def test_tb3d_matches_fused_golden_tm(chunk):
    print(_compare(dict(CASES['d3']), 90, chunk))


@pytest.mark.gpu
def test_tb3d_matches_fused_te_odd_sizes():
    c = dict(CASES['d3'], pol='s', Nx=71, Ny=37, Nz=61)
    print(_compare(c, 60, 13))


@pytest.mark.gpu
def test_tb3d_odd_span_uses_one_single_step():
    import torch
    from lens_sensor_b200 import engine as E
    c = dict(CASES['d3'])
    a, s, _ = _grid(c, True)
    b, _, _ = _grid(c, False)
    tab = E.StepTable(0, 31, s['dt'], s['src'].omega, 2 * np.pi * s['f0'], E.cw_envelope(s['f0']))
    a.step_tb(tab, 0, 31)
    b.step(tab, 0, 31)
    torch.cuda.synchronize()
    assert _rel(a.view('ey'), b.view('ey')) <= TOL


@pytest.mark.gpu
def test_tb3d_refuses_odd_steps_and_missing_scratch():
    import ctypes
    from lens_sensor_b200 import _native as N
    from lens_sensor_b200 import engine as E
    lib = N.load()
    g, s, _ = _grid(dict(CASES['d3']), True)
    tab = E.StepTable(0, 8, s['dt'], s['src'].omega, 2 * np.pi * s['f0'], E.cw_envelope(s['f0']))
    assert lib.lens_fdtd3d_step_tb(ctypes.byref(g.s), ctypes.byref(g.tb), ctypes.byref(tab.s), None, 0, 3, None) == -1
    t = N.TB3D()
    t.chunk = 40
    assert lib.lens_fdtd3d_step_tb(ctypes.byref(g.s), ctypes.byref(t), ctypes.byref(tab.s), None, 0, 2, None) == -1


@pytest.mark.gpu
def test_tb3d_full_size_config1_start():
    """The config-1 grid (480 x 192 x 256, lossy, two beads) over 60 steps."""
    import torch
    from lens_sensor_b200.solver3d import Solve3D
    from lens_sensor_b200.workloads import waveguide3d_tm
    sp, _ = waveguide3d_tm()
    a = Solve3D(sp, 60, comps=(0, 1, 2), engine='fused')
    a.run()
    geo = a.geo
    b = Solve3D(sp, 60, comps=(0, 1, 2), engine='tb', geo=geo)
    b.run()
    torch.cuda.synchronize()
    # against the norm of the whole E (a weak component's own norm is small)
    tot = float(torch.sqrt(sum(torch.linalg.norm(a.grid.view(n).double()) ** 2 for n in ('ex', 'ey', 'ez'))))
    for n in ('ex', 'ey', 'ez'):
        d = float(torch.linalg.norm(b.grid.view(n).double() - a.grid.view(n).double()))
        assert d <= TOL * tot, (n, d / tot)
    ra, rb = a.results(), b.results()
    for k in ('P_in', 'P_out'):
        np.testing.assert_allclose(rb[k], ra[k], rtol=TOL_ACC)
