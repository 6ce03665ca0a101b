"""Failure detection without a GPU fault.

* The fused 3D step bounds every pipeline wait; lens_fdtd3d_watchdog_test runs
  one step in which one CTA's wait runs out (a copy that is never issued, with
  the bound cut to a few hundred tries): the launch must end normally, bit 1 of
  the grid's flag must be set (the host raises on it), and the grid must step
  correctly afterwards.
* A NaN planted in the fields on the host reaches a detector box: the box
  reduction sets bit 2 of the flag and the host raises instead of returning
  numbers.
* A solve with no fault leaves the flag at 0.
No test here faults, traps or hangs a GPU.
"""
import ctypes
import json
import os

import numpy as np
import pytest

from oracle import harness as H

CASES = json.load(open(os.path.join(os.path.dirname(__file__), 'golden', 'cases.json')))


def _grid():
    from lens_sensor_b200 import engine as E
    c = dict(CASES['d3'])
    s = H.setup_3d(c)
    src = dict(ix=s['src'].ix, amp=s['src'].amp, ph1=s['src'].ph1, ph2=s['src'].ph2)
    g = E.Grid3D(c['Nx'], c['Ny'], c['Nz'], s['dx'], s['dt'], (s['ce_x'], s['ce_y'], s['ce_z']), s['da'],
                 s['cpml'], src, src_comp=1, fused=True)
    tab = E.StepTable(0, 64, s['dt'], s['src'].omega, 2 * np.pi * s['f0'], E.cw_envelope(s['f0']))
    return g, tab, s


@pytest.mark.gpu
def test_watchdog_timeout_sets_the_flag_and_the_grid_recovers():
    import torch
    from lens_sensor_b200 import _native as N
    lib = N.load()
    g, tab, _ = _grid()
    g.step(tab, 0, 20)
    torch.cuda.synchronize()
    assert int(g.flag.item()) == 0
    saved = {b: {f: t.clone() for f, t in buf.items()} for b, buf in enumerate(g.bufs)}
    psi = {b: {q: t.clone() for q, t in p.items()} for b, p in enumerate(g.psi)}
    cur = g.s.cur
    st = lib.lens_fdtd3d_watchdog_test(ctypes.byref(g.s), ctypes.byref(tab.s), 20, 1, None)
    assert st == 0                      # the launch itself succeeded
    torch.cuda.synchronize()            # and ended: the context is usable
    assert int(g.flag.item()) & 1
    with pytest.raises(N.LensError, match='timed out'):
        g.check_flag()
    # restore the state of step 20 and the flag; the next steps match an untouched grid
    for b, buf in enumerate(g.bufs):
        for f, t in buf.items():
            t.copy_(saved[b][f])
    for b, p in enumerate(g.psi):
        for q, t in p.items():
            t.copy_(psi[b][q])
    g.s.cur = cur
    g.flag.zero_()
    g.step(tab, 20, 24)
    ref, _, _ = _grid()
    ref.step(tab, 0, 44)
    torch.cuda.synchronize()
    assert int(g.flag.item()) == 0 and int(ref.flag.item()) == 0
    for f in g.FIELDS:
        assert torch.equal(g.view(f), ref.view(f)), f


@pytest.mark.gpu
def test_watchdog_arguments_are_checked():
    from lens_sensor_b200 import _native as N
    lib = N.load()
    g, tab, _ = _grid()
    assert lib.lens_fdtd3d_watchdog_test(ctypes.byref(g.s), ctypes.byref(tab.s), 0, 2, None) == -1
    g.s.flag = None
    assert lib.lens_fdtd3d_watchdog_test(ctypes.byref(g.s), ctypes.byref(tab.s), 0, 1, None) == -1


@pytest.mark.gpu
def test_nan_in_a_detector_box_is_reported():
    import torch
    from lens_sensor_b200 import _native as N
    from lens_sensor_b200 import engine as E
    g, tab, s = _grid()
    nsp = s['n_sp']
    ep = E.Epi3D(g, boxes=[(36, 44, 20, 34, nsp, -nsp)])
    g.step(tab, 0, 10, ep)
    torch.cuda.synchronize()
    g.check_flag()                                  # clean so far
    g.ey[40, 25, 18] = float('nan')                 # planted on the host side of the API
    g.step(tab, 10, 2, ep)
    torch.cuda.synchronize()
    assert int(g.flag.item()) & 2
    with pytest.raises(N.LensError, match='not finite'):
        g.check_flag()
