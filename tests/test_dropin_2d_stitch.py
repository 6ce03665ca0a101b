"""The 2D stitch drop-in (run_beads(method='stitch') -> run_beads_stitched)
against the reference driver's own outputs.

tests/golden/dropin_2d_stitch.json holds, for two whole-driver cases, the result
scalars, the TM <|E|^2> and Ex amplitude arrays and summaries of everything
run_beads_stitched + save_results wrote in the reference
(planar_beads/fdtd2d_core.py:1197-1583, 2085-2265): 'te' 3 windows on the
characterization stack, the last flush with the domain end; 'tm' 4 windows on
an absorbing stack with KAPPA on the core, an input gap, a tilted offset source
and a bead across a seam.

* CPU: the driver on tests/_oracle_engine.py (oracle FP32 stepper; the
  reference's complex64 window sums, the FP64 drive expression before the PEC
  termination): everything to the last digits.
* GPU: the same driver on the CUDA engine (drive fused into the E pass, on-device
  handoff): FP32 in another operation order, values to the stated tolerances.
"""
import glob
import json
import os
import pickle
import re

import numpy as np
import pytest

import _oracle_engine
from lens_sensor_b200 import fdtd2d_core as D2

HERE = os.path.dirname(__file__)
GOLD = json.load(open(os.path.join(HERE, 'golden', 'dropin_2d_stitch.json')))
WALL_CLOCK = {'meta', 'total_time'}

# (scalar rtol, array abs-sum/abs-max rtol, signed-sum tolerance / abs-sum)
TOL_CPU = (1e-6, 1e-5, 1e-6)
TOL_GPU = (1e-3, 2e-3, 3e-3)


def _run(name, engine, tmp_path, monkeypatch):
    case = GOLD[name]
    monkeypatch.chdir(tmp_path)
    monkeypatch.setattr(D2, 'KAPPA', dict(case['kappa']))
    if engine is not None:
        monkeypatch.setattr(D2, 'E', engine)
    kw = dict(case['kw'])
    if case['stack']:
        kw['stack'] = [dict(L, n=complex(*L['n'])) for L in case['stack']]
    r = D2.run_beads(**kw)
    keep = {k: r[k] for k in ('transmission', 'P_in', 'P_out', 'transmission_intensity')}
    arrays = {k: np.array(r[k]) for k in ('Iavg', 'Ex_cw_amp') if r.get(k) is not None}
    D2.save_results(r)
    z = np.load(glob.glob('results/*_frames.npz')[0])
    with open(glob.glob('results/*.pkl')[0], 'rb') as f:
        pk = pickle.load(f)
    left = sorted(re.sub(r'_\d+_\d+\.npy$', '_{tag}.npy', f) for f in os.listdir('results'))
    return keep, arrays, z, pk, left


def _summ_check(a, w, tol, key):
    rs, ra, rsum = tol
    if w['kind'] == 'str':
        assert [str(x) for x in np.asarray(a).ravel()] == w['value'], key
        return
    a = np.asarray(a)
    assert str(a.dtype) == w['dtype'] and list(a.shape) == w['shape'], (key, a.dtype, a.shape)
    if key in WALL_CLOCK or not a.size:
        return
    c = a.astype(np.complex128)
    t = rs if a.size == 1 else ra
    np.testing.assert_allclose(np.abs(c).max(), w['absmax'], rtol=t, err_msg=key)
    np.testing.assert_allclose(np.abs(c).sum(), w['abssum'], rtol=t, err_msg=key)
    bound = (rs if a.size == 1 else rsum) * w['abssum'] + 1e-300
    assert abs(c.real.sum() - w['sum'][0]) <= bound, (key, c.real.sum(), w['sum'])
    assert abs(c.imag.sum() - w['sum'][1]) <= bound, (key, c.imag.sum(), w['sum'])


def _check(name, keep, arrays, z, pk, left, tol):
    g = GOLD[name]
    for k, want in g['result'].items():
        np.testing.assert_allclose(keep[k], want, rtol=tol[0], err_msg=k)
    assert sorted(arrays) == sorted(g['arrays'])
    for k, w in g['arrays'].items():
        _summ_check(arrays[k], w, tol, k)
    assert left == g['files_left'], left
    assert sorted(z.files) == sorted(g['npz']), set(z.files) ^ set(g['npz'])
    for k, w in g['npz'].items():
        _summ_check(z[k], w, tol, k)
    for k, want in g['pkl'].items():
        if k in WALL_CLOCK:
            continue
        got = pk[k]
        if isinstance(want, list):
            np.testing.assert_allclose([np.real(got), np.imag(got)], want, rtol=tol[0], err_msg=k)
        elif isinstance(want, float):
            np.testing.assert_allclose(float(np.real(got)), want, rtol=tol[0], err_msg=k)
        else:
            assert got == want, (k, got, want)
    assert sorted(k for k in pk if k in g['pkl']) == sorted(g['pkl'])


@pytest.mark.parametrize('name', sorted(GOLD))
def test_stitch2d_driver_on_oracle_engine(name, tmp_path, monkeypatch):
    _check(name, *_run(name, _oracle_engine, tmp_path, monkeypatch), TOL_CPU)


def test_stitch2d_unsupported_paths_refuse():
    with pytest.raises(NotImplementedError):
        D2.run_beads('pmma', 'polystyrol', 0.5, method='stitch', boundary='mur1')


@pytest.mark.gpu
@pytest.mark.parametrize('name', sorted(GOLD))
def test_stitch2d_driver_on_gpu(name, tmp_path, monkeypatch):
    _check(name, *_run(name, None, tmp_path, monkeypatch), TOL_GPU)
