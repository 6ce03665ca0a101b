"""The 2D Fourier pulse stitch drop-in (run_beads(method='stitch',
source_type='pulse') -> run_beads_stitched_pulse) against the reference
driver's own outputs.

tests/golden/dropin_2d_pulse.json holds, for two whole-driver cases, the
result scalars, the transmission spectrum, a summary of the synthesised time
frames and summaries of everything run_beads_stitched_pulse + save_results
wrote in the reference (planar_beads/fdtd2d_core.py:1866-2017, 2085-2265):
'te_disp' 5 frequencies with the core's n following n(lambda_k); 'tm_fixed' 5
frequencies with every index held at lambda0, an absorbing stack, KAPPA on the
core, an input gap, a tilted offset source and a set t_max.  Each frequency is a
CW stitch on the engine; the frames are synthesised on the device.

* CPU: the driver on tests/_oracle_engine.py: to the last digits (the device
  synthesis runs in torch complex128, the reference's in numpy).
* GPU: the same driver on the CUDA engine: values to the stated tolerances.
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
GOLD = json.load(open(os.path.join(HERE, 'golden', 'dropin_2d_pulse.json')))
WALL_CLOCK = {'meta', 'total_time'}
PID_PATHS = {'frames_memmap', 'cw_frames_memmap'}

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
    keep = {k: r[k] for k in case['result']}
    spec = {k: np.asarray(r['spectrum'][k], np.float64) for k in case['spectrum']}
    frames = np.array(np.load(r['frames_memmap'], mmap_mode='r')[:len(r['frames'])])
    D2.save_results(r)
    z = np.load(glob.glob('results/*_frames.npz')[0])
    with open(glob.glob('results/*.pkl')[0], 'rb') as f:
        pk = pickle.load(f)
    left = sorted(re.sub(r'_\d+_\d+\.npy$', '_{tag}.npy', f) for f in os.listdir('results'))
    return keep, spec, frames, z, pk, left


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


def _check(name, keep, spec, frames, z, pk, left, tol):
    g = GOLD[name]
    for k, want in g['result'].items():
        np.testing.assert_allclose(keep[k], want, rtol=tol[0], err_msg=k)
    for k, want in g['spectrum'].items():
        np.testing.assert_allclose(spec[k], want, rtol=tol[0], err_msg=k)
    _summ_check(frames, g['frames'], tol, 'frames')
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
        elif k in PID_PATHS:          # temporary stream files carry the process id
            pid = lambda v: re.sub(r'_\d+\.npy$', '_{pid}.npy', str(v))
            assert pid(got) == pid(want), (k, got, want)
        else:
            assert got == want, (k, got, want)
    assert sorted(k for k in pk if k in g['pkl']) == sorted(g['pkl'])


@pytest.mark.parametrize('name', sorted(GOLD))
def test_pulse_stitch_driver_on_oracle_engine(name, tmp_path, monkeypatch):
    _check(name, *_run(name, _oracle_engine, tmp_path, monkeypatch), TOL_CPU)


def test_time_domain_pulse_stitch_refuses():
    with pytest.raises(NotImplementedError):
        D2.run_beads('pmma', 'polystyrol', 0.5, method='stitch', source_type='pulse', pulse_mode='td')


@pytest.mark.gpu
@pytest.mark.parametrize('name', sorted(GOLD))
def test_pulse_stitch_driver_on_gpu(name, tmp_path, monkeypatch):
    _check(name, *_run(name, None, tmp_path, monkeypatch), TOL_GPU)
