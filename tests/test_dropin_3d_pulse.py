"""The 3D Fourier pulse stitch drop-in (run_3d_stitched_pulse) against the
reference driver's outputs.

tests/golden/dropin_3d_pulse.json holds, for two whole-driver cases, the
result scalars, the transmission spectrum, summaries of the synthesised frame
volumes, <E^2> and the centre-frequency CW set, and of everything
run_3d_stitched_pulse + save_results_3d wrote in the reference
(planar_3d/fdtd3d_core.py:2087-2215, 2218-2461): 'te_disp' 3 frequencies with
the core's n from n(lambda_k); 'tm_fixed' 3 frequencies with the indices held,
an absorbing stack, a channel core and a set t_max.  Each frequency is a CW
run_3d_stitched on the engine; the frames are synthesised on the device in
complex64, as the reference sums them.

* CPU: the driver on tests/_oracle_engine.py: to the last digits (torch and
  numpy may round a complex64 product differently in the last bit).
* GPU: the same driver on the CUDA engine: values to the stated tolerances.
"""
import glob
import json
import os
import pickle

import numpy as np
import pytest

import _oracle_engine
from lens_sensor_b200 import fdtd3d_core as D3
from test_dropin_2d_stitch import _summ_check
from test_dropin_3d import _check_arrays

HERE = os.path.dirname(__file__)
GOLD = json.load(open(os.path.join(HERE, 'golden', 'dropin_3d_pulse.json')))
WALL_CLOCK = {'meta', 'times', 'total_time'}

# (scalar rtol, array abs-sum/abs-max rtol, signed-sum tolerance / abs-sum, unused)
TOL_CPU = (1e-6, 1e-5, 1e-6, 0.0)
TOL_GPU = (1e-3, 2e-3, 3e-3, 0.0)


def _run(name, engine, tmp_path, monkeypatch):
    case = GOLD[name]
    monkeypatch.chdir(tmp_path)
    monkeypatch.setattr(D3, 'KAPPA', dict(case['kappa']))
    if engine is not None:
        monkeypatch.setattr(D3, 'E', engine)
    kw = dict(case['kw'])
    if case['stack']:
        kw['stack'] = [dict(L, n=complex(*L['n'])) for L in case['stack']]
    r = D3.run_3d_stitched_pulse(**kw)
    keep = {k: r[k] for k in case['result']}
    spec = {k: np.asarray(r['spectrum'][k], np.float64) for k in case['spectrum']}
    arrays = dict(vols=np.array(r['vols_array']), Iavg=np.array(r['Iavg']), cw_vol=np.array(r['cw_vol']))
    D3.save_results_3d(r)
    files = {os.path.basename(f).replace(kw['label'], '{label}'): np.load(f) for f in glob.glob('results/*.npz')}
    with open(glob.glob('results/*.pkl')[0], 'rb') as f:
        pk = pickle.load(f)
    left = sorted(os.listdir('results'))
    return keep, spec, arrays, files, pk, left


def _check(name, keep, spec, arrays, files, pk, left, tol):
    g = GOLD[name]
    rs = tol[0]
    for k, want in g['result'].items():
        np.testing.assert_allclose(keep[k], want, rtol=rs, atol=1e-300, err_msg=k)
    for k, want in g['spectrum'].items():
        np.testing.assert_allclose(spec[k], want, rtol=rs, err_msg=k)
    for k, w in g['arrays'].items():
        _summ_check(arrays[k], w, tol[:3], k)
    assert left == g['files_left'], left
    assert sorted(files) == sorted(g['npz'])
    for fname, want in g['npz'].items():
        _check_arrays(name, files[fname], want, tol, fname)
    for k, want in g['pkl'].items():
        if k in WALL_CLOCK:
            continue
        got = pk[k]
        if isinstance(want, list):
            np.testing.assert_allclose([np.real(got), np.imag(got)], want, rtol=rs, err_msg=k)
        elif isinstance(want, float):
            np.testing.assert_allclose(float(np.real(got)), want, rtol=rs, err_msg=k)
        else:
            assert got == want, (k, got, want)


@pytest.mark.parametrize('name', sorted(GOLD))
def test_pulse_stitch_3d_on_oracle_engine(name, tmp_path, monkeypatch):
    _check(name, *_run(name, _oracle_engine, tmp_path, monkeypatch), TOL_CPU)


def test_pulse_stitch_3d_refuses_cad():
    with pytest.raises(NotImplementedError):
        D3.run_3d_stitched_pulse('x', 1.49, cad=object())


@pytest.mark.gpu
@pytest.mark.parametrize('name', sorted(GOLD))
def test_pulse_stitch_3d_on_gpu(name, tmp_path, monkeypatch):
    _check(name, *_run(name, None, tmp_path, monkeypatch), TOL_GPU)
