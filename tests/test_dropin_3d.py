"""The 3D drop-in driver against the reference driver's own outputs.

tests/golden/dropin_3d.json holds, for three whole-driver cases, summaries of
everything fdtd3d_core.run_3d + save_results_3d wrote in the reference
(planar_3d/fdtd3d_core.py:793-1308, 2218-2461): both NPZ files key by key
(strings verbatim, arrays as dtype/shape/sum/abs-sum/abs-max) and every scalar
of the PKL summary.  'golden3d' is the reference's characterization case
(tests/test_characterization.py:73-84 there).

* CPU: the driver runs on tests/_oracle_engine.py (the oracle's FP32 stepper
  with the reference's accumulation order): schedule, geometry, convergence
  extension and file writers must reproduce the reference to the last digits.
* GPU: the same driver on the CUDA engine, FP32 in another operation order:
  values to the stated tolerances; keys, shapes, strings and step counts exact.
"""
import glob
import json
import os
import pickle

import numpy as np
import pytest

import _oracle_engine
from lens_sensor_b200 import fdtd3d_core as D3

HERE = os.path.dirname(__file__)
GOLD = json.load(open(os.path.join(HERE, 'golden', 'dropin_3d.json')))
WALL_CLOCK = {'meta', 'times', 'total_time'}

# (scalar rtol, array abs-sum/abs-max rtol, signed-sum tolerance / abs-sum, cw_rel_change abs)
TOL_CPU = (1e-6, 1e-5, 1e-6, 1e-6)
TOL_GPU = (5e-4, 2e-3, 2e-3, 2e-4)


def _run(name, engine, tmp_path, monkeypatch):
    case = GOLD[name]
    monkeypatch.chdir(tmp_path)
    monkeypatch.setattr(D3, 'KAPPA', dict(case['kappa']))
    if engine is not None:
        monkeypatch.setattr(D3, 'E', engine)
    kw = dict(case['kw'])
    if case['stack']:
        kw['stack'] = [dict(L, n=complex(*L['n'])) for L in case['stack']]
    r = D3.run_3d(**kw)
    keep = dict(steps_total=r['steps_total'], transmission=r['transmission'], P_in=r['P_in'], P_out=r['P_out'],
                Iavg=np.array(r['Iavg']), vols=np.array(r['vols_array']))
    D3.save_results_3d(r)
    files = {os.path.basename(f).replace(kw['label'], '{label}'): np.load(f) for f in glob.glob('results/*.npz')}
    with open(glob.glob('results/*.pkl')[0], 'rb') as f:
        pk = pickle.load(f)
    left = [p for p in glob.glob('results/_stream3d_*')]
    return keep, files, pk, left


def _check_arrays(name, z, want, tol, fname):
    rs, ra, rsum, _ = tol
    assert sorted(z.files) == sorted(want), (fname, set(z.files) ^ set(want))
    for k, w in want.items():
        a = np.asarray(z[k])
        if w['kind'] == 'str':
            assert [str(x) for x in a.ravel()] == w['value'], (fname, k)
            continue
        assert str(a.dtype) == w['dtype'] and list(a.shape) == w['shape'], (fname, k, a.dtype, a.shape)
        if k in WALL_CLOCK or not a.size:
            continue
        c = a.astype(np.complex128)
        t = rs if a.size == 1 else ra
        np.testing.assert_allclose(np.abs(c).max(), w['absmax'], rtol=t, err_msg=f'{fname}:{k}')
        np.testing.assert_allclose(np.abs(c).sum(), w['abssum'], rtol=t, err_msg=f'{fname}:{k}')
        bound = (rs if a.size == 1 else rsum) * w['abssum'] + 1e-300
        assert abs(c.real.sum() - w['sum'][0]) <= bound, (fname, k, c.real.sum(), w['sum'])
        assert abs(c.imag.sum() - w['sum'][1]) <= bound, (fname, k, c.imag.sum(), w['sum'])


def _check(name, files, pk, tol):
    g = GOLD[name]
    assert sorted(files) == sorted(g['npz'])
    for fname, want in g['npz'].items():
        _check_arrays(name, files[fname], want, tol, fname)
    rs, _, _, rcw = tol
    for k, want in g['pkl'].items():
        if k in WALL_CLOCK:
            continue
        got = pk[k]
        if k == 'cw_rel_change':
            assert abs(got - want) <= rcw, (k, got, want)
        elif isinstance(want, list):
            np.testing.assert_allclose([np.real(got), np.imag(got)], want, rtol=rs, err_msg=k)
        elif isinstance(want, float):
            np.testing.assert_allclose(float(np.real(got)), want, rtol=rs, err_msg=k)
        else:
            assert got == want, (k, got, want)


@pytest.mark.parametrize('name', sorted(GOLD))
def test_driver_on_oracle_engine(name, tmp_path, monkeypatch):
    keep, files, pk, left = _run(name, _oracle_engine, tmp_path, monkeypatch)
    _check(name, files, pk, TOL_CPU)
    assert not left, left            # the temporary stream files are removed


def test_characterization_known_answer(tmp_path, monkeypatch):
    """The reference's own golden-master numbers (characterization.json, case_3d)."""
    ch = json.load(open(os.path.join(HERE, 'golden', 'characterization.json')))['case_3d']
    keep, _, _, _ = _run('golden3d', _oracle_engine, tmp_path, monkeypatch)
    for k in ('transmission', 'P_in', 'P_out'):
        np.testing.assert_allclose(keep[k], ch[k], rtol=1e-6)
    for k, key in (('Iavg', 'Iavg'), ('vols', 'vols')):
        a = keep[k].astype(np.float64)
        assert list(a.shape) == ch[key]['shape']
        np.testing.assert_allclose([a.sum(), np.abs(a).max(), a.mean()],
                                   [ch[key]['sum'], ch[key]['absmax'], ch[key]['mean']], rtol=1e-6)


def test_unsupported_paths_refuse():
    with pytest.raises(NotImplementedError):
        D3.run_3d('x', 1.49, source_type='pulse')
    with pytest.raises(NotImplementedError):
        D3.run_3d('x', 1.49, boundary='sponge')


@pytest.mark.gpu
@pytest.mark.parametrize('name', sorted(GOLD))
def test_driver_on_gpu(name, tmp_path, monkeypatch):
    keep, files, pk, left = _run(name, None, tmp_path, monkeypatch)
    _check(name, files, pk, TOL_GPU)
