"""The 2D drop-in driver against the reference driver's own outputs.

tests/golden/dropin_2d.json holds, for three whole-driver cases, summaries of
everything fdtd2d_core.run_beads + save_results wrote in the reference
(planar_beads/fdtd2d_core.py:531-927, 2085-2265): every NPZ key (strings
verbatim, arrays as dtype/shape/sum/abs-sum/abs-max) and every scalar of the
PKL summary.  The 'te' case is the reference's characterization case
(tests/test_characterization.py:93-106 there).

* CPU: the driver runs on tests/_oracle_engine.py (the oracle's FP32 stepper
  with the reference's accumulation order), so the schedule, geometry and file
  writer must reproduce the reference to the last digits.
* GPU: the same driver on the CUDA engine; FP32 fields in another operation
  order, so values agree to the stated tolerances, keys/shapes/strings/step
  counts exactly.
"""
import json
import os
import pickle
import glob

import numpy as np
import pytest

import _oracle_engine
from lens_sensor_b200 import fdtd2d_core as D2

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), 'golden', 'dropin_2d.json')))
WALL_CLOCK = {'meta', 'total_time'}     # frame wall times differ run to run

# tolerances: (scalar rtol, array abs-sum/abs-max rtol, signed-sum tolerance as a
# fraction of the abs-sum, cw_rel_change absolute)
TOL_CPU = (1e-6, 1e-5, 1e-6, 1e-6)
TOL_GPU = (5e-4, 2e-3, 2e-3, 2e-4)


def _kwargs(case):
    kw = dict(case['kw'])
    if case['stack']:
        kw['stack'] = [dict(L, n=complex(*L['n'])) for L in case['stack']]
    return kw


def _run(name, engine, tmp_path, monkeypatch):
    case = GOLD[name]
    monkeypatch.chdir(tmp_path)
    monkeypatch.setattr(D2, 'KAPPA', dict(case['kappa']))
    if engine is not None:
        monkeypatch.setattr(D2, 'E', engine)
    r = D2.run_beads(**_kwargs(case))
    # the frame stream file is removed by save_results (as the reference does): keep its frames
    r['_frames_before_save'] = np.array(np.load(r['frames_memmap'], mmap_mode='r')[:len(r['frames'])])
    npz = D2.save_results(r)
    with open(glob.glob('results/*.pkl')[0], 'rb') as f:
        pk = pickle.load(f)
    return r, np.load(npz), pk


def _check(name, z, pk, tol):
    rs, ra, rsum, rcw = tol
    g = GOLD[name]
    assert sorted(z.files) == sorted(g['npz']), (set(z.files) ^ set(g['npz']))
    for k, want in g['npz'].items():
        a = np.asarray(z[k])
        if want['kind'] == 'str':
            assert [str(x) for x in a.ravel()] == want['value'], k
            continue
        assert str(a.dtype) == want['dtype'] and list(a.shape) == want['shape'], k
        if k in WALL_CLOCK or not a.size:
            continue
        c = a.astype(np.complex128)
        tol_a = rs if a.size == 1 else ra
        np.testing.assert_allclose(np.abs(c).max(), want['absmax'], rtol=tol_a, err_msg=k)
        np.testing.assert_allclose(np.abs(c).sum(), want['abssum'], rtol=tol_a, err_msg=k)
        bound = (rs if a.size == 1 else rsum) * want['abssum'] + 1e-300
        assert abs(c.real.sum() - want['sum'][0]) <= bound, (k, c.real.sum(), want['sum'])
        assert abs(c.imag.sum() - want['sum'][1]) <= bound, (k, c.imag.sum(), want['sum'])
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
    r, z, pk = _run(name, _oracle_engine, tmp_path, monkeypatch)
    _check(name, z, pk, TOL_CPU)


def test_characterization_known_answer(tmp_path, monkeypatch):
    """The reference's own golden-master numbers (characterization.json, case_2d)."""
    ch = json.load(open(os.path.join(os.path.dirname(__file__), 'golden', 'characterization.json')))['case_2d']
    r, z, pk = _run('te', _oracle_engine, tmp_path, monkeypatch)
    for k in ('transmission', 'P_in', 'P_out'):
        np.testing.assert_allclose(r[k], ch[k], rtol=1e-6)
    ez = np.asarray(r['_frames_before_save'], np.float64)
    assert list(ez.shape) == ch['frames']['shape']
    np.testing.assert_allclose([ez.sum(), np.abs(ez).max(), ez.mean()],
                               [ch['frames']['sum'], ch['frames']['absmax'], ch['frames']['mean']], rtol=1e-6)


def test_unsupported_paths_refuse():
    with pytest.raises(NotImplementedError):
        D2.run_beads('pmma', 'polystyrol', 0.5, method='stitch', source_type='pulse', pulse_mode='td')
    with pytest.raises(NotImplementedError):
        D2.run_beads('pmma', 'polystyrol', 0.5, boundary='mur')


@pytest.mark.gpu
@pytest.mark.parametrize('name', sorted(GOLD))
def test_driver_on_gpu(name, tmp_path, monkeypatch):
    r, z, pk = _run(name, None, tmp_path, monkeypatch)
    _check(name, z, pk, TOL_GPU)
