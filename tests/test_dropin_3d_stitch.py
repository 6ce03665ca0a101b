"""The 3D stitch drop-in (run_3d_stitched) against the reference driver's outputs.

tests/golden/dropin_3d_stitch.json holds, for two whole-driver cases, the
result scalars and summaries of everything fdtd3d_core.run_3d_stitched +
save_results_3d wrote in the reference (planar_3d/fdtd3d_core.py:1311-1782,
2218-2461): both NPZ files key by key and every scalar of the PKL summary.
'goldenstitch' is the reference's characterization case
(tests/test_characterization.py:87-99 there); 'tm_stack' runs 4 windows on an
absorbing stack with a channel core, a bead across a window seam and a tilted,
offset source behind an input gap.

* CPU: the driver runs on tests/_oracle_engine.py, which steps with the
  oracle's FP32 stepper and accumulates exactly as the reference's stitch loop
  (float32 re/im volume DFT, complex64 overlap handoff, taper drive): window
  plan, geometry of each window, handoff, assembly and file writers must
  reproduce the reference to the last digits.
* GPU: the same driver on the CUDA engine (fused step, drive kernel, on-device
  handoff); FP32 in another operation order, values to the stated tolerances,
  keys, shapes, strings and step counts exact.
"""
import glob
import json
import os
import pickle

import numpy as np
import pytest

import _oracle_engine
from lens_sensor_b200 import fdtd3d_core as D3
from test_dropin_3d import _check_arrays

HERE = os.path.dirname(__file__)
GOLD = json.load(open(os.path.join(HERE, 'golden', 'dropin_3d_stitch.json')))
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
    r = D3.run_3d_stitched(**kw)
    keep = {k: r[k] for k in ('transmission', 'P_in', 'P_out', 'transmission_intensity', 'steps_total')}
    keep.update(Iavg=np.array(r['Iavg']), vols=np.array(r['vols_array']))
    D3.save_results_3d(r)
    files = {os.path.basename(f).replace(kw['label'], '{label}'): np.load(f) for f in glob.glob('results/*.npz')}
    with open(glob.glob('results/*.pkl')[0], 'rb') as f:
        pk = pickle.load(f)
    left = sorted(os.listdir('results'))
    return keep, files, pk, left


def _check(name, keep, files, pk, left, tol):
    g = GOLD[name]
    rs = tol[0]
    for k, want in g['result'].items():
        if isinstance(want, int):
            assert keep[k] == want, (k, keep[k], want)
        else:
            np.testing.assert_allclose(keep[k], want, rtol=rs, atol=1e-300, err_msg=k)
    assert left == g['files_left'], left          # stream memmaps removed, the Efull temp too
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
def test_stitch_driver_on_oracle_engine(name, tmp_path, monkeypatch):
    keep, files, pk, left = _run(name, _oracle_engine, tmp_path, monkeypatch)
    _check(name, keep, files, pk, left, TOL_CPU)


def test_stitch_characterization_known_answer(tmp_path, monkeypatch):
    """The reference's own golden-master numbers (characterization.json, case_3d_stitch)."""
    ch = json.load(open(os.path.join(HERE, 'golden', 'characterization.json')))['case_3d_stitch']
    keep, _, _, _ = _run('goldenstitch', _oracle_engine, tmp_path, monkeypatch)
    for k in ('transmission', 'P_in', 'P_out'):
        np.testing.assert_allclose(keep[k], ch[k], rtol=1e-6)
    a = keep['Iavg'].astype(np.float64)
    assert list(a.shape) == ch['Iavg']['shape']
    np.testing.assert_allclose([a.sum(), np.abs(a).max(), a.mean()],
                               [ch['Iavg']['sum'], ch['Iavg']['absmax'], ch['Iavg']['mean']], rtol=1e-6)
    assert list(keep['vols'].shape) == ch['vols_shape']
    np.testing.assert_allclose(np.abs(keep['vols'].astype(np.float64)).max(), ch['vols_absmax'], rtol=1e-6)


def test_stitch_unsupported_paths_refuse():
    with pytest.raises(NotImplementedError):
        D3.run_3d_stitched('x', 1.49, boundary='sponge')
    with pytest.raises(NotImplementedError):
        D3.run_3d_stitched('x', 1.49, cad=object())


@pytest.mark.gpu
@pytest.mark.parametrize('name', sorted(GOLD))
def test_stitch_driver_on_gpu(name, tmp_path, monkeypatch):
    keep, files, pk, left = _run(name, None, tmp_path, monkeypatch)
    _check(name, keep, files, pk, left, TOL_GPU)
