"""Pin the oracle to the reference: every setup array and every field/phasor of the
golden cases must match what the reference's own code produced
(tests/golden/make_golden.py).  CPU only."""
import json
import os

import numpy as np
import pytest

from oracle import harness as H
from oracle import fdtd_oracle as O

G = os.path.join(os.path.dirname(__file__), 'golden')
CASES = json.load(open(os.path.join(G, 'cases.json')))


def _load(name):
    return dict(np.load(os.path.join(G, name)))


@pytest.fixture(scope='module', params=['te', 'tm'])
def case2d(request):
    c = CASES['d2'][request.param]
    return request.param, c, _load(f'g2d_{request.param}.npz'), H.run_2d(c)


def test_setup_2d_bitwise(case2d):
    name, c, g, r = case2d
    s = H.setup_2d(c)
    for k in ('eps', 'sig', 'ce_e', 'ce_h', 'src_amp', 'src_ph1', 'src_ph2'):
        np.testing.assert_array_equal(s[k], g[k], err_msg=k)
    if c['pol'] == 'p':
        for k in ('ca_x', 'ca_y', 'da_x', 'da_y'):
            np.testing.assert_array_equal(s[k], g[k], err_msg=k)
    for ax in 'xy':
        for t in ('k', 'b', 'c'):
            for st in 'eh':
                np.testing.assert_array_equal(s['c' + ax][t + st], g[f'cpml_{t}{st}{ax}'])


def test_fields_2d_match_reference(case2d):
    name, c, g, r = case2d
    names = ('Ex', 'Ey', 'Hz') if c['pol'] == 'p' else ('Ez', 'Hx', 'Hy')
    for nm in names:
        for n in (c['steps'] // 2, c['steps']):
            np.testing.assert_array_equal(r[f'{nm}_n{n}'], g[f'{nm}_n{n}'], err_msg=f'{nm}_n{n}')
    np.testing.assert_array_equal(r['acc'], g['acc'])
    np.testing.assert_array_equal(r['acc_I'], g['acc_I'])
    if c['pol'] == 'p':
        np.testing.assert_array_equal(r['acc_ex'], g['acc_ex'])
    np.testing.assert_allclose(r['P_box'], g['P_box'], rtol=1e-12)
    for k in ('flux_in', 'flux_up', 'flux_dn'):
        np.testing.assert_allclose(r[k], g[k], rtol=1e-9, err_msg=k)


@pytest.fixture(scope='module')
def case3d():
    c = CASES['d3']
    return c, _load('g3d_tm.npz'), H.run_3d(c)


def test_setup_3d_bitwise(case3d):
    c, g, r = case3d
    s = H.setup_3d(c)
    for k in ('eps', 'ce_x', 'ce_y', 'ce_z', 'da_x', 'da_y', 'da_z', 'src_amp', 'src_ph1', 'src_ph2'):
        np.testing.assert_array_equal(s[k], g[k], err_msg=k)
    assert s['n_sp'] == int(g['n_sp']) and s['src_ix'] == int(g['src_ix'])
    for i, ax in enumerate('xyz'):
        for t in ('b', 'c', 'k'):
            for st in 'eh':
                np.testing.assert_array_equal(s['cpml'][i][t + st], g[f'cpml_{t}{ax}{st}'])


def test_fields_3d_match_reference(case3d):
    c, g, r = case3d
    for nm in ('Ex', 'Ey', 'Ez', 'Hx', 'Hy', 'Hz', 'acc', 'Iavg'):
        np.testing.assert_array_equal(r[nm], g[nm], err_msg=nm)
    np.testing.assert_allclose(r['P_box'], g['P_box'], rtol=1e-12)
    for k in ('flux_in', 'flux_up', 'flux_dn'):
        np.testing.assert_allclose(r[k], g[k], rtol=1e-9, err_msg=k)


def test_fp64_oracle_close_to_fp32_reference(case3d):
    """The FP64 oracle differs from the float32 reference only by float32 rounding."""
    c, g, _ = case3d
    r64 = H.run_3d(c, dtype=np.float64)
    a, b = r64['acc'], g['acc'].astype(np.complex128)
    rel = np.linalg.norm(a - b) / np.linalg.norm(a)
    assert rel < 1e-4, rel


def test_cpml_profiles_outside_pml_are_identity():
    p = O.cpml_axis(50, 10, 10, 25e-9, 4e-17)
    assert np.all(p['be'][11:39] == 1) and np.all(p['ce'][11:39] == 0)
    assert np.all(p['ke'] == 1)
    q = O.cpml_axis(50, 0, 0, 25e-9, 4e-17)
    assert np.all(q['ce'] == 0) and np.all(q['bh'] == 1)
