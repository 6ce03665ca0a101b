"""The product's host setup (lens_sensor_b200.geometry) must produce the same
float32 coefficient, damping, CPML and source arrays as the reference-pinned
oracle, bit for bit.  CPU only."""
import json
import os

import numpy as np
import pytest

from lens_sensor_b200 import geometry as G
from oracle import harness as H

GD = os.path.join(os.path.dirname(__file__), 'golden')
CASES = json.load(open(os.path.join(GD, 'cases.json')))


def _cplx(v):
    return complex(v[0], v[1]) if isinstance(v, (list, tuple)) else v


def spec2d(c):
    st = G.Stack(c['wg_n'], c['wg_um'], [(t, _cplx(n)) for t, n in c['stack']], c['n_sub'])
    return G.Spec2D(c['pol'], c['Nx'], c['Ny'], c['dx'], st, c['tear_m'],
                    G.Bead2D(c['bead']['x_um'], c['bead']['d_um'], c.get('bead_n', 1.59)),
                    npml=c['npml'], lam_nm=c['lam_nm'], waist_um=c.get('waist_um', 3.0))


def spec3d(c):
    st = G.Stack(c['wg_n'], c['t_wg_um'], [(t, _cplx(n)) for t, n in c['stack']], c['n_sub'])
    beads = c.get('beads') or ([c['bead']] if c.get('bead') else [])
    sph = [G.Sphere(b['x_um'], b['d_um'], b.get('n', 1.59), b.get('y_um'), b.get('z_um', 0.0)) for b in beads]
    return G.Spec3D(c['pol'], c['Nx'], c['Ny'], c['Nz'], c['dx_nm'], st, c['tear_um'], sph,
                    npml=c['npml'], lam_nm=c['lam_nm'], waist_um=c.get('waist_um', 1.0))


@pytest.mark.parametrize('name', ['te', 'tm'])
def test_2d_setup_bitwise(name):
    c = CASES['d2'][name]
    o = H.setup_2d(c)
    p = G.build_2d(spec2d(c))
    keys = ['eps', 'sig', 'ce_e', 'ce_h'] + (['ca_x', 'ca_y', 'da_x', 'da_y'] if c['pol'] == 'p' else [])
    for k in keys:
        np.testing.assert_array_equal(p[k], o[k], err_msg=k)
    for k, ok in (('amp', 'src_amp'), ('ph1', 'src_ph1'), ('ph2', 'src_ph2')):
        np.testing.assert_array_equal(p['src'][k], o[ok], err_msg=k)
    assert p['src']['ix'] == o['src'].ix and p['src']['omega'] == o['src'].omega
    for ax in ('cx', 'cy'):
        for k in o[ax]:
            np.testing.assert_array_equal(p[ax][k], o[ax][k], err_msg=ax + k)


def _check3d(c):
    o = H.setup_3d(c)
    sp = spec3d(c)
    p = G.build_3d(sp)
    for a, k in enumerate(('ce_x', 'ce_y', 'ce_z')):
        np.testing.assert_array_equal(p['ce'][a], o[k], err_msg=k)
    if o['da'] is None:
        assert p['da'] is None
    else:
        for a in range(3):
            np.testing.assert_array_equal(p['da'][a], o['da'][a], err_msg=f'da{a}')
    for k, ok in (('amp', 'src_amp'), ('ph1', 'src_ph1'), ('ph2', 'src_ph2')):
        np.testing.assert_array_equal(p['src'][k], o[ok], err_msg=k)
    assert p['src']['ix'] == o['src'].ix and p['src']['omega'] == o['src'].omega
    assert sp.n_sp == o['n_sp']
    for a in range(3):
        for k in o['cpml'][a]:
            np.testing.assert_array_equal(p['cpml'][a][k], o['cpml'][a][k])


def test_3d_setup_bitwise_golden():
    _check3d(CASES['d3'])


def test_3d_setup_bitwise_two_beads_lossless_te():
    c = dict(CASES['d3'], pol='s', Nx=90, stack=[[0.6, 1.333], [0.3, 1.34]],
             beads=[dict(x_um=1.6, d_um=0.5, n=1.59, z_um=0.2), dict(x_um=3.4, d_um=0.6, n=1.59, z_um=-0.3)])
    c.pop('bead')
    _check3d(c)


def test_3d_setup_bitwise_two_beads_lossy():
    c = dict(CASES['d3'], Nx=90, beads=[dict(x_um=1.6, d_um=0.5, n=1.59, z_um=0.2),
                                         dict(x_um=3.4, d_um=0.6, n=1.59, z_um=-0.3)])
    c.pop('bead')
    _check3d(c)


def test_3d_setup_same_on_any_thread_count(monkeypatch):
    """The volume builders split the x range over host threads; the arrays do
    not depend on how many (1, 3 and 7 threads, uneven slabs)."""
    c = dict(CASES['d3'], Nx=113, beads=[dict(x_um=1.6, d_um=0.5, n=1.59, z_um=0.2),
                                          dict(x_um=3.4, d_um=0.6, n=1.59, z_um=-0.3)])
    c.pop('bead')
    sp = spec3d(c)
    out = []
    for n in (1, 3, 7):
        monkeypatch.setattr(G, 'HOST_THREADS', n)
        out.append(G.build_3d(sp))
    for p in out[1:]:
        for a in range(3):
            np.testing.assert_array_equal(p['ce'][a], out[0]['ce'][a])
            np.testing.assert_array_equal(p['da'][a], out[0]['da'][a])


def test_slabs_cover_the_range_once():
    seen = []
    G._slabs(101, lambda a, b: seen.append((a, b)), min_rows=4)
    seen.sort()
    assert seen[0][0] == 0 and seen[-1][1] == 101
    assert all(p[1] == q[0] for p, q in zip(seen, seen[1:]))
    one = []
    G._slabs(10, lambda a, b: one.append((a, b)), min_rows=16)
    assert one == [(0, 10)]
