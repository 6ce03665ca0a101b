"""The CW convergence extension of the 2D drop-in driver against the reference
(planar_beads/fdtd2d_core.py:859-873): after the last step the phasor change
between the last two DFT windows is compared with CW_TOL; above it the run
grows by one window at a time, up to CW_MAX_EXTEND x its step count.

tests/golden/dropin_2d_extend.json (`make_golden.py extend2d`) holds two
whole-driver cases run by the reference with a tighter CW_TOL: 'te_extend'
(1e-4) extends four times and stops at the step limit; 'tm_extend' (1e-3, KAPPA
losses, the Ex phasor) extends once and converges.  The driver runs on the
oracle engine (tests/_oracle_engine.py) and must reproduce every NPZ key, PKL
scalar and step count of the reference.  (The restart of the device DFT windows
itself runs on the GPU in the 'te' case of test_dropin_2d.py, which extends once
under the default CW_TOL.)
"""
import json
import os

import pytest

import _oracle_engine
import test_dropin_2d as T
from lens_sensor_b200 import fdtd2d_core as D2

EXT = json.load(open(os.path.join(os.path.dirname(__file__), 'golden', 'dropin_2d_extend.json')))


@pytest.mark.parametrize('name', sorted(EXT))
def test_cw_extension_on_oracle_engine(name, tmp_path, monkeypatch):
    monkeypatch.setitem(T.GOLD, name, EXT[name])
    monkeypatch.setattr(D2, 'CW_TOL', EXT[name]['cw_tol'])
    r, z, pk = T._run(name, _oracle_engine, tmp_path, monkeypatch)
    T._check(name, z, pk, T.TOL_CPU)
    base = T.GOLD['te' if name == 'te_extend' else 'tm_kappa']['pkl']['steps_total']
    assert pk['steps_total'] > base          # the window was extended
