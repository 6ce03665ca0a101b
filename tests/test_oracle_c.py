"""The C++ restatement of the oracle's 3D step (oracle/o3.cpp via
oracle/fast3d.Grid3DC) against the NumPy oracle, bit for bit, in float32 and
float64, both polarisations, lossy, with a bead.  Grid3DC makes the FP64 runs of
full-size workloads affordable (tests/golden/make_fp64.py); this pins it to the
oracle that the reference's own fixtures pin.  CPU only."""
import json
import os

import numpy as np
import pytest

from oracle import fdtd_oracle as O
from oracle import harness as H
from oracle.fast3d import Grid3DC

CASES = json.load(open(os.path.join(os.path.dirname(__file__), 'golden', 'cases.json')))


@pytest.mark.parametrize('pol', ['p', 's'])
@pytest.mark.parametrize('dtype', [np.float32, np.float64])
def test_c_stepper_matches_numpy_oracle(pol, dtype):
    c = dict(CASES['d3'], pol=pol)
    s = H.setup_3d(c)
    comp = 'Ey' if pol == 'p' else 'Ez'
    args = (c['Nx'], c['Ny'], c['Nz'], s['dx'], s['dt'], s['cpml'], (s['ce_x'], s['ce_y'], s['ce_z']), s['da'],
            s['src'], comp, dtype)
    a, b = O.Grid3D(*args), Grid3DC(*args)
    for n in range(80):
        env = O.cw_envelope(n * s['dt'], s['f0'])
        a.step(n, env)
        b.step(n, env)
    for k, x in a.fields().items():
        y = b.fields()[k]
        assert np.array_equal(x, y), (k, float(np.abs(x - y).max()))
    assert float(np.abs(a.Ey if pol == 'p' else a.Ez).max()) > 0.1    # the wave is there
