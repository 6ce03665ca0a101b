"""Geometry edge cases of the 2D drop-in driver against the reference
(`make_golden.py edges2d`): 'te_nobead' is the reference run without a bead
(place_bead=False, planar_beads/fdtd2d_core.py:218-219: label suffix '_ref',
bead keys still written); 'tm_bead_outside' places the bead centre beyond the
domain end, which the reference's material builder skips (:224).  The driver
runs on the oracle engine and must reproduce every NPZ key, PKL scalar and step
count of the reference; the product's own geometry builder makes the grid."""
import json
import os

import pytest

import _oracle_engine
import test_dropin_2d as T

EDGES = json.load(open(os.path.join(os.path.dirname(__file__), 'golden', 'dropin_2d_edges.json')))


@pytest.mark.parametrize('name', sorted(EDGES))
def test_geometry_edge_cases_on_oracle_engine(name, tmp_path, monkeypatch):
    monkeypatch.setitem(T.GOLD, name, EDGES[name])
    r, z, pk = T._run(name, _oracle_engine, tmp_path, monkeypatch)
    T._check(name, z, pk, T.TOL_CPU)
