"""Geometry edge cases of the 3D drop-in driver against the reference
(`make_golden.py edges3d`): 'te_nobead' runs without a bead (bead=None);
'tm_bead_clipped' places a bead whose sphere crosses the z end of the domain,
so its sub-pixel box (and the Farjadpour tensor patches around it) is clipped
there (planar_3d/fdtd3d_core.py:119-292, 305-378).  The driver runs on the
oracle engine with the product's geometry builder and must reproduce every NPZ
array summary, PKL scalar and step count of the reference."""
import json
import os

import pytest

import _oracle_engine
import test_dropin_3d as T

EDGES = json.load(open(os.path.join(os.path.dirname(__file__), 'golden', 'dropin_3d_edges.json')))


@pytest.mark.parametrize('name', sorted(EDGES))
def test_geometry_edge_cases_on_oracle_engine(name, tmp_path, monkeypatch):
    monkeypatch.setitem(T.GOLD, name, EDGES[name])
    keep, files, pk, left = T._run(name, _oracle_engine, tmp_path, monkeypatch)
    T._check(name, files, pk, T.TOL_CPU)
    assert not left, left
