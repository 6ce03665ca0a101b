"""CPU checks of the C ABI: the shared library builds, loads without a GPU,
exports every entry point that include/lens_fdtd.h declares, and the ctypes
mirrors have the C struct sizes.  No compute is launched."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope='module')
def lib():
    from lens_sensor_b200 import build, _native
    build.build()
    return _native.load()


def _declared():
    txt = open(os.path.join(ROOT, 'include', 'lens_fdtd.h')).read()
    txt = re.sub(r'/\*.*?\*/', '', txt, flags=re.S)
    return sorted(set(re.findall(r'\b(lens_\w+)\s*\(', txt)))


def test_header_declares_entry_points():
    names = _declared()
    assert 'lens_te2d_step' in names and 'lens_fdtd3d_step' in names


def test_every_declared_symbol_is_exported(lib):
    for name in _declared():
        assert hasattr(lib, name), name


def test_bindings_cover_every_declared_symbol():
    from lens_sensor_b200 import _native
    assert set(_declared()) <= set(_native.SIGNATURES), set(_declared()) - set(_native.SIGNATURES)


def test_abi_sizes_match(lib):
    from lens_sensor_b200 import _native
    n = len(_native.MIRRORS)
    sizes = (ctypes.c_int * n)()
    assert lib.lens_abi_sizes(sizes, n) == n
    assert list(sizes) == [ctypes.sizeof(m) for m in _native.MIRRORS]


def test_status_strings(lib):
    assert lib.lens_status_string(0) == b'ok'
    assert lib.lens_status_string(-1) == b'invalid argument'


def test_invalid_arguments_are_rejected_without_launch(lib):
    """NULL grids and empty tables return LENS_ERR_ARG before touching the GPU."""
    from lens_sensor_b200 import _native as N
    assert lib.lens_te2d_step(None, None, None, 0, 1, None) == -1
    assert lib.lens_tm2d_step(None, None, None, 0, 1, None) == -1
    assert lib.lens_fdtd3d_step(None, None, None, 0, 1, None) == -1
    g = N.Grid3D()
    assert lib.lens_fdtd3d_step(ctypes.byref(g), None, None, 0, 1, None) == -1
    inst = (N.Inst2D * 2)()
    blk = (ctypes.c_int * 3)()
    assert lib.lens_batch2d_plan(inst, 2, 8, blk, None) == -1    # empty descriptors
    assert lib.lens_batch2d_step(inst, None, None, None, 2, 0, 8, None, 0, 1, None) == -1
    assert lib.lens_fdtd3d_accum_e2(ctypes.byref(g), 1, 0, None, None) == -1
    assert lib.lens_te2d_step_driven(None, None, None, None, 0, 1, None) == -1
    assert lib.lens_tm2d_step_driven(None, None, None, None, 0, 1, None) == -1
    d = N.Drive3D()
    assert lib.lens_fdtd3d_step_driven(ctypes.byref(g), None, None, None, 0, 1, None) == -1
    assert lib.lens_fdtd3d_step_driven(ctypes.byref(g), None, None, ctypes.byref(d), 0, 1, None) == -1
