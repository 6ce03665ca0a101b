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


# Addresses that are never dereferenced: every call below either fails its
# argument check or runs zero steps, so nothing is launched or copied.
_FAKE = 0x7f0000000000


def _fake(k):
    return _FAKE + 256 * k


def _axis(n, lo, hi, k0):
    from lens_sensor_b200 import _native as N
    a = N.Axis()
    for q, (tag, m) in enumerate((('e', n), ('h', n - 1))):
        p = getattr(a, tag)
        p.b, p.c, p.ik = _fake(k0 + 3 * q), _fake(k0 + 3 * q + 1), _fake(k0 + 3 * q + 2)
        p.n, p.lo, p.hi = m, lo, hi
    return a


def _table(n=8):
    from lens_sensor_b200 import _native as N
    t = N.StepTable()
    t.wt, t.env, t.t0, t.n_table = _fake(40), _fake(41), 0, n
    return t


def _grid2d(pol, wx=4, wy=5, nx=40, ny=30):
    from lens_sensor_b200 import _native as N
    g = N.TE2D() if pol == 's' else N.TM2D()
    g.nx, g.ny, g.pitch = nx, ny, 32
    names = ('ez', 'hx', 'hy', 'ce_e', 'ce_h') if pol == 's' else ('ex', 'ey', 'hz', 'ca_x', 'ca_y')
    for k, nm in enumerate(names):
        setattr(g, nm, _fake(k))
    g.ax, g.ay = _axis(nx, wx, wx, 10), _axis(ny, wy, wy, 20)
    for k, nm in enumerate(_PSI2D[pol]):
        setattr(g, nm, _fake(30 + k))
    g.src.ix = -1
    return g


# the psi array of each 2D kernel with the profile whose strip it serves
_PSI2D = {'s': ('psi_hxy', 'psi_hyx', 'psi_ezx', 'psi_ezy'), 'p': ('psi_hzx', 'psi_hzy', 'psi_exy', 'psi_eyx')}
_STRIP2D = {'s': (('ay', 'h'), ('ax', 'h'), ('ax', 'e'), ('ay', 'e')),
            'p': (('ax', 'h'), ('ay', 'h'), ('ay', 'e'), ('ax', 'e'))}


@pytest.mark.parametrize('pol', ['s', 'p'])
def test_2d_step_requires_the_psi_of_every_strip(lib, pol):
    """A grid whose profile has a strip must carry that strip's psi array; a
    profile without one needs none.  Zero steps: nothing is launched."""
    step = lib.lens_te2d_step if pol == 's' else lib.lens_tm2d_step
    tab = _table()
    g = _grid2d(pol)
    assert step(ctypes.byref(g), ctypes.byref(tab), None, 0, 0, None) != -1
    for nm, (ax, tag) in zip(_PSI2D[pol], _STRIP2D[pol]):
        g = _grid2d(pol)
        setattr(g, nm, None)
        assert step(ctypes.byref(g), ctypes.byref(tab), None, 0, 0, None) == -1, nm
        p = getattr(getattr(g, ax), tag)
        p.lo = p.hi = 0
        assert step(ctypes.byref(g), ctypes.byref(tab), None, 0, 0, None) != -1, nm


@pytest.mark.parametrize('pol', [0, 1])
def test_batch_plan_requires_the_psi_of_every_strip(lib, pol):
    """lens_batch2d_plan (host only) checks each instance like the step does."""
    from lens_sensor_b200 import _native as N

    def inst():
        s = N.Inst2D()
        s.pol, s.nx, s.ny, s.pitch = pol, 40, 30, 32
        for q in range(3):
            s.f[q] = _fake(q)
        s.c[0], s.c[1] = _fake(3), _fake(4)
        s.ax, s.ay = _axis(40, 4, 4, 10), _axis(30, 5, 5, 20)
        for q in range(4):
            s.psi[q] = _fake(30 + q)
        s.src.ix = -1
        return s

    blk = (ctypes.c_int * 2)()
    one = (N.Inst2D * 1)(inst())
    assert lib.lens_batch2d_plan(one, 1, 8, blk, None) > 0
    strips = _STRIP2D['s' if pol == 0 else 'p']
    for q, (ax, tag) in enumerate(strips):
        s = inst()
        s.psi[q] = None
        one = (N.Inst2D * 1)(s)
        assert lib.lens_batch2d_plan(one, 1, 8, blk, None) == -1, q
        p = getattr(getattr(s, ax), tag)
        p.lo = p.hi = 0
        one = (N.Inst2D * 1)(s)
        assert lib.lens_batch2d_plan(one, 1, 8, blk, None) > 0, q


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    """No CPU fallback: without the built library the bindings raise."""
    from lens_sensor_b200 import _native as N
    monkeypatch.setattr(N, '_lib', None)
    with pytest.raises(N.LensError, match='not found'):
        N.load(str(tmp_path / 'liblens_fdtd.so'))


def test_abi_mismatch_fails_loudly(lib, monkeypatch):
    """A library built from another header than the bindings is refused."""
    from lens_sensor_b200 import _native as N

    class Wrong(ctypes.Structure):
        _fields_ = [('x', ctypes.c_char * 3)]
    monkeypatch.setattr(N, '_lib', None)
    monkeypatch.setattr(N, 'MIRRORS', (Wrong,) + tuple(N.MIRRORS[1:]))
    with pytest.raises(N.LensError, match='ABI mismatch'):
        N.load()


def test_grids_need_a_cuda_device():
    """Constructing a grid without a CUDA device raises instead of falling back."""
    import torch
    if torch.cuda.is_available():
        pytest.skip('a CUDA device is present')
    from lens_sensor_b200 import _native as N
    from lens_sensor_b200 import engine as E
    with pytest.raises(N.LensError, match='no CPU fallback'):
        E.StepTable(0, 4, 1e-17, 1e15, 1e15, E.cw_envelope(3e14))
