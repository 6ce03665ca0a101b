"""Host read-back of the 3D phasors (Solve3D.phasors_host): complex64 host
arrays in each component's shape, equal to the complex128 device phasor up to
the float32 rounding of the (2/N) scale (fdtd3d_core.py:1271 keeps the CW
amplitude in complex64)."""
import numpy as np
import pytest

from lens_sensor_b200.geometry import Spec3D, Sphere, Stack


@pytest.mark.gpu
@pytest.mark.parametrize('pol', ['p', 's'])
def test_host_phasors_match_device_phasors(pol):
    from lens_sensor_b200.solver3d import Solve3D
    st = Stack(1.49, 1.0, [(1.0, complex(1.333, 0.001))], 1.376)
    sp = Spec3D(pol, 64, 48, 40, 100.0, st, 2.0, [Sphere(3.0, 0.6, 1.59, -0.3, 0.2)])
    s = Solve3D(sp, 240, comps=(0, 1, 2))
    s.stage_host((0, 1, 2)).run()
    host = s.phasors_host()
    assert sorted(host) == [0, 1, 2]
    for c in (0, 1, 2):
        d = s.phasor(c).cpu().numpy()
        h = host[c]
        assert h.dtype == np.complex64 and h.shape == d.shape, (c, h.dtype, h.shape, d.shape)
        assert np.linalg.norm(d) > 0
        assert np.linalg.norm(h - d) <= 1e-6 * np.linalg.norm(d), c
    assert s.d2h_bytes == sum(64 * 48 * 64 * 8 for _ in range(3))


@pytest.mark.gpu
def test_host_phasors_without_staging_and_partial():
    """Without stage_host(), and for a subset of the components staged in
    page-locked buffers."""
    from lens_sensor_b200.solver3d import Solve3D
    st = Stack(1.49, 1.0, [(1.0, 1.333)], 1.376)
    sp = Spec3D('p', 48, 40, 36, 100.0, st, 2.0)
    s = Solve3D(sp, 200, comps=(0, 1, 2)).run()
    a = s.phasors_host((1,))
    s.stage_host((0, 2), pinned=True)
    b = s.phasors_host((2,))
    for c, h in ((1, a[1]), (2, b[2])):
        d = s.phasor(c).cpu().numpy()
        assert h.shape == d.shape and np.linalg.norm(h - d) <= 1e-6 * np.linalg.norm(d), c


def test_read_back_refuses_components_not_accumulated():
    from lens_sensor_b200.solver3d import Solve3D
    s = Solve3D.__new__(Solve3D)       # no device needed for the argument check
    s.comps = (1,)
    assert s._accumulated(None) == (1,)
    assert s._accumulated([1]) == (1,)
    with pytest.raises(ValueError):
        s._accumulated((0, 1))
