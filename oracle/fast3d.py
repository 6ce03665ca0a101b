"""Multi-threaded C++ stepper for the oracle's 3D grid (TEST INFRASTRUCTURE ONLY).

Grid3DC is oracle.fdtd_oracle.Grid3D with its step() done by oracle/o3.cpp
(same operation order, std::thread workers over x-planes); the fields stay NumPy arrays of the
reference's shapes, so the oracle's source injection, detector sums, flux
pairs and |E|^2 averaging run on them unchanged.  tests/test_oracle_c.py checks
Grid3DC against Grid3D bit for bit in float32 and float64.  Used only to make
the FP64 runs of full-size workloads affordable (tests/golden/make_fp64.py).
"""
import ctypes
import os
import subprocess

import numpy as np

from . import fdtd_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, '_build', 'libo3.so')
_lib = None


def build(force=False):
    """Compile oracle/o3.cpp (oracle/Makefile) if the library is missing or older."""
    src = os.path.join(HERE, 'o3.cpp')
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(['make', '-s'] + (['-B'] if force else []) + ['-C', HERE], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(LIB)
        vp = ctypes.c_void_p
        P = ctypes.POINTER
        lib.o3_step.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, P(vp), P(vp),
                                ctypes.c_double, P(vp), P(vp), P(vp), P(vp), P(ctypes.c_int), P(ctypes.c_int),
                                P(ctypes.c_int), P(ctypes.c_int)]
        lib.o3_step.restype = None
        _lib = lib
    return _lib


def _strip_range(strip, N):
    """(lo, hi) strip widths of an oracle _Strip along its axis of length N."""
    lo = hi = 0
    for sl, *_ in strip.parts:
        s = next(x for x in sl if x != slice(None))
        if s.start == 0:
            lo = s.stop
        else:
            hi = N - s.start
    if lo >= N:
        return N, 0
    return lo, hi


class Grid3DC(O.Grid3D):
    """oracle Grid3D stepped by oracle/o3.cpp."""

    # psi order of o3.cpp: (oracle attribute, axis, cpml axis, staggering, cut)
    _PSI = (('p_hx_z', 2, 'h', False), ('p_hx_y', 1, 'h', False), ('p_hy_x', 0, 'h', False),
            ('p_hy_z', 2, 'h', False), ('p_hz_y', 1, 'h', False), ('p_hz_x', 0, 'h', False),
            ('p_ex_y', 1, 'e', True), ('p_ex_z', 2, 'e', True), ('p_ey_z', 2, 'e', True),
            ('p_ey_x', 0, 'e', True), ('p_ez_x', 0, 'e', True), ('p_ez_y', 1, 'e', True))

    def __init__(self, Nx, Ny, Nz, dx, dt, cpml, ce, da, src, src_comp, dtype=np.float32,
                 faces=('xmin', 'xmax', 'ymin', 'ymax', 'zmin', 'zmax')):
        super().__init__(Nx, Ny, Nz, dx, dt, cpml, ce, da, src, src_comp, dtype, faces)
        self._coef32 = [np.ascontiguousarray(a, np.float32) for a in ce] + \
            ([np.ascontiguousarray(a, np.float32) for a in da] if da is not None else [None] * 3)
        sH = {'p_hx': (Nx, Ny - 1, Nz - 1), 'p_hy': (Nx - 1, Ny, Nz - 1), 'p_hz': (Nx - 1, Ny - 1, Nz),
              'p_ex': (Nx - 1, Ny - 2, Nz - 2), 'p_ey': (Nx - 2, Ny - 1, Nz - 2), 'p_ez': (Nx - 2, Ny - 2, Nz - 1)}
        up = lambda a: np.asarray(a).astype(dtype)
        self._psi, self._prof, self._len, self._lo, self._hi = [], [], [], [], []
        for name, ax, t, cut in self._PSI:
            shape = sH[name[:4]]
            strip = getattr(self, name)
            P = {k: up(v) for k, v in cpml[ax].items()}
            b, c, k = P['b' + t], P['c' + t], P['k' + t]
            if cut:
                b, c, k = b[1:-1], c[1:-1], k[1:-1]
            km = (1.0 / k - 1.0)
            N = shape[ax]
            lo, hi = _strip_range(strip, N)
            self._psi.append(np.zeros(shape, dtype) if lo + hi > 0 else np.zeros(1, dtype))
            self._prof.append(tuple(np.ascontiguousarray(a) for a in (b, c, km)))
            self._len.append(N)
            self._lo.append(lo)
            self._hi.append(hi)
        f = self.faces
        self._pec = [int(s in f) for s in ('xmin', 'xmax', 'ymin', 'ymax', 'zmin', 'zmax')]

    def step(self, n, env):
        lib = load()
        vp = ctypes.c_void_p
        arr = lambda xs: (vp * len(xs))(*[None if x is None else x.ctypes.data for x in xs])
        ints = lambda xs: (ctypes.c_int * len(xs))(*xs)
        fields = [self.Ex, self.Ey, self.Ez, self.Hx, self.Hy, self.Hz]
        assert all(a.flags.c_contiguous and a.dtype == self.dtype for a in fields)
        lib.o3_step(int(self.fp64), self.Nx, self.Ny, self.Nz, arr(fields), arr(self._coef32), float(self.ch),
                    arr(self._psi), arr([p[0] for p in self._prof]), arr([p[1] for p in self._prof]),
                    arr([p[2] for p in self._prof]), ints(self._len), ints(self._lo), ints(self._hi),
                    ints(self._pec))
        self.src.inject(getattr(self, self.src_comp), n * self.dt, env, self.fp64)
