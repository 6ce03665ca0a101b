"""ctypes binding of liblens_fdtd.so (include/lens_fdtd.h).

The structs below mirror the C declarations field by field; ``load()`` checks
their sizes against ``lens_abi_sizes`` so a layout drift fails loudly.  There
is no fallback: if the library is missing the import of the engine raises.
"""
import ctypes
import os
from ctypes import POINTER, c_float, c_int, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, '_lib', 'liblens_fdtd.so')

MAX_BOX = 4
MAX_CTYPE = 4
MAX_PLANE = 4


class Profile(ctypes.Structure):
    _fields_ = [('b', c_void_p), ('c', c_void_p), ('ik', c_void_p),
                ('n', c_int), ('lo', c_int), ('hi', c_int)]


class Axis(ctypes.Structure):
    _fields_ = [('e', Profile), ('h', Profile)]


class StepTable(ctypes.Structure):
    _fields_ = [('wt', c_void_p), ('env', c_void_p), ('pe', c_void_p), ('ph', c_void_p),
                ('t0', c_int), ('n_table', c_int)]


class Source(ctypes.Structure):
    _fields_ = [('ix', c_int), ('amp', c_void_p), ('ph1', c_void_p), ('ph2', c_void_p),
                ('nj', c_int), ('nk', c_int), ('pitch_k', c_int)]


class TE2D(ctypes.Structure):
    _fields_ = [('nx', c_int), ('ny', c_int), ('pitch', c_int),
                ('ez', c_void_p), ('hx', c_void_p), ('hy', c_void_p),
                ('ce_e', c_void_p), ('ce_h', c_void_p), ('ch', c_float),
                ('ax', Axis), ('ay', Axis),
                ('psi_hxy', c_void_p), ('psi_hyx', c_void_p), ('psi_ezx', c_void_p),
                ('psi_ezy', c_void_p), ('pec', c_int * 4), ('src', Source)]


class TM2D(ctypes.Structure):
    _fields_ = [('nx', c_int), ('ny', c_int), ('pitch', c_int),
                ('ex', c_void_p), ('ey', c_void_p), ('hz', c_void_p),
                ('ca_x', c_void_p), ('ca_y', c_void_p), ('da_x', c_void_p), ('da_y', c_void_p),
                ('ch', c_float), ('ax', Axis), ('ay', Axis),
                ('psi_hzx', c_void_p), ('psi_hzy', c_void_p), ('psi_exy', c_void_p),
                ('psi_eyx', c_void_p), ('pec', c_int * 4), ('src', Source)]


class Epi2D(ctypes.Structure):
    _fields_ = [('nbox', c_int), ('box', (c_int * 4) * MAX_BOX), ('box_acc', c_void_p),
                ('dft_n0', c_int), ('dft_n1', c_int), ('dft', c_void_p), ('dft_ex', c_void_p),
                ('prev_n0', c_int), ('prev_n1', c_int), ('dft_prev', c_void_p),
                ('iavg_n0', c_int), ('iavg', c_void_p),
                ('nplane', c_int), ('plane', c_int * MAX_PLANE), ('plane_acc', c_void_p),
                ('dft_raw', c_void_p), ('ex2', c_void_p),
                ('nsx', c_int), ('sx_plane', c_int * MAX_PLANE), ('sx_acc', c_void_p)]


NPSI = 12
PSI_NAMES = ('hx_z', 'hx_y', 'hy_x', 'hy_z', 'hz_y', 'hz_x',
             'ex_y', 'ex_z', 'ey_z', 'ey_x', 'ez_x', 'ez_y')   # LENS_PSI_* order


class Grid3D(ctypes.Structure):
    _fields_ = [('nx', c_int), ('ny', c_int), ('nz', c_int), ('pitch', c_int),
                ('f', (c_void_p * 6) * 2), ('psi', (c_void_p * NPSI) * 2), ('cur', c_int),
                ('ce_x', c_void_p), ('ce_y', c_void_p), ('ce_z', c_void_p),
                ('da_x', c_void_p), ('da_y', c_void_p), ('da_z', c_void_p),
                ('ch', c_float), ('ax', Axis), ('ay', Axis), ('az', Axis),
                ('pec', c_int * 6), ('src', Source), ('src_comp', c_int), ('flag', c_void_p),
                ('ctype', c_void_p), ('ctab', c_void_p), ('cexpl', c_void_p), ('ntype', c_int)]


class Epi3D(ctypes.Structure):
    _fields_ = [('nbox', c_int), ('box', (c_int * 6) * MAX_BOX), ('box_acc', c_void_p),
                ('dft_n0', c_int), ('dft_n1', c_int), ('dft', c_void_p * 3),
                ('conv_k', c_int), ('prev_n0', c_int), ('prev_n1', c_int),
                ('conv_prev', c_void_p), ('conv_last', c_void_p),
                ('nplane', c_int), ('plane', c_int * MAX_PLANE), ('plane_acc', c_void_p)]


F32, F16, BF16 = 0, 1, 2   # LENS_F32 / LENS_F16 / LENS_BF16 field storage


class Inst2D(ctypes.Structure):
    _fields_ = [('pol', c_int), ('nx', c_int), ('ny', c_int), ('pitch', c_int),
                ('f', c_void_p * 3), ('c', c_void_p * 4), ('ch', c_float),
                ('ax', Axis), ('ay', Axis), ('psi', c_void_p * 4), ('pec', c_int * 4),
                ('src', Source), ('dft_n0', c_int), ('dft_n1', c_int), ('dft', c_void_p), ('n_start', c_int),
                ('rtype', c_void_p), ('ctab', c_void_p)]


class TB2D(ctypes.Structure):
    _fields_ = [('g', Inst2D), ('f1', c_void_p * 3), ('psi1', c_void_p * 4), ('psi_lv', c_void_p),
                ('dft_kahan', c_int)]


TB_K = 4


class TB3D(ctypes.Structure):
    _fields_ = [('psi_lv', c_void_p * 12), ('chunk', c_int)]


class RsOut2D(ctypes.Structure):
    _fields_ = [('frames', c_void_p), ('every', c_int), ('nframes', c_int), ('kahan', c_int)]


RS_MAX_INST = 32


TB3_K = 2


class Drive3D(ctypes.Structure):
    _fields_ = [('nplanes', c_int), ('taper', c_void_p), ('hand', c_void_p * 3)]


class Drive2D(ctypes.Structure):
    _fields_ = [('nplanes', c_int), ('taper', c_void_p), ('hand', c_void_p), ('tab', c_void_p)]


MIRRORS = (Profile, Axis, StepTable, Source, TE2D, TM2D, Epi2D, Grid3D, Epi3D, Inst2D, Drive3D, Drive2D, TB2D, TB3D,
           RsOut2D)

# Every exported entry point with its ctypes signature (checked by the tests
# against include/lens_fdtd.h).
SIGNATURES = {
    'lens_te2d_step': (c_int, [POINTER(TE2D), POINTER(StepTable), POINTER(Epi2D), c_int, c_int, c_void_p]),
    'lens_tm2d_step': (c_int, [POINTER(TM2D), POINTER(StepTable), POINTER(Epi2D), c_int, c_int, c_void_p]),
    'lens_te2d_step_driven': (c_int, [POINTER(TE2D), POINTER(StepTable), POINTER(Epi2D), POINTER(Drive2D), c_int,
                                      c_int, c_void_p]),
    'lens_tm2d_step_driven': (c_int, [POINTER(TM2D), POINTER(StepTable), POINTER(Epi2D), POINTER(Drive2D), c_int,
                                      c_int, c_void_p]),
    'lens_fdtd3d_step': (c_int, [POINTER(Grid3D), POINTER(StepTable), POINTER(Epi3D), c_int, c_int, c_void_p]),
    'lens_fdtd3d_step_driven': (c_int, [POINTER(Grid3D), POINTER(StepTable), POINTER(Epi3D), POINTER(Drive3D),
                                        c_int, c_int, c_void_p]),
    'lens_fdtd3d_accum_e2': (c_int, [POINTER(Grid3D), c_int, c_int, c_void_p, c_void_p]),
    'lens_fdtd3d_step_tb': (c_int, [POINTER(Grid3D), POINTER(TB3D), POINTER(StepTable), POINTER(Epi3D), c_int, c_int,
                                    c_void_p]),
    'lens_fdtd3d_watchdog_test': (c_int, [POINTER(Grid3D), POINTER(StepTable), c_int, c_int, c_void_p]),
    'lens_batch2d_plan': (c_int, [POINTER(Inst2D), c_int, c_int, POINTER(c_int), POINTER(c_int)]),
    'lens_batch2d_step': (c_int, [POINTER(Inst2D), c_void_p, c_void_p, c_void_p, c_int, c_int, c_int,
                                  POINTER(StepTable), c_int, c_int, c_void_p]),
    'lens_batch2d_run': (c_int, [POINTER(Inst2D), c_void_p, c_void_p, c_void_p, c_int, c_int, c_int,
                                 POINTER(StepTable), c_int, c_int, c_void_p, c_void_p, c_void_p]),
    'lens_batch2d_step_noalloc': (c_int, [POINTER(Inst2D), c_int, c_int, c_int, POINTER(StepTable), c_int,
                                          c_int, c_void_p]),
    'lens_tb2d_plan': (c_int, [POINTER(TB2D), c_int, c_int, POINTER(c_int)]),
    'lens_tb2d_step': (c_int, [POINTER(TB2D), c_void_p, c_void_p, c_int, c_int, c_int, POINTER(StepTable), c_int,
                               c_int, c_void_p]),
    'lens_rs2d_plan': (c_int, [POINTER(Inst2D), c_int, POINTER(c_int), POINTER(c_int), POINTER(c_int)]),
    'lens_rs2d_bands': (c_int, [POINTER(Inst2D), c_int, c_int, c_int, POINTER(ctypes.c_short), c_int]),
    'lens_rs2d_scratch_bytes': (ctypes.c_size_t, [c_int, c_int]),
    'lens_rs2d_run': (c_int, [POINTER(Inst2D), c_void_p, POINTER(RsOut2D), c_int, POINTER(StepTable), c_int, c_int,
                              c_void_p, ctypes.c_size_t, c_void_p, c_void_p]),
    'lens_rs2d_watchdog_test': (c_int, [POINTER(Inst2D), c_void_p, c_int, POINTER(StepTable), c_int, c_int,
                                        c_void_p, ctypes.c_size_t, c_void_p, c_void_p]),
    'lens_version': (c_int, []),
    'lens_status_string': (ctypes.c_char_p, [c_int]),
    'lens_abi_sizes': (c_int, [POINTER(c_int), c_int]),
}

_lib = None


class LensError(RuntimeError):
    pass


def load(path=LIB_PATH):
    """Load the engine library once; raise if it is missing or its ABI differs."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise LensError(f'{path} not found: build it with `python -m lens_sensor_b200.build` '
                        '(there is no CPU fallback)')
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    sizes = (c_int * len(MIRRORS))()
    lib.lens_abi_sizes(sizes, len(MIRRORS))
    mine = [ctypes.sizeof(m) for m in MIRRORS]
    if list(sizes) != mine:
        raise LensError(f'ABI mismatch between liblens_fdtd.so {list(sizes)} and bindings {mine}')
    _lib = lib
    return lib


def check(status):
    if status != 0:
        raise LensError(f'liblens_fdtd: {load().lens_status_string(status).decode()} ({status})')
