"""Compile the sm_100a CUDA engine into lens_sensor_b200/_lib/liblens_fdtd.so.

The library is built in-tree with nvcc (no JIT cache), so the file travels with
the source tree to the machine that runs it.  Usage:

    python -m lens_sensor_b200.build          # or lens_sensor_b200.build.build()
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, 'csrc')
LIBDIR = os.path.join(HERE, '_lib')
LIB = os.path.join(LIBDIR, 'liblens_fdtd.so')
SOURCES = ['fdtd2d.cu', 'fdtd2d_batch.cu', 'fdtd2d_resident.cu', 'fdtd2d_tb.cu', 'fdtd3d.cu', 'fdtd3d_tb.cu']
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']


def nvcc():
    for c in (os.environ.get('NVCC'), '/usr/local/cuda/bin/nvcc', 'nvcc'):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return 'nvcc'


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(ROOT, 'include', 'lens_fdtd.h'))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    """Compile the shared library if any source is newer than it."""
    if not force and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    cmd = [nvcc(), '-O3', '-std=c++17', '-lineinfo', *ARCH, '-shared', '-Xcompiler', '-fPIC',
           '-I', os.path.join(ROOT, 'include'), '-I', CSRC, '--expt-relaxed-constexpr',
           *extra, '-o', LIB + '.tmp'] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(' '.join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError('nvcc failed:\n' + r.stdout + r.stderr)
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    os.replace(LIB + '.tmp', LIB)
    return LIB


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose=True,
                extra=(['-Xptxas', '-v'] if '--ptxas' in sys.argv else [])))
