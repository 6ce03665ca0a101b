"""FP64 oracle runs of the benchmark workloads at full size (fixture generator).

The FP64 oracle is the reference algorithm (oracle/, pinned bit for bit to the
reference on the golden cases) with float64 fields, psi and accumulators over
the same float32 coefficients; the FP32 oracle is the reference algorithm in
the reference's own float32.  Both replay the GPU solves' schedules
(lens_sensor_b200.solver2d.schedule_2d, solver3d.schedule_3d, batch2d's
8-period window) on the seeded workloads of lens_sensor_b200.workloads:

  c0     planar2d_te      2D TE 1600 x 480, 6000 steps, one-period CW phasor,
                          Ez snapshots every 200 steps
  c1     waveguide3d_tm   3D TM 480 x 192 x 256, 4000 steps, Ex/Ey/Ez phasors over
                          8 periods, detector boxes, flux planes, Iavg
  sw<q>  sweep2d[q]       batched-sweep instances q = 10, 17, 18, 23 (TE, TM, TE,
                          TM), 4000 steps, 8-period phasor

The 3D runs use oracle/fast3d.py (the oracle's step in C++, checked bit for bit
against the NumPy oracle by tests/test_oracle_c.py).  The FP32 oracle's error
against FP64 is computed here on the whole fields and recorded beside the
fixtures, as the reference algorithm's own float32 error.

Fixtures (tests/golden/fp64/): the whole c0 phasor; for the larger fields a
hashed sample of the cells (sample_mask: 1 cell in 2^s by a multiplicative hash
of the flat index) plus the z mid-plane of each c1 component, and the whole-field
norms; scalars and the FP32 errors in fp64.json.

  python tests/golden/make_fp64.py run c1 f64 RAW     # one run -> RAW/c1_f64.npz
  python tests/golden/make_fp64.py pack RAW           # RAW/*.npz -> tests/golden/fp64/
  python tests/golden/make_fp64.py all RAW            # every run (2 at a time), then pack
"""
import json
import os
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import fdtd_oracle as O  # noqa: E402
from oracle import harness as H  # noqa: E402

OUT = os.path.join(HERE, 'fp64')
SWEEP_Q = (10, 17, 18, 23)
C0_STEPS, C1_STEPS, SW_STEPS = 6000, 4000, 4000


def sample_mask(n, shift):
    """1 cell in 2^shift of a flat array of n cells: (i * 2654435761 mod 2^32) >> (32 - shift) == 0."""
    i = np.arange(n, dtype=np.uint64)
    return (((i * np.uint64(2654435761)) & np.uint64(0xFFFFFFFF)) >> np.uint64(32 - shift)) == 0


def case2d(sp):
    st = sp.stack
    return dict(pol=sp.pol, Nx=sp.nx, Ny=sp.ny, dx=sp.dx, lam_nm=sp.lam_nm, npml=sp.npml, tear_m=sp.tear_m,
                wg_n=complex(st.wg_n).real, wg_um=st.t_wg_um, n_sub=st.n_sub, waist_um=sp.waist_um,
                stack=[[t, [complex(n).real, complex(n).imag]] for t, n in st.layers],
                bead=dict(x_um=sp.bead.x_um, d_um=sp.bead.d_um, y_um=sp.bead.y_um),
                bead_n=complex(sp.bead.n).real)


def case3d(sp):
    st = sp.stack
    return dict(pol=sp.pol, Nx=sp.nx, Ny=sp.ny, Nz=sp.nz, dx_nm=sp.dx_nm, t_wg_um=st.t_wg_um, tear_um=sp.tear_um,
                stack=[[t, [complex(n).real, complex(n).imag]] for t, n in st.layers], n_sub=st.n_sub,
                wg_n=st.wg_n, npml=sp.npml, lam_nm=sp.lam_nm, waist_um=sp.waist_um,
                beads=[dict(x_um=b.x_um, d_um=b.d_um, n=b.n, y_um=b.y_um, z_um=b.z_um) for b in sp.beads])


def _check_same(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape or not np.array_equal(a, b):
        raise SystemExit(f'{what}: the oracle setup differs from the product geometry for this workload')


# ----------------------------------------------------------------------------- 2D runs
def run2d(sp, steps, dtype, n_acc, snaps=()):
    """Oracle 2D solve of `steps` steps: phasor (2/n_acc) sum F e^{-iwt} of the node
    field over the last n_acc steps, snapshots of the raw driven component."""
    from lens_sensor_b200 import geometry as G
    c = case2d(sp)
    s = H.setup_2d(c)
    geo = G.build_2d(sp)
    keys = ['ce_e', 'ce_h'] if sp.pol == 's' else ['ca_x', 'ca_y', 'da_x', 'da_y']
    for k in keys:
        if k in s or geo.get(k) is not None:
            _check_same(geo.get(k), s.get(k), k)
    for k, ok in (('amp', 'src_amp'), ('ph1', 'src_ph1'), ('ph2', 'src_ph2')):
        _check_same(geo['src'][k], s[ok], k)
    for ax in ('cx', 'cy'):
        for k in s[ax]:
            _check_same(geo[ax][k], s[ax][k], ax + k)
    coef = {k: s[k] for k in keys if k in s}
    g = O.Grid2D(sp.pol, sp.nx, sp.ny, s['dx'], s['dt'], s['cx'], s['cy'], s['src'], coef, dtype)
    omega = 2 * np.pi * s['f0']
    cdt = np.complex128 if dtype == np.float64 else np.complex64
    acc = np.zeros((sp.nx, sp.ny), cdt)
    snap = []
    comp = 'Ez' if sp.pol == 's' else 'Ey'
    for n in range(steps):
        t = n * s['dt']
        g.step(n, O.cw_envelope(t, s['f0'], sp.ramp_periods))
        if n >= steps - n_acc:
            acc += g.field().astype(cdt) * np.exp(-1j * omega * t)
        if n + 1 in snaps:
            snap.append(getattr(g, comp).astype(np.float64))
    return dict(phasor=(2.0 / n_acc) * acc.astype(np.complex128), snaps=np.array(snap))


def run_c0(dtype):
    from lens_sensor_b200.solver2d import schedule_2d
    from lens_sensor_b200.workloads import planar2d_te
    sp, steps = planar2d_te()
    sc = schedule_2d(sp, steps)
    return run2d(sp, steps, dtype, sc['n_acc'], set(sc['snaps']))


def run_sw(q, dtype):
    from lens_sensor_b200.workloads import sweep2d
    specs, steps = sweep2d()
    sp = specs[q]
    steps_per_T = max(4, int(round((1.0 / sp.f0) / sp.dt)))
    return run2d(sp, steps, dtype, min(steps, 8 * steps_per_T))


# ----------------------------------------------------------------------------- 3D run
def run_c1(dtype):
    from lens_sensor_b200 import geometry as G
    from lens_sensor_b200.solver3d import schedule_3d
    from lens_sensor_b200.workloads import waveguide3d_tm
    from oracle.fast3d import Grid3DC
    sp, steps = waveguide3d_tm()
    s = H.setup_3d(case3d(sp))
    geo = G.build_3d(sp)
    for a, k in enumerate(('ce_x', 'ce_y', 'ce_z')):
        _check_same(geo['ce'][a], s[k], k)
        _check_same(geo['da'][a], s['da'][a], f'da{a}')
        for k in s['cpml'][a]:
            _check_same(geo['cpml'][a][k], s['cpml'][a][k], f'cpml{a}{k}')
    for k, ok in (('amp', 'src_amp'), ('ph1', 'src_ph1'), ('ph2', 'src_ph2')):
        _check_same(geo['src'][k], s[ok], k)
    sc = schedule_3d(sp, steps, geo['x_facet_um'])
    comp = 'Ey' if sp.pol == 'p' else 'Ez'
    g = Grid3DC(sp.nx, sp.ny, sp.nz, s['dx'], s['dt'], s['cpml'], (s['ce_x'], s['ce_y'], s['ce_z']), s['da'],
                s['src'], comp, dtype)
    cdt = np.complex128 if dtype == np.float64 else np.complex64
    omega = sc['omega']
    d0, d1 = sc['dft']
    p0, p1 = sc['prev']
    F = getattr(g, comp)
    kc = F.shape[2] // 2
    acc = {c: np.zeros(getattr(g, c).shape, cdt) for c in ('Ex', 'Ey', 'Ez')}
    conv_last = np.zeros(F.shape[:2], cdt)
    conv_prev = np.zeros(F.shape[:2], cdt)
    Iavg = np.zeros(F.shape, dtype)
    P = np.zeros(2, np.float64)
    flux = O.PlaneFlux(omega, s['dt'], dtype)
    boxes = [(slice(b[0], b[1]), slice(b[2], b[3]), slice(b[4], b[5])) for b in sc['boxes']]
    iav = set(range(sc['n_avg0'], steps, sc['m_I']))
    t0 = time.time()
    for n in range(steps):
        t = n * s['dt']
        g.step(n, O.cw_envelope(t, s['f0'], sp.ramp_periods))
        for q, b in enumerate(boxes):
            P[q] += g.box_e2(*b)
        if n in iav:
            O.accum_e2(Iavg, g.Ex, g.Ey, g.Ez)
        ph = np.exp(-1j * omega * t)
        if d0 <= n < d1:
            for c in acc:
                acc[c] += getattr(g, c).astype(cdt) * ph
            conv_last += F[:, :, kc].astype(cdt) * ph
            for k, il in sc['planes'].items():
                flux.add(k, t, g.flux_pairs(il))
        elif p0 <= n < p1:
            conv_prev += F[:, :, kc].astype(cdt) * ph
        if n % 500 == 0:
            print(f'c1 {np.dtype(dtype).name} step {n} {time.time() - t0:.0f} s', flush=True)
    na, nb = d1 - d0, p1 - p0
    ca, cb = conv_last / na, conv_prev / max(nb, 1)
    rel = float(np.linalg.norm(ca - cb) / max(np.linalg.norm(ca), 1e-300))
    dx = s['dx']
    S = {k: flux.flux(k) for k in sc['planes']}
    out = {f'phasor_{c}': (2.0 / na) * acc[c].astype(np.complex128) for c in acc}
    out.update(Iavg=Iavg.astype(np.float64), P_in=P[0] * dx ** 3, P_out=P[1] * dx ** 3,
               S_in=S['in'], S_out=S['out'], S_up=S['src_up'], S_dn=S['src_dn'],
               transmission=S['out'] / S['in'], cw_rel_change=rel, n_iavg=len(iav))
    return out


# ----------------------------------------------------------------------------- driver
def run(name, prec, raw):
    dtype = np.float64 if prec == 'f64' else np.float32
    t0 = time.time()
    if name == 'c0':
        out = run_c0(dtype)
    elif name == 'c1':
        out = run_c1(dtype)
    elif name.startswith('sw'):
        out = run_sw(int(name[2:]), dtype)
    else:
        raise SystemExit(f'unknown run {name}')
    os.makedirs(raw, exist_ok=True)
    np.savez(os.path.join(raw, f'{name}_{prec}.npz'), **out)
    print(f'{name} {prec}: {time.time() - t0:.0f} s', flush=True)


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def pack(raw):
    os.makedirs(OUT, exist_ok=True)
    meta = dict(generator='tests/golden/make_fp64.py', hash_multiplier=2654435761, runs={})
    ld = lambda n, p: np.load(os.path.join(raw, f'{n}_{p}.npz'))
    # c0: the whole phasor; snapshots by their norms and a 1/8 sample of the last
    a, b = ld('c0', 'f64'), ld('c0', 'f32')
    ph, sn = a['phasor'], a['snaps']
    m8 = sample_mask(sn[-1].size, 3)
    np.savez_compressed(os.path.join(OUT, 'c0.npz'), phasor=ph.astype(np.complex64),
                        snap_norms=np.linalg.norm(sn.reshape(len(sn), -1), axis=1),
                        snap_last_sample=sn[-1].ravel()[m8].astype(np.float32))
    meta['runs']['c0'] = dict(workload='planar2d_te', steps=C0_STEPS, n_snaps=int(len(sn)),
                              phasor_norm=float(np.linalg.norm(ph)),
                              ref_fp32_err=dict(phasor=rel(b['phasor'], ph), snap_last=rel(b['snaps'][-1], sn[-1]),
                                                snap_all=rel(b['snaps'], sn)))
    # sweep instances: 1/8 samples of the phasor
    for q in SWEEP_Q:
        a, b = ld(f'sw{q}', 'f64'), ld(f'sw{q}', 'f32')
        ph = a['phasor']
        m = sample_mask(ph.size, 3)
        np.savez_compressed(os.path.join(OUT, f'sw{q}.npz'), phasor_sample=ph.ravel()[m].astype(np.complex64))
        meta['runs'][f'sw{q}'] = dict(workload=f'sweep2d[{q}]', steps=SW_STEPS, shape=list(ph.shape), sample_shift=3,
                                      phasor_norm=float(np.linalg.norm(ph)),
                                      ref_fp32_err=dict(phasor=rel(b['phasor'], ph),
                                                        phasor_sample=rel(b['phasor'].ravel()[m], ph.ravel()[m])))
    # c1: z mid-planes, 1/256 samples and norms of the three phasors; Iavg likewise
    a, b = ld('c1', 'f64'), ld('c1', 'f32')
    fx, r1 = {}, dict(workload='waveguide3d_tm', steps=C1_STEPS, sample_shift=8, ref_fp32_err={})
    vec64 = np.sqrt(sum(np.linalg.norm(a[f'phasor_{c}']) ** 2 for c in ('Ex', 'Ey', 'Ez')))
    for c in ('Ex', 'Ey', 'Ez'):
        ph, p32 = a[f'phasor_{c}'], b[f'phasor_{c}']
        m = sample_mask(ph.size, 8)
        kz = ph.shape[2] // 2
        fx[f'{c}_zmid'] = ph[:, :, kz].astype(np.complex64)
        fx[f'{c}_sample'] = ph.ravel()[m].astype(np.complex64)
        r1[f'{c}_shape'] = list(ph.shape)
        r1[f'{c}_norm'] = float(np.linalg.norm(ph))
        r1['ref_fp32_err'][c] = dict(own=rel(p32, ph), vector=float(np.linalg.norm(p32 - ph) / vec64),
                                     sample=rel(p32.ravel()[m], ph.ravel()[m]))
    I = a['Iavg']
    m = sample_mask(I.size, 8)
    fx['Iavg_zmid'] = I[:, :, I.shape[2] // 2].astype(np.float32)
    fx['Iavg_sample'] = I.ravel()[m].astype(np.float32)
    r1['Iavg_norm'] = float(np.linalg.norm(I))
    r1['ref_fp32_err']['Iavg'] = rel(b['Iavg'], I)
    r1['vector_norm'] = float(vec64)
    for k in ('P_in', 'P_out', 'S_in', 'S_out', 'S_up', 'S_dn', 'transmission', 'cw_rel_change', 'n_iavg'):
        r1[k] = float(a[k])
        r1['ref_fp32_err'][k] = float(abs(float(b[k]) - float(a[k])) / max(abs(float(a[k])), 1e-300))
    np.savez_compressed(os.path.join(OUT, 'c1.npz'), **fx)
    meta['runs']['c1'] = r1
    with open(os.path.join(OUT, 'fp64.json'), 'w') as f:
        json.dump(meta, f, indent=1)
    print(json.dumps(meta, indent=1))


def all_runs(raw):
    jobs = [('c1', 'f64'), ('c1', 'f32'), ('c0', 'f64'), ('c0', 'f32')] + \
        [(f'sw{q}', p) for q in SWEEP_Q for p in ('f64', 'f32')]
    env = dict(os.environ, O3_THREADS=str(max(1, (os.cpu_count() or 2) // 2)))
    running = []
    for name, prec in jobs:
        if len(running) >= 2:
            running.pop(0).wait()
        running.append(subprocess.Popen([sys.executable, __file__, 'run', name, prec, raw], env=env))
    for p in running:
        p.wait()
    pack(raw)


if __name__ == '__main__':
    cmd = sys.argv[1]
    if cmd == 'run':
        run(sys.argv[2], sys.argv[3], sys.argv[4])
    elif cmd == 'pack':
        pack(sys.argv[2])
    else:
        all_runs(sys.argv[2])
