"""Write the golden fixtures in this folder by running the REFERENCE's own code.

Run from the repository root, in a container where the reference checkout is
available (it is read only, nothing is written there):

    LENS_REF=<path of the reference checkout> python tests/golden/make_golden.py

The reference (s1alknau/lens_sensor) is pure NumPy here (CuPy absent), so its
primitives are imported and driven for a fixed number of steps in the loop order
of planar_beads/fdtd2d_core.py:781-847 and planar_3d/fdtd3d_core.py:1106-1158.
The fixtures pin the oracle (tests/test_oracle_golden.py) and give the GPU
parity tests seeded inputs whose reference outputs are known.

Outputs:
  g2d_te.npz, g2d_tm.npz, g3d_tm.npz   setup arrays + fields/phasors after N steps
  characterization.json                run_beads / run_3d / run_3d_stitched known
                                       answers at the reference HEAD
  dropin_2d.json                       run_beads + save_results outputs (NPZ / PKL
                                       summaries) of three whole-driver cases
  dropin_3d.json                       the same for run_3d + save_results_3d
  dropin_3d_stitch.json                the same for run_3d_stitched + save_results_3d
  dropin_2d_stitch.json                the same for run_beads(method='stitch') + save_results
  dropin_2d_sliding.json, dropin_2d_pulse.json, dropin_3d_pulse.json
                                       the co-moving window and the pulse stitches
  dropin_2d_extend.json                run_beads with a tighter CW_TOL (window extensions)
  dropin_2d_edges.json, dropin_3d_edges.json
                                       no bead; a bead beyond or across the domain end

`python tests/golden/make_golden.py dropin` stops after the two JSON files;
`python tests/golden/make_golden.py stitch` writes only the 3D stitch fixtures
(adds case_3d_stitch to characterization.json, writes dropin_3d_stitch.json);
`python tests/golden/make_golden.py stitch2d` writes dropin_2d_stitch.json.
`python tests/golden/make_golden.py sliding2d` writes dropin_2d_sliding.json.
`python tests/golden/make_golden.py pulse2d` writes dropin_2d_pulse.json.
`python tests/golden/make_golden.py pulse3d` writes dropin_3d_pulse.json.
`python tests/golden/make_golden.py extend2d` writes dropin_2d_extend.json.
`python tests/golden/make_golden.py edges2d` writes dropin_2d_edges.json.
`python tests/golden/make_golden.py edges3d` writes dropin_3d_edges.json.
"""
import json
import os
import shutil
import sys
import tempfile

import numpy as np

REF = os.environ.get('LENS_REF')
if not REF or not os.path.isdir(REF):
    raise SystemExit('set LENS_REF to the path of the reference (s1alknau/lens_sensor) checkout')
OUT = os.path.dirname(os.path.abspath(__file__))
os.environ['PYTHONDONTWRITEBYTECODE'] = '1'
sys.dont_write_bytecode = True
for p in (REF, os.path.join(REF, 'planar_beads'), os.path.join(REF, 'planar_3d')):
    sys.path.insert(0, p)

import fdtd2d_core as d2                     # noqa: E402
import fdtd3d_core as d3                     # noqa: E402
from boundaries import make_boundary          # noqa: E402
from boundaries3d import make_boundary_3d     # noqa: E402
from common import vcsel                      # noqa: E402
from common.flux import PlaneFluxDFT, pairs_2d, pairs_3d  # noqa: E402

C0, EPS0, MU0 = d2.C0, d2.EPS0, d2.MU0


def _stack(spec):
    return [dict(name=f'L{i}', t_um=t, n=complex(n), kappa=complex(n).imag, mat=None)
            for i, (t, n) in enumerate(spec)]


# --------------------------------------------------------------------------- 2D
CASE_2D = dict(
    te=dict(pol='s', Nx=140, Ny=96, dx=50e-9, tear_m=2.0e-6, wg_n=1.49, wg_um=1.2,
            stack=[(0.9, 1.333), (0.4, 1.34)], n_sub=1.376, bead=dict(d_um=0.6, x_um=3.3),
            npml=10, steps=240, lam_nm=850.0, ramp=None, seed=11),
    tm=dict(pol='p', Nx=140, Ny=96, dx=50e-9, tear_m=2.0e-6, wg_n=1.49, wg_um=1.2,
            stack=[(0.9, complex(1.333, 0.002)), (0.4, 1.34)], n_sub=1.376,
            bead=dict(d_um=0.6, x_um=3.3), npml=12, steps=240, lam_nm=850.0, ramp=None, seed=12),
)


def run_2d(c):
    d2.TEAR_BUFFER = c['tear_m']
    d2.LAM_LOSS = c['lam_nm'] * 1e-9
    Nx, Ny, dx = c['Nx'], c['Ny'], c['dx']
    dt = 0.5 * dx / (C0 * np.sqrt(2))
    src_ix = c['npml'] + 2
    x_facet_um, air, zsrc = d2._vcsel_geom_2d(src_ix, dx, 0.0)
    stack = _stack(c['stack'])
    bp = {}
    T_WG = c['wg_um'] * 1e-6
    eps, sig = d2.build_materials(Nx, Ny, dx, c['wg_n'], 1.59, T_WG, c['bead']['x_um'],
                                  c['bead']['d_um'], 0.0, True, n_cornea=c['n_sub'],
                                  input_gap_um=x_facet_um, length_um=Nx * dx * 1e6,
                                  tm_patch=(bp if c['pol'] == 'p' else None), stack=stack)
    ce_e, ce_h = d2._coeffs(eps, sig, dt, dx)
    out = dict(eps=eps, sig=sig, ce_e=ce_e, ce_h=ce_h, dt=dt, dx=dx, src_ix=src_ix,
               x_facet_um=x_facet_um, zsrc=zsrc)
    da_x = da_y = None
    if c['pol'] == 'p':
        ca_x, ca_y, ch_tm = d2._tm_coeffs(eps, dt, dx)
        d2._apply_bead_tm(bp, ca_x, ca_y, dt, dx)
        da_x, da_y = d2._tm_loss(eps, sig, ca_x, ca_y, dt)
        out.update(ca_x=ca_x, ca_y=ca_y)
        if da_x is not None:
            out.update(da_x=da_x, da_y=da_y)
    f0 = C0 / (c['lam_nm'] * 1e-9)
    sigma_t = 4 / (2 * np.pi * f0)
    y0 = -c['tear_m']
    iy, vs, vs_ey = d2._vcsel_source_2d(Ny, dx, dt, T_WG, src_ix, 0.0, 3.0, c['lam_nm'], 0.0,
                                        1.0, zsrc, f0, y0_m=y0)
    src = vs_ey if c['pol'] == 'p' else vs
    out.update(src_amp=src.amp, src_ph1=src.ph1, src_ph2=src.ph2)
    bnd = make_boundary('cpml', c['pol'], Nx, Ny, dx, dt, npml=c['npml'], lam_m=c['lam_nm'] * 1e-9)
    for nm in ('kex', 'bex', 'cex', 'khx', 'bhx', 'chx', 'key', 'bey', 'cey', 'khy', 'bhy', 'chy'):
        out['cpml_' + nm] = getattr(bnd, nm)
    Ch = np.float32(dt / (MU0 * dx))
    Ez = np.zeros((Nx, Ny), np.float32)
    Hx = np.zeros((Nx, Ny - 1), np.float32)
    Hy = np.zeros((Nx - 1, Ny), np.float32)
    Ex = np.zeros((Nx - 1, Ny), np.float32)
    Ey = np.zeros((Nx, Ny - 1), np.float32)
    Hz = np.zeros((Nx - 1, Ny - 1), np.float32)
    omega = 2 * np.pi * f0
    steps = c['steps']
    n_dft = 48
    acc = np.zeros((Nx, Ny), np.complex64)
    acc_ex = np.zeros((Nx, Ny), np.complex64)
    acc_I = np.zeros((Nx, Ny), np.float32)
    box = (slice(40, 60), slice(30, 60))
    P = np.zeros((), np.float64)
    flux = PlaneFluxDFT(omega, dt)
    planes = {'in': 70, 'src_up': src.plane_up, 'src_dn': src.plane_dn}
    snaps = {}
    for n in range(steps):
        t = n * dt
        env = float(1 - np.exp(-((t / (2 * sigma_t)) ** 2)))
        if c['pol'] == 'p':
            bnd.update_H(Ex, Ey, Hz, Ch)
            if da_x is not None:
                Ex *= da_x
                Ey *= da_y
            bnd.update_E(Ex, Ey, Hz, ca_x, ca_y)
            src.inject(Ey, t, env)
            bnd.terminate(Ex, Ey)
            field = d2._tm_node_field(Ey)
            I_E = field * field + d2._tm_ex2_node(Ex)
        else:
            bnd.update_H(Ez, Hx, Hy, Ch)
            bnd.update_E(Ez, Hx, Hy, ce_e, ce_h)
            src.inject(Ez, t, env)
            bnd.terminate(Ez)
            field = Ez
            I_E = field * field
        P += np.sum(I_E[box], dtype=np.float64)
        if n >= steps - n_dft:
            acc += field.astype(np.complex64) * np.exp(-1j * omega * t)
            if c['pol'] == 'p':
                acc_ex += d2._tm_ex_node(Ex).astype(np.complex64) * np.exp(-1j * omega * t)
            for k, il in planes.items():
                flux.add(k, t, pairs_2d(c['pol'], il, Ez=Ez, Hy=Hy, Ey=Ey, Hz=Hz))
        if n >= steps // 2:
            acc_I += I_E
        if n + 1 in (steps // 2, steps):
            tag = f'_n{n + 1}'
            if c['pol'] == 'p':
                snaps.update({'Ex' + tag: Ex.copy(), 'Ey' + tag: Ey.copy(), 'Hz' + tag: Hz.copy()})
            else:
                snaps.update({'Ez' + tag: Ez.copy(), 'Hx' + tag: Hx.copy(), 'Hy' + tag: Hy.copy()})
    out.update(snaps)
    out.update(acc=acc, acc_I=acc_I, P_box=P, n_dft=n_dft,
               flux_in=flux.flux('in'), flux_up=flux.flux('src_up'), flux_dn=flux.flux('src_dn'))
    if c['pol'] == 'p':
        out['acc_ex'] = acc_ex
    return out


# --------------------------------------------------------------------------- 3D
CASE_3D = dict(pol='p', Nx=64, Ny=48, Nz=40, dx_nm=50.0, t_wg_um=0.8, air_um=0.5,
               tear_um=1.1, stack=[(0.6, complex(1.333, 0.003)), (0.3, 1.34)], n_sub=1.376,
               wg_n=1.49, bead=dict(x_um=1.9, d_um=0.5, n=1.59, z_um=0.1), npml=10,
               steps=90, lam_nm=850.0)


def run_3d_case(c):
    Nx, Ny, Nz = c['Nx'], c['Ny'], c['Nz']
    dx_um = c['dx_nm'] / 1000.0
    dx = c['dx_nm'] * 1e-9
    dt = 0.5 * dx / (C0 * np.sqrt(3))
    LAM = c['lam_nm'] * 1e-9
    d3.LAM_LOSS = LAM
    y0_um = -c['tear_um']
    z0_um = -Nz * dx_um / 2.0
    n_sp = d3._sponge_cells(None, 1.2, dx_um, (Nx, Ny, Nz), warn=False)
    x_src_um, x_wg_start_um, air, zsrc = d3._vcsel_geom_3d(n_sp, dx_um, 0.0)
    stack = _stack(c['stack'])
    tp = {}
    eps = d3.build_eps3d(Nx, Ny, Nz, dx_um, y0_um, z0_um, c['wg_n'], c['t_wg_um'],
                         0.0, 0.0, 0.0, 1.48, 1.333, 1.34, c['n_sub'], c['bead'],
                         x_wg_start_um=x_wg_start_um, tensor_patch=tp, stack=stack)
    eps_r, eim = d3._split_eps3(eps)
    inv, da = d3._inv_loss(eps_r, eim, dt, dx, LAM)
    ce_x, ce_y, ce_z = d3._ce_arrays(inv, tp, dt, dx, dx_um, da=da)
    da3 = d3._stagger_da(da)
    pol, Nj, Nk = d3._resolve_pol(c['pol'], Ny, Nz)
    src_ix, j_src, k_src, vs = d3._build_gauss_source(
        n_sp, c['t_wg_um'], y0_um, z0_um, dx_um, dx, LAM, Nj, Nk, 1.0, 1.0, 0.0, 0.0, 0.0,
        n_src_fn=lambda j, k: 1.0, pol=pol, dt=dt, z_prop_um=zsrc)
    bnd = make_boundary_3d('cpml', dx, dt, d3.ALL_FACES, shape=(Nx, Ny, Nz), lam_m=LAM)
    Ch = np.float32(dt / (MU0 * dx))
    Ex = np.zeros((Nx - 1, Ny, Nz), np.float32)
    Ey = np.zeros((Nx, Ny - 1, Nz), np.float32)
    Ez = np.zeros((Nx, Ny, Nz - 1), np.float32)
    Hx = np.zeros((Nx, Ny - 1, Nz - 1), np.float32)
    Hy = np.zeros((Nx - 1, Ny, Nz - 1), np.float32)
    Hz = np.zeros((Nx - 1, Ny - 1, Nz), np.float32)
    f0 = C0 / LAM
    omega = 2 * np.pi * f0
    sigma_t = 4 / (2 * np.pi * f0)
    steps = c['steps']
    n_dft = 30
    acc = np.zeros_like(Ey, dtype=np.complex64)
    Iavg = np.zeros_like(Ey)
    P = np.zeros((), np.float64)
    zs = slice(n_sp, -n_sp) if 2 * n_sp < Nz else slice(0, Nz)
    box = (slice(36, 44), slice(20, 34), zs)
    flux = PlaneFluxDFT(omega, dt)
    planes = {'in': 40, 'src_up': vs.plane_up, 'src_dn': vs.plane_dn}
    out = dict(eps=eps, ce_x=ce_x, ce_y=ce_y, ce_z=ce_z, dt=dt, dx=dx, n_sp=n_sp,
               src_ix=src_ix, x_wg_start_um=x_wg_start_um, zsrc=zsrc,
               src_amp=vs.amp, src_ph1=vs.ph1, src_ph2=vs.ph2)
    if da3 is not None:
        out.update(da_x=da3[0], da_y=da3[1], da_z=da3[2])
    for ax in 'xyz':
        for t in ('b', 'c', 'k'):
            for s in ('e', 'h'):
                out[f'cpml_{t}{ax}{s}'] = getattr(bnd, f'{t}{ax}{s}')
    for n in range(steps):
        t = n * dt
        env = float(1 - np.exp(-((t / (2 * sigma_t)) ** 2)))
        bnd.step(Ex, Ey, Ez, Hx, Hy, Hz, ce_x, ce_y, ce_z, Ch, da=da3)
        vs.inject(Ey, t, env)
        P += d3._box_E2(Ex, Ey, Ez, *box)
        if n >= steps // 2 and (n - steps // 2) % 3 == 0:
            d3._accum_E2(Iavg, Ex, Ey, Ez)
        if n >= steps - n_dft:
            acc += Ey.astype(np.complex64) * np.exp(-1j * omega * t)
            for k, il in planes.items():
                flux.add(k, t, pairs_3d(il, Ey, Ez, Hy, Hz))
    out.update(Ex=Ex, Ey=Ey, Ez=Ez, Hx=Hx, Hy=Hy, Hz=Hz, acc=acc, Iavg=Iavg, P_box=P,
               n_dft=n_dft, flux_in=flux.flux('in'), flux_up=flux.flux('src_up'),
               flux_dn=flux.flux('src_dn'))
    return out


def characterization():
    """The reference's own golden-master cases (tests/test_characterization.py:73-116)
    re-run at HEAD; its stored constants are stale, these are the live values."""
    sys.path.insert(0, os.path.join(REF, 'tests'))
    import test_characterization as tc
    prev = os.getcwd()
    tmp = tempfile.mkdtemp(prefix='lens_golden_')
    try:
        os.chdir(tmp)
        r3 = tc._run_3d_case()
        r2 = tc._run_2d_case()
    finally:
        os.chdir(prev)
        shutil.rmtree(tmp, ignore_errors=True)
    return dict(case_3d=r3, case_2d=r2)


def characterization_stitch():
    """The reference's 3D stitch golden-master case (tests/test_characterization.py:87-99)
    re-run at HEAD."""
    sys.path.insert(0, os.path.join(REF, 'tests'))
    import test_characterization as tc
    prev = os.getcwd()
    tmp = tempfile.mkdtemp(prefix='lens_golden_')
    try:
        os.chdir(tmp)
        return tc._run_3d_stitch_case()
    finally:
        os.chdir(prev)
        shutil.rmtree(tmp, ignore_errors=True)


# ------------------------------------------------------------- drop-in run_beads
# Whole-driver cases: fdtd2d_core.run_beads + save_results (method='full', CPML, CW).
# 'te' is the reference's characterization case; 'tm_kappa' adds KAPPA losses on the
# legacy aqueous layer and the core (TM loss split, Ex phasor); 'tm_stack' runs a
# custom absorbing layer stack (auto tear buffer, stack keys in the output).
DROPIN_2D = dict(
    te=dict(kw=dict(wg_mat='pmma', bead_mat='polystyrol', bead_d_um=0.5, dx_nm=100.0,
                    save_frames=True, n_snapshots=2, wg_thickness_um=1.0, lambda_nm=850.0,
                    method='full', length_um=8.0, bead_x_um=4.0), kappa={}),
    tm_kappa=dict(kw=dict(wg_mat='pmma', bead_mat='polystyrol', bead_d_um=0.6, dx_nm=80.0,
                          save_frames=True, n_snapshots=3, wg_thickness_um=1.2, lambda_nm=850.0,
                          method='full', length_um=7.0, bead_x_um=3.6, polarization='p',
                          t_aqueous_um=1.5, t_lipid_um=0.1), kappa=dict(aq=0.002, wg=0.0005)),
    tm_stack=dict(kw=dict(wg_mat='pmma', bead_mat='polystyrol', bead_d_um=0.5, dx_nm=100.0,
                          save_frames=True, n_snapshots=2, wg_thickness_um=1.0, lambda_nm=850.0,
                          method='full', length_um=8.0, bead_x_um=4.0, polarization='p',
                          stack=[dict(name='Aqueous', t_um=6.0, n=complex(1.333, 0.001), kappa=0.001,
                                      mat=None),
                                 dict(name='Mucin', t_um=3.5, n=complex(1.342, 0.0), kappa=0.0,
                                      mat=None)]), kappa={}),
)


def _summ(v):
    """JSON summary of one NPZ / PKL value: strings verbatim, arrays reduced."""
    a = np.asarray(v)
    if a.dtype.kind in 'USO':
        return dict(kind='str', value=[str(x) for x in a.ravel()])
    d = dict(kind='num', dtype=str(a.dtype), shape=list(a.shape))
    if a.size:
        c = a.astype(np.complex128)
        d.update(sum=[float(c.real.sum()), float(c.imag.sum())], abssum=float(np.abs(c).sum()),
                 absmax=float(np.abs(c).max()))
    return d


# The CW convergence extension (fdtd2d_core.py:859-873): with the tolerance on the
# phasor change between DFT windows set below what these short runs reach, the
# driver extends the run window by window up to CW_MAX_EXTEND x its step count.
DROPIN_2D_EXTEND = dict(
    te_extend=dict(DROPIN_2D['te'], cw_tol=1e-4),
    tm_extend=dict(DROPIN_2D['tm_kappa'], cw_tol=1e-3),
)


# Geometry edge cases of run_beads: the reference run without a bead
# (place_bead=False, fdtd2d_core.py:218-219, label suffix '_ref'), and a bead
# whose centre lies beyond the domain end, which build_materials skips (:224).
DROPIN_2D_EDGES = dict(
    te_nobead=dict(DROPIN_2D['te'], kw=dict(DROPIN_2D['te']['kw'], place_bead=False)),
    tm_bead_outside=dict(DROPIN_2D['tm_kappa'], kw=dict(DROPIN_2D['tm_kappa']['kw'], bead_x_um=9.5)),
)


def dropin_2d(cases=None):
    """Run the reference driver end to end for DROPIN_2D (or `cases`) and
    summarise its outputs; a case's 'cw_tol' replaces the module's CW_TOL."""
    import glob
    import pickle
    out = {}
    for name, c in (DROPIN_2D if cases is None else cases).items():
        prev, tmp = os.getcwd(), tempfile.mkdtemp(prefix='lens_dropin_')
        old_k, old_tol = d2.KAPPA, d2.CW_TOL
        try:
            os.chdir(tmp)
            d2.KAPPA = dict(c['kappa'])
            d2.CW_TOL = c.get('cw_tol', old_tol)
            r = d2.run_beads(**c['kw'])
            d2.save_results(r)
            z = np.load(glob.glob('results/*_frames.npz')[0])
            npz = {k: _summ(z[k]) for k in z.files}
            with open(glob.glob('results/*.pkl')[0], 'rb') as f:
                pk = pickle.load(f)
        finally:
            d2.KAPPA, d2.CW_TOL = old_k, old_tol
            os.chdir(prev)
            shutil.rmtree(tmp, ignore_errors=True)
        scal = {k: (v if isinstance(v, (str, bool, int)) or v is None else
                    [float(np.real(v)), float(np.imag(v))] if isinstance(v, complex) else float(v))
                for k, v in pk.items() if isinstance(v, (str, bool, int, float, complex, np.floating))
                or v is None}
        out[name] = dict(kw={k: v for k, v in c['kw'].items() if k != 'stack'}, kappa=c['kappa'],
                         stack=[dict(L, n=[L['n'].real, L['n'].imag]) for L in c['kw'].get('stack', [])],
                         npz=npz, pkl=scal)
        if 'cw_tol' in c:
            out[name]['cw_tol'] = c['cw_tol']
    return out


# ------------------------------------------------------------- drop-in run_3d
# Whole-driver cases: fdtd3d_core.run_3d + save_results_3d (CPML, CW).  'golden3d' is
# the reference's characterization case (TE, legacy tear film); 'tm_stack' a TM run on
# a custom absorbing stack with a displaced bead; 'te_kappa' KAPPA losses with a lipid
# layer, astigmatic tilted offset source, input gap and end facet.
DROPIN_3D = dict(
    golden3d=dict(kw=dict(label='golden3d', wg_n=1.491, lx_um=4.0, air_um=1.0, tear_um=2.0, lz_um=2.0,
                          dx_nm=100.0, t_wg_um=1.0, t_aq_um=1.0, t_mu_um=0.5, lam_nm=850.0, n_snapshots=2,
                          steps_factor=1.0, vcsel_waist_um=1.0, vcsel_waist_z_um=1.0,
                          bead=dict(x_um=2.0, d_um=0.5, n=1.59), n_sponge=8), kappa={}),
    tm_stack=dict(kw=dict(label='tm_stack', wg_n=1.49, lx_um=4.2, air_um=0.8, lz_um=2.4, dx_nm=100.0,
                          t_wg_um=0.9, lam_nm=850.0, n_snapshots=3, steps_factor=1.0, vcsel_waist_um=1.2,
                          vcsel_waist_z_um=0.9, bead=dict(x_um=2.3, d_um=0.6, n=1.59, z_um=0.2),
                          n_sponge=8, polarization='p',
                          stack=[dict(name='Aqueous', t_um=1.2, n=complex(1.333, 0.002), kappa=0.002, mat=None),
                                 dict(name='Mucin', t_um=0.4, n=complex(1.342, 0.0), kappa=0.0, mat=None)]),
                  kappa={}),
    te_kappa=dict(kw=dict(label='te_kappa', wg_n=1.49, lx_um=4.0, air_um=0.8, tear_um=2.2, lz_um=2.0,
                          dx_nm=100.0, t_wg_um=1.0, t_lip_um=0.2, t_aq_um=0.9, t_mu_um=0.4, lam_nm=850.0,
                          n_snapshots=2, steps_factor=1.0, vcsel_waist_um=1.1, vcsel_waist_z_um=0.8,
                          vcsel_tilt_deg=3.0, vcsel_offset_y_um=0.1, vcsel_offset_z_um=-0.1,
                          input_gap_um=1.5, end_facet_um=0.5, bead=dict(x_um=2.1, d_um=0.5, n=1.59),
                          n_sponge=8), kappa=dict(aq=0.003, wg=0.0005)),
)


# Geometry edge cases of run_3d: no bead (bead=None), and a bead whose sphere
# crosses the z end of the domain, so its sub-pixel box is clipped there.
DROPIN_3D_EDGES = dict(
    te_nobead=dict(DROPIN_3D['golden3d'], kw=dict(DROPIN_3D['golden3d']['kw'], label='te_nobead', bead=None)),
    tm_bead_clipped=dict(DROPIN_3D['tm_stack'],
                         kw=dict(DROPIN_3D['tm_stack']['kw'], label='tm_bead_clipped',
                                 bead=dict(x_um=2.3, d_um=0.6, n=1.59, z_um=1.05))),
)


def dropin_3d(cases=None):
    """Run the reference 3D driver end to end for DROPIN_3D (or `cases`) and
    summarise its outputs."""
    import glob
    import pickle
    out = {}
    for name, c in (DROPIN_3D if cases is None else cases).items():
        prev, tmp = os.getcwd(), tempfile.mkdtemp(prefix='lens_dropin3d_')
        old_k = d3.KAPPA
        try:
            os.chdir(tmp)
            d3.KAPPA = dict(c['kappa'])
            r = d3.run_3d(**c['kw'])
            d3.save_results_3d(r)
            files = {}
            for f in sorted(glob.glob('results/*.npz')):
                z = np.load(f)
                files[os.path.basename(f).replace(c['kw']['label'], '{label}')] = {k: _summ(z[k]) for k in z.files}
            with open(glob.glob('results/*.pkl')[0], 'rb') as f:
                pk = pickle.load(f)
        finally:
            d3.KAPPA = old_k
            os.chdir(prev)
            shutil.rmtree(tmp, ignore_errors=True)
        scal = {k: (v if isinstance(v, (str, bool, int)) or v is None else
                    [float(np.real(v)), float(np.imag(v))] if isinstance(v, complex) else float(v))
                for k, v in pk.items() if isinstance(v, (str, bool, int, float, complex, np.floating))
                or v is None}
        kw = {k: v for k, v in c['kw'].items() if k != 'stack'}
        out[name] = dict(kw=kw, kappa=c['kappa'],
                         stack=[dict(L, n=[L['n'].real, L['n'].imag]) for L in c['kw'].get('stack', [])],
                         npz=files, pkl=scal)
    return out


# ------------------------------------------------------ drop-in run_3d_stitched
# Whole-driver cases: fdtd3d_core.run_3d_stitched + save_results_3d.  'goldenstitch' is
# the reference's characterization case (TE, 3 windows, the last one flush with the
# domain end so two windows assemble the same planes); 'tm_stack' a TM run over 4
# windows on an absorbing custom stack, a rectangular channel, a bead across a window
# seam, an input gap and a tilted offset source.
DROPIN_3D_STITCH = dict(
    goldenstitch=dict(kw=dict(label='goldenstitch', wg_n=1.491, window_w_um=2.0, slide_um=1.2, lx_um=4.0,
                              air_um=1.0, tear_um=2.0, lz_um=2.0, dx_nm=100.0, t_wg_um=1.0, t_aq_um=1.0,
                              t_mu_um=0.5, lam_nm=850.0, n_snapshots=2, vcsel_waist_um=1.0,
                              vcsel_waist_z_um=1.0, bead=dict(x_um=2.0, d_um=0.5, n=1.59), n_sponge=8),
                      kappa={}),
    tm_stack=dict(kw=dict(label='tm_stack', wg_n=1.49, window_w_um=2.2, slide_um=1.0, lx_um=5.0, air_um=0.6,
                          tear_um=2.0, lz_um=2.0, dx_nm=100.0, t_wg_um=0.9, lam_nm=850.0, n_snapshots=3,
                          vcsel_waist_um=0.9, vcsel_waist_z_um=0.7, vcsel_tilt_deg=2.0, vcsel_offset_y_um=0.05,
                          vcsel_offset_z_um=-0.1, input_gap_um=1.5, wg_width_um=1.2, n_clad_side=1.33,
                          bead=dict(x_um=2.1, d_um=0.6, n=1.59, z_um=0.15), n_sponge=8, polarization='p',
                          stack=[dict(name='Aqueous', t_um=1.0, n=complex(1.333, 0.002), kappa=0.002, mat=None),
                                 dict(name='Mucin', t_um=0.3, n=complex(1.342, 0.0), kappa=0.0, mat=None)]),
                  kappa={}),
)


def dropin_3d_stitch():
    """Run the reference stitch driver end to end for DROPIN_3D_STITCH and summarise."""
    import glob
    import pickle
    out = {}
    for name, c in DROPIN_3D_STITCH.items():
        prev, tmp = os.getcwd(), tempfile.mkdtemp(prefix='lens_stitch_')
        old_k = d3.KAPPA
        try:
            os.chdir(tmp)
            d3.KAPPA = dict(c['kappa'])
            r = d3.run_3d_stitched(**c['kw'])
            res = dict(transmission=float(r['transmission']), P_in=float(r['P_in']), P_out=float(r['P_out']),
                       transmission_intensity=float(r['transmission_intensity']),
                       steps_total=int(r['steps_total']))
            d3.save_results_3d(r)
            files = {}
            for f in sorted(glob.glob('results/*.npz')):
                z = np.load(f)
                files[os.path.basename(f).replace(c['kw']['label'], '{label}')] = {k: _summ(z[k]) for k in z.files}
            with open(glob.glob('results/*.pkl')[0], 'rb') as f:
                pk = pickle.load(f)
            left = sorted(os.listdir('results'))
        finally:
            d3.KAPPA = old_k
            os.chdir(prev)
            shutil.rmtree(tmp, ignore_errors=True)
        scal = {k: (v if isinstance(v, (str, bool, int)) or v is None else
                    [float(np.real(v)), float(np.imag(v))] if isinstance(v, complex) else float(v))
                for k, v in pk.items() if isinstance(v, (str, bool, int, float, complex, np.floating))
                or v is None}
        kw = {k: v for k, v in c['kw'].items() if k != 'stack'}
        out[name] = dict(kw=kw, kappa=c['kappa'],
                         stack=[dict(L, n=[L['n'].real, L['n'].imag]) for L in c['kw'].get('stack', [])],
                         result=res, npz=files, pkl=scal, files_left=left)
    return out


# ------------------------------------------------------ drop-in run_beads_stitched
# Whole-driver cases: fdtd2d_core.run_beads(method='stitch') + save_results.  'te' runs 3
# windows on the characterization stack (the last one flush with the domain end); 'tm'
# 4 windows on an absorbing custom stack with KAPPA on the core, an input gap, a tilted
# offset source and a bead across a seam (TM: Ey handoff, <Ex^2> and Ex amplitude).
DROPIN_2D_STITCH = dict(
    te=dict(kw=dict(wg_mat='pmma', bead_mat='polystyrol', bead_d_um=0.5, dx_nm=100.0, save_frames=True,
                    n_snapshots=2, wg_thickness_um=1.0, lambda_nm=850.0, method='stitch', length_um=12.0,
                    bead_x_um=5.0, window_w_um=5.0, slide_um=3.5), kappa={}),
    tm=dict(kw=dict(wg_mat='pmma', bead_mat='polystyrol', bead_d_um=0.6, dx_nm=100.0, save_frames=True,
                    n_snapshots=3, wg_thickness_um=1.2, lambda_nm=850.0, method='stitch', length_um=14.0,
                    bead_x_um=6.3, window_w_um=5.0, slide_um=3.2, polarization='p', input_gap_um=1.5,
                    vcsel_tilt=2.0, vcsel_offset=0.1, vcsel_waist=1.2,
                    stack=[dict(name='Aqueous', t_um=2.0, n=complex(1.333, 0.002), kappa=0.002, mat=None),
                           dict(name='Mucin', t_um=0.5, n=complex(1.342, 0.0), kappa=0.0, mat=None)]),
            kappa=dict(wg=0.0005)),
)


def dropin_2d_stitch():
    """Run the reference 2D stitch end to end for DROPIN_2D_STITCH and summarise its outputs."""
    import glob
    import pickle
    import re
    out = {}
    for name, c in DROPIN_2D_STITCH.items():
        prev, tmp = os.getcwd(), tempfile.mkdtemp(prefix='lens_stitch2d_')
        old_k = d2.KAPPA
        try:
            os.chdir(tmp)
            d2.KAPPA = dict(c['kappa'])
            r = d2.run_beads(**c['kw'])
            res = dict(transmission=float(r['transmission']), P_in=float(r['P_in']), P_out=float(r['P_out']),
                       transmission_intensity=float(r['transmission_intensity']))
            arrays = {}
            for key in ('Iavg', 'Ex_cw_amp'):
                if r.get(key) is not None:
                    arrays[key] = _summ(np.asarray(r[key]))
            d2.save_results(r)
            z = np.load(glob.glob('results/*_frames.npz')[0])
            npz = {k: _summ(z[k]) for k in z.files}
            with open(glob.glob('results/*.pkl')[0], 'rb') as f:
                pk = pickle.load(f)
            left = sorted(re.sub(r'_\d+_\d+\.npy$', '_{tag}.npy', f) for f in os.listdir('results'))
        finally:
            d2.KAPPA, d2.CW_TOL = old_k, old_tol
            os.chdir(prev)
            shutil.rmtree(tmp, ignore_errors=True)
        scal = {k: (v if isinstance(v, (str, bool, int)) or v is None else
                    [float(np.real(v)), float(np.imag(v))] if isinstance(v, complex) else float(v))
                for k, v in pk.items() if isinstance(v, (str, bool, int, float, complex, np.floating))
                or v is None}
        out[name] = dict(kw={k: v for k, v in c['kw'].items() if k != 'stack'}, kappa=c['kappa'],
                         stack=[dict(L, n=[L['n'].real, L['n'].imag]) for L in c['kw'].get('stack', [])],
                         result=res, arrays=arrays, npz=npz, pkl=scal, files_left=left)
    return out


# ------------------------------------------------------- drop-in 2D sliding window
# run_beads(method='sliding') -> run_beads_sliding + save_results: 'te_pulse' a
# Gaussian pulse (3 cycles) through 4 slides of an 8 um window with a bead;
# 'tm_cw' a CW VCSEL through 4 slides on an absorbing stack with KAPPA on the
# core, an input gap and a tilted offset source.  Both with a 2 um air buffer
# (module AIR_BUFFER) and a 3 um tear buffer to keep the runs small.
DROPIN_2D_SLIDING = dict(
    te_pulse=dict(kw=dict(wg_mat='pmma', bead_mat='polystyrol', bead_d_um=0.5, dx_nm=25.0, save_frames=True,
                          n_snapshots=4, wg_thickness_um=1.0, lambda_nm=850.0, method='sliding', length_um=16.0,
                          bead_x_um=7.0, window_w_um=8.0, slide_um=4.0, source_type='pulse', pulse_cycles=3.0,
                          tear_buffer_um=3.0),
                  kappa={}, air_um=2.0),
    tm_cw=dict(kw=dict(wg_mat='pmma', bead_mat='polystyrol', bead_d_um=0.6, dx_nm=25.0, save_frames=True,
                       n_snapshots=3, wg_thickness_um=1.2, lambda_nm=850.0, method='sliding', length_um=14.0,
                       bead_x_um=6.3, window_w_um=7.0, slide_um=3.5, polarization='p', input_gap_um=1.5,
                       vcsel_tilt=2.0, vcsel_offset=0.1, vcsel_waist=1.2, tear_buffer_um=4.5,
                       stack=[dict(name='Aqueous', t_um=2.0, n=complex(1.333, 0.002), kappa=0.002, mat=None),
                              dict(name='Mucin', t_um=0.5, n=complex(1.342, 0.0), kappa=0.0, mat=None)]),
               kappa=dict(wg=0.0005), air_um=2.0),
)


def dropin_2d_sliding():
    """Run the reference co-moving window end to end for DROPIN_2D_SLIDING and summarise its outputs."""
    import glob
    import pickle
    out = {}
    for name, c in DROPIN_2D_SLIDING.items():
        prev, tmp = os.getcwd(), tempfile.mkdtemp(prefix='lens_sliding2d_')
        old_k, old_air = d2.KAPPA, d2.AIR_BUFFER
        try:
            os.chdir(tmp)
            d2.KAPPA = dict(c['kappa'])
            d2.AIR_BUFFER = c['air_um'] * 1e-6
            r = d2.run_beads(**c['kw'])
            res = {k: float(r[k]) for k in ('transmission', 'P_in', 'P_out', 'transmission_intensity')}
            res.update({k: float(r[k]) for k in ('coupling_efficiency', 'facet_reflection') if k in r})
            fr = np.load(r['frames_memmap'], mmap_mode='r')[:len(r['frames'])]
            frames = _summ(np.asarray(fr))
            d2.save_results(r)
            z = np.load(glob.glob('results/*_frames.npz')[0])
            npz = {k: _summ(z[k]) for k in z.files}
            with open(glob.glob('results/*.pkl')[0], 'rb') as f:
                pk = pickle.load(f)
            left = sorted(os.listdir('results'))
        finally:
            d2.KAPPA, d2.AIR_BUFFER = old_k, old_air
            os.chdir(prev)
            shutil.rmtree(tmp, ignore_errors=True)
        scal = {k: (v if isinstance(v, (str, bool, int)) or v is None else
                    [float(np.real(v)), float(np.imag(v))] if isinstance(v, complex) else float(v))
                for k, v in pk.items() if isinstance(v, (str, bool, int, float, complex, np.floating))
                or v is None}
        out[name] = dict(kw={k: v for k, v in c['kw'].items() if k != 'stack'}, kappa=c['kappa'],
                         air_um=c['air_um'],
                         stack=[dict(L, n=[L['n'].real, L['n'].imag]) for L in c['kw'].get('stack', [])],
                         result=res, frames=frames, npz=npz, pkl=scal, files_left=left)
    return out


# ------------------------------------------------- drop-in 2D Fourier pulse stitch
# run_beads(method='stitch', source_type='pulse') -> run_beads_stitched_pulse +
# save_results: 'te_disp' 5 frequencies with material dispersion (the core's n
# follows n(lambda_k)) on the characterization stack; 'tm_fixed' 4 frequencies
# with every index held at lambda0, an absorbing stack, KAPPA on the core, an
# input gap and a tilted offset source, frames at a set t_max.
DROPIN_2D_PULSE = dict(
    te_disp=dict(kw=dict(wg_mat='pmma', bead_mat='polystyrol', bead_d_um=0.5, dx_nm=100.0, save_frames=True,
                         n_snapshots=2, wg_thickness_um=1.0, lambda_nm=850.0, method='stitch', length_um=12.0,
                         bead_x_um=5.0, window_w_um=5.0, slide_um=3.5, source_type='pulse', pulse_cycles=3.0,
                         pulse_nfreq=5), kappa={}),
    tm_fixed=dict(kw=dict(wg_mat='pmma', bead_mat='polystyrol', bead_d_um=0.6, dx_nm=100.0, save_frames=True,
                          n_snapshots=3, wg_thickness_um=1.2, lambda_nm=850.0, method='stitch', length_um=11.0,
                          bead_x_um=5.3, window_w_um=5.0, slide_um=3.2, polarization='p', input_gap_um=1.5,
                          vcsel_tilt=2.0, vcsel_offset=0.1, vcsel_waist=1.2, source_type='pulse', pulse_cycles=4.0,
                          pulse_nfreq=4, pulse_dispersion=False, pulse_tmax_fs=120.0,
                          stack=[dict(name='Aqueous', t_um=2.0, n=complex(1.333, 0.002), kappa=0.002, mat=None),
                                 dict(name='Mucin', t_um=0.5, n=complex(1.342, 0.0), kappa=0.0, mat=None)]),
                  kappa=dict(wg=0.0005)),
)


def dropin_2d_pulse():
    """Run the reference Fourier pulse stitch end to end for DROPIN_2D_PULSE and summarise its outputs."""
    import glob
    import pickle
    import re
    out = {}
    for name, c in DROPIN_2D_PULSE.items():
        prev, tmp = os.getcwd(), tempfile.mkdtemp(prefix='lens_pulse2d_')
        old_k = d2.KAPPA
        try:
            os.chdir(tmp)
            d2.KAPPA = dict(c['kappa'])
            r = d2.run_beads(**c['kw'])
            res = {k: float(r[k]) for k in ('transmission', 'P_in', 'P_out', 'transmission_intensity')}
            spec = {k: [float(v) for v in np.asarray(r['spectrum'][k])] for k in ('lam_nm', 'T', 'P_out', 'weight')}
            fr = _summ(np.asarray(np.load(r['frames_memmap'], mmap_mode='r')[:len(r['frames'])]))
            d2.save_results(r)
            z = np.load(glob.glob('results/*_frames.npz')[0])
            npz = {k: _summ(z[k]) for k in z.files}
            with open(glob.glob('results/*.pkl')[0], 'rb') as f:
                pk = pickle.load(f)
            left = sorted(re.sub(r'_\d+_\d+\.npy$', '_{tag}.npy', f) for f in os.listdir('results'))
        finally:
            d2.KAPPA, d2.CW_TOL = old_k, old_tol
            os.chdir(prev)
            shutil.rmtree(tmp, ignore_errors=True)
        scal = {k: (v if isinstance(v, (str, bool, int)) or v is None else
                    [float(np.real(v)), float(np.imag(v))] if isinstance(v, complex) else float(v))
                for k, v in pk.items() if isinstance(v, (str, bool, int, float, complex, np.floating))
                or v is None}
        out[name] = dict(kw={k: v for k, v in c['kw'].items() if k != 'stack'}, kappa=c['kappa'],
                         stack=[dict(L, n=[L['n'].real, L['n'].imag]) for L in c['kw'].get('stack', [])],
                         result=res, spectrum=spec, frames=fr, npz=npz, pkl=scal, files_left=left)
    return out


# ------------------------------------------------- drop-in 3D Fourier pulse stitch
# fdtd3d_core.run_3d_stitched_pulse + save_results_3d: 'te_disp' the
# characterization stitch geometry, 3 frequencies, the core's n from n(lambda_k)
# (disp_map); 'tm_fixed' the absorbing-stack channel case, 3 frequencies with the
# indices held, a set t_max and 8 frames.
DROPIN_3D_PULSE = dict(
    te_disp=dict(kw=dict(label='te_disp', wg_n=1.491, window_w_um=2.0, slide_um=1.2, lx_um=4.0, air_um=1.0,
                         tear_um=2.0, lz_um=2.0, dx_nm=100.0, t_wg_um=1.0, t_aq_um=1.0, t_mu_um=0.5, lam_nm=850.0,
                         n_snapshots=2, vcsel_waist_um=1.0, vcsel_waist_z_um=1.0,
                         bead=dict(x_um=2.0, d_um=0.5, n=1.59), n_sponge=8, pulse_cycles=3.0, pulse_nfreq=3,
                         disp_map=dict(wg_n='pmma')), kappa={}),
    tm_fixed=dict(kw=dict(label='tm_fixed', wg_n=1.49, window_w_um=2.2, slide_um=1.0, lx_um=5.0, air_um=0.6,
                          tear_um=2.0, lz_um=2.0, dx_nm=100.0, t_wg_um=0.9, lam_nm=850.0, n_snapshots=3,
                          vcsel_waist_um=0.9, vcsel_waist_z_um=0.7, vcsel_tilt_deg=2.0, vcsel_offset_y_um=0.05,
                          vcsel_offset_z_um=-0.1, input_gap_um=1.5, wg_width_um=1.2, n_clad_side=1.33,
                          bead=dict(x_um=2.1, d_um=0.6, n=1.59, z_um=0.15), n_sponge=8, polarization='p',
                          pulse_cycles=4.0, pulse_nfreq=3, pulse_dispersion=False, pulse_tmax_fs=90.0,
                          stack=[dict(name='Aqueous', t_um=1.0, n=complex(1.333, 0.002), kappa=0.002, mat=None),
                                 dict(name='Mucin', t_um=0.3, n=complex(1.342, 0.0), kappa=0.0, mat=None)]),
                  kappa={}),
)


def dropin_3d_pulse():
    """Run the reference 3D Fourier pulse stitch end to end for DROPIN_3D_PULSE and summarise."""
    import glob
    import pickle
    out = {}
    for name, c in DROPIN_3D_PULSE.items():
        prev, tmp = os.getcwd(), tempfile.mkdtemp(prefix='lens_pulse3d_')
        old_k = d3.KAPPA
        try:
            os.chdir(tmp)
            d3.KAPPA = dict(c['kappa'])
            r = d3.run_3d_stitched_pulse(**c['kw'])
            res = dict(transmission=float(r['transmission']), P_in=float(r['P_in']), P_out=float(r['P_out']))
            spec = {k: [float(v) for v in np.asarray(r['spectrum'][k])] for k in ('lam_nm', 'T', 'weight')}
            arrays = dict(vols=_summ(np.asarray(r['vols_array'])), Iavg=_summ(np.asarray(r['Iavg'])),
                          cw_vol=_summ(np.asarray(r['cw_vol'])))
            d3.save_results_3d(r)
            files = {}
            for f in sorted(glob.glob('results/*.npz')):
                z = np.load(f)
                files[os.path.basename(f).replace(c['kw']['label'], '{label}')] = {k: _summ(z[k]) for k in z.files}
            with open(glob.glob('results/*.pkl')[0], 'rb') as f:
                pk = pickle.load(f)
            left = sorted(os.listdir('results'))
        finally:
            d3.KAPPA = old_k
            os.chdir(prev)
            shutil.rmtree(tmp, ignore_errors=True)
        scal = {k: (v if isinstance(v, (str, bool, int)) or v is None else
                    [float(np.real(v)), float(np.imag(v))] if isinstance(v, complex) else float(v))
                for k, v in pk.items() if isinstance(v, (str, bool, int, float, complex, np.floating))
                or v is None}
        kw = {k: v for k, v in c['kw'].items() if k != 'stack'}
        out[name] = dict(kw=kw, kappa=c['kappa'],
                         stack=[dict(L, n=[L['n'].real, L['n'].imag]) for L in c['kw'].get('stack', [])],
                         result=res, spectrum=spec, arrays=arrays, npz=files, pkl=scal, files_left=left)
    return out


def main():
    if 'edges3d' in sys.argv[1:]:
        with open(os.path.join(OUT, 'dropin_3d_edges.json'), 'w') as f:
            json.dump(dropin_3d(DROPIN_3D_EDGES), f, indent=1)
        print('wrote dropin_3d_edges.json')
        return
    if 'edges2d' in sys.argv[1:]:
        with open(os.path.join(OUT, 'dropin_2d_edges.json'), 'w') as f:
            json.dump(dropin_2d(DROPIN_2D_EDGES), f, indent=1)
        print('wrote dropin_2d_edges.json')
        return
    if 'extend2d' in sys.argv[1:]:
        with open(os.path.join(OUT, 'dropin_2d_extend.json'), 'w') as f:
            json.dump(dropin_2d(DROPIN_2D_EXTEND), f, indent=1)
        print('wrote dropin_2d_extend.json')
        return
    if 'pulse3d' in sys.argv[1:]:
        with open(os.path.join(OUT, 'dropin_3d_pulse.json'), 'w') as f:
            json.dump(dropin_3d_pulse(), f, indent=1)
        print('wrote dropin_3d_pulse.json')
        return
    if 'pulse2d' in sys.argv[1:]:
        with open(os.path.join(OUT, 'dropin_2d_pulse.json'), 'w') as f:
            json.dump(dropin_2d_pulse(), f, indent=1)
        print('wrote dropin_2d_pulse.json')
        return
    if 'sliding2d' in sys.argv[1:]:
        with open(os.path.join(OUT, 'dropin_2d_sliding.json'), 'w') as f:
            json.dump(dropin_2d_sliding(), f, indent=1)
        print('wrote dropin_2d_sliding.json')
        return
    if 'stitch2d' in sys.argv[1:]:
        with open(os.path.join(OUT, 'dropin_2d_stitch.json'), 'w') as f:
            json.dump(dropin_2d_stitch(), f, indent=1)
        print('wrote dropin_2d_stitch.json')
        return
    if 'stitch' in sys.argv[1:]:
        path = os.path.join(OUT, 'characterization.json')
        ch = json.load(open(path))
        ch['case_3d_stitch'] = characterization_stitch()
        with open(path, 'w') as f:
            json.dump(ch, f, indent=1)
        with open(os.path.join(OUT, 'dropin_3d_stitch.json'), 'w') as f:
            json.dump(dropin_3d_stitch(), f, indent=1)
        print('wrote case_3d_stitch, dropin_3d_stitch.json')
        return
    ch = characterization()          # first: the cases below change module globals
    with open(os.path.join(OUT, 'characterization.json'), 'w') as f:
        json.dump(ch, f, indent=1)
    print('wrote characterization.json')
    with open(os.path.join(OUT, 'dropin_2d.json'), 'w') as f:
        json.dump(dropin_2d(), f, indent=1)
    print('wrote dropin_2d.json')
    with open(os.path.join(OUT, 'dropin_3d.json'), 'w') as f:
        json.dump(dropin_3d(), f, indent=1)
    print('wrote dropin_3d.json')
    if 'dropin' in sys.argv[1:]:
        return
    for name, c in CASE_2D.items():
        o = run_2d(c)
        o = {k: (np.asarray(v) if not isinstance(v, (int, float)) else np.asarray(v)) for k, v in o.items()}
        np.savez_compressed(os.path.join(OUT, f'g2d_{name}.npz'), **o)
        print('wrote', name, sorted(o))
    o = run_3d_case(CASE_3D)
    np.savez_compressed(os.path.join(OUT, 'g3d_tm.npz'), **{k: np.asarray(v) for k, v in o.items()})
    print('wrote g3d_tm')
    with open(os.path.join(OUT, 'cases.json'), 'w') as f:
        json.dump(dict(d2=CASE_2D, d3=CASE_3D), f, indent=1, default=lambda v: [v.real, v.imag])


if __name__ == '__main__':
    main()
