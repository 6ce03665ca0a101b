"""Oracle drivers for fixed-step solves (TEST INFRASTRUCTURE ONLY).

Builds a case with the oracle's setup functions and runs it for a fixed number
of steps in the reference loop order (planar_beads/fdtd2d_core.py:781-850,
planar_3d/fdtd3d_core.py:1106-1158).  A case is a plain dict (see
tests/golden/cases.json): geometry in the reference's own parameters, so the
same dict drives the reference (tests/golden/make_golden.py), this oracle and
the GPU engine.
"""

import numpy as np

from . import fdtd_oracle as O

F32 = np.float32


def _cplx(v):
    return complex(v[0], v[1]) if isinstance(v, (list, tuple)) else v


def sponge_cells(dx_um, shape, sponge_um=1.2):
    """fdtd3d_core.py:262-275 with n_sponge=None."""
    n = max(8, int(np.ceil(float(sponge_um) / dx_um)))
    cap = max(8, min(s // 6 for s in shape))
    return min(n, cap)


def air_path_um(distance_um, dx_um):
    """vcsel.py:64-70."""
    return max(float(distance_um or 0.0), max(1.0, 8 * float(dx_um)))


# ----------------------------------------------------------------------------- 2D
def setup_2d(c):
    Nx, Ny, dx = c['Nx'], c['Ny'], c['dx']
    dt = 0.5 * dx / (O.C0 * np.sqrt(2))
    lam_m = c['lam_nm'] * 1e-9
    src_ix = c['npml'] + 2
    air = air_path_um(0.0, dx * 1e6)
    x_facet_um = src_ix * dx * 1e6 + air
    zsrc = 0.0 - air
    stack = [(t, _cplx(n)) for t, n in c['stack']]
    T_WG = c['wg_um'] * 1e-6
    r = c['bead']['d_um'] * 1e-6 / 2.0
    yc = c['bead']['y_um'] * 1e-6 if c['bead'].get('y_um') is not None else -r
    bead = dict(xc=c['bead']['x_um'] * 1e-6, yc=yc, r=r, n=c.get('bead_n', 1.59))
    tm = c['pol'] == 'p'
    eps, sig, patch = O.materials_2d(Nx, Ny, dx, -c['tear_m'], c['wg_n'], T_WG, stack, c['n_sub'],
                                     bead, x_wg=(x_facet_um * 1e-6, Nx * dx * 1e6 * 1e-6),
                                     lam_m=lam_m, tm=tm)
    ce_e, ce_h = O.te_coeffs(eps, sig, dt, dx)
    out = dict(eps=eps, sig=sig, ce_e=ce_e, ce_h=ce_h, dt=dt, dx=dx, src_ix=src_ix,
               x_facet_um=x_facet_um, zsrc=zsrc)
    if tm:
        ca_x, ca_y, da_x, da_y = O.tm_coeffs(eps, sig, dt, dx, patch)
        out.update(ca_x=ca_x, ca_y=ca_y)
        if da_x is not None:
            out.update(da_x=da_x, da_y=da_y)
    f0 = O.C0 / lam_m
    y0 = -c['tear_m']
    yc = T_WG / 2
    y_um = (y0 + np.arange(Ny) * dx) * 1e6
    amp, ph = O.profile_1d(y_um, yc * 1e6, zsrc, c.get('waist_um', 3.0), c['lam_nm'], 1.0, 0.0)
    kdx = O.kx_dx(c['lam_nm'], dx, O.C0 * dt, 1.0, 0.0)
    src = O.Huygens(src_ix, amp, ph, 2 * np.pi * f0, kdx)
    if tm:
        src = src.on_ey_grid()
    out.update(src=src, src_amp=src.amp, src_ph1=src.ph1, src_ph2=src.ph2, f0=f0)
    npml = c['npml']
    out['cx'] = O.cpml_axis(Nx, npml, npml, dx, dt, lam_m)
    out['cy'] = O.cpml_axis(Ny, npml, npml, dx, dt, lam_m)
    return out


def run_2d(c, dtype=F32, steps=None, n_dft=48, box=(slice(40, 60), slice(30, 60)),
           planes=None, setup=None, envelope=None):
    """The golden 2D loop of tests/golden/make_golden.py, on the oracle."""
    s = setup or setup_2d(c)
    Nx, Ny = c['Nx'], c['Ny']
    steps = c['steps'] if steps is None else steps
    coef = {k: s[k] for k in ('ce_e', 'ce_h', 'ca_x', 'ca_y', 'da_x', 'da_y') if k in s}
    g = O.Grid2D(c['pol'], Nx, Ny, s['dx'], s['dt'], s['cx'], s['cy'], s['src'], coef, dtype)
    f0 = s['f0']
    omega = 2 * np.pi * f0
    sigma_t = 4 / (2 * np.pi * f0)
    cdt = np.complex128 if dtype == np.float64 else np.complex64
    acc = np.zeros((Nx, Ny), cdt)
    acc_ex = np.zeros((Nx, Ny), cdt)
    acc_I = np.zeros((Nx, Ny), dtype)
    P = np.zeros((), np.float64)
    flux = O.PlaneFlux(omega, s['dt'], dtype)
    if planes is None:
        planes = {'in': 70, 'src_up': s['src'].ix - 1, 'src_dn': s['src'].ix + 3}
    out = {}
    for n in range(steps):
        t = n * s['dt']
        env = envelope(n) if envelope else float(1 - np.exp(-((t / (2 * sigma_t)) ** 2)))
        g.step(n, env)
        field = g.field()
        I_E = g.intensity(field)
        P += np.sum(I_E[box], dtype=np.float64)
        if n >= steps - n_dft:
            ph = np.exp(-1j * omega * t)        # complex128 scalar, as in the reference
            acc += field.astype(cdt) * ph
            if c['pol'] == 'p':
                acc_ex += g.ex_node().astype(cdt) * ph
            for k, il in planes.items():
                flux.add(k, t, g.flux_pairs(il))
        if n >= steps // 2:
            acc_I += I_E
        if n + 1 in (steps // 2, steps):
            tag = f'_n{n + 1}'
            names = ('Ex', 'Ey', 'Hz') if c['pol'] == 'p' else ('Ez', 'Hx', 'Hy')
            out.update({nm + tag: getattr(g, nm).copy() for nm in names})
    out.update(acc=acc, acc_I=acc_I, P_box=P, flux_in=flux.flux('in'),
               flux_up=flux.flux('src_up'), flux_dn=flux.flux('src_dn'), grid=g)
    if c['pol'] == 'p':
        out['acc_ex'] = acc_ex
    return out


# ----------------------------------------------------------------------------- 3D
def setup_3d(c):
    Nx, Ny, Nz = c['Nx'], c['Ny'], c['Nz']
    dx_um = c['dx_nm'] / 1000.0
    dx = c['dx_nm'] * 1e-9
    dt = 0.5 * dx / (O.C0 * np.sqrt(3))
    LAM = c['lam_nm'] * 1e-9
    y0_um = -c['tear_um']
    z0_um = -Nz * dx_um / 2.0
    n_sp = sponge_cells(dx_um, (Nx, Ny, Nz))
    x_src_um = (n_sp + 6) * dx_um
    air = air_path_um(0.0, dx_um)
    x_wg_start_um = x_src_um + air
    zsrc = 0.0 - air
    stack = [(t, _cplx(n)) for t, n in c['stack']]
    beads = c.get('beads')
    if beads is None:
        beads = [c['bead']] if c.get('bead') else []
    eps, tp = O.eps_3d(Nx, Ny, Nz, dx_um, y0_um, z0_um, c['wg_n'], c['t_wg_um'], stack,
                       c['n_sub'], beads, x_wg_start_um=x_wg_start_um)
    ce_x, ce_y, ce_z, da = O.coeffs_3d(eps, tp, dt, dx, dx_um, LAM)
    pol = c['pol']
    Nj, Nk = (Ny - 1, Nz) if pol == 'p' else (Ny, Nz - 1)
    src_ix = n_sp + 6
    yc = c['t_wg_um'] / 2
    zc = 0.0
    yv = y0_um + (np.arange(Nj) + (0.5 if pol == 'p' else 0.0)) * dx_um
    zv = z0_um + (np.arange(Nk) + (0.5 if pol == 's' else 0.0)) * dx_um
    w = c.get('waist_um', 1.0)
    amp, ph = O.profile_2d(yv, zv, yc, zc, zsrc, w, w, c['lam_nm'], 1.0, 0.0)
    kdx = O.kx_dx(c['lam_nm'], dx, O.C0 * dt, 1.0, 0.0)
    src = O.Huygens(src_ix, amp, ph, 2 * np.pi * O.C0 / LAM, kdx)
    npml = c['npml']
    cp = [O.cpml_axis(N, npml, npml, dx, dt, LAM) for N in (Nx, Ny, Nz)]
    out = dict(eps=eps, ce_x=ce_x, ce_y=ce_y, ce_z=ce_z, dt=dt, dx=dx, n_sp=n_sp, src_ix=src_ix,
               x_wg_start_um=x_wg_start_um, zsrc=zsrc, src=src, src_amp=src.amp,
               src_ph1=src.ph1, src_ph2=src.ph2, cpml=cp, f0=O.C0 / LAM, da=da)
    if da is not None:
        out.update(da_x=da[0], da_y=da[1], da_z=da[2])
    return out


def run_3d(c, dtype=F32, steps=None, n_dft=30, box=None, planes=None, setup=None,
           iavg_every=3, envelope=None):
    """The golden 3D loop of tests/golden/make_golden.py, on the oracle."""
    s = setup or setup_3d(c)
    Nx, Ny, Nz = c['Nx'], c['Ny'], c['Nz']
    steps = c['steps'] if steps is None else steps
    comp = 'Ey' if c['pol'] == 'p' else 'Ez'
    g = O.Grid3D(Nx, Ny, Nz, s['dx'], s['dt'], s['cpml'], (s['ce_x'], s['ce_y'], s['ce_z']),
                 s['da'], s['src'], comp, dtype)
    f0 = s['f0']
    omega = 2 * np.pi * f0
    sigma_t = 4 / (2 * np.pi * f0)
    cdt = np.complex128 if dtype == np.float64 else np.complex64
    F = getattr(g, comp)
    acc = np.zeros(F.shape, cdt)
    Iavg = np.zeros(F.shape, dtype)
    P = np.zeros((), np.float64)
    n_sp = s['n_sp']
    if box is None:
        zs = slice(n_sp, -n_sp) if 2 * n_sp < Nz else slice(0, Nz)
        box = (slice(36, 44), slice(20, 34), zs)
    if planes is None:
        planes = {'in': 40, 'src_up': s['src'].ix - 1, 'src_dn': s['src'].ix + 3}
    flux = O.PlaneFlux(omega, s['dt'], dtype)
    for n in range(steps):
        t = n * s['dt']
        env = envelope(n) if envelope else float(1 - np.exp(-((t / (2 * sigma_t)) ** 2)))
        g.step(n, env)
        P += g.box_e2(*box)
        if iavg_every and n >= steps // 2 and (n - steps // 2) % iavg_every == 0:
            O.accum_e2(Iavg, g.Ex, g.Ey, g.Ez)
        if n >= steps - n_dft:
            acc += F.astype(cdt) * np.exp(-1j * omega * t)
            for k, il in planes.items():
                flux.add(k, t, g.flux_pairs(il))
    out = dict(g.fields())
    out.update(acc=acc, Iavg=Iavg, P_box=P, flux_in=flux.flux('in'), flux_up=flux.flux('src_up'),
               flux_dn=flux.flux('src_dn'), grid=g)
    return out
